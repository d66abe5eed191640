// File formats of the reference, host code only:
//  - body files source%04d.dat / target%04d.dat (exafmm include/dataset.h:
//    313-372): one value per line, x y z q per body (targets: pot ax ay az),
//    written with the stream's default formatting (6 significant digits);
//    reading continues at a caller-held stream position, as the reference's
//    Dataset::filePosition does across calls;
//  - the example's per-step report main.csv (ex/tapas_exafmm.cxx:651-677) and
//    the partition report of cpp/include/tapas/hot/report.h:40-152, in the
//    column layout of tapas::util::CSV / RankCSV (cpp/include/tapas/util.h:
//    113-316): a Rank column first, every field right-aligned to 14
//    characters (one blank after a field that fills its width, except the
//    last), doubles in std::scientific, integers as they print.
#include <unistd.h>

#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"

namespace tb {
namespace {

std::string body_file(const char *dir, const char *stem, int rank) {
  std::ostringstream name;
  if (dir && *dir) name << dir << '/';
  name << stem << std::setfill('0') << std::setw(4) << rank << ".dat";
  return name.str();
}

int write_columns(const char *dir, const char *stem, int rank, int64_t n,
                  const double *const cols[4], int stride, int digits) {
  if (rank < 0 || n < 0 || (n > 0 && !cols[0])) {
    set_error(nullptr, "write %s: bad rank, count or null array", stem);
    return TAPAS_B200_ERR_ARG;
  }
  const std::string path = body_file(dir, stem, rank);
  std::ofstream f(path.c_str(), std::ios::out);
  if (!f.good()) {
    set_error(nullptr, "write %s: cannot open %s", stem, path.c_str());
    return TAPAS_B200_ERR_ARG;
  }
  if (digits > 0) f << std::setprecision(digits);
  for (int64_t i = 0; i < n; i++)
    for (int c = 0; c < 4; c++) f << cols[c][(size_t)i * stride] << std::endl;
  f.close();
  if (!f) {
    set_error(nullptr, "write %s: write to %s failed", stem, path.c_str());
    return TAPAS_B200_ERR_ARG;
  }
  return TAPAS_B200_OK;
}

int read_columns(const char *dir, const char *stem, int rank, int64_t n, double *const cols[4],
                 int stride, int64_t *position) {
  if (rank < 0 || n < 0 || (n > 0 && !cols[0])) {
    set_error(nullptr, "read %s: bad rank, count or null array", stem);
    return TAPAS_B200_ERR_ARG;
  }
  const std::string path = body_file(dir, stem, rank);
  std::ifstream f(path.c_str(), std::ios::in);
  if (!f.good()) {
    set_error(nullptr, "read %s: cannot open %s", stem, path.c_str());
    return TAPAS_B200_ERR_ARG;
  }
  if (position) f.seekg((std::streamoff)*position);
  for (int64_t i = 0; i < n; i++)
    for (int c = 0; c < 4; c++) {
      if (!(f >> cols[c][(size_t)i * stride])) {
        set_error(nullptr, "read %s: %s holds fewer than %lld bodies after the start position",
                  stem, path.c_str(), (long long)n);
        return TAPAS_B200_ERR_ARG;
      }
    }
  if (position) *position = (int64_t)f.tellg();
  return TAPAS_B200_OK;
}

// One CSV field as tapas::util::Format prints it.
std::string fmt_field(double v) {
  std::ostringstream s;
  s << std::scientific << v;
  return s.str();
}
std::string fmt_field(uint64_t v) { return std::to_string(v); }
std::string fmt_field(int64_t v) { return std::to_string(v); }
std::string fmt_field(const std::string &v) { return v; }

constexpr int kCsvWidth = 14;  // CSV::kDefaultWidth

// A header line and one row in CSV::DumpHeader / CSV::Dump's layout.
int write_csv(const std::string &path, const std::vector<std::string> &cols,
              const std::vector<std::string> &vals) {
  std::ofstream f(path.c_str(), std::ios::out);
  if (!f.good()) {
    set_error(nullptr, "report: cannot open %s", path.c_str());
    return TAPAS_B200_ERR_ARG;
  }
  for (const auto &c : cols) {
    for (int i = (int)c.size(); i < kCsvWidth; i++) f << ' ';
    f << c;
  }
  f << '\n';
  for (size_t k = 0; k < vals.size(); k++) {
    const int npad = kCsvWidth - (int)vals[k].size();
    for (int i = 0; i < npad; i++) f << ' ';
    f << vals[k];
    if (k + 1 < vals.size() && npad <= 0) f << ' ';
  }
  f << '\n';
  f.close();
  if (!f) {
    set_error(nullptr, "report: write to %s failed", path.c_str());
    return TAPAS_B200_ERR_ARG;
  }
  return TAPAS_B200_OK;
}

}  // namespace
}  // namespace tb

using namespace tb;

extern "C" {

int tapas_b200_write_sources(const char *dir, int rank, int64_t n, const double *x,
                             const double *y, const double *z, const double *q, int digits) {
  if (n > 0 && (!x || !y || !z || !q)) {
    set_error(nullptr, "write_sources: null array");
    return TAPAS_B200_ERR_ARG;
  }
  const double *cols[4] = {x, y, z, q};
  return write_columns(dir, "source", rank, n, cols, 1, digits);
}

int tapas_b200_write_targets(const char *dir, int rank, int64_t n, const double *trg4,
                             int digits) {
  const double *cols[4] = {trg4, trg4 ? trg4 + 1 : nullptr, trg4 ? trg4 + 2 : nullptr,
                           trg4 ? trg4 + 3 : nullptr};
  return write_columns(dir, "target", rank, n, cols, 4, digits);
}

int tapas_b200_read_sources(const char *dir, int rank, int64_t n, double *x, double *y,
                            double *z, double *q, int64_t *position) {
  if (n > 0 && (!x || !y || !z || !q)) {
    set_error(nullptr, "read_sources: null array");
    return TAPAS_B200_ERR_ARG;
  }
  double *cols[4] = {x, y, z, q};
  return read_columns(dir, "source", rank, n, cols, 1, position);
}

int tapas_b200_read_targets(const char *dir, int rank, int64_t n, double *trg4,
                            int64_t *position) {
  double *cols[4] = {trg4, trg4 ? trg4 + 1 : nullptr, trg4 ? trg4 + 2 : nullptr,
                     trg4 ? trg4 + 3 : nullptr};
  return read_columns(dir, "target", rank, n, cols, 4, position);
}

int tapas_b200_write_main_csv(const char *path, int rank, double total, double upward,
                              double traverse, double downward, double tree, uint64_t num_p2p,
                              uint64_t num_m2l) {
  if (!path || !*path) {
    set_error(nullptr, "write_main_csv: empty path");
    return TAPAS_B200_ERR_ARG;
  }
  return write_csv(path,
                   {"Rank", "total", "upward", "traverse", "downward", "tree", "numP2P",
                    "numM2L"},
                   {fmt_field((int64_t)rank), fmt_field(total), fmt_field(upward),
                    fmt_field(traverse), fmt_field(downward), fmt_field(tree),
                    fmt_field(num_p2p), fmt_field(num_m2l)});
}

int tapas_b200_write_report(tapas_b200_ctx *ctx, const char *prefix, const char *suffix) {
  if (!ctx) {
    set_error(nullptr, "write_report: null context");
    return TAPAS_B200_ERR_ARG;
  }
  if (!ctx->have_tree) {
    set_error(ctx, "write_report: nothing evaluated");
    return TAPAS_B200_ERR_STATE;
  }
  // TAPAS_REPORT_PREFIX / TAPAS_REPORT_SUFFIX when not given, as the example does
  const char *ep = getenv("TAPAS_REPORT_PREFIX"), *es = getenv("TAPAS_REPORT_SUFFIX");
  const std::string pre = prefix ? prefix : (ep ? ep : "");
  const std::string suf = suffix ? suffix : (es ? es : "");
  const tapas_b200_timings &t = ctx->timings;
  const double s = 1e-3;  // phase timings are milliseconds; the reports hold seconds
  const double tree = s * (t.upload + t.bbox_keys + t.sort + t.tree);
  const double up = s * t.upward;
  const double trav = s * (t.traverse + t.list_sort + t.m2l + t.p2p);
  const double down = s * t.downward;
  const double total = tree + up + trav + down + s * t.download;
  // The example's counters count functor calls.  Non-mutual lists: one call
  // per listed pair and per body pair.  Mutual: one M2L call per unordered
  // pair (the lists hold both directions) and, for P2P, one call per body pair
  // of two leaves plus j <= i within a leaf; every non-empty leaf has its self
  // pair, so that is (directed body pairs + bodies) / 2.
  uint64_t np2p = 0, nm2l = 0;
  if (ctx->have_lists) {
    np2p = ctx->mutual ? (ctx->n_p2p_int + (uint64_t)ctx->n) / 2 : ctx->n_p2p_int;
    nm2l = ctx->mutual ? (uint64_t)ctx->n_m2l / 2 : (uint64_t)ctx->n_m2l;
  }
  TB_TRY(tapas_b200_write_main_csv((pre + "main" + suf + ".csv").c_str(), 0, total, up, trav,
                                   down, tree, np2p, nm2l));
  // hot/report.h on one rank: no sampling, exchange, global tree or LET
  char host[200] = {0};
  if (gethostname(host, sizeof host - 1) != 0) host[0] = '\0';
  TB_TRY(write_csv(pre + "hostnames" + suf + ".csv", {"Rank", "Hostname"},
                   {fmt_field((int64_t)0), std::string(host)}));
  TB_TRY(write_csv(pre + "misc" + suf + ".csv", {"SamplingRate", "NB"},
                   {fmt_field(1.0), fmt_field((int64_t)ctx->n)}));
  const int64_t nonleaf = (ctx->ncells - 1) / 8;
  TB_TRY(write_csv(pre + "load_balancing" + suf + ".csv",
                   {"Rank", "NumBodies1", "NumBodies2", "NumLeaves", "NumCells"},
                   {fmt_field((int64_t)0), fmt_field((int64_t)ctx->n), fmt_field((int64_t)ctx->n),
                    fmt_field(ctx->ncells - nonleaf), fmt_field(ctx->ncells)}));
  TB_TRY(write_csv(pre + "tree_construction" + suf + ".csv",
                   {"Rank", "all", "sample", "exchange", "grow-local", "grow-global"},
                   {fmt_field((int64_t)0), fmt_field(tree), fmt_field(0.0), fmt_field(0.0),
                    fmt_field(s * (t.bbox_keys + t.sort + t.tree)), fmt_field(0.0)}));
  TB_TRY(write_csv(pre + "map2" + suf + ".csv",
                   {"Rank", "all", "let", "net_traverse", "device_call"},
                   {fmt_field((int64_t)0), fmt_field(trav), fmt_field(0.0),
                    fmt_field(s * (t.traverse + t.list_sort)), fmt_field(s * (t.m2l + t.p2p))}));
  return TAPAS_B200_OK;
}

}  // extern "C"
