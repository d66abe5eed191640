// Test oracle driver around the UNMODIFIED reference Tapas ExaFMM example.
//
// This translation unit includes the reference's own example program
// (sample/exafmm-dev-13274dd4ac68/examples/tapas_exafmm.cxx) with its `main`
// renamed, so the reference's FMM_Upward / FMM_DTT / FMM_Downward functors,
// P2M/M2M/M2L/L2L/L2P/P2P callbacks, octree build and mappers run exactly as
// shipped.  Only the input (bodies read from a file instead of the example's
// built-in dataset generator) and the output (binary dump) differ from the
// example's main() at tapas_exafmm.cxx:448-712.
//
// It is test infrastructure: built by oracle/Makefile into oracle/_ref/, run
// only by tests/, tests/golden/make_golden.py and bench.py's reference arm.
//
// Usage:  tapas_exafmm_ref IN OUT [repeat [mutual]]
//   IN : int64 n, int32 ncrit, float64 theta, then n x {x,y,z,q} float64
//   mutual: 0 (default) or 1, the example's -m option (SetOptMutual and the
//           FMM_DTT mutual argument, tapas_exafmm.cxx:507-515,604-606)
//   OUT: see write_output() below.

#define main tapas_exafmm_reference_main
#include "tapas_exafmm.cxx"
#undef main

#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <vector>

namespace {

bool read_input(const char *path, Bodies &bodies, int &ncrit, double &theta) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  int64_t n = 0;
  int32_t nc = 0;
  double th = 0;
  bool ok = fread(&n, 8, 1, f) == 1 && fread(&nc, 4, 1, f) == 1 && fread(&th, 8, 1, f) == 1;
  std::vector<double> buf((size_t)n * 4);
  ok = ok && fread(buf.data(), 8, buf.size(), f) == buf.size();
  fclose(f);
  if (!ok) return false;
  bodies.resize((size_t)n);
  for (int64_t i = 0; i < n; i++) {
    Body &b = bodies[(size_t)i];
    b.X[0] = buf[4 * i + 0];
    b.X[1] = buf[4 * i + 1];
    b.X[2] = buf[4 * i + 2];
    b.SRC = buf[4 * i + 3];
    b.IBODY = (int)i;
    b.IRANK = 0;
    b.ICELL = 0;
    b.WEIGHT = 1;
    b.TRG = 0;
  }
  ncrit = nc;
  theta = th;
  return true;
}

template <class T>
void put(FILE *f, const T &v) { fwrite(&v, sizeof(T), 1, f); }

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s IN OUT [repeat [mutual]]\n", argv[0]);
    return 2;
  }
  int repeat = argc > 3 ? atoi(argv[3]) : 1;
  const int mutual = argc > 4 ? (atoi(argv[4]) != 0) : 0;
  Bodies input;
  int ncrit = 0;
  double theta = 0;
  if (!read_input(argv[1], input, ncrit, theta)) {
    fprintf(stderr, "cannot read %s\n", argv[1]);
    return 1;
  }
  MPI_Init(&argc, &argv);

  double t_tree = 0, t_up = 0, t_dtt = 0, t_down = 0, t_total = 0;
  Bodies bodies;
  TapasFMM::Cell *root = nullptr;
  for (int r = 0; r < repeat; r++) {
    bodies = input;
    ResetCount();
    // Same phase sequence and timers as tapas_exafmm.cxx:551-650.
    double total_bt = GetTime();
    double bt = GetTime();
    root = TapasFMM::Partition(bodies.data(), bodies.size(), ncrit);
    double et = GetTime();
    double tt = et - bt;
    root->SetOptMutual(mutual);
    bt = GetTime();
    TapasFMM::Map(FMM_Upward(), *root, (real_t)theta);
    et = GetTime();
    double tu = et - bt;
    bt = GetTime();
    TapasFMM::Map(FMM_DTT(), tapas::Product(*root, *root), mutual, 0, (real_t)theta);
    et = GetTime();
    double td = et - bt;
    bt = GetTime();
    TapasFMM::Map(FMM_Downward(), *root);
    et = GetTime();
    double tw = et - bt;
    CopyBackResult(bodies, root);
    double total_et = GetTime();
    double tot = total_et - total_bt;
    if (r == 0 || tot < t_total) {
      t_total = tot; t_tree = tt; t_up = tu; t_dtt = td; t_down = tw;
    }
  }

  // Output.
  FILE *f = fopen(argv[2], "wb");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", argv[2]);
    return 1;
  }
  auto &ht = root->data().ht_;
  std::vector<uint64_t> keys;
  keys.reserve(ht.size());
  for (auto &kv : ht) keys.push_back(kv.first);
  std::sort(keys.begin(), keys.end());

  int64_t n = (int64_t)bodies.size();
  int64_t ncells = (int64_t)keys.size();
  int32_t nterm = NTERM;
#ifdef COUNT
  uint64_t np2p = numP2P, nm2l = numM2L;
#else
  uint64_t np2p = 0, nm2l = 0;
#endif
  put(f, n);
  put(f, ncells);
  put(f, nterm);
  put(f, (int32_t)P);
  put(f, np2p);
  put(f, nm2l);
  put(f, t_tree); put(f, t_up); put(f, t_dtt); put(f, t_down); put(f, t_total);
  // Bodies in the reference's (Morton) order: original index, X, SRC, TRG.
  for (int64_t i = 0; i < n; i++) {
    const Body &b = bodies[(size_t)i];
    put(f, (int64_t)b.IBODY);
    put(f, (double)b.X[0]); put(f, (double)b.X[1]); put(f, (double)b.X[2]);
    put(f, (double)b.SRC);
    for (int d = 0; d < 4; d++) put(f, (double)b.TRG[d]);
  }
  // Cells sorted by key: key, leaf flag, nb, body offset, center, width, M, L.
  const Body *b0 = &root->local_body(0);
  for (uint64_t k : keys) {
    TapasFMM::Cell *c = ht[k];
    put(f, k);
    put(f, (int32_t)(c->IsLeaf() ? 1 : 0));
    put(f, (int32_t)c->local_nb());
    int64_t bid = c->IsLeaf() ? (int64_t)(&c->local_body(0) - b0) : 0;
    put(f, bid);
    for (int d = 0; d < 3; d++) put(f, (double)c->center()[d]);
    for (int d = 0; d < 3; d++) put(f, (double)c->width(d));
    for (int t = 0; t < NTERM; t++) { put(f, c->attr().M[t].real()); put(f, c->attr().M[t].imag()); }
    for (int t = 0; t < NTERM; t++) { put(f, c->attr().L[t].real()); put(f, c->attr().L[t].imag()); }
  }
  fclose(f);
  MPI_Finalize();
  return 0;
}
