// A Tapas program in the shape of the reference's drivers, built against
// include/tapas_b200/tapas.hpp and libtapas_b200.so.
//
//   fmm: the timestep of sample/exafmm-dev-13274dd4ac68/examples/
//        tapas_exafmm.cxx:560-641 (Partition, Map(FMM_Upward), Map(FMM_DTT,
//        Product(root, root), mutual, nspawn, theta), Map(FMM_Downward),
//        CopyBackResult)
//   bh:  calc() of sample/barnes-hut/bh.cc:228-245 (Partition, Map(Approximate),
//        Map(interact, Product(root, root), theta), read local_body_attr)
//
// usage: tapas_api_driver fmm|bh <in.bin> <out.bin> <P> <ncrit> <theta> <mixed>
//   in.bin:  int64 n, then x[n], y[n], z[n], q[n] (FP64)
//   out.bin: int64 n, then per body in the tree's order: int64 original
//            index, 4 FP64 results
// Exit status 0 on success, 3 when the library reports an error (message on
// stderr).
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tapas_b200/tapas.hpp"

// ExaFMM's body as the example uses it (exafmm include/types.h:62-75): the
// coordinates, the charge SRC, the original index IBODY and the result TRG.
struct kvec4 {
  double v[4];
  double &operator[](int i) { return v[i]; }
  const double &operator[](int i) const { return v[i]; }
};
struct Body {
  double X[3];
  double SRC;
  int64_t IBODY;
  kvec4 TRG;
};
struct CellAttr {};
static const size_t kBodyCoordOffset = offsetof(Body, X);
struct FMM_Params : public tapas::HOT<3, double, Body, kBodyCoordOffset, kvec4, CellAttr> {};
using TapasFMM = tapas::Tapas<FMM_Params>;

// The Barnes-Hut sample's body and attribute type (bh.cc:30-35, 72-78).
struct float4 {
  double x, y, z, w;
};
struct BH_Params : public tapas::HOT<3, double, float4, 0, float4, float4> {};
using TapasBH = tapas::Tapas<BH_Params>;
using Vec3 = tapas::Vec<3, double>;

static void CopyBackResult(std::vector<Body> &bodies, TapasFMM::Cell *root) {
  bodies.clear();
  Body *beg = &root->local_body(0);
  bodies.assign(beg, beg + root->local_nb());
  for (size_t i = 0; i < bodies.size(); i++) bodies[i].TRG = root->local_body_attr((long)i);
}

static bool read_input(const char *path, std::vector<double> &x, std::vector<double> &y,
                       std::vector<double> &z, std::vector<double> &q) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  int64_t n = 0;
  bool ok = std::fread(&n, 8, 1, f) == 1 && n > 0;
  if (ok) {
    x.resize(n);
    y.resize(n);
    z.resize(n);
    q.resize(n);
    for (auto *a : {&x, &y, &z, &q}) ok = ok && std::fread(a->data(), 8, n, f) == (size_t)n;
  }
  std::fclose(f);
  return ok;
}

static bool write_output(const char *path, const std::vector<int64_t> &idx,
                         const std::vector<double> &res) {
  FILE *f = std::fopen(path, "wb");
  if (!f) return false;
  const int64_t n = (int64_t)idx.size();
  bool ok = std::fwrite(&n, 8, 1, f) == 1;
  for (int64_t i = 0; ok && i < n; i++)
    ok = std::fwrite(&idx[i], 8, 1, f) == 1 && std::fwrite(&res[4 * i], 8, 4, f) == 4;
  return std::fclose(f) == 0 && ok;
}

int main(int argc, char **argv) {
  if (argc != 8) {
    std::fprintf(stderr, "usage: %s fmm|bh in.bin out.bin P ncrit theta mixed\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  const int P = std::atoi(argv[4]);
  const int ncrit = std::atoi(argv[5]);
  const double theta = std::atof(argv[6]);
  tapas::b200::options().P = P;
  tapas::b200::options().precision = std::atoi(argv[7]) ? TAPAS_B200_MIXED : TAPAS_B200_FP64;

  std::vector<double> x, y, z, q;
  if (!read_input(argv[2], x, y, z, q)) {
    std::fprintf(stderr, "cannot read %s\n", argv[2]);
    return 2;
  }
  const size_t n = x.size();
  std::vector<int64_t> idx(n);
  std::vector<double> res(4 * n);
  try {
    if (mode == "fmm") {
      std::vector<Body> bodies(n);
      for (size_t i = 0; i < n; i++) {
        bodies[i].X[0] = x[i];
        bodies[i].X[1] = y[i];
        bodies[i].X[2] = z[i];
        bodies[i].SRC = q[i];
        bodies[i].IBODY = (int64_t)i;
      }
      TapasFMM::Cell *root = TapasFMM::Partition(bodies.data(), (long)bodies.size(), ncrit);
      root->SetOptMutual(false);
      TapasFMM::Map(tapas::FMM_Upward(), *root, theta);
      const int mutual = 0, nspawn = 1000;
      TapasFMM::Map(tapas::FMM_DTT(), tapas::Product(*root, *root), mutual, nspawn, theta);
      TapasFMM::Map(tapas::FMM_Downward(), *root);
      CopyBackResult(bodies, root);
      delete root;
      for (size_t i = 0; i < n; i++) {
        idx[i] = bodies[i].IBODY;
        for (int k = 0; k < 4; k++) res[4 * i + k] = bodies[i].TRG[k];
      }
    } else if (mode == "bh") {
      std::vector<float4> source(n);
      for (size_t i = 0; i < n; i++) source[i] = float4{x[i], y[i], z[i], q[i]};
      TapasBH::Region r(Vec3(0.0, 0.0, 0.0), Vec3(1.0, 1.0, 1.0));
      (void)r;
      TapasBH::Cell *root = TapasBH::Partition(source.data(), (long)source.size(), ncrit);
      TapasBH::Map(tapas::Approximate(), *root);
      TapasBH::Map(tapas::interact(), tapas::Product(*root, *root), theta);
      const long nb = (long)root->local_nb();
      std::vector<float4> out(&root->local_body_attr(0), &root->local_body_attr(0) + nb);
      source = std::vector<float4>(&root->local_body(0), &root->local_body(0) + nb);
      root->Report();
      // The sample's bodies carry no index: recover it from the tree's order.
      std::vector<int64_t> orig(n);
      if (tapas_b200_get_sorted(root->context(), orig.data(), nullptr) != TAPAS_B200_OK) {
        std::fprintf(stderr, "get_sorted failed\n");
        return 3;
      }
      delete root;
      for (size_t i = 0; i < n; i++) {
        idx[i] = orig[i];
        const double v[4] = {out[i].x, out[i].y, out[i].z, out[i].w};
        std::memcpy(&res[4 * i], v, sizeof v);
      }
    } else {
      std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
      return 2;
    }
  } catch (const tapas::b200::Error &e) {
    std::fprintf(stderr, "tapas_b200 error %d: %s\n", e.code, e.what());
    return 3;
  }
  if (!write_output(argv[3], idx, res)) {
    std::fprintf(stderr, "cannot write %s\n", argv[3]);
    return 2;
  }
  return 0;
}
