// User functors on the GPU through include/tapas_b200/device.cuh and the
// Tapas header, compiled by nvcc the way the reference's CUDA build compiles
// its examples.
//
//  1. FMM_DTT_With<P2P>: the example's timestep with the near field computed
//     by a user P2P functor written like the reference's CUDA one
//     (sample/exafmm-dev-13274dd4ac68/examples/LaplaceP2PCPU_tapas.h:23-44,
//     accumulating through tapas::Accumulate), against the same timestep with
//     the library's own P2P kernel;
//  2. MapReduce: per-cell charge-weighted position sums and charge (the
//     Barnes-Hut sample's centre-of-mass pass, bh_reduce.cc:155-190), against
//     sums over each cell's body range on the host;
//  3. MapCells + Reduce: cells per level counted with atomic reduces, against
//     the level table.
//
// usage: device_api_test N P NCRIT THETA  -> one JSON line; exit 0 when every
// check is within its tolerance, 1 otherwise, 3 on a library error.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tapas_b200/tapas.hpp"

struct kvec4 {
  double v[4];
  __host__ __device__ double &operator[](int i) { return v[i]; }
  __host__ __device__ const double &operator[](int i) const { return v[i]; }
};
struct Body {
  double X[3];
  double SRC;
  int64_t IBODY;
  kvec4 TRG;
};
struct CellAttr {};
struct FMM_Params : public tapas::HOT<3, double, Body, 0, kvec4, CellAttr> {};
using TapasFMM = tapas::Tapas<FMM_Params>;

struct Vec3d {
  double v[3];
};

// The reference's CUDA P2P functor, in this program's types: pot += qi qj / r,
// acc -= qi qj dX / r^3, r = 0 skipped, no softening.
struct P2P {
  template <class B, class A>
  __host__ __device__ void operator()(B &bi, A &ai, B &bj, A &, Vec3d xp, int) const {
    double d[3];
    for (int k = 0; k < 3; k++) d[k] = bi.X[k] - bj.X[k] - xp.v[k];
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 != 0) {
      const double inv_r2 = 1.0 / r2;
      const double qq_r = bi.SRC * bj.SRC * sqrt(inv_r2);
      const double s = inv_r2 * qq_r;
      tapas::Accumulate(ai[0], qq_r);
      tapas::Accumulate(ai[1], -d[0] * s);
      tapas::Accumulate(ai[2], -d[1] * s);
      tapas::Accumulate(ai[3], -d[2] * s);
    }
  }
};
// the reference's extra (Xperiodic, mutual) arguments, bound
struct P2PBound {
  P2P f;
  template <class B, class A>
  __device__ void operator()(B &bi, A &ai, B &bj, A &aj) const {
    f(bi, ai, bj, aj, Vec3d{{0, 0, 0}}, 0);
  }
};

struct Moment {
  double x, y, z, w;
};
struct LeafMoment {
  __device__ Moment operator()(const tapas::b200::CellView &, const Body *b, int nb) const {
    Moment m{0, 0, 0, 0};
    for (int i = 0; i < nb; i++) {
      m.x += b[i].SRC * b[i].X[0];
      m.y += b[i].SRC * b[i].X[1];
      m.z += b[i].SRC * b[i].X[2];
      m.w += b[i].SRC;
    }
    return m;
  }
};
struct AddMoment {
  __device__ Moment operator()(Moment a, Moment b) const {
    return Moment{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w};
  }
};
struct KeepMoment {
  __device__ Moment operator()(const tapas::b200::CellView &, Moment m) const { return m; }
};
struct AddInt {
  __device__ unsigned long long operator()(unsigned long long a, unsigned long long b) const {
    return a + b;
  }
};
struct CountLevel {
  unsigned long long *count;
  __device__ void operator()(const tapas::b200::CellView &c, int) const {
    tapas::b200::Reduce(count[c.level], 1ull, AddInt());
  }
};

int main(int argc, char **argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s N P NCRIT THETA\n", argv[0]);
    return 2;
  }
  const int64_t n = atoll(argv[1]);
  const int P = atoi(argv[2]), ncrit = atoi(argv[3]);
  const double theta = atof(argv[4]);
  std::vector<Body> bodies((size_t)n);
  uint64_t s = 12345;
  auto next = [&]() {  // 53-bit uniform [0, 1) from a 64-bit LCG
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int64_t i = 0; i < n; i++) {
    Body &b = bodies[(size_t)i];
    for (int k = 0; k < 3; k++) b.X[k] = 2 * next() - 1;
    b.SRC = next() + 0.01;
    b.IBODY = i;
  }
  tapas::b200::options().P = P;
  try {
    // 1. user P2P functor vs the library's P2P
    TapasFMM::Cell *a = TapasFMM::Partition(bodies.data(), n, ncrit);
    TapasFMM::Map(tapas::FMM_Upward(), *a, theta);
    TapasFMM::Map(tapas::FMM_DTT_With<P2PBound>{}, tapas::Product(*a, *a), 0, 0, theta);
    TapasFMM::Map(tapas::FMM_Downward(), *a);
    TapasFMM::Cell *b = TapasFMM::Partition(bodies.data(), n, ncrit);
    TapasFMM::Map(tapas::FMM_Upward(), *b, theta);
    TapasFMM::Map(tapas::FMM_DTT(), tapas::Product(*b, *b), 0, 0, theta);
    TapasFMM::Map(tapas::FMM_Downward(), *b);
    double num = 0, den = 0;
    for (int64_t i = 0; i < n; i++)
      for (int k = 0; k < 4; k++) {
        num = fmax(num, fabs(a->local_body_attr(i)[k] - b->local_body_attr(i)[k]));
        den = fmax(den, fabs(b->local_body_attr(i)[k]));
      }
    const double rel_p2p = num / den;
    // 2. MapReduce moments vs host sums over the cells' body ranges
    std::vector<Moment> mom =
        TapasFMM::MapReduce<Moment>(*a, LeafMoment(), AddMoment(), KeepMoment());
    const int64_t C = a->tree_info().n_cells;
    std::vector<int32_t> nb(C), bbeg(C);
    tapas::b200::check(tapas_b200_get_cells(a->context(), nullptr, nullptr, nb.data(),
                                            bbeg.data(), nullptr, nullptr, nullptr, nullptr),
                       a->context());
    double rel_mom = 0;
    for (int64_t c = 0; c < C; c++) {
      double h[4] = {0, 0, 0, 0}, habs = 0;
      for (int32_t i = bbeg[c]; i < bbeg[c] + nb[c]; i++) {
        const Body &bd = a->local_body(i);
        for (int k = 0; k < 3; k++) h[k] += bd.SRC * bd.X[k];
        h[3] += bd.SRC;
        habs += bd.SRC * (1 + fabs(bd.X[0]) + fabs(bd.X[1]) + fabs(bd.X[2]));
      }
      const double g[4] = {mom[c].x, mom[c].y, mom[c].z, mom[c].w};
      for (int k = 0; k < 4; k++)
        if (habs > 0) rel_mom = fmax(rel_mom, fabs(g[k] - h[k]) / habs);
    }
    // 3. cells per level with Reduce
    tapas_b200_device_view v;
    tapas::b200::check(tapas_b200_get_device_view(a->context(), &v), a->context());
    unsigned long long *dcount = nullptr;
    cudaMalloc(&dcount, sizeof(unsigned long long) * TAPAS_B200_MAX_LEVELS);
    cudaMemset(dcount, 0, sizeof(unsigned long long) * TAPAS_B200_MAX_LEVELS);
    tapas::b200::check(tapas::b200::MapCells(a->context(), CountLevel{dcount}, true),
                       a->context());
    std::vector<unsigned long long> count(TAPAS_B200_MAX_LEVELS);
    cudaDeviceSynchronize();
    cudaMemcpy(count.data(), dcount, sizeof(unsigned long long) * count.size(),
               cudaMemcpyDeviceToHost);
    cudaFree(dcount);
    bool count_ok = true;
    for (int64_t l = 0; l < v.n_levels; l++)
      count_ok = count_ok &&
                 count[(size_t)l] == (unsigned long long)(v.level_off[l + 1] - v.level_off[l]);
    printf("{\"max_rel_user_p2p\": %.3e, \"max_rel_mapreduce\": %.3e, \"reduce_levels_ok\": %s, "
           "\"levels\": %lld, \"cells\": %lld}\n",
           rel_p2p, rel_mom, count_ok ? "true" : "false", (long long)v.n_levels, (long long)C);
    delete a;
    delete b;
    return (rel_p2p < 1e-12 && rel_mom < 1e-13 && count_ok) ? 0 : 1;
  } catch (const tapas::b200::Error &e) {
    fprintf(stderr, "library error %d: %s\n", e.code, e.what());
    return 3;
  }
}
