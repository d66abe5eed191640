// tapas_b200/tapas.hpp - C++ host side of libtapas_b200 in the shape of the
// reference's Tapas API, for the ExaFMM Laplace-spherical and Barnes-Hut
// paths.
//
// A program written against the reference (sample/exafmm-dev-13274dd4ac68/
// examples/tapas_exafmm.cxx, sample/barnes-hut/bh.cc) keeps its calls:
//
//   using TapasFMM = tapas::Tapas<FMM_Params>;          // FMM_Params : tapas::HOT<...>
//   TapasFMM::Cell *root = TapasFMM::Partition(bodies.data(), bodies.size(), ncrit);
//   TapasFMM::Map(FMM_Upward(), *root, theta);
//   TapasFMM::Map(FMM_DTT(), tapas::Product(*root, *root), mutual, nspawn, theta);
//   TapasFMM::Map(FMM_Downward(), *root);
//   ... root->local_body(i), root->local_body_attr(i)    // CopyBackResult
//
// and replaces the reference headers (tapas.h, tapas_exafmm.h and the ExaFMM
// callback headers) with this one.  The functor types FMM_Upward, FMM_DTT,
// FMM_Downward (and Approximate, interact for Barnes-Hut) are provided here as
// tags: their bodies run as sm_100a kernels, so a Map over a functor the
// library has no kernel for does not compile (static_assert), and there is no
// CPU fallback.
//
// Mapping of the reference's types and calls:
//   tapas::HOT<3, double, Body, ofst, BodyAttr, CellAttr>  cpp/include/tapas/hot.h:1308-1330
//   tapas::Tapas<TSP>::Partition                           hot.h:1349-1352
//   tapas::Tapas<TSP>::Map (cell, product, ...)             hot.h:1354-1396
//   tapas::Product(Cell&, Cell&)                            hot.h:1296-1305
//   Cell::local_nb / local_body / local_body_attr           hot.h:319-345
// The body charge is read through tapas::b200::BodyCharge<Body> (default: the
// ExaFMM member SRC); the coordinates at the TSP's byte offset, as the
// reference's ParticlePosOffset does (basic_types.h:110-118).
// Expansion order and arithmetic: tapas::b200::options() (the reference fixes
// the order at compile time with EXPANSION).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../tapas_b200.h"
#ifdef __CUDACC__
#include "device.cuh"
#endif

namespace tapas {

using index_t = long;

namespace b200 {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const tapas_b200_ctx *ctx) {
  if (rc != TAPAS_B200_OK) throw Error(rc, tapas_b200_last_error(ctx));
}

struct Options {
  int P = 10;                        // expansion order (2..16)
  int precision = TAPAS_B200_FP64;   // or TAPAS_B200_MIXED
  int device = 0;
  double bh_eps2 = 1e-6;             // Barnes-Hut softening (bh.cc:21)
};
inline Options &options() {
  static Options o;
  return o;
}

// Charge (FMM) or mass (Barnes-Hut) of a body: the member SRC of an ExaFMM
// Body (exafmm include/types.h:62-66), else the member w of the Barnes-Hut
// sample's float4 (bh.cc:30-35).  Specialise for other bodies.
template <class Body, class = void>
struct BodyCharge {
  static double get(const Body &b) { return (double)b.w; }
};
template <class Body>
struct BodyCharge<Body, decltype((void)std::declval<const Body &>().SRC)> {
  static double get(const Body &b) { return (double)b.SRC; }
};

// Stores one body's four results (ax, ay, az, potential in the Barnes-Hut
// sample's x, y, z, w; potential, ax, ay, az in ExaFMM's kvec4 TRG).
template <class Attr, class = void>
struct AttrStore {
  static void set(Attr &a, const double *t) {
    for (int k = 0; k < 4; k++) a[k] = t[k];
  }
};
template <class Attr>
struct AttrStore<Attr, decltype((void)std::declval<Attr &>().w)> {
  static void set(Attr &a, const double *t) {
    a.x = t[0];
    a.y = t[1];
    a.z = t[2];
    a.w = t[3];
  }
};

// Kernel kinds behind the functor tags below.
enum class Kind { None, FmmUpward, FmmDTT, FmmDownward, BhApproximate, BhInteract };
template <class F>
struct KindOf {
  static constexpr Kind value = Kind::None;
};

}  // namespace b200

// Tags of the reference example's functors (ex/tapas_exafmm.cxx:87-286) and
// of the Barnes-Hut sample's (bh.cc:155-224).
struct FMM_Upward {};
struct FMM_DTT {};
struct FMM_Downward {};
struct Approximate {};
struct interact {};

namespace b200 {
template <> struct KindOf<FMM_Upward> { static constexpr Kind value = Kind::FmmUpward; };
template <> struct KindOf<FMM_DTT> { static constexpr Kind value = Kind::FmmDTT; };
template <> struct KindOf<FMM_Downward> { static constexpr Kind value = Kind::FmmDownward; };
template <> struct KindOf<Approximate> { static constexpr Kind value = Kind::BhApproximate; };
template <> struct KindOf<interact> { static constexpr Kind value = Kind::BhInteract; };
}  // namespace b200

// Small fixed vector and region (cpp/include/tapas/vec.h, basic_types.h:
// Region).  The partition computes its own bounding cube, as the reference's
// HOT partition does; a Region is accepted and kept only for source
// compatibility.
template <int DIM, class FP>
struct Vec {
  FP v[DIM];
  template <class... T>
  Vec(T... a) : v{(FP)a...} {
    static_assert(sizeof...(T) == DIM, "one value per dimension");
  }
  FP &operator[](int i) { return v[i]; }
  const FP &operator[](int i) const { return v[i]; }
};

template <int DIM, class FP>
struct Region {
  Vec<DIM, FP> min, max;
  Region(const Vec<DIM, FP> &lo, const Vec<DIM, FP> &hi) : min(lo), max(hi) {}
};

// Tapas static parameters (hot.h:1308-1330).
template <int DIM, class FP, class BODY, size_t BODY_COORD_OFST, class BODY_ATTR, class CELL_ATTR>
struct HOT {
  static_assert(DIM == 3, "the B200 path is three-dimensional");
  static_assert(std::is_same<FP, double>::value, "bodies are FP64");
  static constexpr int Dim = DIM;
  static constexpr size_t kBodyCoordOffset = BODY_COORD_OFST;
  using FP_ = FP;
  using Body = BODY;
  using BodyAttr = BODY_ATTR;
  using CellAttr = CELL_ATTR;
};

template <class TSP>
class Cell {
 public:
  using Body = typename TSP::Body;
  using BodyAttr = typename TSP::BodyAttr;

  Cell() {
    check_(tapas_b200_ctx_create(b200::options().device, &ctx_));
  }
  ~Cell() { tapas_b200_ctx_destroy(ctx_); }
  Cell(const Cell &) = delete;
  Cell &operator=(const Cell &) = delete;

  bool IsRoot() const { return true; }
  bool IsLeaf() const { return info_.n_cells == 1; }
  size_t local_nb() const { return (size_t)info_.n_bodies; }
  size_t nb() const { return local_nb(); }
  // Bodies and their attributes in the tree's (Morton) order, as the
  // reference's root cell exposes them after the Maps (hot.h:966-1010).
  Body &local_body(index_t i) { return bodies_[(size_t)i]; }
  const Body &local_body(index_t i) const { return bodies_[(size_t)i]; }
  BodyAttr &local_body_attr(index_t i) { return attrs_[(size_t)i]; }
  const BodyAttr &local_body_attr(index_t i) const { return attrs_[(size_t)i]; }
  void SetOptMutual(bool m) { mutual_ = m; }
  bool GetOptMutual() const { return mutual_; }
  void Report() const {}
  tapas_b200_ctx *context() const { return ctx_; }
  const tapas_b200_tree_stats &tree_info() const { return info_; }

  // --- used by Tapas<TSP> ---
  void partition_(const Body *b, index_t nb, int ncrit) {
    const size_t n = (size_t)nb;
    std::vector<double> x(n), y(n), z(n), q(n);
    for (size_t i = 0; i < n; i++) {
      double p[3];
      std::memcpy(p, reinterpret_cast<const char *>(b + i) + TSP::kBodyCoordOffset, sizeof p);
      x[i] = p[0];
      y[i] = p[1];
      z[i] = p[2];
      q[i] = b200::BodyCharge<Body>::get(b[i]);
    }
    check_(tapas_b200_partition(ctx_, x.data(), y.data(), z.data(), q.data(), (int64_t)n, ncrit,
                                TAPAS_B200_HOST));
    check_(tapas_b200_tree_info(ctx_, &info_));
    std::vector<int64_t> orig(n);
    check_(tapas_b200_get_sorted(ctx_, orig.data(), nullptr));
    bodies_.resize(n);
    for (size_t i = 0; i < n; i++) bodies_[i] = b[(size_t)orig[i]];
    attrs_.assign(n, BodyAttr());
  }
  void fetch_results_() {
    const size_t n = bodies_.size();
    std::vector<double> t(4 * n);
    check_(tapas_b200_get_results(ctx_, t.data(), TAPAS_B200_ORDER_SORTED, TAPAS_B200_HOST));
    for (size_t i = 0; i < n; i++) b200::AttrStore<BodyAttr>::set(attrs_[i], &t[4 * i]);
  }
  void check_(int rc) const { b200::check(rc, ctx_); }
#ifdef __CUDACC__
  // The user's P2P functor over the context's leaf pairs, on device copies
  // of the bodies (BodyAttr starts value-initialised); the near field goes
  // back to the library for the L2P.  BodyAttr must be the four doubles of
  // ExaFMM's kvec4 (pot, ax, ay, az).
  template <class F>
  void user_p2p_(F f) {
    static_assert(sizeof(BodyAttr) == 4 * sizeof(double),
                  "the near field is four doubles per body (ExaFMM kvec4)");
    const size_t n = bodies_.size();
    Body *db = nullptr;
    BodyAttr *da = nullptr;
    const std::vector<BodyAttr> zero(n, BodyAttr());
    int rc = cudaMalloc(&db, sizeof(Body) * n) == cudaSuccess &&
                     cudaMalloc(&da, sizeof(BodyAttr) * n) == cudaSuccess
                 ? TAPAS_B200_OK
                 : TAPAS_B200_ERR_NOMEM;
    if (rc == TAPAS_B200_OK &&
        (cudaMemcpy(db, bodies_.data(), sizeof(Body) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(da, zero.data(), sizeof(BodyAttr) * n, cudaMemcpyHostToDevice) != cudaSuccess))
      rc = TAPAS_B200_ERR_CUDA;
    if (rc == TAPAS_B200_OK) rc = b200::Map2LeafPairs(ctx_, db, da, f);
    if (rc == TAPAS_B200_OK)
      rc = tapas_b200_set_near_field(ctx_, reinterpret_cast<const double *>(da),
                                     TAPAS_B200_DEVICE);
    void *s = nullptr;
    tapas_b200_get_stream(ctx_, &s);
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(s)) != cudaSuccess && rc == TAPAS_B200_OK)
      rc = TAPAS_B200_ERR_CUDA;
    cudaFree(db);
    cudaFree(da);
    if (rc != TAPAS_B200_OK && rc != TAPAS_B200_ERR_STATE)
      throw b200::Error(rc, std::string("user P2P functor: ") + tapas_b200_last_error(ctx_));
    check_(rc);
  }
  // MapReduce over the tree (device.cuh) with the root's bodies; values in
  // get_cells order.
  template <class T, class LeafF, class Op, class PostF>
  std::vector<T> map_reduce_(LeafF leaf, Op op, PostF post) {
    const size_t n = bodies_.size(), C = (size_t)info_.n_cells;
    Body *db = nullptr;
    T *dv = nullptr;
    std::vector<T> out(C);
    int rc = cudaMalloc(&db, sizeof(Body) * n) == cudaSuccess &&
                     cudaMalloc(&dv, sizeof(T) * C) == cudaSuccess
                 ? TAPAS_B200_OK
                 : TAPAS_B200_ERR_NOMEM;
    if (rc == TAPAS_B200_OK &&
        cudaMemcpy(db, bodies_.data(), sizeof(Body) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = TAPAS_B200_ERR_CUDA;
    if (rc == TAPAS_B200_OK) rc = b200::MapReduce(ctx_, db, dv, leaf, op, post);
    void *s = nullptr;
    tapas_b200_get_stream(ctx_, &s);
    if (rc == TAPAS_B200_OK &&
        (cudaStreamSynchronize(static_cast<cudaStream_t>(s)) != cudaSuccess ||
         cudaMemcpy(out.data(), dv, sizeof(T) * C, cudaMemcpyDeviceToHost) != cudaSuccess))
      rc = TAPAS_B200_ERR_CUDA;
    cudaFree(db);
    cudaFree(dv);
    check_(rc);
    return out;
  }
#endif

 private:
  tapas_b200_ctx *ctx_ = nullptr;
  tapas_b200_tree_stats info_{};
  std::vector<Body> bodies_;
  std::vector<BodyAttr> attrs_;
  bool mutual_ = false;
};

#ifdef __CUDACC__
// FMM_DTT with the user's own body-pair functor for the near field, the
// reference's P2P offload through its vectormap (the traversal's leaf pairs
// go to Map2LeafPairs; include/tapas_b200/device.cuh).  The functor is called
// as p2p(Body &bi, BodyAttr &ai, Body &bj, BodyAttr &aj) on the device, one
// thread per target body; a reference functor with the extra (Xperiodic,
// mutual) arguments is wrapped by a functor that passes them.
template <class P2PFunctor>
struct FMM_DTT_With {
  P2PFunctor p2p;
};
#endif

template <class CELL>
struct ProductIterator {
  CELL &t1_;
  CELL &t2_;
};

template <class TSP>
ProductIterator<Cell<TSP>> Product(Cell<TSP> &c1, Cell<TSP> &c2) {
  return ProductIterator<Cell<TSP>>{c1, c2};
}

template <class TSP>
struct Tapas {
  using Cell = tapas::Cell<TSP>;
  using Body = typename TSP::Body;
  using Region = tapas::Region<TSP::Dim, typename TSP::FP_>;

  // hot.h:1349-1352.  The returned root owns the GPU state; delete it (or
  // keep it) as the reference program's lifetime requires.
  static Cell *Partition(Body *b, index_t nb, int max_nb) {
    std::unique_ptr<Cell> c(new Cell());
    c->partition_(b, nb, max_nb);
    return c.release();
  }

  // Map over a cell: upward / downward passes (hot.h:1393-1396).
  template <class Funct, class... Args>
  static void Map(Funct, Cell &c, Args... args) {
    constexpr b200::Kind k = b200::KindOf<Funct>::value;
    static_assert(k == b200::Kind::FmmUpward || k == b200::Kind::FmmDownward ||
                      k == b200::Kind::BhApproximate,
                  "no sm_100a kernel for this functor in a cell Map");
    const b200::Options &o = b200::options();
    if (k == b200::Kind::FmmUpward) {
      c.check_(tapas_b200_upward(c.context(), o.P, o.precision));
    } else if (k == b200::Kind::FmmDownward) {
      c.check_(tapas_b200_downward(c.context(), o.precision));
      c.fetch_results_();
    } else {
      c.check_(tapas_b200_bh_upward(c.context()));
    }
    (void)sizeof...(args);
  }

  // Map over the root x root product: the dual-tree traversal with M2L and
  // P2P (FMM_DTT, args: mutual, nspawn, theta) or the Barnes-Hut walk
  // (interact, args: theta) (hot.h:1354-1360).
  template <class Funct, class... Args>
  static void Map(Funct, ProductIterator<Cell> prod, Args... args) {
    constexpr b200::Kind k = b200::KindOf<Funct>::value;
    static_assert(k == b200::Kind::FmmDTT || k == b200::Kind::BhInteract,
                  "no sm_100a kernel for this functor in a product Map");
    if (&prod.t1_ != &prod.t2_) throw b200::Error(TAPAS_B200_ERR_ARG, "Product(root, root) only");
    const b200::Options &o = b200::options();
    const double a[] = {(double)args...};
    if (k == b200::Kind::FmmDTT) {
      static_assert(k != b200::Kind::FmmDTT || sizeof...(args) == 3,
                    "FMM_DTT takes (mutual, nspawn, theta)");
      prod.t1_.check_(tapas_b200_traverse(prod.t1_.context(), a[2], (int)a[0], o.precision));
    } else {
      static_assert(k != b200::Kind::BhInteract || sizeof...(args) == 1, "interact takes (theta)");
      prod.t1_.check_(tapas_b200_bh_interact(prod.t1_.context(), a[0], o.bh_eps2, o.precision));
      prod.t1_.fetch_results_();
    }
  }

#ifdef __CUDACC__
  // FMM_DTT with the user's P2P functor (args: mutual, nspawn, theta): lists
  // and M2L by the library, the near field by the functor on the device.
  template <class F, class... Args>
  static void Map(FMM_DTT_With<F> fn, ProductIterator<Cell> prod, Args... args) {
    static_assert(sizeof...(args) == 3, "FMM_DTT takes (mutual, nspawn, theta)");
    if (&prod.t1_ != &prod.t2_) throw b200::Error(TAPAS_B200_ERR_ARG, "Product(root, root) only");
    const double a[] = {(double)args...};
    Cell &c = prod.t1_;
    c.check_(tapas_b200_build_lists(c.context(), a[2], (int)a[0]));
    c.check_(tapas_b200_m2l(c.context(), b200::options().precision));
    c.user_p2p_(fn.p2p);
  }

  // MapReduce (the reference's proposed Reduce API, bh_reduce.cc:186):
  // per cell, children before parents, leaf(cell, bodies, nb) at leaves and
  // op folded over the 8 children in order elsewhere, then post(cell, value);
  // device functors; values in get_cells order.
  template <class T, class LeafF, class Op, class PostF>
  static std::vector<T> MapReduce(Cell &c, LeafF leaf, Op op, PostF post) {
    return c.template map_reduce_<T>(leaf, op, post);
  }
#endif
};

}  // namespace tapas
