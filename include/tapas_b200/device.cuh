// tapas_b200/device.cuh - user functors on the GPU over libtapas_b200's tree
// and lists, compiled into the user's program by nvcc (sm_100a).
//
// The reference offloads any __host__ __device__ body-pair functor through
// its vectormap: the traversal collects leaf pairs (map2), and Finish2 runs
// the functor over every body pair on the GPU (cpp/include/tapas/
// vectormap_cuda.h:645-1005, kernel :219-280, accumulation through
// tapas::Accumulate's atomics, map.h:159-211).  Its unfinished Reduce /
// MapReduce (sample/barnes-hut/bh_reduce.cc:186, bh_accumulate.cc:190-193,
// examples/tapas_exafmm_reduce.cxx:109,162) folds children into parents.
// Here:
//
//   Map2LeafPairs(ctx, bodies, attrs, f, args...)
//       f(const Body &bi, Attr &ai, const Body &bj, const Attr &aj, args...)
//       for every body pair of every (target leaf, source leaf) pair of the
//       context's P2P list, on device arrays of the caller's Body / Attr
//       types in the tree's (Morton) order.  One thread owns each target body
//       and keeps its attribute in registers, so f writes ai without atomics.
//   MapCells(ctx, f, up)
//       f(const CellView &c, int cell) for every cell, level by level
//       (children before parents when up, parents first otherwise).
//   MapReduce(ctx, bodies, vals, leaf, op, post)
//       per cell, children before parents: a leaf's value is
//       leaf(cell, bodies + bbeg, nb), a parent's is op folded over its 8
//       children in child order (a fixed order: deterministic); then
//       vals[cell] = post(cell, value).
//   Reduce(dst, v, op)   (device)
//       dst = op(dst, v) as one atomic step (compare-and-swap loop), for
//       4- and 8-byte T: the reference's out-of-order reduce into a shared
//       parent attribute.
//
// All launches go on the context's stream; the functions return the
// library's status codes (TAPAS_B200_ERR_CUDA on a launch failure).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <type_traits>

#include "../tapas_b200.h"

namespace tapas {

// The reference's tapas::Accumulate (cpp/include/tapas/map.h:159-211) adds
// with a compare-and-swap loop because its kernel shares target attributes
// between threads.  Map2LeafPairs gives every target body to one thread, so
// an accumulation is a plain add (and works on the register copy it passes).
template <class T>
__host__ __device__ inline void Accumulate(T &to, T v) {
  to += v;
}

namespace b200 {

// What a cell functor sees of a cell.
struct CellView {
  int32_t index, nb, bbeg, leaf, level, parent, child0;
  double center[3], width;
};

__device__ __forceinline__ CellView cell_view(const tapas_b200_device_view &v, int c) {
  CellView cv;
  cv.index = c;
  cv.nb = v.nb[c];
  cv.bbeg = v.bbeg[c];
  cv.leaf = v.leaf[c];
  cv.level = v.level[c];
  cv.parent = v.parent[c];
  cv.child0 = v.child0[c];
  for (int d = 0; d < 3; d++) cv.center[d] = v.center3[3 * c + d];
  cv.width = v.max3[3 * c] - v.min3[3 * c];
  return cv;
}

// dst = op(dst, v), atomically (compare-and-swap on the value's bits).
template <class T, class Op>
__device__ inline T Reduce(T &dst, T v, Op op) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "Reduce works on 4- and 8-byte values");
  static_assert(std::is_trivially_copyable<T>::value, "Reduce needs a trivially copyable type");
  using U = typename std::conditional<sizeof(T) == 4, unsigned int, unsigned long long>::type;
  U *addr = reinterpret_cast<U *>(&dst);
  U old = *addr, assumed;
  do {
    assumed = old;
    T cur;
    memcpy(&cur, &assumed, sizeof(T));
    const T nv = op(cur, v);
    U bits;
    memcpy(&bits, &nv, sizeof(T));
    old = atomicCAS(addr, assumed, bits);
  } while (old != assumed);
  T res;
  memcpy(&res, &old, sizeof(T));
  return res;
}

namespace detail {

template <class Body, class Attr, class F, class... Args>
__global__ void map2_leaf_pairs(tapas_b200_device_view v, const Body *__restrict__ bodies,
                                Attr *__restrict__ attrs, F f, Args... args) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t smask = (1ull << v.list_shift) - 1;
  for (int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < v.n_cells;
       t += warps) {
    const int e0 = v.p2p_off[t], e1 = v.p2p_off[t + 1];
    if (e0 == e1) continue;
    const int tb0 = v.bbeg[t], nt = v.nb[t];
    for (int i0 = 0; i0 < nt; i0 += 32) {
      const int i = tb0 + i0 + lane;
      const bool mine = i0 + lane < nt;
      Body bi;
      Attr ai;
      if (mine) {
        bi = bodies[i];
        ai = attrs[i];
      }
      for (int e = e0; e < e1; e++) {
        const int s = (int)(v.p2p_list[e] & smask);
        const int sb0 = v.bbeg[s], ns = v.nb[s];
        if (mine)
          for (int j = sb0; j < sb0 + ns; j++) {
            // lvalue copies: the reference's functors take non-const references
            // (a write to the source's attribute is not kept)
            Body bj = bodies[j];
            Attr aj = attrs[j];
            f(bi, ai, bj, aj, args...);
          }
      }
      if (mine) attrs[i] = ai;
    }
  }
}

template <class F>
__global__ void map_cells_range(tapas_b200_device_view v, int64_t c0, int64_t c1, F f) {
  for (int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < c1;
       c += (int64_t)gridDim.x * blockDim.x)
    f(cell_view(v, (int)c), (int)c);
}

template <class Body, class T, class LeafF, class Op, class PostF>
__global__ void reduce_cells_range(tapas_b200_device_view v, int64_t c0, int64_t c1,
                                   const Body *__restrict__ bodies, T *__restrict__ vals,
                                   LeafF leaf, Op op, PostF post) {
  for (int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < c1;
       c += (int64_t)gridDim.x * blockDim.x) {
    const CellView cv = cell_view(v, (int)c);
    T r;
    if (cv.leaf) {
      r = leaf(cv, bodies + cv.bbeg, cv.nb);
    } else {
      r = vals[cv.child0];
      for (int k = 1; k < 8; k++) r = op(r, vals[cv.child0 + k]);
    }
    vals[c] = post(cv, r);
  }
}

inline int grid_for(int64_t n, int block) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return (int)g;
}

inline int launch_status() {
  return cudaGetLastError() == cudaSuccess ? TAPAS_B200_OK : TAPAS_B200_ERR_CUDA;
}

}  // namespace detail

// f over every body pair of the context's P2P leaf pairs (after build_lists
// or traverse).  bodies / attrs: device arrays of n_bodies in Morton order.
template <class Body, class Attr, class F, class... Args>
int Map2LeafPairs(tapas_b200_ctx *ctx, const Body *bodies, Attr *attrs, F f, Args... args) {
  tapas_b200_device_view v;
  int rc = tapas_b200_get_device_view(ctx, &v);
  if (rc != TAPAS_B200_OK) return rc;
  if (!v.p2p_off) return TAPAS_B200_ERR_STATE;
  void *s = nullptr;
  tapas_b200_get_stream(ctx, &s);
  constexpr int kBlock = 128;  // 4 warps, one target leaf each
  detail::map2_leaf_pairs<Body, Attr, F, Args...>
      <<<detail::grid_for(v.n_cells * 32, kBlock), kBlock, 0, static_cast<cudaStream_t>(s)>>>(
          v, bodies, attrs, f, args...);
  return detail::launch_status();
}

// f(cell, index) for every cell, a level at a time: children before parents
// when up, parents before children otherwise.
template <class F>
int MapCells(tapas_b200_ctx *ctx, F f, bool up) {
  tapas_b200_device_view v;
  int rc = tapas_b200_get_device_view(ctx, &v);
  if (rc != TAPAS_B200_OK) return rc;
  void *s = nullptr;
  tapas_b200_get_stream(ctx, &s);
  for (int64_t k = 0; k < v.n_levels; k++) {
    const int64_t l = up ? v.n_levels - 1 - k : k;
    const int64_t c0 = v.level_off[l], c1 = v.level_off[l + 1];
    if (c1 <= c0) continue;
    detail::map_cells_range<<<detail::grid_for(c1 - c0, 256), 256, 0,
                              static_cast<cudaStream_t>(s)>>>(v, c0, c1, f);
    if ((rc = detail::launch_status()) != TAPAS_B200_OK) return rc;
  }
  return TAPAS_B200_OK;
}

// The upward fold described above; vals: device array of n_cells values.
template <class Body, class T, class LeafF, class Op, class PostF>
int MapReduce(tapas_b200_ctx *ctx, const Body *bodies, T *vals, LeafF leaf, Op op, PostF post) {
  tapas_b200_device_view v;
  int rc = tapas_b200_get_device_view(ctx, &v);
  if (rc != TAPAS_B200_OK) return rc;
  void *s = nullptr;
  tapas_b200_get_stream(ctx, &s);
  for (int64_t l = v.n_levels - 1; l >= 0; l--) {
    const int64_t c0 = v.level_off[l], c1 = v.level_off[l + 1];
    if (c1 <= c0) continue;
    detail::reduce_cells_range<<<detail::grid_for(c1 - c0, 256), 256, 0,
                                 static_cast<cudaStream_t>(s)>>>(v, c0, c1, bodies, vals, leaf,
                                                                 op, post);
    if ((rc = detail::launch_status()) != TAPAS_B200_OK) return rc;
  }
  return TAPAS_B200_OK;
}

}  // namespace b200
}  // namespace tapas
