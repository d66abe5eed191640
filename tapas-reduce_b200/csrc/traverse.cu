// Dual-tree traversal on the GPU: builds the M2L and P2P work lists.
//
// The reference runs FMM_DTT (sample/exafmm-dev-13274dd4ac68/examples/
// tapas_exafmm.cxx:209-286) recursively from (root, root).  Each visit is a
// pure function of the two cells, so the recursion is replaced by a
// breadth-first frontier of (target, source) pairs: every step classifies all
// pending pairs at once and emits
//   - an M2L pair   if R2 > (Ri + Rj)^2  (R2 = squared centre distance,
//                   geometry.h:81-83; Ri = (max width / 2 * 1.00001) / theta),
//   - a P2P pair    if both are leaves (skipped when either is empty: the
//                   reference's Map over an empty body product is a no-op,
//                   cpp/include/tapas/hot.h:1362-1369),
//   - 8 new pairs   otherwise, splitting by tapas_splitCell (:252-285): split
//                   the non-leaf side, and if both are non-leaves the one with
//                   the larger R, ties -> target.
// With mutual = 1 (the example's -m option) a pair (c, c) of a non-leaf cell
// with itself splits both sides and visits only the 36 child pairs (c_i, c_j),
// i <= j (tapas_splitCell's `mutual && Ci == Cj` branch; the product map's
// AllowMutualInteraction rule, cpp/include/tapas/hot/mapper.h:28-121 and
// iterator.h:98-100,165-167,279-281).  Every unordered cell pair is then
// visited once and acts both ways (M2L both ways, LaplaceSphericalCPU_tapas.h:
// 208-273; P2P both ways, LaplaceP2PCPU_tapas.h:48-74).  Here the unordered
// pairs are expanded into the two directed pairs before the lists are
// ordered, so the evaluation kernels see ordinary (target, source) lists.
// The acceptance test is evaluated with separately rounded FP64 operations so
// every decision matches the reference bit for bit; the lists are therefore
// equal as sets.  They are then sorted by (target, source) so the evaluation
// order, and so every result, is deterministic.
#include <algorithm>

#include "primitives.cuh"
#include "traverse.cuh"

namespace tb {
namespace {

constexpr int kBlock = 256;

// What one visit reads of a cell, packed so a visit touches two sectors per
// cell: geometry {cx, cy, cz, R} with R = (max width / 2 * 1.00001) / theta,
// and {nb, first child or -1 for a leaf}.
struct TravCells {
  const double4 *geo;
  const int2 *meta;
};

// The traversal's cell records for this theta, with the reference's
// operations in its order for R (max over the widths, halve, * 1.00001,
// / theta), computed once per traversal instead of twice per visited pair.
__global__ void trav_cells(int64_t ncells, const double *__restrict__ mn,
                           const double *__restrict__ mx, const double *__restrict__ cen,
                           const int32_t *__restrict__ nb, const int32_t *__restrict__ leaf,
                           const int32_t *__restrict__ child, double theta,
                           double4 *__restrict__ geo, int2 *__restrict__ meta) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncells;
       i += (int64_t)gridDim.x * blockDim.x) {
    double w = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double wd = __dsub_rn(mx[3 * i + d], mn[3 * i + d]);
      w = (w < wd) ? wd : w;  // std::max(R, w)
    }
    const double R = __ddiv_rn(__dmul_rn(w / 2, 1.00001), theta);
    geo[i] = make_double4(cen[3 * i + 0], cen[3 * i + 1], cen[3 * i + 2], R);
    meta[i] = make_int2(nb[i], leaf[i] ? -1 : child[i]);
  }
}

// Per-thread output counts packed in one word for the block scan: M2L pairs
// in bits 0-8, P2P pairs in bits 9-17, new frontier pairs in bits 18-31
// (at most 256, 256 and 36 * 256 per block; 36 for a mutual self split).
constexpr int kWarpsPerBlock = kBlock / 32;
constexpr int kSelfSplit = 36;  // child pairs (i, j), i <= j, of a cell with itself
static_assert(kBlock <= 256, "packed per-block counts hold at most 256 threads");
static_assert(kSelfSplit * kBlock < (1 << 14), "frontier count field is 14 bits");

// counters: [0] next frontier size, [1] m2l size, [2] p2p size,
//           [3] p2p body-pair interactions, [4] overflow bits (1: a list,
//           2: the next frontier; [0] still counts the frontier's full size)
// Slots in the three outputs are reserved once per block (one atomic per
// counter per block), the block's threads taking consecutive slots.
__global__ void __launch_bounds__(kBlock) dtt_step(TravCells c, const int2 *__restrict__ front,
                                                   int64_t nfront, int2 *__restrict__ next,
                                                   int64_t next_cap, uint64_t *__restrict__ m2l,
                                                   int64_t m2l_cap, uint64_t *__restrict__ p2p,
                                                   int64_t p2p_cap,
                                                   unsigned long long *__restrict__ counters,
                                                   int prune_empty, int mutual) {
  __shared__ uint32_t wsum[kWarpsPerBlock];
  __shared__ unsigned long long wint[kWarpsPerBlock];
  __shared__ unsigned long long bbase[3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nfront;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = base + threadIdx.x;
    int kind = 0;  // 0 none, 1 m2l, 2 p2p, 3 split target, 4 split source, 5 split both
    int t = 0, s = 0, split_child = 0;
    unsigned long long inter = 0;
    if (i < nfront) {
      const int2 pr = front[i];
      t = pr.x;
      s = pr.y;
      const int2 mt = c.meta[t], ms = c.meta[s];
      // An empty cell (and so all of its descendants) contributes nothing as a
      // source and receives nothing used later as a target.
      if (!prune_empty || (mt.x != 0 && ms.x != 0)) {
        const double4 gt = c.geo[t], gs = c.geo[s];
        const double dx = __dsub_rn(gt.x, gs.x);
        const double dy = __dsub_rn(gt.y, gs.y);
        const double dz = __dsub_rn(gt.z, gs.z);
        double R2 = __dadd_rn(0.0, __dmul_rn(dx, dx));
        R2 = __dadd_rn(R2, __dmul_rn(dy, dy));
        R2 = __dadd_rn(R2, __dmul_rn(dz, dz));
        const double Ri = gt.w, Rj = gs.w;
        const double RR = __dadd_rn(Ri, Rj);
        const bool lt = mt.y < 0, ls = ms.y < 0;
        if (R2 > __dmul_rn(RR, RR)) {
          kind = 1;
        } else if (lt && ls) {
          if (mt.x > 0 && ms.x > 0) {
            kind = 2;
            // body pairs evaluated: both directions of a mutual pair of two leaves
            inter = (unsigned long long)mt.x * (unsigned long long)ms.x;
            if (mutual && t != s) inter *= 2;
          }
        } else if (ls) {
          kind = 3;
        } else if (lt) {
          kind = 4;
        } else if (mutual && t == s) {
          kind = 5;
        } else {
          kind = (Ri >= Rj) ? 3 : 4;
        }
        split_child = kind == 3 ? mt.y : ms.y;
      }
    }
    const uint32_t mine = (kind == 1 ? 1u : 0u) | (kind == 2 ? 1u << 9 : 0u) |
                          (kind == 3 || kind == 4 ? 8u << 18 : 0u) |
                          (kind == 5 ? (uint32_t)kSelfSplit << 18 : 0u);
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    unsigned long long w = inter;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (lane == 31) wsum[warp] = incl;
    if (lane == 0) wint[warp] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      unsigned long long tot = 0;
#pragma unroll
      for (int k = 0; k < kWarpsPerBlock; k++) {
        const uint32_t v = wsum[k];
        wsum[k] = run;
        run += v;
        tot += wint[k];
      }
      const uint32_t n1 = run & 511u, n2 = (run >> 9) & 511u, n3 = run >> 18;
      bbase[0] = n1 ? atomicAdd(counters + 1, (unsigned long long)n1) : 0;
      bbase[1] = n2 ? atomicAdd(counters + 2, (unsigned long long)n2) : 0;
      bbase[2] = n3 ? atomicAdd(counters + 0, (unsigned long long)n3) : 0;
      if (tot) atomicAdd(counters + 3, tot);
    }
    __syncthreads();
    const uint32_t off = wsum[warp] + incl - mine;
    if (kind == 1) {
      const unsigned long long dst = bbase[0] + (off & 511u);
      if ((int64_t)dst < m2l_cap) m2l[dst] = ((uint64_t)(uint32_t)t << 32) | (uint32_t)s;
      else atomicOr(counters + 4, 1ull);
    } else if (kind == 2) {
      const unsigned long long dst = bbase[1] + ((off >> 9) & 511u);
      if ((int64_t)dst < p2p_cap) p2p[dst] = ((uint64_t)(uint32_t)t << 32) | (uint32_t)s;
      else atomicOr(counters + 4, 1ull);
    } else if (kind == 5) {
      const unsigned long long dst = bbase[2] + (off >> 18);
      if ((int64_t)(dst + kSelfSplit) <= next_cap) {
        int2 *o = next + dst;
        int k = 0;
        for (int a = 0; a < 8; a++)
          for (int b2 = a; b2 < 8; b2++) o[k++] = make_int2(split_child + a, split_child + b2);
      } else {
        atomicOr(counters + 4, 2ull);
      }
    } else if (kind >= 3) {
      const unsigned long long dst = bbase[2] + (off >> 18);
      if ((int64_t)(dst + 8) <= next_cap) {
        int4 *o4 = reinterpret_cast<int4 *>(next + dst);  // dst is even (8 and 36 are)
        if (kind == 3) {
#pragma unroll
          for (int k = 0; k < 8; k += 2)
            o4[k / 2] = make_int4(split_child + k, s, split_child + k + 1, s);
        } else {
#pragma unroll
          for (int k = 0; k < 8; k += 2)
            o4[k / 2] = make_int4(t, split_child + k, t, split_child + k + 1);
        }
      } else {
        atomicOr(counters + 4, 2ull);
      }
    }
    __syncthreads();  // wsum / bbase are rewritten by the next round
  }
}

// The directed pairs of a mutual list: (t, s) and (s, t) for t != s, a self
// pair (t, t) once.  Slots are reserved once per warp; the order is set by the
// (target, source) sort that follows.
__global__ void expand_mutual(const uint64_t *__restrict__ in, int64_t n,
                              uint64_t *__restrict__ out, int64_t cap,
                              unsigned long long *__restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += stride) {
    const int64_t i = base + lane;
    uint64_t x = 0;
    int k = 0;
    if (i < n) {
      x = in[i];
      k = ((x >> 32) != (x & 0xFFFFFFFFull)) ? 2 : 1;
    }
    int incl = k;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int tot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long b0 = 0;
    if (lane == 0) b0 = atomicAdd(cnt, (unsigned long long)tot);
    b0 = __shfl_sync(0xffffffffu, b0, 0);
    const int64_t dst = (int64_t)b0 + incl - k;
    if (k >= 1 && dst < cap) out[dst] = x;
    if (k == 2 && dst + 1 < cap) out[dst + 1] = (x << 32) | (x >> 32);
  }
}

// Packs (t << 32 | s) into (t << b | s) for a narrower sort key.
__global__ void pack_pairs(uint64_t *__restrict__ v, int64_t n, int b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t x = v[i];
    v[i] = ((x >> 32) << b) | (x & 0xFFFFFFFFull);
  }
}

// ---------------------------------------------------------------------------
// List ordering.  The traversal emits pairs in an order set by its atomics;
// the lists are put in (target, source) order by a counting sort on the
// target (the counts' scan is the lists' CSR offsets) followed by a bitonic
// sort of each target's sources in shared memory: one warp per segment of up
// to kWarpSegMax pairs, one block per longer segment up to kSegSortMax, and
// the radix sort of the whole list when a segment is longer still.  Every
// (target, source) pair is visited at most once (the split rule is a function
// of the pair, so two visiting paths from (root, root) cannot diverge), so a
// segment's sources are distinct.
// ---------------------------------------------------------------------------
constexpr int kWarpSegMax = 512;
constexpr int kSegSortMax = 8192;
constexpr int kSegWarps = 8;
constexpr int kLongThreads = 1024;

__global__ void target_counts(const uint64_t *__restrict__ v, int64_t n, int32_t *__restrict__ cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + (v[i] >> 32), 1);
}

// *mx = max over c of off[c + 1] - off[c].
__global__ void segment_max(const int32_t *__restrict__ off, int64_t ncells,
                            unsigned long long *__restrict__ mx) {
  unsigned m = 0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncells;
       c += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (unsigned)(off[c + 1] - off[c]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(mx, (unsigned long long)m);
}

// Places each pair's source in its target's segment (order inside it
// arbitrary).  cur starts as the segment offsets.
__global__ void scatter_by_target(const uint64_t *__restrict__ v, int64_t n,
                                  int32_t *__restrict__ cur, uint32_t *__restrict__ src) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t x = v[i];
    const int32_t pos = atomicAdd(cur + (x >> 32), 1);
    src[pos] = (uint32_t)x;
  }
}

// Ascending bitonic sort of a[0, np), np a power of two, by threads
// tid = 0 .. nthr-1 of a warp (kBlockLevel false) or of the block.
template <bool kBlockLevel>
__device__ __forceinline__ void bitonic_sort(uint32_t *a, int np, int tid, int nthr) {
  for (int k = 2; k <= np; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int c = tid; c < (np >> 1); c += nthr) {
        const int lo = ((c & ~(j - 1)) << 1) | (c & (j - 1));
        const int hi = lo + j;
        const uint32_t x = a[lo], y = a[hi];
        if ((x > y) == ((lo & k) == 0)) {
          a[lo] = y;
          a[hi] = x;
        }
      }
      if (kBlockLevel) __syncthreads(); else __syncwarp();
    }
  }
}

__device__ __forceinline__ int pow2_at_least(int n) {
  int p = 2;
  while (p < n) p <<= 1;
  return p;
}

// One warp per target segment of at most kWarpSegMax sources; longer segments
// are listed for sort_long_segments.  out[i] = t << b | sorted source.
__global__ void __launch_bounds__(kSegWarps * 32) sort_segments(
    const uint32_t *__restrict__ src, const int32_t *__restrict__ off, int64_t ncells, int b,
    uint64_t *__restrict__ out, int32_t *__restrict__ long_list,
    unsigned long long *__restrict__ long_cnt) {
  __shared__ uint32_t buf[kSegWarps][kWarpSegMax];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *a = buf[warp];
  const int64_t warps = (int64_t)gridDim.x * kSegWarps;
  for (int64_t c = (int64_t)blockIdx.x * kSegWarps + warp; c < ncells; c += warps) {
    const int32_t a0 = off[c], len = off[c + 1] - a0;
    const uint64_t th = (uint64_t)c << b;
    if (len == 0) continue;
    if (len > kWarpSegMax) {
      if (lane == 0) long_list[atomicAdd(long_cnt, 1ull)] = (int32_t)c;
      continue;
    }
    if (len == 1) {
      if (lane == 0) out[a0] = th | src[a0];
      continue;
    }
    const int np = pow2_at_least(len);
    for (int i = lane; i < np; i += 32) a[i] = i < len ? src[a0 + i] : 0xFFFFFFFFu;
    __syncwarp();
    bitonic_sort<false>(a, np, lane, 32);
    for (int i = lane; i < len; i += 32) out[a0 + i] = th | a[i];
    __syncwarp();
  }
}

// One block per listed segment of kWarpSegMax < length <= kSegSortMax.
__global__ void __launch_bounds__(kLongThreads) sort_long_segments(
    const uint32_t *__restrict__ src, const int32_t *__restrict__ off, int b,
    uint64_t *__restrict__ out, const int32_t *__restrict__ long_list,
    const unsigned long long *__restrict__ long_cnt) {
  __shared__ uint32_t a[kSegSortMax];
  const int64_t nl = (int64_t)*long_cnt;
  for (int64_t k = blockIdx.x; k < nl; k += gridDim.x) {
    const int32_t c = long_list[k];
    const int32_t a0 = off[c], len = off[c + 1] - a0;
    const uint64_t th = (uint64_t)c << b;
    const int np = pow2_at_least(len);
    for (int i = threadIdx.x; i < np; i += kLongThreads) a[i] = i < len ? src[a0 + i] : 0xFFFFFFFFu;
    __syncthreads();
    bitonic_sort<true>(a, np, threadIdx.x, kLongThreads);
    for (int i = threadIdx.x; i < len; i += kLongThreads) out[a0 + i] = th | a[i];
    __syncthreads();
  }
}

// out[i] = c << b | src[i] over each target segment, sources in the order
// the scatter left them (one warp per target).
__global__ void __launch_bounds__(kSegWarps * 32) pack_segments(
    const uint32_t *__restrict__ src, const int32_t *__restrict__ off, int64_t ncells, int b,
    uint64_t *__restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * kSegWarps;
  for (int64_t c = (int64_t)blockIdx.x * kSegWarps + warp; c < ncells; c += warps) {
    const int32_t a0 = off[c], a1 = off[c + 1];
    const uint64_t th = (uint64_t)c << b;
    for (int32_t i = a0 + lane; i < a1; i += 32) out[i] = th | src[i];
  }
}

__global__ void list_sources(const uint64_t *__restrict__ v, int64_t n, uint64_t mask,
                             uint32_t *__restrict__ src) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    src[i] = (uint32_t)(v[i] & mask);
}

int bits_for(int64_t x) {
  int b = 1;
  while (((int64_t)1 << b) <= x) b++;
  return b;
}

// Sorts each target segment of list w (0: M2L, 1: P2P) by source, given the
// sources in segment order in ctx->list_src and the longest segment.
int sort_segment_sources(tapas_b200_ctx *ctx, int w, unsigned long long longest) {
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  const int b = ctx->list_shift;
  tb::DBuf<uint64_t> &L = w ? ctx->p2p : ctx->m2l;
  const int32_t *off = w ? ctx->p2p_off.p : ctx->m2l_off.p;
  TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p + 7, 0, sizeof(unsigned long long), s));
  // the per-target cursors are spent: their buffer holds the long-segment list
  sort_segments<<<grid_for(C, kSegWarps, ctx->num_sms * 8), kSegWarps * 32, 0, s>>>(
      ctx->list_src.p, off, C, b, L.p, ctx->list_cnt.p, ctx->counters.p + 7);
  TB_LAUNCH_CHECK(ctx);
  if (longest > (unsigned long long)kWarpSegMax) {
    sort_long_segments<<<ctx->num_sms, kLongThreads, 0, s>>>(ctx->list_src.p, off, b, L.p,
                                                              ctx->list_cnt.p,
                                                              ctx->counters.p + 7);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

}  // namespace

int sort_list_sources(tapas_b200_ctx *ctx, int w) {
  if (!ctx->have_lists || ctx->sources_sorted[w]) return TAPAS_B200_OK;
  const int64_t n = w ? ctx->n_p2p : ctx->n_m2l;
  if (n > 0) {
    cudaStream_t s = ctx->stream;
    TB_CUDA(ctx, ctx->list_src.ensure(n + 1, s));
    TB_CUDA(ctx, ctx->list_cnt.ensure(ctx->ncells + 1, s));
    list_sources<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
        w ? ctx->p2p.p : ctx->m2l.p, n, (1ull << ctx->list_shift) - 1, ctx->list_src.p);
    TB_LAUNCH_CHECK(ctx);
    TB_TRY(sort_segment_sources(ctx, w, ctx->longest_segment[w]));
  }
  ctx->sources_sorted[w] = true;
  return TAPAS_B200_OK;
}

int sort_list_sources(tapas_b200_ctx *ctx) {
  TB_TRY(sort_list_sources(ctx, 0));
  return sort_list_sources(ctx, 1);
}

int build_lists(tapas_b200_ctx *ctx, double theta, int mutual, bool sort_sources) {
  if (!ctx->have_tree) {
    set_error(ctx, "build_lists: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  if (!(theta > 0)) {
    set_error(ctx, "build_lists: theta must be > 0");
    return TAPAS_B200_ERR_ARG;
  }
  if (mutual != 0 && mutual != 1) {
    set_error(ctx, "build_lists: mutual must be 0 or 1");
    return TAPAS_B200_ERR_ARG;
  }
  ctx->mutual = mutual;
  cudaStream_t s = ctx->stream;
  ctx->theta = theta;
  ctx->have_lists = false;
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->trav_geo.ensure(C + 1, s));
  TB_CUDA(ctx, ctx->trav_meta.ensure(C + 1, s));
  trav_cells<<<grid_for(C, kBlock), kBlock, 0, s>>>(C, ctx->cmin.p, ctx->cmax.p, ctx->ccen.p,
                                                    ctx->cnb.p, ctx->cleaf.p, ctx->cchild.p, theta,
                                                    ctx->trav_geo.p, ctx->trav_meta.p);
  TB_LAUNCH_CHECK(ctx);
  const TravCells cv{ctx->trav_geo.p, ctx->trav_meta.p};
  TB_CUDA(ctx, ctx->counters.ensure(8, s));
  TB_CUDA(ctx, ctx->pinned.ensure(256));
  unsigned long long *hc = reinterpret_cast<unsigned long long *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, 8 * sizeof(unsigned long long), s));
  {
    PhaseTimer tm(ctx, &ctx->timings.traverse);
    TB_CUDA(ctx, ctx->front_a.ensure(1024, s));
    const int2 root = make_int2(0, 0);
    TB_CUDA(ctx, cudaMemcpyAsync(ctx->front_a.p, &root, sizeof(int2), cudaMemcpyHostToDevice, s));
    int64_t nfront = 1, n_m2l = 0, n_p2p = 0, visited = 0;
    unsigned long long n_int = 0;
    int iters = 0;
    unsigned long long *hset = hc + 16;  // counter values restored before a step
    while (nfront > 0) {
      visited += nfront;
      // Each visited pair adds at most one M2L or P2P pair; the next frontier
      // gets 2 * nfront slots first, and a step that needs more is run again
      // with the size its reservations counted.
      TB_CUDA(ctx, ctx->m2l.ensure(n_m2l + nfront, s, true, n_m2l));
      TB_CUDA(ctx, ctx->p2p.ensure(n_p2p + nfront, s, true, n_p2p));
      TB_CUDA(ctx, ctx->front_b.ensure(std::max<int64_t>(2 * nfront, 1024), s));
      for (int attempt = 0;; attempt++) {
        hset[0] = 0;
        hset[1] = (unsigned long long)n_m2l;
        hset[2] = (unsigned long long)n_p2p;
        hset[3] = n_int;
        hset[4] = 0;
        TB_CUDA(ctx, cudaMemcpyAsync(ctx->counters.p, hset, 5 * sizeof(unsigned long long),
                                     cudaMemcpyHostToDevice, s));
        dtt_step<<<grid_for(nfront, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
            cv, ctx->front_a.p, nfront, ctx->front_b.p, (int64_t)ctx->front_b.cap, ctx->m2l.p,
            (int64_t)ctx->m2l.cap, ctx->p2p.p, (int64_t)ctx->p2p.cap, ctx->counters.p,
            ctx->reference_lists ? 0 : 1, mutual);
        TB_LAUNCH_CHECK(ctx);
        TB_CUDA(ctx, cudaMemcpyAsync(hc, ctx->counters.p, 5 * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, s));
        TB_CUDA(ctx, cudaStreamSynchronize(s));
        if (hc[4] & 1) {
          set_error(ctx, "traversal: work list capacity exceeded");
          return TAPAS_B200_ERR_CAPACITY;
        }
        if (!(hc[4] & 2)) break;
        if (attempt > 0) {
          set_error(ctx, "traversal: frontier capacity exceeded after resizing");
          return TAPAS_B200_ERR_CAPACITY;
        }
        TB_CUDA(ctx, ctx->front_b.ensure((size_t)hc[0], s));
      }
      nfront = (int64_t)hc[0];
      n_m2l = (int64_t)hc[1];
      n_p2p = (int64_t)hc[2];
      n_int = hc[3];
      std::swap(ctx->front_a, ctx->front_b);
      if (++iters > 4 * (kMaxDepth + 2)) {
        set_error(ctx, "traversal did not terminate within its iteration bound");
        return TAPAS_B200_ERR_CAPACITY;
      }
    }
    ctx->n_m2l_visited = n_m2l;
    ctx->n_p2p_visited = n_p2p;
    if (mutual) {
      // unordered pairs -> directed pairs (M2L has no self pairs; P2P has one
      // self pair per non-empty leaf)
      tb::DBuf<uint64_t> *lists[2] = {&ctx->m2l, &ctx->p2p};
      int64_t *counts[2] = {&n_m2l, &n_p2p};
      for (int w = 0; w < 2; w++) {
        const int64_t n = *counts[w];
        if (n == 0) continue;
        TB_CUDA(ctx, ctx->list_alt.ensure(2 * n, s));
        TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p + 5, 0, sizeof(unsigned long long), s));
        expand_mutual<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
            lists[w]->p, n, ctx->list_alt.p, 2 * n, ctx->counters.p + 5);
        TB_LAUNCH_CHECK(ctx);
        TB_CUDA(ctx, cudaMemcpyAsync(hc + 5, ctx->counters.p + 5, sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, s));
        TB_CUDA(ctx, cudaStreamSynchronize(s));
        *counts[w] = (int64_t)hc[5];
        std::swap(lists[w]->p, ctx->list_alt.p);
        std::swap(lists[w]->cap, ctx->list_alt.cap);
      }
    }
    ctx->n_m2l = n_m2l;
    ctx->n_p2p = n_p2p;
    ctx->n_p2p_int = n_int;
    ctx->trav_iters = iters;
    ctx->trav_pairs = visited;
  }
  {
    PhaseTimer tm(ctx, &ctx->timings.list_sort);
    const int b = bits_for(C);
    ctx->list_shift = b;
    TB_CUDA(ctx, ctx->m2l_off.ensure(C + 1, s));
    TB_CUDA(ctx, ctx->p2p_off.ensure(C + 1, s));
    TB_CUDA(ctx, ctx->list_cnt.ensure(C + 1, s));
    const int64_t nlist[2] = {ctx->n_m2l, ctx->n_p2p};
    tb::DBuf<uint64_t> *lists[2] = {&ctx->m2l, &ctx->p2p};
    tb::DBuf<int32_t> *offs[2] = {&ctx->m2l_off, &ctx->p2p_off};
    // 1. per-target counts -> CSR offsets, and the longest segment
    TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p + 5, 0, 2 * sizeof(unsigned long long), s));
    for (int w = 0; w < 2; w++) {
      TB_CUDA(ctx, cudaMemsetAsync(ctx->list_cnt.p, 0, sizeof(int32_t) * (C + 1), s));
      if (nlist[w] > 0) {
        target_counts<<<grid_for(nlist[w], kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
            lists[w]->p, nlist[w], ctx->list_cnt.p);
        TB_LAUNCH_CHECK(ctx);
      }
      TB_TRY(scan_exclusive(ctx, ctx->list_cnt.p, offs[w]->p, C, offs[w]->p + C));
      segment_max<<<grid_for(C, kBlock, ctx->num_sms * 8), kBlock, 0, s>>>(offs[w]->p, C,
                                                                          ctx->counters.p + 5 + w);
      TB_LAUNCH_CHECK(ctx);
    }
    TB_CUDA(ctx, cudaMemcpyAsync(hc + 5, ctx->counters.p + 5, 2 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    for (int w = 0; w < 2; w++) {
      ctx->longest_segment[w] = hc[5 + w];
      ctx->sources_sorted[w] = true;
    }
    // 2. counting sort by target, then each target's sources
    for (int w = 0; w < 2; w++) {
      tb::DBuf<uint64_t> &L = *lists[w];
      const int64_t n = nlist[w];
      if (n == 0) continue;
      if (hc[5 + w] <= (unsigned long long)kSegSortMax) {
        TB_CUDA(ctx, ctx->list_src.ensure(n + 1, s));
        TB_CUDA(ctx, cudaMemcpyAsync(ctx->list_cnt.p, offs[w]->p, sizeof(int32_t) * C,
                                     cudaMemcpyDeviceToDevice, s));
        scatter_by_target<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
            L.p, n, ctx->list_cnt.p, ctx->list_src.p);
        TB_LAUNCH_CHECK(ctx);
        if (!sort_sources) {
          // grouped by target only; sort_list_sources() completes the order
          // when a caller needs it
          pack_segments<<<grid_for(C, kSegWarps, ctx->num_sms * 8), kSegWarps * 32, 0, s>>>(
              ctx->list_src.p, offs[w]->p, C, b, L.p);
          TB_LAUNCH_CHECK(ctx);
          ctx->sources_sorted[w] = false;
        } else {
          TB_TRY(sort_segment_sources(ctx, w, hc[5 + w]));
        }
      } else {
        TB_CUDA(ctx, ctx->list_alt.ensure(n + 1, s));
        pack_pairs<<<grid_for(n, kBlock), kBlock, 0, s>>>(L.p, n, b);
        TB_LAUNCH_CHECK(ctx);
        uint64_t *k = L.p, *ka = ctx->list_alt.p;
        uint32_t *nv = nullptr, *nva = nullptr;
        TB_TRY(radix_sort(ctx, k, ka, nv, nva, n, 0, 2 * b));
        if (k != L.p) {
          std::swap(L.p, ctx->list_alt.p);
          std::swap(L.cap, ctx->list_alt.cap);
        }
      }
    }
  }
  ctx->have_lists = true;
  return TAPAS_B200_OK;
}

}  // namespace tb
