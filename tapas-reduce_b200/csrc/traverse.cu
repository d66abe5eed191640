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
//   - 8 new pairs   otherwise, splitting by tapas_splitCell (:252-285; with
//                   mutual = 0: split the non-leaf side, and if both are
//                   non-leaves the one with the larger R, ties -> target).
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

struct CellView {
  const int32_t *leaf, *nb, *child;
  const double *cen;
  const double *R;  // per cell: (max width / 2 * 1.00001) / theta
};

// R of every cell for this theta, with the reference's operations in its
// order (max over the widths, halve, * 1.00001, / theta), computed once per
// traversal instead of twice per visited pair.
__global__ void cell_radii(int64_t ncells, const double *__restrict__ mn,
                           const double *__restrict__ mx, double theta, double *__restrict__ R) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncells;
       i += (int64_t)gridDim.x * blockDim.x) {
    double w = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double wd = __dsub_rn(mx[3 * i + d], mn[3 * i + d]);
      w = (w < wd) ? wd : w;  // std::max(R, w)
    }
    R[i] = __ddiv_rn(__dmul_rn(w / 2, 1.00001), theta);
  }
}

// Warp-aggregated reservation of `cnt` slots per lane in a global counter.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long *ctr, unsigned cnt,
                                                           unsigned &my_off) {
  const unsigned lane = threadIdx.x & 31;
  // Inclusive prefix of cnt across the warp.
  unsigned incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += t;
  }
  unsigned total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && total) base = atomicAdd(ctr, (unsigned long long)total);
  base = __shfl_sync(0xffffffffu, base, 31);
  my_off = incl - cnt;
  return base;
}

// counters: [0] next frontier size, [1] m2l size, [2] p2p size,
//           [3] p2p body-pair interactions, [4] overflow flag
__global__ void __launch_bounds__(kBlock) dtt_step(CellView c, double theta,
                                                   const int2 *__restrict__ front, int64_t nfront,
                                                   int2 *__restrict__ next, int64_t next_cap,
                                                   uint64_t *__restrict__ m2l, int64_t m2l_cap,
                                                   uint64_t *__restrict__ p2p, int64_t p2p_cap,
                                                   unsigned long long *__restrict__ counters,
                                                   int prune_empty) {
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nfront;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = base + threadIdx.x;
    int kind = 0;  // 0 none, 1 m2l, 2 p2p, 3 split target, 4 split source
    int t = 0, s = 0;
    unsigned long long inter = 0;
    bool live = i < nfront;
    if (live) {
      int2 pr = front[i];
      t = pr.x;
      s = pr.y;
      // An empty cell (and so all of its descendants) contributes nothing as a
      // source and receives nothing used later as a target.
      if (prune_empty && (c.nb[t] == 0 || c.nb[s] == 0)) live = false;
    }
    if (live) {
      const double dx = __dsub_rn(c.cen[3 * t + 0], c.cen[3 * s + 0]);
      const double dy = __dsub_rn(c.cen[3 * t + 1], c.cen[3 * s + 1]);
      const double dz = __dsub_rn(c.cen[3 * t + 2], c.cen[3 * s + 2]);
      double R2 = __dadd_rn(0.0, __dmul_rn(dx, dx));
      R2 = __dadd_rn(R2, __dmul_rn(dy, dy));
      R2 = __dadd_rn(R2, __dmul_rn(dz, dz));
      const double Ri = c.R[t], Rj = c.R[s];
      const double RR = __dadd_rn(Ri, Rj);
      const bool lt = c.leaf[t] != 0, ls = c.leaf[s] != 0;
      if (R2 > __dmul_rn(RR, RR)) {
        kind = 1;
      } else if (lt && ls) {
        const int nt = c.nb[t], ns = c.nb[s];
        if (nt > 0 && ns > 0) {
          kind = 2;
          inter = (unsigned long long)nt * (unsigned long long)ns;
        }
      } else if (ls) {
        kind = 3;
      } else if (lt) {
        kind = 4;
      } else {
        kind = (Ri >= Rj) ? 3 : 4;
      }
    }
    unsigned off;
    // M2L
    unsigned long long b1 = warp_reserve(counters + 1, kind == 1, off);
    if (kind == 1) {
      unsigned long long dst = b1 + off;
      if ((int64_t)dst < m2l_cap) m2l[dst] = ((uint64_t)(uint32_t)t << 32) | (uint32_t)s;
      else counters[4] = 1;
    }
    unsigned long long b2 = warp_reserve(counters + 2, kind == 2, off);
    if (kind == 2) {
      unsigned long long dst = b2 + off;
      if ((int64_t)dst < p2p_cap) p2p[dst] = ((uint64_t)(uint32_t)t << 32) | (uint32_t)s;
      else counters[4] = 1;
    }
    unsigned long long b3 = warp_reserve(counters + 0, (kind >= 3) ? 8u : 0u, off);
    if (kind >= 3) {
      unsigned long long dst = b3 + off;
      if ((int64_t)(dst + 8) <= next_cap) {
        if (kind == 3) {
          const int c0 = c.child[t];
#pragma unroll
          for (int k = 0; k < 8; k++) next[dst + k] = make_int2(c0 + k, s);
        } else {
          const int c0 = c.child[s];
#pragma unroll
          for (int k = 0; k < 8; k++) next[dst + k] = make_int2(t, c0 + k);
        }
      } else {
        counters[4] = 1;
      }
    }
    // p2p interaction count
    unsigned long long w = inter;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(counters + 3, w);
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

// off[c] = lower_bound(sorted packed keys, c << b), c in [0, ncells].
__global__ void csr_offsets(const uint64_t *__restrict__ v, int64_t n, int b, int64_t ncells,
                            int32_t *__restrict__ off) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c <= ncells;
       c += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = (uint64_t)c << b;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = lo + ((hi - lo) >> 1);
      if (v[mid] < key) lo = mid + 1; else hi = mid;
    }
    off[c] = (int32_t)lo;
  }
}

int bits_for(int64_t x) {
  int b = 1;
  while (((int64_t)1 << b) <= x) b++;
  return b;
}

}  // namespace

int build_lists(tapas_b200_ctx *ctx, double theta) {
  if (!ctx->have_tree) {
    set_error(ctx, "build_lists: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  if (!(theta > 0)) {
    set_error(ctx, "build_lists: theta must be > 0");
    return TAPAS_B200_ERR_ARG;
  }
  cudaStream_t s = ctx->stream;
  ctx->theta = theta;
  ctx->have_lists = false;
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->cell_r.ensure(C + 1, s));
  cell_radii<<<grid_for(C, kBlock), kBlock, 0, s>>>(C, ctx->cmin.p, ctx->cmax.p, theta,
                                                    ctx->cell_r.p);
  TB_LAUNCH_CHECK(ctx);
  CellView cv{ctx->cleaf.p, ctx->cnb.p, ctx->cchild.p, ctx->ccen.p, ctx->cell_r.p};
  TB_CUDA(ctx, ctx->counters.ensure(8, s));
  TB_CUDA(ctx, ctx->pinned.ensure(256));
  unsigned long long *hc = reinterpret_cast<unsigned long long *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, 8 * sizeof(unsigned long long), s));
  {
    PhaseTimer tm(ctx, &ctx->timings.traverse);
    TB_CUDA(ctx, ctx->front_a.ensure(1024, s));
    const int2 root = make_int2(0, 0);
    TB_CUDA(ctx, cudaMemcpyAsync(ctx->front_a.p, &root, sizeof(int2), cudaMemcpyHostToDevice, s));
    int64_t nfront = 1, n_m2l = 0, n_p2p = 0;
    int iters = 0;
    while (nfront > 0) {
      TB_CUDA(ctx, ctx->front_b.ensure(8 * nfront, s));
      TB_CUDA(ctx, ctx->m2l.ensure(n_m2l + nfront, s, true, n_m2l));
      TB_CUDA(ctx, ctx->p2p.ensure(n_p2p + nfront, s, true, n_p2p));
      TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, sizeof(unsigned long long), s));
      dtt_step<<<grid_for(nfront, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
          cv, theta, ctx->front_a.p, nfront, ctx->front_b.p, (int64_t)ctx->front_b.cap, ctx->m2l.p,
          (int64_t)ctx->m2l.cap, ctx->p2p.p, (int64_t)ctx->p2p.cap, ctx->counters.p,
          ctx->reference_lists ? 0 : 1);
      TB_LAUNCH_CHECK(ctx);
      TB_CUDA(ctx, cudaMemcpyAsync(hc, ctx->counters.p, 5 * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, s));
      TB_CUDA(ctx, cudaStreamSynchronize(s));
      if (hc[4]) {
        set_error(ctx, "traversal: work list capacity exceeded");
        return TAPAS_B200_ERR_CAPACITY;
      }
      nfront = (int64_t)hc[0];
      n_m2l = (int64_t)hc[1];
      n_p2p = (int64_t)hc[2];
      std::swap(ctx->front_a, ctx->front_b);
      if (++iters > 4 * (kMaxDepth + 2)) {
        set_error(ctx, "traversal did not terminate within its iteration bound");
        return TAPAS_B200_ERR_CAPACITY;
      }
    }
    ctx->n_m2l = n_m2l;
    ctx->n_p2p = n_p2p;
    ctx->n_p2p_int = hc[3];
    ctx->trav_iters = iters;
  }
  {
    PhaseTimer tm(ctx, &ctx->timings.list_sort);
    const int b = bits_for(C);
    ctx->list_shift = b;
    TB_CUDA(ctx, ctx->m2l_off.ensure(C + 1, s));
    TB_CUDA(ctx, ctx->p2p_off.ensure(C + 1, s));
    for (int which = 0; which < 2; which++) {
      tb::DBuf<uint64_t> &L = which == 0 ? ctx->m2l : ctx->p2p;
      tb::DBuf<int32_t> &off = which == 0 ? ctx->m2l_off : ctx->p2p_off;
      const int64_t n = which == 0 ? ctx->n_m2l : ctx->n_p2p;
      if (n > 0) {
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
      csr_offsets<<<grid_for(C + 1, kBlock), kBlock, 0, s>>>(L.p, n, b, C, off.p);
      TB_LAUNCH_CHECK(ctx);
    }
  }
  ctx->have_lists = true;
  return TAPAS_B200_OK;
}

}  // namespace tb
