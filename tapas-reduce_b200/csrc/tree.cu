// Octree construction on the GPU: bounding cube, Morton keys, key sort, body
// permutation and the level-by-level cell build.
//
// Follows cpp/include/tapas/hot/buildtree.h (SamplingOctree) on one rank:
//  - bbox_*:        the constructor's box, :72-87, including its scalar
//                   broadcast (the box is a cube; body 0 contributes only z).
//  - keys_kernel:   BodiesToKeys, :505-539, with Morton::CalcFinestKey,
//                   sfc_morton.h:387-402.
//  - radix sort:    SortByKeys, common.h:249-273 (stable here; the reference's
//                   std::sort leaves equal keys in unspecified order).
//  - build_level:   GenerateCell, :388-459: a cell's bodies are the sorted
//                   range [lower_bound(k), lower_bound(GetNext(k))); it is a
//                   leaf iff nb <= ncrit; non-leaves get all 8 children.  Cells
//                   are stored breadth first, level after level.
// Layout in HBM: bodies SoA FP64 (x,y,z,q) in input and sorted order; keys
// u64; cells SoA (key, range, parent, first child, leaf, 3x min/max/center).
#include <algorithm>

#include "primitives.cuh"
#include "tree.cuh"

namespace tb {
namespace {

constexpr int kBlock = 256;

// Exact FP64 operations: the reference is compiled for x86-64 without FMA, so
// every product/sum that decides a key bit or a cell boundary must round
// separately (no contraction).
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// std::max(p, hi) = p < hi ? hi : p ;  std::min(p, lo) = lo < p ? lo : p
__device__ __forceinline__ void mm_update(double p, double &lo, double &hi) {
  hi = (p < hi) ? hi : p;
  lo = (lo < p) ? lo : p;
}

__global__ void __launch_bounds__(kBlock) bbox_partial(const double *__restrict__ x,
                                                       const double *__restrict__ y,
                                                       const double *__restrict__ z, int64_t n,
                                                       double *__restrict__ part) {
  // Initialise from body 0's z (the value the reference's box starts from).
  double lo = z[0], hi = z[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    mm_update(x[i], lo, hi);
    mm_update(y[i], lo, hi);
    mm_update(z[i], lo, hi);
  }
  for (int o = 16; o > 0; o >>= 1) {
    double l2 = __shfl_down_sync(0xffffffffu, lo, o);
    double h2 = __shfl_down_sync(0xffffffffu, hi, o);
    lo = fmin(lo, l2);
    hi = fmax(hi, h2);
  }
  __shared__ double sl[kBlock / 32], sh[kBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sl[warp] = lo; sh[warp] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kBlock / 32; w++) { lo = fmin(lo, sl[w]); hi = fmax(hi, sh[w]); }
    part[2 * blockIdx.x] = lo;
    part[2 * blockIdx.x + 1] = hi;
  }
}

__global__ void bbox_final(const double *__restrict__ part, int nparts, double *__restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double lo = part[0], hi = part[1];
    for (int i = 1; i < nparts; i++) {
      lo = fmin(lo, part[2 * i]);
      hi = fmax(hi, part[2 * i + 1]);
    }
    out[0] = lo;
    out[1] = hi;
  }
}

// Keys of the bodies, and each body packed as one 32-byte record (x, y, z, q)
// so the gather into key order reads one sector per body; with q null the
// charge is packed later (pack_charges).
__global__ void __launch_bounds__(kBlock) keys_kernel(const double *__restrict__ x,
                                                      const double *__restrict__ y,
                                                      const double *__restrict__ z,
                                                      const double *__restrict__ q, int64_t n,
                                                      const double *__restrict__ box,
                                                      uint64_t *__restrict__ keys,
                                                      uint32_t *__restrict__ idx,
                                                      double4 *__restrict__ packed) {
  const double lo = box[0], hi = box[1];
  const int nfc = 1 << kMaxDepth;
  const double pitch = ddiv(dsub(hi, lo), (double)nfc);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int a[3];
    const double p[3] = {x[i], y[i], z[i]};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double o = ddiv(dsub(p[d], lo), pitch);
      a[d] = to_int_x86(o);
      if (a[d] == nfc) a[d]--;
    }
    keys[i] = finest_key(a[0], a[1], a[2]);
    idx[i] = (uint32_t)i;
    packed[i] = make_double4(p[0], p[1], p[2], q ? q[i] : 0.0);
  }
}

__global__ void pack_charges(const double *__restrict__ q, int64_t n,
                             double4 *__restrict__ packed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    packed[i].w = q[i];
}

__global__ void __launch_bounds__(kBlock) gather_bodies(
    const double4 *__restrict__ packed, const uint32_t *__restrict__ idx, int64_t n,
    double *__restrict__ sx, double *__restrict__ sy, double *__restrict__ sz,
    double *__restrict__ sq) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 b = packed[idx[i]];
    sx[i] = b.x;
    sy[i] = b.y;
    sz[i] = b.z;
    sq[i] = b.w;
  }
}

__global__ void init_root(int64_t n, int ncrit, const double *__restrict__ box,
                          uint64_t *ckey, int32_t *cbeg, int32_t *cnb, int32_t *cparent,
                          int32_t *cchild, int32_t *cleaf, int32_t *clevel, double *cmin,
                          double *cmax, double *ccen) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  ckey[0] = 0;
  cbeg[0] = 0;
  cnb[0] = (int32_t)n;
  cparent[0] = -1;
  cchild[0] = -1;
  cleaf[0] = n <= ncrit ? 1 : 0;
  clevel[0] = 0;
  for (int d = 0; d < 3; d++) {
    cmin[d] = box[0];
    cmax[d] = box[1];
    ccen[d] = dadd(box[1], box[0]) / 2;  // (max + min) / 2, hot.h:232-238
  }
}

// split flag of each cell of a level
__global__ void level_flags(const int32_t *__restrict__ cleaf, int64_t a, int64_t cnt,
                            int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = cleaf[a + i] ? 0 : 1;
}

__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t *__restrict__ a, int64_t lo,
                                                   int64_t hi, uint64_t v) {
  while (lo < hi) {
    int64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// One thread per child of the non-leaf cells of level [a, a+cnt).
__global__ void __launch_bounds__(kBlock) build_children(
    int64_t a, int64_t cnt, int64_t child_base, const int32_t *__restrict__ flag,
    const int32_t *__restrict__ flag_scan, const uint64_t *__restrict__ keys, int ncrit,
    uint64_t *__restrict__ ckey, int32_t *__restrict__ cbeg, int32_t *__restrict__ cnb,
    int32_t *__restrict__ cparent, int32_t *__restrict__ cchild, int32_t *__restrict__ cleaf,
    int32_t *__restrict__ clevel, double *__restrict__ cmin, double *__restrict__ cmax,
    double *__restrict__ ccen) {
  const int64_t total = cnt * 8;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t li = t >> 3;   // cell within the level
    const int ci = (int)(t & 7);
    if (!flag[li]) continue;
    const int64_t p = a + li;
    const int64_t c = child_base + 8 * (int64_t)flag_scan[li] + ci;
    if (ci == 0) cchild[p] = (int32_t)c;
    const uint64_t pk = ckey[p];
    const uint64_t k = key_child(pk, ci);
    const int64_t pb = cbeg[p], pe = pb + cnb[p];
    const int64_t rb = lower_bound_u64(keys, pb, pe, k);
    const int64_t re = lower_bound_u64(keys, rb, pe, key_next(k));
    const int nb = (int)(re - rb);
    const int depth = key_depth(k);
    ckey[c] = k;
    cbeg[c] = (int32_t)rb;
    cnb[c] = nb;
    cparent[c] = (int32_t)p;
    cchild[c] = -1;
    // Leaf iff nb <= ncrit.  Cells at the deepest key level are leaves too:
    // the reference's child-key shift is undefined there.
    cleaf[c] = (nb <= ncrit || depth >= kMaxDepth) ? 1 : 0;
    clevel[c] = depth;
    // Region: parent's box halved once (CalcRegion, sfc_morton.h:536-557).
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double mn = cmin[3 * p + d], mx = cmax[3 * p + d];
      const double mid = dadd(mx, mn) / 2;
      double lo, hi;
      if ((ci >> d) & 1) { lo = mid; hi = mx; } else { lo = mn; hi = mid; }
      cmin[3 * c + d] = lo;
      cmax[3 * c + d] = hi;
      ccen[3 * c + d] = dadd(hi, lo) / 2;
    }
  }
}

__global__ void collect_leaves(const int32_t *__restrict__ cleaf, const int32_t *__restrict__ cnb,
                               int64_t ncells, int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncells;
       i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = (cleaf[i] && cnb[i] > 0) ? 1 : 0;
}

__global__ void compact_indices(const int32_t *__restrict__ flag,
                                const int32_t *__restrict__ scan, int64_t n,
                                int32_t *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (flag[i]) out[scan[i]] = (int32_t)i;
}

__global__ void leaf_depth_hist(const int32_t *__restrict__ leaves, int64_t nleaves,
                                const int32_t *__restrict__ clevel, const int32_t *__restrict__ cnb,
                                int nbins, unsigned long long *__restrict__ hist) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nleaves;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int c = leaves[w];
    const int d = min(clevel[c], nbins - 1);
    atomicAdd(hist + d, (unsigned long long)cnb[c]);
  }
}

}  // namespace

int leaf_depth_histogram(tapas_b200_ctx *ctx, int nbins, int64_t *out) {
  if (!ctx->have_tree) {
    set_error(ctx, "leaf_depth_histogram: no tree");
    return TAPAS_B200_ERR_STATE;
  }
  if (nbins < 1 || nbins > 64 || !out) {
    set_error(ctx, "leaf_depth_histogram: nbins must be 1..64");
    return TAPAS_B200_ERR_ARG;
  }
  cudaStream_t s = ctx->stream;
  TB_CUDA(ctx, ctx->counters.ensure(64, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, 64 * sizeof(unsigned long long), s));
  const int64_t nl = ctx->n_nonempty_leaves;
  if (nl > 0) {
    leaf_depth_hist<<<grid_for(nl, kBlock), kBlock, 0, s>>>(ctx->leaf_list.p, nl, ctx->clevel.p,
                                                             ctx->cnb.p, nbins, ctx->counters.p);
    TB_LAUNCH_CHECK(ctx);
  }
  TB_CUDA(ctx, cudaMemcpyAsync(out, ctx->counters.p, nbins * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  return TAPAS_B200_OK;
}

int ensure_cells(tapas_b200_ctx *ctx, int64_t need, int64_t used) {
  cudaStream_t s = ctx->stream;
  if ((size_t)need <= ctx->ckey.cap) return TAPAS_B200_OK;
  TB_CUDA(ctx, ctx->ckey.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->cbeg.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->cnb.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->cparent.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->cchild.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->cleaf.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->clevel.ensure(need, s, true, used));
  TB_CUDA(ctx, ctx->cmin.ensure(3 * need, s, true, 3 * used));
  TB_CUDA(ctx, ctx->cmax.ensure(3 * need, s, true, 3 * used));
  TB_CUDA(ctx, ctx->ccen.ensure(3 * need, s, true, 3 * used));
  return TAPAS_B200_OK;
}

int build_tree(tapas_b200_ctx *ctx, int ncrit) {
  cudaStream_t s = ctx->stream;
  const int64_t n = ctx->n;
  if (n <= 0) {
    set_error(ctx, "partition: no bodies");
    return TAPAS_B200_ERR_ARG;
  }
  ctx->have_tree = ctx->have_lists = ctx->have_M = ctx->have_L = false;
  ctx->level_ops_P = 0;  // translation operators belong to the previous tree
  ctx->ncrit = ncrit;
  TB_CUDA(ctx, ctx->keys.ensure(n, s));
  TB_CUDA(ctx, ctx->keys_alt.ensure(n, s));
  TB_CUDA(ctx, ctx->idx.ensure(n, s));
  TB_CUDA(ctx, ctx->idx_alt.ensure(n, s));
  TB_CUDA(ctx, ctx->sx.ensure(n, s));
  TB_CUDA(ctx, ctx->sy.ensure(n, s));
  TB_CUDA(ctx, ctx->sz.ensure(n, s));
  TB_CUDA(ctx, ctx->sq.ensure(n, s));
  TB_CUDA(ctx, ctx->body_pack.ensure(n, s));
  TB_CUDA(ctx, ctx->trg.ensure(4 * n, s));
  TB_CUDA(ctx, ctx->bbox.ensure(2, s));

  {
    PhaseTimer t(ctx, &ctx->timings.bbox_keys);
    const int nparts = grid_for(n, kBlock, ctx->num_sms * 4);
    TB_CUDA(ctx, ctx->scratch_d.ensure(2 * nparts + 2, s));
    bbox_partial<<<nparts, kBlock, 0, s>>>(ctx->x.p, ctx->y.p, ctx->z.p, n, ctx->scratch_d.p);
    TB_LAUNCH_CHECK(ctx);
    bbox_final<<<1, 32, 0, s>>>(ctx->scratch_d.p, nparts, ctx->bbox.p);
    TB_LAUNCH_CHECK(ctx);
    keys_kernel<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
        ctx->x.p, ctx->y.p, ctx->z.p, ctx->q_pending ? nullptr : ctx->q.p, n, ctx->bbox.p,
        ctx->keys.p, ctx->idx.p, ctx->body_pack.p);
    TB_LAUNCH_CHECK(ctx);
  }
  {
    PhaseTimer t(ctx, &ctx->timings.sort);
    uint64_t *k = ctx->keys.p, *ka = ctx->keys_alt.p;
    uint32_t *v = ctx->idx.p, *va = ctx->idx_alt.p;
    // Depth bits (4..0) are 19 for every body key; sort on bits 5..61.
    TB_TRY(radix_sort(ctx, k, ka, v, va, n, kDepthBits, kDepthBits + 3 * kMaxDepth));
    if (k != ctx->keys.p) { std::swap(ctx->keys.p, ctx->keys_alt.p); std::swap(ctx->keys.cap, ctx->keys_alt.cap); }
    if (v != ctx->idx.p) { std::swap(ctx->idx.p, ctx->idx_alt.p); std::swap(ctx->idx.cap, ctx->idx_alt.cap); }
    if (ctx->q_pending) {  // the charges' copy ran alongside the keys and the sort
      TB_CUDA(ctx, cudaStreamWaitEvent(s, ctx->q_ready, 0));
      pack_charges<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(ctx->q.p, n,
                                                                            ctx->body_pack.p);
      TB_LAUNCH_CHECK(ctx);
      ctx->q_pending = false;
    }
    gather_bodies<<<grid_for(n, kBlock, ctx->num_sms * 16), kBlock, 0, s>>>(
        ctx->body_pack.p, ctx->idx.p, n, ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p);
    TB_LAUNCH_CHECK(ctx);
  }
  PhaseTimer t(ctx, &ctx->timings.tree);
  // Level-by-level build.  Estimate capacity: ~ 8/7 * 8 * n / ncrit cells.
  int64_t est = 64 + (int64_t)(2.5 * 8.0 * (double)n / (double)std::max(ncrit, 1));
  TB_TRY(ensure_cells(ctx, est, 0));
  TB_CUDA(ctx, ctx->pinned.ensure(64));
  init_root<<<1, 32, 0, s>>>(n, ncrit, ctx->bbox.p, ctx->ckey.p, ctx->cbeg.p, ctx->cnb.p,
                             ctx->cparent.p, ctx->cchild.p, ctx->cleaf.p, ctx->clevel.p,
                             ctx->cmin.p, ctx->cmax.p, ctx->ccen.p);
  TB_LAUNCH_CHECK(ctx);
  ctx->level_off.assign(1, 0);
  ctx->level_off.push_back(1);
  int64_t a = 0, cnt = 1;
  int depth = 0;
  int32_t *h_total = reinterpret_cast<int32_t *>(ctx->pinned.p);
  while (true) {
    TB_CUDA(ctx, ctx->flag.ensure(cnt + 1, s));
    TB_CUDA(ctx, ctx->flag_scan.ensure(cnt + 1, s));
    level_flags<<<grid_for(cnt, kBlock), kBlock, 0, s>>>(ctx->cleaf.p, a, cnt, ctx->flag.p);
    TB_LAUNCH_CHECK(ctx);
    TB_TRY(scan_exclusive(ctx, ctx->flag.p, ctx->flag_scan.p, cnt, ctx->flag_scan.p + cnt));
    TB_CUDA(ctx, cudaMemcpyAsync(h_total, ctx->flag_scan.p + cnt, sizeof(int32_t),
                                 cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    const int64_t nsplit = *h_total;
    if (nsplit == 0) break;
    const int64_t child_base = a + cnt;
    const int64_t nchild = 8 * nsplit;
    TB_TRY(ensure_cells(ctx, child_base + nchild, child_base));
    build_children<<<grid_for(cnt * 8, kBlock, ctx->num_sms * 32), kBlock, 0, s>>>(
        a, cnt, child_base, ctx->flag.p, ctx->flag_scan.p, ctx->keys.p, ncrit, ctx->ckey.p,
        ctx->cbeg.p, ctx->cnb.p, ctx->cparent.p, ctx->cchild.p, ctx->cleaf.p, ctx->clevel.p,
        ctx->cmin.p, ctx->cmax.p, ctx->ccen.p);
    TB_LAUNCH_CHECK(ctx);
    a = child_base;
    cnt = nchild;
    depth++;
    ctx->level_off.push_back(a + cnt);
    if (depth > kMaxDepth) {
      set_error(ctx, "tree build exceeded the maximum key depth");
      return TAPAS_B200_ERR_CAPACITY;
    }
  }
  ctx->ncells = a + cnt;
  ctx->max_depth = depth;
  // Non-empty leaves (the P2M / L2P / P2P work units).
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->flag.ensure(C + 1, s));
  TB_CUDA(ctx, ctx->flag_scan.ensure(C + 1, s));
  TB_CUDA(ctx, ctx->leaf_list.ensure(C + 1, s));
  collect_leaves<<<grid_for(C, kBlock), kBlock, 0, s>>>(ctx->cleaf.p, ctx->cnb.p, C, ctx->flag.p);
  TB_LAUNCH_CHECK(ctx);
  TB_TRY(scan_exclusive(ctx, ctx->flag.p, ctx->flag_scan.p, C, ctx->flag_scan.p + C));
  compact_indices<<<grid_for(C, kBlock), kBlock, 0, s>>>(ctx->flag.p, ctx->flag_scan.p, C,
                                                         ctx->leaf_list.p);
  TB_LAUNCH_CHECK(ctx);
  double *hb = reinterpret_cast<double *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemcpyAsync(hb, ctx->bbox.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaMemcpyAsync(reinterpret_cast<int32_t *>(hb + 2), ctx->flag_scan.p + C,
                               sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->box_lo = hb[0];
  ctx->box_hi = hb[1];
  ctx->n_nonempty_leaves = *reinterpret_cast<int32_t *>(hb + 2);
  ctx->have_tree = true;
  return TAPAS_B200_OK;
}

}  // namespace tb
