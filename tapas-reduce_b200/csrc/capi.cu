// C ABI of libtapas_b200 (declared in include/tapas_b200.h).
#include <algorithm>
#include <cstring>
#include <new>

#include "common.cuh"
#include "kernels.cuh"
#include "m2l_tc.cuh"
#include "traverse.cuh"
#include "tree.cuh"

namespace tb {

static thread_local std::string g_last_error;

void set_error(tapas_b200_ctx *ctx, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) ctx->last_error = buf;
  g_last_error = buf;
}

namespace {

__global__ void scatter_results(const double *__restrict__ trg, const uint32_t *__restrict__ idx,
                                int64_t n, double *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 v = reinterpret_cast<const double4 *>(trg)[i];
    reinterpret_cast<double4 *>(out)[idx[i]] = v;
  }
}

__global__ void widen_idx(const uint32_t *__restrict__ idx, int64_t n, int64_t *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = idx[i];
}

// FP64 direct sum, field form, one block per target (original indices).
__global__ void __launch_bounds__(256) direct_kernel(const double *__restrict__ x,
                                                     const double *__restrict__ y,
                                                     const double *__restrict__ z,
                                                     const double *__restrict__ q, int64_t n,
                                                     const int64_t *__restrict__ tg,
                                                     double *__restrict__ out) {
  const int64_t i = tg[blockIdx.x];
  const double xi = x[i], yi = y[i], zi = z[i];
  double p = 0, ax = 0, ay = 0, az = 0;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    const double dx = xi - x[j], dy = yi - y[j], dz = zi - z[j];
    const double R2 = dx * dx + dy * dy + dz * dz;
    if (R2 != 0) {
      const double invR = 1.0 / sqrt(R2);
      const double qr = q[j] * invR;
      const double s3 = qr * invR * invR;
      p += qr;
      ax -= dx * s3;
      ay -= dy * s3;
      az -= dz * s3;
    }
  }
  __shared__ double red[4][8];
  for (int o = 16; o > 0; o >>= 1) {
    p += __shfl_down_sync(0xffffffffu, p, o);
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
    az += __shfl_down_sync(0xffffffffu, az, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = p; red[1][w] = ax; red[2][w] = ay; red[3][w] = az; }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0;
    for (int k = 0; k < 8; k++) s += red[threadIdx.x][k];
    out[4 * blockIdx.x + threadIdx.x] = s;
  }
}

// The non-empty leaves whose ownership mask has bit 1 (their bodies are
// evaluated here); order is irrelevant (every leaf is independent).
__global__ void select_owned_leaves(const int32_t *__restrict__ leaves, int64_t nl,
                                    const uint8_t *__restrict__ own, int32_t *__restrict__ out,
                                    int *__restrict__ count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nl;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = leaves[i];
    if (own[c] & 2) out[atomicAdd(count, 1)] = c;
  }
}

int copy_in(tapas_b200_ctx *ctx, double *dst, const double *src, int64_t n, int mem) {
  TB_CUDA(ctx, cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)n,
                               mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyHostToDevice,
                               ctx->stream));
  return TAPAS_B200_OK;
}

int check_ctx(tapas_b200_ctx *ctx) {
  if (!ctx) {
    set_error(nullptr, "null context");
    return TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaSetDevice(ctx->device));
  return TAPAS_B200_OK;
}

int check_mem(tapas_b200_ctx *ctx, int mem) {
  if (mem != TAPAS_B200_HOST && mem != TAPAS_B200_DEVICE) {
    set_error(ctx, "mem must be TAPAS_B200_HOST or TAPAS_B200_DEVICE");
    return TAPAS_B200_ERR_ARG;
  }
  return TAPAS_B200_OK;
}

int check_precision(tapas_b200_ctx *ctx, int precision) {
  if (precision != TAPAS_B200_FP64 && precision != TAPAS_B200_MIXED) {
    set_error(ctx, "precision must be TAPAS_B200_FP64 or TAPAS_B200_MIXED");
    return TAPAS_B200_ERR_ARG;
  }
  return TAPAS_B200_OK;
}

}  // namespace
}  // namespace tb

using namespace tb;

extern "C" {

int tapas_b200_ctx_create(int device, tapas_b200_ctx **out) {
  if (!out) {
    set_error(nullptr, "ctx_create: null output pointer");
    return TAPAS_B200_ERR_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error(nullptr, "ctx_create: no CUDA device (%s)", cudaGetErrorString(e));
    return TAPAS_B200_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) {
    set_error(nullptr, "ctx_create: device %d outside 0..%d", device, ndev - 1);
    return TAPAS_B200_ERR_ARG;
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    set_error(nullptr, "ctx_create: %s", cudaGetErrorString(e));
    return TAPAS_B200_ERR_CUDA;
  }
  if (prop.major != 10) {
    set_error(nullptr, "ctx_create: device %d is sm_%d%d; this library is built for sm_100a",
              device, prop.major, prop.minor);
    return TAPAS_B200_ERR_UNSUPPORTED;
  }
  tapas_b200_ctx *ctx = new (std::nothrow) tapas_b200_ctx();
  if (!ctx) {
    set_error(nullptr, "ctx_create: out of host memory");
    return TAPAS_B200_ERR_NOMEM;
  }
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error(nullptr, "ctx_create: %s", cudaGetErrorString(e));
    delete ctx;
    return TAPAS_B200_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  *out = ctx;
  return TAPAS_B200_OK;
}

int tapas_b200_ctx_destroy(tapas_b200_ctx *ctx) {
  if (!ctx) return TAPAS_B200_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto *b : {&ctx->x, &ctx->y, &ctx->z, &ctx->q, &ctx->sx, &ctx->sy, &ctx->sz, &ctx->sq,
                  &ctx->trg, &ctx->trg_out, &ctx->bbox, &ctx->scratch_d, &ctx->cmin, &ctx->cmax,
                  &ctx->ccen})
    b->release();
  for (auto *b : {&ctx->keys, &ctx->keys_alt, &ctx->ckey, &ctx->m2l, &ctx->p2p, &ctx->list_alt})
    b->release();
  for (auto *b : {&ctx->idx, &ctx->idx_alt, &ctx->sort_hist}) b->release();
  for (auto *b : {&ctx->scan_tmp, &ctx->cbeg, &ctx->cnb, &ctx->cparent, &ctx->cchild, &ctx->cleaf,
                  &ctx->clevel, &ctx->flag, &ctx->flag_scan, &ctx->leaf_list, &ctx->list_cnt,
                  &ctx->m2l_off, &ctx->p2p_off, &ctx->m2l_tlist, &ctx->p2p_tlist})
    b->release();
  ctx->front_a.release();
  ctx->front_b.release();
  ctx->counters.release();
  ctx->trav_geo.release();
  ctx->body_pack.release();
  ctx->trav_meta.release();
  ctx->list_src.release();
  ctx->M.release();
  ctx->L.release();
  ctx->op_m2m.release();
  ctx->op_l2l.release();
  ctx->op_part.release();
  // mixed-form state: near-field offsets, P2P work items, tensor-core M2L
  for (auto *b : {&ctx->rel4, &ctx->rel_lo}) b->release();
  for (auto *b : {&ctx->p2p_wkey, &ctx->p2p_wkey_alt}) b->release();
  for (auto *b : {&ctx->p2p_order, &ctx->p2p_order_alt}) b->release();
  for (auto *b : {&ctx->p2p_kcnt, &ctx->p2p_koff, &ctx->p2p_psz, &ctx->p2p_poff}) b->release();
  ctx->p2p_counter.release();
  ctx->p2p_items.release();
  ctx->p2p_part.release();
  for (auto *b : {&ctx->l2p_body_leaf}) b->release();
  ctx->l2p_lf.release();
  ctx->l2p_geo.release();
  ctx->tc.release();
  mlp_release(ctx);
  ctx->bh_attr.release();
  ctx->bh_attr32.release();
  ctx->pinned.release();
  for (int k = 0; k < kGemmSlabs; k++) {
    if (ctx->gemm_streams[k]) cudaStreamDestroy(ctx->gemm_streams[k]);
    if (ctx->gemm_join[k]) cudaEventDestroy(ctx->gemm_join[k]);
  }
  if (ctx->gemm_fork) cudaEventDestroy(ctx->gemm_fork);
  if (ctx->upload_stream) cudaStreamDestroy(ctx->upload_stream);
  if (ctx->q_ready) cudaEventDestroy(ctx->q_ready);
  if (ctx->upload_fork) cudaEventDestroy(ctx->upload_fork);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return TAPAS_B200_OK;
}

int tapas_b200_set_stream(tapas_b200_ctx *ctx, void *stream) {
  TB_TRY(check_ctx(ctx));
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return TAPAS_B200_OK;
}

int tapas_b200_set_profiling(tapas_b200_ctx *ctx, int on) {
  TB_TRY(check_ctx(ctx));
  ctx->profiling = on != 0;
  return TAPAS_B200_OK;
}

int tapas_b200_set_reference_lists(tapas_b200_ctx *ctx, int on) {
  TB_TRY(check_ctx(ctx));
  ctx->reference_lists = on != 0;  // applies to the next list construction
  return TAPAS_B200_OK;
}

int tapas_b200_set_wait_limit(tapas_b200_ctx *ctx, int64_t cycles) {
  TB_TRY(check_ctx(ctx));
  ctx->tc_wait_limit = cycles > 0 ? (long long)cycles : 4000000000LL;
  return TAPAS_B200_OK;
}

int tapas_b200_get_timings(tapas_b200_ctx *ctx, tapas_b200_timings *out) {
  TB_TRY(check_ctx(ctx));
  if (!out) return TAPAS_B200_ERR_ARG;
  *out = ctx->timings;
  return TAPAS_B200_OK;
}

const char *tapas_b200_last_error(const tapas_b200_ctx *ctx) {
  return ctx ? ctx->last_error.c_str() : g_last_error.c_str();
}

int64_t tapas_b200_kernel_launches(tapas_b200_ctx *ctx, int reset) {
  if (!ctx) return -1;
  int64_t v = ctx->launches;
  if (reset) ctx->launches = 0;
  return v;
}

int tapas_b200_partition(tapas_b200_ctx *ctx, const double *x, const double *y, const double *z,
                         const double *q, int64_t n, int ncrit, int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (n <= 0 || n > (int64_t)0x7FFFFFFF || !x || !y || !z || !q) {
    set_error(ctx, "partition: need 1 <= n < 2^31 and non-null body arrays (n=%lld)",
              (long long)n);
    return TAPAS_B200_ERR_ARG;
  }
  if (ncrit < 1) {
    set_error(ctx, "partition: ncrit must be >= 1");
    return TAPAS_B200_ERR_ARG;
  }
  cudaStream_t s = ctx->stream;
  ctx->timings = tapas_b200_timings{};  // a partition starts a new step's timings
  {
    PhaseTimer t(ctx, &ctx->timings.upload);
    TB_CUDA(ctx, ctx->x.ensure(n, s));
    TB_CUDA(ctx, ctx->y.ensure(n, s));
    TB_CUDA(ctx, ctx->z.ensure(n, s));
    TB_CUDA(ctx, ctx->q.ensure(n, s));
    TB_TRY(copy_in(ctx, ctx->x.p, x, n, mem));
    TB_TRY(copy_in(ctx, ctx->y.p, y, n, mem));
    TB_TRY(copy_in(ctx, ctx->z.p, z, n, mem));
    ctx->q_pending = false;
  }
  if (mem == TAPAS_B200_DEVICE) {
    PhaseTimer t(ctx, &ctx->timings.upload);
    TB_TRY(copy_in(ctx, ctx->q.p, q, n, mem));
  } else {
    // The charges are first read when the sorted bodies are gathered: their
    // copy from the host runs on a side stream while the keys are built and
    // sorted.
    if (!ctx->upload_stream) {
      TB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->upload_stream, cudaStreamNonBlocking));
      TB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->q_ready, cudaEventDisableTiming));
      TB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->upload_fork, cudaEventDisableTiming));
    }
    TB_CUDA(ctx, cudaEventRecord(ctx->upload_fork, s));  // q's buffer is free from here
    TB_CUDA(ctx, cudaStreamWaitEvent(ctx->upload_stream, ctx->upload_fork, 0));
    TB_CUDA(ctx, cudaMemcpyAsync(ctx->q.p, q, sizeof(double) * (size_t)n,
                                 cudaMemcpyHostToDevice, ctx->upload_stream));
    TB_CUDA(ctx, cudaEventRecord(ctx->q_ready, ctx->upload_stream));
    ctx->q_pending = true;
  }
  ctx->n = n;
  ctx->have_bh_attr = false;
  ctx->sharded = false;  // an ownership mask belongs to one tree
  ctx->tc.mt_ready = false;
  return build_tree(ctx, ncrit);
}

int tapas_b200_get_device_view(tapas_b200_ctx *ctx, tapas_b200_device_view *out) {
  TB_TRY(check_ctx(ctx));
  if (!out) {
    set_error(ctx, "get_device_view: null output");
    return TAPAS_B200_ERR_ARG;
  }
  if (!ctx->have_tree) {
    set_error(ctx, "get_device_view: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  TB_TRY(sort_list_sources(ctx));  // the view's lists: sources in order per target
  *out = tapas_b200_device_view{};
  out->n_bodies = ctx->n;
  out->n_cells = ctx->ncells;
  const int64_t nlev = std::min<int64_t>((int64_t)ctx->level_off.size() - 1,
                                         TAPAS_B200_MAX_LEVELS);
  out->n_levels = nlev;
  for (int64_t l = 0; l <= nlev; l++) out->level_off[l] = ctx->level_off[(size_t)l];
  out->nb = ctx->cnb.p;
  out->bbeg = ctx->cbeg.p;
  out->leaf = ctx->cleaf.p;
  out->parent = ctx->cparent.p;
  out->child0 = ctx->cchild.p;
  out->level = ctx->clevel.p;
  out->center3 = ctx->ccen.p;
  out->min3 = ctx->cmin.p;
  out->max3 = ctx->cmax.p;
  out->x = ctx->sx.p;
  out->y = ctx->sy.p;
  out->z = ctx->sz.p;
  out->q = ctx->sq.p;
  out->orig_index = ctx->idx.p;
  if (ctx->have_lists) {
    out->p2p_off = ctx->p2p_off.p;
    out->m2l_off = ctx->m2l_off.p;
    out->p2p_list = ctx->p2p.p;
    out->m2l_list = ctx->m2l.p;
    out->n_p2p = ctx->n_p2p;
    out->n_m2l = ctx->n_m2l;
    out->list_shift = ctx->list_shift;
  }
  return TAPAS_B200_OK;
}

int tapas_b200_set_near_field(tapas_b200_ctx *ctx, const double *trg4, int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (!trg4) {
    set_error(ctx, "set_near_field: null input");
    return TAPAS_B200_ERR_ARG;
  }
  if (!ctx->have_tree) {
    set_error(ctx, "set_near_field: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  TB_CUDA(ctx, cudaMemcpyAsync(ctx->trg.p, trg4, sizeof(double) * 4 * (size_t)ctx->n,
                               mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyHostToDevice,
                               ctx->stream));
  ctx->near_precision = TAPAS_B200_FP64;  // sums carry q_i: the L2P divides by it
  return TAPAS_B200_OK;
}

int tapas_b200_get_stream(tapas_b200_ctx *ctx, void **stream) {
  TB_TRY(check_ctx(ctx));
  if (!stream) return TAPAS_B200_ERR_ARG;
  *stream = ctx->stream;
  return TAPAS_B200_OK;
}

int tapas_b200_set_owned_cells(tapas_b200_ctx *ctx, const uint8_t *mask, int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (!ctx->have_tree) {
    set_error(ctx, "set_owned_cells: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  ctx->have_M = ctx->have_L = ctx->have_lists = false;
  if (!mask) {
    ctx->sharded = false;
    return TAPAS_B200_OK;
  }
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells, nl = ctx->n_nonempty_leaves;
  TB_CUDA(ctx, ctx->cell_own.ensure(C + 1, s));
  TB_CUDA(ctx, cudaMemcpyAsync(ctx->cell_own.p, mask, (size_t)C,
                               mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyHostToDevice,
                               s));
  TB_CUDA(ctx, ctx->leaf_own.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->counters.ensure(8, s));
  int *cnt = reinterpret_cast<int *>(ctx->counters.p);
  TB_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int), s));
  if (nl > 0) {
    select_owned_leaves<<<grid_for(nl, 256), 256, 0, s>>>(ctx->leaf_list.p, nl, ctx->cell_own.p,
                                                           ctx->leaf_own.p, cnt);
    TB_LAUNCH_CHECK(ctx);
  }
  TB_CUDA(ctx, ctx->pinned.ensure(256));
  int *h = reinterpret_cast<int *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemcpyAsync(h, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->n_owned_leaves = h[0];
  ctx->sharded = true;
  return TAPAS_B200_OK;
}

int tapas_b200_bh_upward(tapas_b200_ctx *ctx) {
  TB_TRY(check_ctx(ctx));
  return bh_upward(ctx);
}

int tapas_b200_bh_interact(tapas_b200_ctx *ctx, double theta, double eps2, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  return bh_interact(ctx, theta, eps2, precision);
}

int tapas_b200_bh_counts(tapas_b200_ctx *ctx, uint64_t *n_approx, uint64_t *n_direct) {
  TB_TRY(check_ctx(ctx));
  if (n_approx) *n_approx = ctx->bh_napprox;
  if (n_direct) *n_direct = ctx->bh_ndirect;
  return TAPAS_B200_OK;
}

int tapas_b200_bh_evaluate(tapas_b200_ctx *ctx, const double *x, const double *y, const double *z,
                           const double *m, int64_t n, int ncrit, double theta, double eps2,
                           int precision, double *out4, int order, int mem) {
  TB_TRY(tapas_b200_partition(ctx, x, y, z, m, n, ncrit, mem));
  TB_TRY(tapas_b200_bh_upward(ctx));
  TB_TRY(tapas_b200_bh_interact(ctx, theta, eps2, precision));
  return tapas_b200_get_results(ctx, out4, order, mem);
}

int tapas_b200_tree_info(tapas_b200_ctx *ctx, tapas_b200_tree_stats *out) {
  TB_TRY(check_ctx(ctx));
  if (!out) return TAPAS_B200_ERR_ARG;
  if (!ctx->have_tree) {
    set_error(ctx, "tree_info: no tree");
    return TAPAS_B200_ERR_STATE;
  }
  // leaves = cells - non-leaves; every non-leaf has 8 children: C = 1 + 8 * nonleaf
  const int64_t nonleaf = (ctx->ncells - 1) / 8;
  out->n_bodies = ctx->n;
  out->n_cells = ctx->ncells;
  out->n_leaves = ctx->ncells - nonleaf;
  out->max_depth = ctx->max_depth;
  out->ncrit = ctx->ncrit;
  out->box_lo = ctx->box_lo;
  out->box_hi = ctx->box_hi;
  return TAPAS_B200_OK;
}

int tapas_b200_get_cells(tapas_b200_ctx *ctx, uint64_t *key, int32_t *leaf, int32_t *nb,
                         int32_t *bbeg, int32_t *parent, int32_t *child0, double *center3,
                         double *width3) {
  TB_TRY(check_ctx(ctx));
  if (!ctx->have_tree) {
    set_error(ctx, "get_cells: no tree");
    return TAPAS_B200_ERR_STATE;
  }
  const int64_t C = ctx->ncells;
  cudaStream_t s = ctx->stream;
  auto d2h = [&](void *h, const void *d, size_t bytes) -> int {
    if (!h) return TAPAS_B200_OK;
    TB_CUDA(ctx, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
    return TAPAS_B200_OK;
  };
  TB_TRY(d2h(key, ctx->ckey.p, 8 * C));
  TB_TRY(d2h(leaf, ctx->cleaf.p, 4 * C));
  TB_TRY(d2h(nb, ctx->cnb.p, 4 * C));
  TB_TRY(d2h(bbeg, ctx->cbeg.p, 4 * C));
  TB_TRY(d2h(parent, ctx->cparent.p, 4 * C));
  TB_TRY(d2h(child0, ctx->cchild.p, 4 * C));
  TB_TRY(d2h(center3, ctx->ccen.p, 24 * C));
  if (width3) {
    std::vector<double> mn(3 * C), mx(3 * C);
    TB_TRY(d2h(mn.data(), ctx->cmin.p, 24 * C));
    TB_TRY(d2h(mx.data(), ctx->cmax.p, 24 * C));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    for (int64_t i = 0; i < 3 * C; i++) width3[i] = mx[i] - mn[i];
  }
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  return TAPAS_B200_OK;
}

int tapas_b200_leaf_depth_histogram(tapas_b200_ctx *ctx, int nbins, int64_t *hist) {
  TB_TRY(check_ctx(ctx));
  return leaf_depth_histogram(ctx, nbins, hist);
}

int tapas_b200_get_sorted(tapas_b200_ctx *ctx, int64_t *orig_index, uint64_t *keys) {
  TB_TRY(check_ctx(ctx));
  if (!ctx->have_tree) {
    set_error(ctx, "get_sorted: no tree");
    return TAPAS_B200_ERR_STATE;
  }
  cudaStream_t s = ctx->stream;
  const int64_t n = ctx->n;
  if (keys) TB_CUDA(ctx, cudaMemcpyAsync(keys, ctx->keys.p, 8 * n, cudaMemcpyDeviceToHost, s));
  if (orig_index) {
    std::vector<uint32_t> tmp(n);
    TB_CUDA(ctx, cudaMemcpyAsync(tmp.data(), ctx->idx.p, 4 * n, cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    for (int64_t i = 0; i < n; i++) orig_index[i] = tmp[i];
  }
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  return TAPAS_B200_OK;
}

int tapas_b200_upward(tapas_b200_ctx *ctx, int P, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  if (!ctx->have_tree) {
    set_error(ctx, "upward: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  if (P < kMinP || P > kMaxP) {
    set_error(ctx, "upward: expansion order P=%d outside %d..%d", P, kMinP, kMaxP);
    return TAPAS_B200_ERR_UNSUPPORTED;
  }
  PhaseTimer t(ctx, &ctx->timings.upward);
  ctx->have_M = ctx->have_L = false;
  ctx->P = P;
  ctx->precision = precision;
  ctx->have_leaf_M = false;
  ctx->tc.mt_ready = false;
  if (precision == TAPAS_B200_MIXED) {
    TB_TRY(p2m_only(ctx, P, true));
    PhaseTimer tm(ctx, &ctx->timings.m2m);
    TB_TRY(tc_tree_upward(ctx));
  } else {
    TB_TRY(upward_fp64(ctx, P));
  }
  ctx->have_M = true;
  return TAPAS_B200_OK;
}

int tapas_b200_p2m(tapas_b200_ctx *ctx, int P, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  if (!ctx->have_tree) {
    set_error(ctx, "p2m: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  if (P < kMinP || P > kMaxP) {
    set_error(ctx, "p2m: expansion order P=%d outside %d..%d", P, kMinP, kMaxP);
    return TAPAS_B200_ERR_UNSUPPORTED;
  }
  PhaseTimer t(ctx, &ctx->timings.upward);
  ctx->have_M = ctx->have_L = false;
  ctx->P = P;
  ctx->precision = precision;
  ctx->tc.mt_ready = false;
  TB_TRY(p2m_only(ctx, P, precision == TAPAS_B200_MIXED));
  ctx->have_leaf_M = true;
  return TAPAS_B200_OK;
}

int tapas_b200_m2m(tapas_b200_ctx *ctx) {
  TB_TRY(check_ctx(ctx));
  if (!ctx->have_leaf_M) {
    set_error(ctx, "m2m: needs p2m first");
    return TAPAS_B200_ERR_STATE;
  }
  PhaseTimer t(ctx, &ctx->timings.m2m);
  if (ctx->precision == TAPAS_B200_MIXED) TB_TRY(tc_tree_upward(ctx));
  else TB_TRY(m2m_only(ctx));
  ctx->have_leaf_M = false;
  ctx->have_M = true;
  return TAPAS_B200_OK;
}

int tapas_b200_get_multipoles(tapas_b200_ctx *ctx, double *M, int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (!M || !(ctx->have_M || ctx->have_leaf_M)) {
    set_error(ctx, "get_multipoles: null output or no multipoles");
    return M ? TAPAS_B200_ERR_STATE : TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaMemcpyAsync(M, ctx->M.p, sizeof(double2) * (size_t)ctx->ncells * nterm_of(ctx->P),
                               mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyDeviceToHost,
                               ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TAPAS_B200_OK;
}

int tapas_b200_set_multipoles(tapas_b200_ctx *ctx, const double *M, int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (!M || !(ctx->have_M || ctx->have_leaf_M)) {
    set_error(ctx, "set_multipoles: null input or no expansion order set (p2m first)");
    return M ? TAPAS_B200_ERR_STATE : TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaMemcpyAsync(ctx->M.p, M, sizeof(double2) * (size_t)ctx->ncells * nterm_of(ctx->P),
                               mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyHostToDevice,
                               ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TAPAS_B200_OK;
}

int tapas_b200_build_lists(tapas_b200_ctx *ctx, double theta, int mutual) {
  TB_TRY(check_ctx(ctx));
  return build_lists(ctx, theta, mutual);
}

int tapas_b200_list_info(tapas_b200_ctx *ctx, tapas_b200_list_stats *out) {
  TB_TRY(check_ctx(ctx));
  if (!out) return TAPAS_B200_ERR_ARG;
  if (!ctx->have_lists) {
    set_error(ctx, "list_info: no lists");
    return TAPAS_B200_ERR_STATE;
  }
  out->n_m2l = ctx->n_m2l;
  out->n_p2p = ctx->n_p2p;
  out->n_p2p_interactions = ctx->n_p2p_int;
  out->traverse_iterations = ctx->trav_iters;
  out->n_m2l_tc = ctx->n_m2l_tc;
  out->tc_classes = ctx->tc_classes;
  out->tc_tiles = ctx->tc_tiles;
  out->pairs_visited = ctx->trav_pairs;
  return TAPAS_B200_OK;
}

int tapas_b200_get_lists(tapas_b200_ctx *ctx, int32_t *m2l_tgt, int32_t *m2l_src,
                         int32_t *p2p_tgt, int32_t *p2p_src) {
  TB_TRY(check_ctx(ctx));
  if (!ctx->have_lists) {
    set_error(ctx, "get_lists: no lists");
    return TAPAS_B200_ERR_STATE;
  }
  TB_TRY(sort_list_sources(ctx));
  const int b = ctx->list_shift;
  const uint64_t mask = (1ull << b) - 1;
  for (int which = 0; which < 2; which++) {
    const int64_t n = which ? ctx->n_p2p : ctx->n_m2l;
    int32_t *t = which ? p2p_tgt : m2l_tgt;
    int32_t *sidx = which ? p2p_src : m2l_src;
    if (!t && !sidx) continue;
    std::vector<uint64_t> h(n);
    if (n)
      TB_CUDA(ctx, cudaMemcpyAsync(h.data(), which ? ctx->p2p.p : ctx->m2l.p, 8 * n,
                                   cudaMemcpyDeviceToHost, ctx->stream));
    TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int64_t i = 0; i < n; i++) {
      if (t) t[i] = (int32_t)(h[i] >> b);
      if (sidx) sidx[i] = (int32_t)(h[i] & mask);
    }
  }
  return TAPAS_B200_OK;
}

int tapas_b200_m2l(tapas_b200_ctx *ctx, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  if (!ctx->have_lists || !ctx->have_M) {
    set_error(ctx, "m2l: needs upward and build_lists first");
    return TAPAS_B200_ERR_STATE;
  }
  PhaseTimer t(ctx, &ctx->timings.m2l);
  if (precision == TAPAS_B200_MIXED) {
    TB_TRY(m2l_tensorcore(ctx));
  } else {
    TB_TRY(sort_list_sources(ctx, 0));  // the FP64 sums run in source order
    TB_TRY(m2l_fp64(ctx));
  }
  ctx->have_L = true;
  return TAPAS_B200_OK;
}

int tapas_b200_p2p(tapas_b200_ctx *ctx, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  if (!ctx->have_lists) {
    set_error(ctx, "p2p: needs build_lists first");
    return TAPAS_B200_ERR_STATE;
  }
  PhaseTimer t(ctx, &ctx->timings.p2p);
  ctx->near_precision = precision;
  if (precision == TAPAS_B200_MIXED) return p2p_mixed(ctx);
  TB_TRY(sort_list_sources(ctx, 1));  // the FP64 sums run in source order
  return p2p_fp64(ctx);
}

int tapas_b200_traverse(tapas_b200_ctx *ctx, double theta, int mutual, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  // the mixed form needs the lists grouped by target, not each target's
  // sources sorted (its M2L regroups the pairs by offset class, its FP32
  // near field sums in any order)
  TB_TRY(build_lists(ctx, theta, mutual, precision != TAPAS_B200_MIXED));
  TB_TRY(tapas_b200_m2l(ctx, precision));
  return tapas_b200_p2p(ctx, precision);
}

int tapas_b200_downward(tapas_b200_ctx *ctx, int precision) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_precision(ctx, precision));
  if (!ctx->have_L) {
    set_error(ctx, "downward: needs traverse first");
    return TAPAS_B200_ERR_STATE;
  }
  PhaseTimer t(ctx, &ctx->timings.downward);
  if (precision == TAPAS_B200_MIXED) return downward_fp32_l2p(ctx);
  return downward_fp64(ctx);
}

int tapas_b200_get_expansions(tapas_b200_ctx *ctx, double *M, double *L) {
  TB_TRY(check_ctx(ctx));
  if (!ctx->have_M) {
    set_error(ctx, "get_expansions: no expansions");
    return TAPAS_B200_ERR_STATE;
  }
  const size_t bytes = sizeof(double2) * (size_t)ctx->ncells * nterm_of(ctx->P);
  if (M) TB_CUDA(ctx, cudaMemcpyAsync(M, ctx->M.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (L && ctx->have_L)
    TB_CUDA(ctx, cudaMemcpyAsync(L, ctx->L.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TAPAS_B200_OK;
}

int tapas_b200_get_results(tapas_b200_ctx *ctx, double *trg4, int order, int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (!trg4 || (order != TAPAS_B200_ORDER_SORTED && order != TAPAS_B200_ORDER_ORIGINAL)) {
    set_error(ctx, "get_results: bad output pointer or order");
    return TAPAS_B200_ERR_ARG;
  }
  if (!ctx->have_tree) {
    set_error(ctx, "get_results: nothing evaluated");
    return TAPAS_B200_ERR_STATE;
  }
  PhaseTimer t(ctx, &ctx->timings.download);
  cudaStream_t s = ctx->stream;
  const int64_t n = ctx->n;
  const double *src = ctx->trg.p;
  if (order == TAPAS_B200_ORDER_ORIGINAL) {
    // device output: scattered straight into the caller's buffer
    double *dst = trg4;
    if (mem == TAPAS_B200_HOST) {
      TB_CUDA(ctx, ctx->trg_out.ensure(4 * n, s));
      dst = ctx->trg_out.p;
    }
    scatter_results<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(ctx->trg.p, ctx->idx.p, n,
                                                                         dst);
    TB_LAUNCH_CHECK(ctx);
    if (mem == TAPAS_B200_DEVICE) {
      TB_CUDA(ctx, cudaStreamSynchronize(s));
      return TAPAS_B200_OK;
    }
    src = ctx->trg_out.p;
  }
  TB_CUDA(ctx, cudaMemcpyAsync(trg4, src, 32 * (size_t)n,
                               mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyDeviceToHost,
                               s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  return TAPAS_B200_OK;
}

int tapas_b200_evaluate(tapas_b200_ctx *ctx, const double *x, const double *y, const double *z,
                        const double *q, int64_t n, int P, int ncrit, double theta, int precision,
                        double *trg4, int order, int mem) {
  TB_TRY(tapas_b200_partition(ctx, x, y, z, q, n, ncrit, mem));
  TB_TRY(tapas_b200_upward(ctx, P, precision));
  TB_TRY(tapas_b200_traverse(ctx, theta, 0, precision));
  TB_TRY(tapas_b200_downward(ctx, precision));
  return tapas_b200_get_results(ctx, trg4, order, mem);
}

int tapas_b200_direct(tapas_b200_ctx *ctx, const int64_t *targets, int64_t k, double *out4,
                      int mem) {
  TB_TRY(check_ctx(ctx));
  TB_TRY(check_mem(ctx, mem));
  if (ctx->n <= 0) {
    set_error(ctx, "direct: no bodies");
    return TAPAS_B200_ERR_STATE;
  }
  if (k <= 0 || !targets || !out4 || k > 0x7FFFFFFF) {
    set_error(ctx, "direct: bad target list");
    return TAPAS_B200_ERR_ARG;
  }
  cudaStream_t s = ctx->stream;
  int64_t *dt = nullptr;
  double *dout = nullptr;
  TB_CUDA(ctx, cudaMallocAsync(&dt, sizeof(int64_t) * k, s));
  cudaError_t e = cudaMallocAsync(&dout, sizeof(double) * 4 * k, s);
  if (e != cudaSuccess) {
    cudaFreeAsync(dt, s);
    TB_CUDA(ctx, e);
  }
  int rc = TAPAS_B200_OK;
  const cudaMemcpyKind in_kind =
      mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind out_kind =
      mem == TAPAS_B200_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  std::vector<int64_t> host_check;
  if (mem == TAPAS_B200_HOST) {
    for (int64_t i = 0; i < k; i++)
      if (targets[i] < 0 || targets[i] >= ctx->n) {
        set_error(ctx, "direct: target index %lld out of range", (long long)targets[i]);
        rc = TAPAS_B200_ERR_ARG;
        break;
      }
  }
  if (rc == TAPAS_B200_OK) {
    e = cudaMemcpyAsync(dt, targets, sizeof(int64_t) * k, in_kind, s);
    if (e == cudaSuccess) {
      direct_kernel<<<(unsigned)k, 256, 0, s>>>(ctx->x.p, ctx->y.p, ctx->z.p, ctx->q.p, ctx->n,
                                                dt, dout);
      count_launch(ctx);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out4, dout, sizeof(double) * 4 * k, out_kind, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      set_error(ctx, "direct: %s", cudaGetErrorString(e));
      rc = TAPAS_B200_ERR_CUDA;
    }
  }
  cudaFreeAsync(dt, s);
  cudaFreeAsync(dout, s);
  return rc;
}

}  // extern "C"
