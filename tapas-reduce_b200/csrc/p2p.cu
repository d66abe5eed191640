// Near field (P2P) over the leaf-pair list, replacing the reference's
// vectormap_cuda_pack_kernel2 (cpp/include/tapas/vectormap_cuda.h:219-280)
// with the P2P functor of ex/LaplaceP2PCPU_tapas.h:23-44.
//
// The reference packs target leaves per source leaf and accumulates every
// pair with four CAS-loop atomics on the target attributes.  Here the list is
// grouped by TARGET leaf (CSR) and one warp owns a target leaf at a time:
//  - warps take target leaves from a global queue ordered by decreasing work
//    (nt * sum of source bodies), so long interaction lists start first;
//  - each lane keeps kR targets in registers (kR = ceil(nt/32), a template
//    parameter, so no issue slot is spent on unused target slots); leaves of
//    <= 16 bodies are replicated over 32/nt lane groups that split the sources;
//  - source bodies are staged in the warp's shared-memory slice and read as
//    broadcasts; each target's sum is written once, without atomics.
//
// FP64 form: the reference's arithmetic (pot += qi qj / r, acc -= qi qj dX/r^3,
// r == 0 skipped), 1/r from rsqrt (1 ulp).
//
// Mixed form: FP32 arithmetic with results per unit charge.  Positions are
// kept as FP32 (hi, lo) offsets from the body's leaf centre; a source is moved
// into the target leaf's frame with an error-free sum (TwoSum) of its hi part
// and the FP64 centre difference, so the separation x_i - x_j is formed from
// ~47-bit operands and rounds once.  1/r is rsqrtf refined by one Newton step.
// Each source leaf is summed in plain FP32 and the partial is Kahan-added into
// the target's (sum, compensation) pair; the final near field is FP64.
#include <algorithm>

#include "kernels.cuh"
#include "primitives.cuh"

namespace tb {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;
constexpr int kStage = 64;   // source bodies staged per warp at a time
constexpr int kMaxR = 4;     // targets per lane: leaves up to 128 bodies per pass

// ---------------------------------------------------------------------------
// work order: target leaves by decreasing nt * sum(ns)
// ---------------------------------------------------------------------------
__global__ void leaf_work_keys(const int32_t *__restrict__ leaves, int64_t nleaves,
                               const int32_t *__restrict__ off, const uint64_t *__restrict__ list,
                               uint64_t src_mask, const int32_t *__restrict__ cnb,
                               uint64_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nleaves;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int c = leaves[w];
    uint64_t ns = 0;
    for (int e = off[c]; e < off[c + 1]; e++) ns += (uint64_t)cnb[(int)(list[e] & src_mask)];
    uint64_t work = ns * (uint64_t)cnb[c];
    if (work > 0xFFFFFFFFull) work = 0xFFFFFFFFull;
    keys[w] = 0xFFFFFFFFull - work;  // ascending sort -> decreasing work
    vals[w] = (uint32_t)c;
  }
}

__device__ __forceinline__ int next_leaf(int *counter, int lane) {
  int w = 0;
  if (lane == 0) w = atomicAdd(counter, 1);
  return __shfl_sync(0xffffffffu, w, 0);
}

// ---------------------------------------------------------------------------
// FP64
// ---------------------------------------------------------------------------
template <int kR>
__device__ __forceinline__ void fp64_tile(int lane, int wi, int tb0, int nt, int e0, int e1,
                                          const uint64_t *__restrict__ list, uint64_t mask,
                                          const int32_t *__restrict__ cbeg,
                                          const int32_t *__restrict__ cnb,
                                          const double *__restrict__ sx,
                                          const double *__restrict__ sy,
                                          const double *__restrict__ sz,
                                          const double *__restrict__ sq, double4 (*src)[32],
                                          double *__restrict__ trg) {
  double xi[kR], yi[kR], zi[kR], qi[kR], pot[kR], ax[kR], ay[kR], az[kR];
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const int i = lane + 32 * r;
    const bool v = i < nt;
    xi[r] = v ? sx[tb0 + i] : 0.0;
    yi[r] = v ? sy[tb0 + i] : 0.0;
    zi[r] = v ? sz[tb0 + i] : 0.0;
    qi[r] = v ? sq[tb0 + i] : 0.0;
    pot[r] = ax[r] = ay[r] = az[r] = 0.0;
  }
  for (int e = e0; e < e1; e++) {
    const int s = (int)(list[e] & mask);
    const int sb0 = cbeg[s], ns = cnb[s];
    for (int chunk = 0; chunk < ns; chunk += 32) {
      const int cnt = min(32, ns - chunk);
      __syncwarp();
      if (lane < cnt) {
        const int j = sb0 + chunk + lane;
        src[wi][lane] = make_double4(sx[j], sy[j], sz[j], sq[j]);
      }
      __syncwarp();
      for (int k = 0; k < cnt; k++) {
        const double4 b = src[wi][k];
#pragma unroll
        for (int r = 0; r < kR; r++) {
          const double dx = xi[r] - b.x, dy = yi[r] - b.y, dz = zi[r] - b.z;
          const double R2 = dx * dx + dy * dy + dz * dz;
          if (R2 != 0) {
            const double invR = rsqrt(R2);
            const double qq = qi[r] * b.w * invR;
            const double s3 = invR * invR * qq;
            pot[r] += qq;
            ax[r] -= dx * s3;
            ay[r] -= dy * s3;
            az[r] -= dz * s3;
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const int i = lane + 32 * r;
    if (i < nt)
      reinterpret_cast<double4 *>(trg)[tb0 + i] = make_double4(pot[r], ax[r], ay[r], az[r]);
  }
}

__global__ void __launch_bounds__(kThreads) p2p_fp64_kernel(
    const uint32_t *__restrict__ order, int64_t nleaves, int *__restrict__ counter,
    const int32_t *__restrict__ off, const uint64_t *__restrict__ list, uint64_t src_mask,
    const int32_t *__restrict__ cbeg, const int32_t *__restrict__ cnb,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, double *__restrict__ trg) {
  __shared__ double4 src[kWarps][32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    const int w = next_leaf(counter, lane);
    if (w >= nleaves) break;
    const int c = (int)order[w];
    const int tb0 = cbeg[c], nt_all = cnb[c];
    const int e0 = off[c], e1 = off[c + 1];
    for (int tbase = 0; tbase < nt_all; tbase += 32 * kMaxR) {
      const int nt = min(nt_all - tbase, 32 * kMaxR);
      const int R = (nt + 31) / 32;
#define TB_FP64_TILE(RR)                                                                    \
  fp64_tile<RR>(lane, wi, tb0 + tbase, nt, e0, e1, list, src_mask, cbeg, cnb, sx, sy, sz, sq, \
                src, trg)
      if (R == 1) TB_FP64_TILE(1);
      else if (R == 2) TB_FP64_TILE(2);
      else if (R == 3) TB_FP64_TILE(3);
      else TB_FP64_TILE(4);
#undef TB_FP64_TILE
    }
  }
}

// ---------------------------------------------------------------------------
// mixed
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) prepare_rel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, float4 *__restrict__ rel_hi, float4 *__restrict__ rel_lo) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = cbeg[c], nb = cnb[c];
  const double cx = ccen[3 * c], cy = ccen[3 * c + 1], cz = ccen[3 * c + 2];
  for (int b = lane; b < nb; b += 32) {
    const int i = b0 + b;
    const double rx = sx[i] - cx, ry = sy[i] - cy, rz = sz[i] - cz;
    const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
    rel_hi[i] = make_float4(hx, hy, hz, (float)sq[i]);
    rel_lo[i] = make_float4((float)(rx - hx), (float)(ry - hy), (float)(rz - hz), 0.f);
  }
}

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  const float y = __fsub_rn(v, comp);
  const float t = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

// a + b = s + e exactly (Knuth's TwoSum)
__device__ __forceinline__ float two_sum(float a, float b, float &e) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return s;
}

template <int kR>
__device__ __forceinline__ void mixed_tile(
    int lane, int wi, int tb0, int nt, int G, int g, int e0, int e1, double tcx, double tcy,
    double tcz, const uint64_t *__restrict__ list, uint64_t mask, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const float4 *__restrict__ rel_hi, const float4 *__restrict__ rel_lo, float4 (*shi)[kStage],
    float4 (*slo)[kStage], double4 (*red)[32], double *__restrict__ trg) {
  const bool active = g < G;
  const int tl = (G > 1) ? lane % nt : lane;
  float txh[kR], tyh[kR], tzh[kR], txl[kR], tyl[kR], tzl[kR];
  float ps[kR], pc[kR], xs[kR], xc[kR], ys[kR], yc[kR], zs[kR], zc[kR];
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const int t = tl + 32 * r;
    const bool v = active && t < nt;
    const float4 h = v ? rel_hi[tb0 + t] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 l = v ? rel_lo[tb0 + t] : make_float4(0.f, 0.f, 0.f, 0.f);
    txh[r] = h.x; tyh[r] = h.y; tzh[r] = h.z;
    txl[r] = l.x; tyl[r] = l.y; tzl[r] = l.z;
    ps[r] = pc[r] = xs[r] = xc[r] = ys[r] = yc[r] = zs[r] = zc[r] = 0.f;
  }
  for (int e = e0; e < e1; e++) {
    const int s = (int)(list[e] & mask);
    const int sb0 = cbeg[s], ns = cnb[s];
    // source frame -> target frame: FP64 centre difference as (hi, lo) floats
    const double dcx = ccen[3 * s] - tcx, dcy = ccen[3 * s + 1] - tcy,
                 dcz = ccen[3 * s + 2] - tcz;
    const float shx = (float)dcx, shy = (float)dcy, shz = (float)dcz;
    const float slx = (float)(dcx - shx), sly = (float)(dcy - shy), slz = (float)(dcz - shz);
    for (int chunk = 0; chunk < ns; chunk += kStage) {
      const int cnt = min(kStage, ns - chunk);
      __syncwarp();
      for (int k = lane; k < cnt; k += 32) {
        const float4 h = rel_hi[sb0 + chunk + k];
        const float4 l = rel_lo[sb0 + chunk + k];
        float ex, ey, ez;
        const float ax = two_sum(h.x, shx, ex), ay = two_sum(h.y, shy, ey),
                    az = two_sum(h.z, shz, ez);
        shi[wi][k] = make_float4(ax, ay, az, h.w);
        slo[wi][k] = make_float4(ex + (l.x + slx), ey + (l.y + sly), ez + (l.z + slz), 0.f);
      }
      __syncwarp();
      float tp[kR], tx[kR], ty[kR], tz[kR];
#pragma unroll
      for (int r = 0; r < kR; r++) tp[r] = tx[r] = ty[r] = tz[r] = 0.f;
      for (int k = g; k < cnt; k += G) {
        const float4 bh = shi[wi][k];
        const float4 bl = slo[wi][k];
#pragma unroll
        for (int r = 0; r < kR; r++) {
          const float dx = (txh[r] - bh.x) + (txl[r] - bl.x);
          const float dy = (tyh[r] - bh.y) + (tyl[r] - bl.y);
          const float dz = (tzh[r] - bh.z) + (tzl[r] - bl.z);
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          float ri = rsqrtf(r2);
          ri = ri * fmaf(-0.5f * r2, ri * ri, 1.5f);  // one Newton step
          ri = r2 > 0.f ? ri : 0.f;
          const float qr = bh.w * ri;
          const float qr3 = qr * ri * ri;
          tp[r] += qr;
          tx[r] = fmaf(dx, qr3, tx[r]);
          ty[r] = fmaf(dy, qr3, ty[r]);
          tz[r] = fmaf(dz, qr3, tz[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < kR; r++) {
        kahan_add(ps[r], pc[r], tp[r]);
        kahan_add(xs[r], xc[r], tx[r]);
        kahan_add(ys[r], yc[r], ty[r]);
        kahan_add(zs[r], zc[r], tz[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kR; r++) {
    double4 v = make_double4((double)ps[r] - (double)pc[r], -((double)xs[r] - (double)xc[r]),
                             -((double)ys[r] - (double)yc[r]), -((double)zs[r] - (double)zc[r]));
    if (G > 1) {
      __syncwarp();
      red[wi][lane] = v;
      __syncwarp();
      if (g == 0) {
        for (int gg = 1; gg < G; gg++) {
          const double4 o = red[wi][lane + gg * nt];
          v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
        }
      }
    }
    const int t = tl + 32 * r;
    if (active && g == 0 && t < nt) reinterpret_cast<double4 *>(trg)[tb0 + t] = v;
  }
}

__global__ void __launch_bounds__(kThreads) p2p_mixed_kernel(
    const uint32_t *__restrict__ order, int64_t nleaves, int *__restrict__ counter,
    const int32_t *__restrict__ off, const uint64_t *__restrict__ list, uint64_t src_mask,
    const int32_t *__restrict__ cbeg, const int32_t *__restrict__ cnb,
    const double *__restrict__ ccen, const float4 *__restrict__ rel_hi,
    const float4 *__restrict__ rel_lo, double *__restrict__ trg) {
  __shared__ float4 shi[kWarps][kStage];
  __shared__ float4 slo[kWarps][kStage];
  __shared__ double4 red[kWarps][32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    const int w = next_leaf(counter, lane);
    if (w >= nleaves) break;
    const int c = (int)order[w];
    const int tb0 = cbeg[c], nt_all = cnb[c];
    const int e0 = off[c], e1 = off[c + 1];
    const double tcx = ccen[3 * c], tcy = ccen[3 * c + 1], tcz = ccen[3 * c + 2];
    for (int tbase = 0; tbase < nt_all; tbase += 32 * kMaxR) {
      const int nt = min(nt_all - tbase, 32 * kMaxR);
      const int G = nt <= 16 ? 32 / nt : 1;
      const int g = nt <= 16 ? lane / nt : 0;
      const int R = (nt + 31) / 32;
#define TB_MIXED_TILE(RR)                                                                     \
  mixed_tile<RR>(lane, wi, tb0 + tbase, nt, G, g, e0, e1, tcx, tcy, tcz, list, src_mask, cbeg, \
                 cnb, ccen, rel_hi, rel_lo, shi, slo, red, trg)
      if (R == 1) TB_MIXED_TILE(1);
      else if (R == 2) TB_MIXED_TILE(2);
      else if (R == 3) TB_MIXED_TILE(3);
      else TB_MIXED_TILE(4);
#undef TB_MIXED_TILE
    }
  }
}

// Builds ctx->p2p_order (target leaves by decreasing work) for the current lists.
int p2p_order(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const int64_t nl = ctx->n_nonempty_leaves;
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  TB_CUDA(ctx, ctx->p2p_wkey.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_wkey_alt.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_order.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_order_alt.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_counter.ensure(4, s));
  leaf_work_keys<<<grid_for(nl, 256), 256, 0, s>>>(ctx->leaf_list.p, nl, ctx->p2p_off.p,
                                                    ctx->p2p.p, mask, ctx->cnb.p,
                                                    ctx->p2p_wkey.p, ctx->p2p_order.p);
  TB_LAUNCH_CHECK(ctx);
  uint64_t *k = ctx->p2p_wkey.p, *ka = ctx->p2p_wkey_alt.p;
  uint32_t *v = ctx->p2p_order.p, *va = ctx->p2p_order_alt.p;
  TB_TRY(radix_sort(ctx, k, ka, v, va, nl, 0, 32));
  if (v != ctx->p2p_order.p) {
    std::swap(ctx->p2p_order.p, ctx->p2p_order_alt.p);
    std::swap(ctx->p2p_order.cap, ctx->p2p_order_alt.cap);
  }
  if (k != ctx->p2p_wkey.p) {
    std::swap(ctx->p2p_wkey.p, ctx->p2p_wkey_alt.p);
    std::swap(ctx->p2p_wkey.cap, ctx->p2p_wkey_alt.cap);
  }
  TB_CUDA(ctx, cudaMemsetAsync(ctx->p2p_counter.p, 0, sizeof(int), s));
  return TAPAS_B200_OK;
}

int p2p_grid(tapas_b200_ctx *ctx) {
  // persistent: enough warps to fill the GPU, never more than the leaves
  const int64_t nl = ctx->n_nonempty_leaves;
  int64_t g = (int64_t)ctx->num_sms * 8;
  const int64_t need = (nl + kWarps - 1) / kWarps;
  return (int)std::max<int64_t>(1, std::min(g, need));
}

}  // namespace

int p2p_fp64(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const int64_t nl = ctx->n_nonempty_leaves;
  if (nl == 0) return TAPAS_B200_OK;
  TB_TRY(p2p_order(ctx));
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  p2p_fp64_kernel<<<p2p_grid(ctx), kThreads, 0, s>>>(
      ctx->p2p_order.p, nl, ctx->p2p_counter.p, ctx->p2p_off.p, ctx->p2p.p, mask, ctx->cbeg.p,
      ctx->cnb.p, ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p, ctx->trg.p);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

int p2p_mixed(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const int64_t nl = ctx->n_nonempty_leaves;
  if (nl == 0) return TAPAS_B200_OK;
  TB_CUDA(ctx, ctx->rel4.ensure(ctx->n, s));
  TB_CUDA(ctx, ctx->rel_lo.ensure(ctx->n, s));
  prepare_rel<<<(unsigned)((nl + 7) / 8), 256, 0, s>>>(ctx->leaf_list.p, nl, ctx->cbeg.p,
                                                      ctx->cnb.p, ctx->ccen.p, ctx->sx.p,
                                                      ctx->sy.p, ctx->sz.p, ctx->sq.p,
                                                      ctx->rel4.p, ctx->rel_lo.p);
  TB_LAUNCH_CHECK(ctx);
  TB_TRY(p2p_order(ctx));
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  p2p_mixed_kernel<<<p2p_grid(ctx), kThreads, 0, s>>>(
      ctx->p2p_order.p, nl, ctx->p2p_counter.p, ctx->p2p_off.p, ctx->p2p.p, mask, ctx->cbeg.p,
      ctx->cnb.p, ctx->ccen.p, ctx->rel4.p, ctx->rel_lo.p, ctx->trg.p);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

}  // namespace tb
