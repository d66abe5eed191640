// Near field (P2P) over the leaf-pair list, replacing the reference's
// vectormap_cuda_pack_kernel2 (cpp/include/tapas/vectormap_cuda.h:219-280)
// with the P2P functor of ex/LaplaceP2PCPU_tapas.h:23-44.
//
// The reference packs target leaves per source leaf and accumulates every
// pair with four CAS-loop atomics on the target attributes.  Here the list is
// grouped by TARGET leaf (CSR), one warp owns a target leaf, each lane keeps
// up to kR targets in registers, source bodies are staged 32 at a time in the
// warp's shared-memory slice and read as broadcasts, and each target's sum is
// written once, without atomics.
//
// FP64 form: the reference's arithmetic (pot += qi qj / r, acc -= qi qj dX/r^3,
// pairs with r == 0 skipped), 1/r via the correctly rounded-to-1-ulp rsqrt.
#include "kernels.cuh"

namespace tb {
namespace {

constexpr int kWarps = 4;
constexpr int kThreads = 32 * kWarps;

template <int kR>
__global__ void __launch_bounds__(kThreads) p2p_fp64_kernel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ off,
    const uint64_t *__restrict__ list, uint64_t src_mask, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ sx, const double *__restrict__ sy,
    const double *__restrict__ sz, const double *__restrict__ sq, double *__restrict__ trg) {
  __shared__ double4 src[kWarps][32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wi;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int tb0 = cbeg[c], nt = cnb[c];
  const int e0 = off[c], e1 = off[c + 1];
  for (int tbase = 0; tbase < nt; tbase += 32 * kR) {
    double xi[kR], yi[kR], zi[kR], qi[kR], pot[kR], ax[kR], ay[kR], az[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) {
      const int i = tbase + lane + 32 * r;
      const bool v = i < nt;
      xi[r] = v ? sx[tb0 + i] : 0.0;
      yi[r] = v ? sy[tb0 + i] : 0.0;
      zi[r] = v ? sz[tb0 + i] : 0.0;
      qi[r] = v ? sq[tb0 + i] : 0.0;
      pot[r] = ax[r] = ay[r] = az[r] = 0.0;
    }
    for (int e = e0; e < e1; e++) {
      const int s = (int)(list[e] & src_mask);
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
      const int i = tbase + lane + 32 * r;
      if (i < nt) {
        double4 *o = reinterpret_cast<double4 *>(trg) + (tb0 + i);
        *o = make_double4(pot[r], ax[r], ay[r], az[r]);
      }
    }
  }
}

}  // namespace

int p2p_fp64(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const int64_t nl = ctx->n_nonempty_leaves;
  if (nl == 0) return TAPAS_B200_OK;
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  const int grid = (int)((nl + kWarps - 1) / kWarps);
  const int R = (ctx->ncrit + 31) / 32;
#define TB_P2P64(RR)                                                                          \
  p2p_fp64_kernel<RR><<<grid, kThreads, 0, s>>>(ctx->leaf_list.p, nl, ctx->p2p_off.p,          \
                                                ctx->p2p.p, mask, ctx->cbeg.p, ctx->cnb.p,     \
                                                ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p,    \
                                                ctx->trg.p)
  if (R <= 1) TB_P2P64(1);
  else if (R <= 2) TB_P2P64(2);
  else if (R <= 3) TB_P2P64(3);
  else TB_P2P64(4);
#undef TB_P2P64
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

// ---------------------------------------------------------------------------
// Mixed form: FP32 arithmetic, compensated accumulation, results per unit
// charge in FP64.
//
// Positions are stored as FP32 offsets from their leaf's centre (computed in
// FP64, rounded once), and a source leaf is brought into the target leaf's
// frame by adding the FP64 centre difference rounded once to FP32, so the
// separation of nearby bodies keeps ~24 bits however far the box is from the
// origin.  Each lane sums one source leaf in plain FP32, then adds that
// partial into a Kahan (sum, compensation) pair.  Targets of a small leaf
// (nt <= 16) are replicated over 32/nt lane groups that split the sources,
// and the groups are combined in FP64 at the end.
// ---------------------------------------------------------------------------
namespace {

constexpr int kStage = 128;  // source bodies staged per warp at a time
constexpr int kMaxR = 4;     // targets per lane (leaves up to 128 bodies per pass)

__global__ void __launch_bounds__(kThreads) prepare_rel4(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, float4 *__restrict__ rel4) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = cbeg[c], nb = cnb[c];
  const double cx = ccen[3 * c], cy = ccen[3 * c + 1], cz = ccen[3 * c + 2];
  for (int b = lane; b < nb; b += 32) {
    const int i = b0 + b;
    rel4[i] = make_float4((float)(sx[i] - cx), (float)(sy[i] - cy), (float)(sz[i] - cz),
                          (float)sq[i]);
  }
}

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  const float y = __fsub_rn(v, comp);
  const float t = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

__global__ void __launch_bounds__(kThreads) p2p_mixed_kernel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ off,
    const uint64_t *__restrict__ list, uint64_t src_mask, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const float4 *__restrict__ rel4, double *__restrict__ trg) {
  __shared__ float4 src[kWarps][kStage];
  __shared__ double4 red[kWarps][32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wi;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int tb0 = cbeg[c], nt_all = cnb[c];
  const int e0 = off[c], e1 = off[c + 1];
  const double tcx = ccen[3 * c], tcy = ccen[3 * c + 1], tcz = ccen[3 * c + 2];
  for (int tbase = 0; tbase < nt_all; tbase += 32 * kMaxR) {
    const int nt = min(nt_all - tbase, 32 * kMaxR);
    // Lane layout: small leaves are replicated over G groups.
    const int G = nt <= 16 ? 32 / nt : 1;
    const int R = nt <= 32 ? 1 : (nt + 31) / 32;
    const int g = nt <= 16 ? lane / nt : 0;
    const bool active = g < G;
    float xi[kMaxR], yi[kMaxR], zi[kMaxR];
    float ps[kMaxR], pc[kMaxR], xs[kMaxR], xc[kMaxR], ys[kMaxR], yc[kMaxR], zs[kMaxR], zc[kMaxR];
#pragma unroll
    for (int r = 0; r < kMaxR; r++) {
      const int t = (nt <= 16 ? lane % nt : lane) + 32 * r;
      const bool v = active && r < R && t < nt;
      const float4 p = v ? rel4[tb0 + tbase + t] : make_float4(0.f, 0.f, 0.f, 0.f);
      xi[r] = p.x; yi[r] = p.y; zi[r] = p.z;
      ps[r] = pc[r] = xs[r] = xc[r] = ys[r] = yc[r] = zs[r] = zc[r] = 0.f;
    }
    for (int e = e0; e < e1; e++) {
      const int s = (int)(list[e] & src_mask);
      const int sb0 = cbeg[s], ns = cnb[s];
      // Source frame -> target frame: FP64 centre difference rounded once.
      const float shx = (float)(ccen[3 * s] - tcx);
      const float shy = (float)(ccen[3 * s + 1] - tcy);
      const float shz = (float)(ccen[3 * s + 2] - tcz);
      for (int chunk = 0; chunk < ns; chunk += kStage) {
        const int cnt = min(kStage, ns - chunk);
        __syncwarp();
        for (int k = lane; k < cnt; k += 32) {
          const float4 b = rel4[sb0 + chunk + k];
          src[wi][k] = make_float4(b.x + shx, b.y + shy, b.z + shz, b.w);
        }
        __syncwarp();
        float tp[kMaxR], tx[kMaxR], ty[kMaxR], tz[kMaxR];
#pragma unroll
        for (int r = 0; r < kMaxR; r++) tp[r] = tx[r] = ty[r] = tz[r] = 0.f;
        for (int k = g; k < cnt; k += G) {
          const float4 b = src[wi][k];
#pragma unroll
          for (int r = 0; r < kMaxR; r++) {
            if (r < R) {
              const float dx = xi[r] - b.x, dy = yi[r] - b.y, dz = zi[r] - b.z;
              const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
              const float ri = r2 > 0.f ? rsqrtf(r2) : 0.f;
              const float qr = b.w * ri;
              const float qr3 = qr * ri * ri;
              tp[r] += qr;
              tx[r] = fmaf(dx, qr3, tx[r]);
              ty[r] = fmaf(dy, qr3, ty[r]);
              tz[r] = fmaf(dz, qr3, tz[r]);
            }
          }
        }
#pragma unroll
        for (int r = 0; r < kMaxR; r++) {
          if (r < R) {
            kahan_add(ps[r], pc[r], tp[r]);
            kahan_add(xs[r], xc[r], tx[r]);
            kahan_add(ys[r], yc[r], ty[r]);
            kahan_add(zs[r], zc[r], tz[r]);
          }
        }
      }
    }
    // Combine (sum - comp) in FP64, then the lane groups.
#pragma unroll
    for (int r = 0; r < kMaxR; r++) {
      if (r >= R) continue;
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
      const int t = (nt <= 16 ? lane % nt : lane) + 32 * r;
      if (active && g == 0 && t < nt)
        reinterpret_cast<double4 *>(trg)[tb0 + tbase + t] = v;
    }
  }
}

}  // namespace

int p2p_mixed(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  const int64_t nl = ctx->n_nonempty_leaves;
  if (nl == 0) return TAPAS_B200_OK;
  const int grid = (int)((nl + kWarps - 1) / kWarps);
  TB_CUDA(ctx, ctx->rel4.ensure(ctx->n, s));
  prepare_rel4<<<grid, kThreads, 0, s>>>(ctx->leaf_list.p, nl, ctx->cbeg.p, ctx->cnb.p,
                                         ctx->ccen.p, ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p,
                                         ctx->rel4.p);
  TB_LAUNCH_CHECK(ctx);
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  p2p_mixed_kernel<<<grid, kThreads, 0, s>>>(ctx->leaf_list.p, nl, ctx->p2p_off.p, ctx->p2p.p,
                                             mask, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p,
                                             ctx->rel4.p, ctx->trg.p);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

}  // namespace tb
