// Barnes-Hut path of the reference's sample (sample/barnes-hut/bh.cc) on the
// same octree (tree.cu), body mass in the charge slot.
//
//  bh_upward_level  Approximate (bh.cc:155-190), one launch per level from the
//                   deepest: an empty leaf is zero, a one-body leaf is that
//                   body, a non-leaf the mass and mass-weighted centre of its 8
//                   children summed in index order (leaves with more bodies,
//                   ncrit > 1, use the same formula over their bodies).
//  bh_walk_kernel   interact + ComputeForce (bh.cc:135-153, 192-224): each
//                   body walks the tree depth first from the root, children
//                   visited 0..7 like the sample's recursion; a warp's 32
//                   bodies (consecutive in Morton order) share one bounded
//                   stack of the union of their walks (below).  A cell is
//                   accepted when width / |centre - body| < theta; a leaf is
//                   summed body by body (the body itself included, as in the
//                   sample).
// The FP64 form uses separately rounded operations in the sample's order, so
// it reproduces the sample bit for bit; the FP32 form ("mixed") walks with FP32
// positions and FP32 copies of the FP64 cell moments.
#include "common.cuh"

namespace tb {
namespace {

constexpr int kStack = 192;  // > 7 pending siblings x 19 levels + 1

__global__ void bh_upward_level(int64_t a, int64_t cnt, const int32_t *__restrict__ cleaf,
                                const int32_t *__restrict__ cnb, const int32_t *__restrict__ cbeg,
                                const int32_t *__restrict__ cchild, const double *__restrict__ sx,
                                const double *__restrict__ sy, const double *__restrict__ sz,
                                const double *__restrict__ sm, double4 *__restrict__ attr) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < cnt;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = a + w;
    double4 r;
    if (cleaf[c]) {
      const int nb = cnb[c], b0 = cbeg[c];
      if (nb == 0) {
        r = make_double4(0, 0, 0, 0);
      } else if (nb == 1) {
        r = make_double4(sx[b0], sy[b0], sz[b0], sm[b0]);
      } else {
        double W = 0, X = 0, Y = 0, Z = 0;
        for (int i = 0; i < nb; i++) {
          const int b = b0 + i;
          W = __dadd_rn(W, sm[b]);
          X = __dadd_rn(X, __dmul_rn(sx[b], sm[b]));
          Y = __dadd_rn(Y, __dmul_rn(sy[b], sm[b]));
          Z = __dadd_rn(Z, __dmul_rn(sz[b], sm[b]));
        }
        r = make_double4(__ddiv_rn(X, W), __ddiv_rn(Y, W), __ddiv_rn(Z, W), W);
      }
    } else {
      double W = 0, X = 0, Y = 0, Z = 0;
      const int ch = cchild[c];
      for (int i = 0; i < 8; i++) {
        const double4 s = attr[ch + i];
        W = __dadd_rn(W, s.w);
        X = __dadd_rn(X, __dmul_rn(s.x, s.w));
        Y = __dadd_rn(Y, __dmul_rn(s.y, s.w));
        Z = __dadd_rn(Z, __dmul_rn(s.z, s.w));
      }
      r = make_double4(__ddiv_rn(X, W), __ddiv_rn(Y, W), __ddiv_rn(Z, W), W);
    }
    attr[c] = r;
  }
}

// ComputeForce (bh.cc:135-153), FP64, the sample's rounding order.
__device__ __forceinline__ void force64(double px, double py, double pz, double ax, double ay,
                                        double az, double aw, double eps2, double4 &o) {
  const double dx = __dsub_rn(ax, px), dy = __dsub_rn(ay, py), dz = __dsub_rn(az, pz);
  double R2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
  R2 = __dadd_rn(__dadd_rn(R2, __dmul_rn(dz, dz)), eps2);
  const double invR = __ddiv_rn(1.0, __dsqrt_rn(R2));
  const double invR3 = __dmul_rn(__dmul_rn(invR, invR), invR);
  o.x = __dadd_rn(o.x, __dmul_rn(__dmul_rn(dx, invR3), aw));
  o.y = __dadd_rn(o.y, __dmul_rn(__dmul_rn(dy, invR3), aw));
  o.z = __dadd_rn(o.z, __dmul_rn(__dmul_rn(dz, invR3), aw));
  o.w = __dadd_rn(o.w, __dmul_rn(invR, aw));
}

__device__ __forceinline__ void force32(float px, float py, float pz, float ax, float ay, float az,
                                        float aw, float eps2, float4 &o) {
  const float dx = ax - px, dy = ay - py, dz = az - pz;
  const float R2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  const float invR = rsqrtf(R2);
  const float wr = aw * invR;
  const float wr3 = wr * invR * invR;
  o.x = fmaf(dx, wr3, o.x);
  o.y = fmaf(dy, wr3, o.y);
  o.z = fmaf(dz, wr3, o.z);
  o.w += wr;
}

struct BhTree {
  const int32_t *leaf, *nb, *beg, *child;
  const double *cmin, *cmax, *ccen;
};

// One walk per warp over the union of its 32 bodies' walks.  The warp keeps
// one stack of (cell, lanes that reach it); at each popped cell the lanes in
// its mask do what their own walk does there (sum a leaf, accept the cell, or
// open it), and the cell's children are pushed for the lanes that opened it.
// Every lane's walk is a depth-first walk with children 0..7 of a subtree of
// the union's, so a lane meets its cells in its own order, takes the sample's
// decisions and sums its interactions in the sample's order; the warp reads
// each cell and each leaf body once for all its lanes, and the bodies, in
// Morton order, share most of their walks.
constexpr int kWalkWarps = 4;
template <bool kFp64>
__global__ void __launch_bounds__(32 * kWalkWarps) bh_walk_kernel(
    BhTree T, int64_t n, const double *__restrict__ sx, const double *__restrict__ sy,
    const double *__restrict__ sz, const double *__restrict__ sm, const double4 *__restrict__ attr,
    const float4 *__restrict__ attr32, const float4 *__restrict__ pos32, double theta,
    double eps2, double *__restrict__ out, unsigned long long *__restrict__ counters) {
  __shared__ int scell[kWalkWarps][kStack];
  __shared__ unsigned smask[kWalkWarps][kStack];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const double theta2 = __dmul_rn(theta, theta);
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = b < n;
  unsigned long long napprox = 0, ndirect = 0, overflow = 0;
  const double px = valid ? sx[b] : 0.0, py = valid ? sy[b] : 0.0, pz = valid ? sz[b] : 0.0;
  double4 o64 = make_double4(0, 0, 0, 0);
  float4 o32 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 p32 = (kFp64 || !valid) ? make_float4(0.f, 0.f, 0.f, 0.f) : pos32[b];
  const unsigned lanes = __ballot_sync(0xffffffffu, valid);
  int sp = 0;  // the same in every lane
  if (lanes) {
    if (lane == 0) {
      scell[wi][0] = 0;
      smask[wi][0] = lanes;
    }
    sp = 1;
    __syncwarp();
  }
  while (sp > 0) {
    --sp;
    const int c = scell[wi][sp];
    const unsigned m = smask[wi][sp];
    __syncwarp();  // read before a push reuses the slot
    const bool mine = (m >> lane) & 1u;
    if (T.leaf[c]) {
      if (mine) {
        const int nb = T.nb[c], b0 = T.beg[c];
        for (int i = 0; i < nb; i++) {
          const int j = b0 + i;
          if (kFp64) force64(px, py, pz, sx[j], sy[j], sz[j], sm[j], eps2, o64);
          else {
            const float4 q = pos32[j];
            force32(p32.x, p32.y, p32.z, q.x, q.y, q.z, q.w, (float)eps2, o32);
          }
        }
        ndirect += (unsigned)nb;
      }
      continue;
    }
    bool open = false;
    if (mine) {
      // the sample's MAC: cell width / |centre - body| < theta
      const double dx = __dsub_rn(px, T.ccen[3 * c]), dy = __dsub_rn(py, T.ccen[3 * c + 1]),
                   dz = __dsub_rn(pz, T.ccen[3 * c + 2]);
      double R = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
      R = __dadd_rn(R, __dmul_rn(dz, dz));
      const double s = __dsub_rn(T.cmax[3 * c], T.cmin[3 * c]);
      // The sample evaluates fl(s / fl(sqrt(R))) < theta.  That value is
      // s/sqrt(R) within ~2.3 ulp, and s^2 against theta^2 R below within
      // ~4 ulp, so outside a relative band of 1e-13 around theta^2 R the
      // squared test decides the same way without the square root and the
      // division; inside it the sample's own operations decide.
      const double s2 = __dmul_rn(s, s), t2R = __dmul_rn(theta2, R);
      bool accept;
      if (s2 < __dmul_rn(t2R, 1.0 - 1e-13)) accept = true;
      else if (s2 > __dmul_rn(t2R, 1.0 + 1e-13)) accept = false;
      else accept = __ddiv_rn(s, __dsqrt_rn(R)) < theta;
      if (accept) {
        if (kFp64) {
          const double4 a = attr[c];
          force64(px, py, pz, a.x, a.y, a.z, a.w, eps2, o64);
        } else {
          const float4 a = attr32[c];
          force32(p32.x, p32.y, p32.z, a.x, a.y, a.z, a.w, (float)eps2, o32);
        }
        napprox++;
      } else {
        open = true;
      }
    }
    const unsigned om = __ballot_sync(0xffffffffu, open);
    if (om) {
      if (sp + 8 > kStack) {
        if (mine) overflow = 1;
        break;
      }
      // children 7..0 from the bottom up, so child 0 is popped first
      if (lane < 8) {
        scell[wi][sp + lane] = T.child[c] + 7 - lane;
        smask[wi][sp + lane] = om;
      }
      sp += 8;
      __syncwarp();
    }
  }
  if (valid) {
    double4 *o = reinterpret_cast<double4 *>(out) + b;
    *o = kFp64 ? o64 : make_double4((double)o32.x, (double)o32.y, (double)o32.z, (double)o32.w);
  }
  for (int s = 16; s > 0; s >>= 1) {
    napprox += __shfl_down_sync(0xffffffffu, napprox, s);
    ndirect += __shfl_down_sync(0xffffffffu, ndirect, s);
    overflow |= __shfl_down_sync(0xffffffffu, overflow, s);
  }
  if (lane == 0) {
    if (napprox) atomicAdd(counters + 0, napprox);
    if (ndirect) atomicAdd(counters + 1, ndirect);
    if (overflow) atomicOr(counters + 2, 1ull);
  }
}

__global__ void bh_to_fp32(int64_t ncells, const double4 *__restrict__ attr,
                           float4 *__restrict__ attr32, int64_t n, const double *__restrict__ sx,
                           const double *__restrict__ sy, const double *__restrict__ sz,
                           const double *__restrict__ sm, float4 *__restrict__ pos32) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncells + n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i < ncells) {
      const double4 a = attr[i];
      attr32[i] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
    } else {
      const int64_t b = i - ncells;
      pos32[b] = make_float4((float)sx[b], (float)sy[b], (float)sz[b], (float)sm[b]);
    }
  }
}

}  // namespace

int bh_upward(tapas_b200_ctx *ctx) {
  if (!ctx->have_tree) {
    set_error(ctx, "bh_upward: no tree (call partition first)");
    return TAPAS_B200_ERR_STATE;
  }
  cudaStream_t s = ctx->stream;
  TB_CUDA(ctx, ctx->bh_attr.ensure(ctx->ncells + 1, s));
  PhaseTimer t(ctx, &ctx->timings.upward);
  for (int lev = (int)ctx->level_off.size() - 2; lev >= 0; lev--) {
    const int64_t a = ctx->level_off[lev], cnt = ctx->level_off[lev + 1] - a;
    if (cnt <= 0) continue;
    bh_upward_level<<<grid_for(cnt, 256), 256, 0, s>>>(
        a, cnt, ctx->cleaf.p, ctx->cnb.p, ctx->cbeg.p, ctx->cchild.p, ctx->sx.p, ctx->sy.p,
        ctx->sz.p, ctx->sq.p, ctx->bh_attr.p);
    TB_LAUNCH_CHECK(ctx);
  }
  ctx->have_bh_attr = true;
  return TAPAS_B200_OK;
}

int bh_interact(tapas_b200_ctx *ctx, double theta, double eps2, int precision) {
  if (!ctx->have_bh_attr) {
    set_error(ctx, "bh_interact: call bh_upward first");
    return TAPAS_B200_ERR_STATE;
  }
  if (!(theta > 0) || !(eps2 >= 0)) {
    set_error(ctx, "bh_interact: need theta > 0 and eps2 >= 0");
    return TAPAS_B200_ERR_ARG;
  }
  cudaStream_t s = ctx->stream;
  const int64_t n = ctx->n, C = ctx->ncells;
  TB_CUDA(ctx, ctx->counters.ensure(8, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->counters.p, 0, 8 * sizeof(unsigned long long), s));
  BhTree T{ctx->cleaf.p, ctx->cnb.p, ctx->cbeg.p, ctx->cchild.p, ctx->cmin.p, ctx->cmax.p,
           ctx->ccen.p};
  PhaseTimer t(ctx, &ctx->timings.p2p);
  const int grid = (int)((n + 32 * kWalkWarps - 1) / (32 * kWalkWarps));
  if (precision == TAPAS_B200_FP64) {
    bh_walk_kernel<true><<<grid, 32 * kWalkWarps, 0, s>>>(T, n, ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p,
                                              ctx->bh_attr.p, nullptr, nullptr, theta, eps2,
                                              ctx->trg.p, ctx->counters.p);
  } else {
    TB_CUDA(ctx, ctx->bh_attr32.ensure(C + 1, s));
    TB_CUDA(ctx, ctx->rel4.ensure(n, s));
    bh_to_fp32<<<grid_for(C + n, 256), 256, 0, s>>>(C, ctx->bh_attr.p, ctx->bh_attr32.p, n,
                                                     ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p,
                                                     ctx->rel4.p);
    TB_LAUNCH_CHECK(ctx);
    bh_walk_kernel<false><<<grid, 32 * kWalkWarps, 0, s>>>(T, n, ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p,
                                               ctx->bh_attr.p, ctx->bh_attr32.p, ctx->rel4.p,
                                               theta, eps2, ctx->trg.p, ctx->counters.p);
  }
  TB_LAUNCH_CHECK(ctx);
  unsigned long long *h = reinterpret_cast<unsigned long long *>(ctx->pinned.p);
  TB_CUDA(ctx, ctx->pinned.ensure(256));
  h = reinterpret_cast<unsigned long long *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemcpyAsync(h, ctx->counters.p, 3 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->bh_napprox = h[0];
  ctx->bh_ndirect = h[1];
  if (h[2]) {
    set_error(ctx, "bh_interact: a walk exceeded its stack bound");
    return TAPAS_B200_ERR_CAPACITY;
  }
  return TAPAS_B200_OK;
}

}  // namespace tb
