// FP64 expansion kernels: P2M, M2M, M2L, L2L, L2P (ExaFMM Laplace spherical
// harmonics, ex/LaplaceSphericalCPU_tapas.h), templated on the order P.
//
// Work mapping (one warp per cell; the warp's lanes split the expansion
// coefficients, the harmonics table of each translation is built by P lanes,
// one Legendre column per lane, into the warp's shared-memory slice):
//   P2M  - warp per non-empty leaf; lanes own bodies, each (n,m) term is a
//          warp shuffle reduction, lane t%32 keeps coefficient t.
//   M2M  - per level, bottom-up; warp per non-leaf cell, 8 children.
//   M2L  - warp per target cell over its CSR list of sources.
//   L2L  - per level, top-down; warp per non-empty cell.
//   L2P  - warp per non-empty leaf; lane per body, harmonics streamed in
//          registers (no table), L of the leaf staged in shared memory.
// Bound: FP64 pipe (M2L ~ 8 sum_j (j+1)(P-j)^2 flop per translation).
#include "expansions.cuh"
#include "kernels.cuh"

namespace tb {
namespace {

constexpr int kWarps = 4;  // warps per block
constexpr int kThreads = 32 * kWarps;

template <int P>
struct Sizes {
  static constexpr int NT = P * (P + 1) / 2;
  static constexpr int NY = P * P;
  static constexpr int R = (NT + 31) / 32;  // coefficients per lane
};

// ---------------------------------------------------------------------------
// P2M (:138-163): M[n,m] = sum_b q_b * conj(Y_n^m(x_b - center))
// ---------------------------------------------------------------------------
// Coefficient index t = n(n+1)/2 + m of position s in P2M's term order
// (m = 0..P-1, then n = m..P-1).
template <int P>
__device__ __forceinline__ int p2m_term_index(int s) {
  int m = 0;
  while (s >= P - m) {
    s -= P - m;
    m++;
  }
  const int n = m + s;
  return n * (n + 1) / 2 + m;
}

// Sums buf[0..15] of every lane over the warp, leaving lane l (and l ^ 1) with
// the total of buf[(l >> 1) & 15]: four halving exchanges (each lane keeps the
// half its lane bit selects and sends the other), then one pairwise add.
// 16 + 8 + 4 + 2 values are exchanged instead of 16 separate 5-step sums.
__device__ __forceinline__ double warp_reduce_scatter16(double (&buf)[16], int lane) {
#pragma unroll
  for (int o = 16, h = 8; o >= 2; o >>= 1, h >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; i++) {
      const double keep = up ? buf[i + h] : buf[i];
      const double send = up ? buf[i] : buf[i + h];
      buf[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return buf[0] + __shfl_xor_sync(0xffffffffu, buf[0], 1);
}

template <int P>
__global__ void __launch_bounds__(kThreads) p2m_kernel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, double2 *__restrict__ M) {
  using S = Sizes<P>;
  constexpr int kGroups = (S::NT + 7) / 8;  // 8 complex terms per reduction
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = cbeg[c], nb = cnb[c];
  const double cx = ccen[3 * c], cy = ccen[3 * c + 1], cz = ccen[3 * c + 2];
  // acc[g]: this lane's share of group g's sums, component (lane >> 1) & 15
  double acc[kGroups];
#pragma unroll
  for (int g = 0; g < kGroups; g++) acc[g] = 0;
  for (int base = 0; base < nb; base += 32) {
    const int b = base + lane;
    const bool valid = b < nb;
    double q = 0, rho = 1, alpha = 0, beta = 0;
    if (valid) {
      q = sq[b0 + b];
      cart2sph(sx[b0 + b] - cx, sy[b0 + b] - cy, sz[b0 + b] - cz, rho, alpha, beta);
    }
    const double x = cos(alpha), y = sin(alpha);
    double sb, cb;
    sincos(beta, &sb, &cb);
    const cd ei{cb, sb};
    // Streamed evalMultipole (:63-99): this body's q*conj(Y_n^m) terms, 8 at a
    // time, summed over the warp's bodies by one reduce-scatter.
    double buf[16];
    int s = 0;
    double fact = 1, pn = 1, rhom = 1;
    cd eim{1.0, 0.0};
#pragma unroll
    for (int m = 0; m < P; m++) {
      double p = pn, p1 = pn;
      double rhon = rhom;
#pragma unroll
      for (int n = m; n < P; n++) {
        if (n > m) rhon *= 1.0 / -(n + m);  // constants after unrolling
        const double sc = q * rhon * p;
        buf[2 * (s & 7)] = sc * eim.x;
        buf[2 * (s & 7) + 1] = -sc * eim.y;
        if ((s & 7) == 7 || s == S::NT - 1) {
#pragma unroll
          for (int i = 2 * (s & 7) + 2; i < 16; i++) buf[i] = 0;
          acc[s >> 3] += warp_reduce_scatter16(buf, lane);
        }
        s++;
        if (n == m) {
          p = x * (2 * m + 1) * p1;
          rhon = rhom * rho;
        } else {
          const double p2 = p1;
          p1 = p;
          p = (x * (2 * n + 1) * p1 - (n + m) * p2) * (1.0 / (n - m + 1));
          rhon *= rho;
        }
      }
      rhom = rhom * rho * (1.0 / (double)(-(2 * m + 2) * (2 * m + 1)));
      pn = -pn * fact * y;
      fact += 2;
      eim = cmul(eim, ei);
    }
  }
  double *Mc = reinterpret_cast<double *>(M + (int64_t)c * S::NT);
  const int d = (lane >> 1) & 15;
  if ((lane & 1) == 0) {
#pragma unroll
    for (int g = 0; g < kGroups; g++) {
      const int sp = 8 * g + (d >> 1);
      if (sp < S::NT) Mc[2 * p2m_term_index<P>(sp) + (d & 1)] = acc[g];
    }
  }
}

// ---------------------------------------------------------------------------
// M2M (:165-206), one level: M[c] = sum over 8 children of the shifted M.
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(kThreads) m2m_kernel(
    int64_t a, int64_t cnt, const int32_t *__restrict__ cleaf, const int32_t *__restrict__ cnb,
    const int32_t *__restrict__ cchild, const double *__restrict__ ccen, double2 *__restrict__ M) {
  using S = Sizes<P>;
  __shared__ cd Ysm[kWarps][S::NY];
  __shared__ cd Msm[kWarps][S::NT];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wi;
  if (w >= cnt) return;
  const int64_t c = a + w;
  if (cleaf[c] || cnb[c] == 0) return;  // an empty cell's M stays zero
  cd *Y = Ysm[wi];
  cd *Mj = Msm[wi];
  cd acc[S::R];
  int jj[S::R], kk[S::R];
#pragma unroll
  for (int r = 0; r < S::R; r++) {
    acc[r] = cd{0, 0};
    jk_of(lane + 32 * r, jj[r], kk[r]);
  }
  const int ch0 = cchild[c];
  for (int ci = 0; ci < 8; ci++) {
    const int cj = ch0 + ci;
    if (cnb[cj] == 0) continue;  // an empty child's M is zero
    const Sph sp = sph_of(ccen[3 * c] - ccen[3 * cj], ccen[3 * c + 1] - ccen[3 * cj + 1],
                          ccen[3 * c + 2] - ccen[3 * cj + 2]);
    __syncwarp();
    if (lane < P) multipole_column<P>(lane, sp.r, sp.x, sp.y, sp.ei, Y);
    for (int t = lane; t < S::NT; t += 32) {
      double2 v = M[(int64_t)cj * S::NT + t];
      Mj[t] = cd{v.x, v.y};
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < S::R; r++) {
      if (lane + 32 * r >= S::NT) continue;
      const int j = jj[r], k = kk[r];
      cd m_acc{0, 0};
      for (int n = 0; n <= j; n++) {
        const int mlo = max(-n, -j + k + n), mhi = min(k - 1, n);
        for (int m = mlo; m <= mhi; m++) {
          const int jnkms = (j - n) * (j - n + 1) / 2 + k - m;
          const int nm = n * n + n - m;
          const double sgn = ((m >= 0) ? 1.0 : oddeven(m)) * oddeven(n);
          cmac(m_acc, scal(sgn, Mj[jnkms]), Y[nm]);
        }
        const int mhi2 = min(n, j + k - n);
        for (int m = k; m <= mhi2; m++) {
          const int jnkms = (j - n) * (j - n + 1) / 2 - k + m;
          const int nm = n * n + n - m;
          cmac(m_acc, scal(oddeven(k + n + m), conjd(Mj[jnkms])), Y[nm]);
        }
      }
      acc[r].x += m_acc.x;
      acc[r].y += m_acc.y;
    }
  }
#pragma unroll
  for (int r = 0; r < S::R; r++) {
    const int t = lane + 32 * r;
    if (t < S::NT) M[c * S::NT + t] = make_double2(acc[r].x, acc[r].y);
  }
}

// ---------------------------------------------------------------------------
// M2L (:208-273, mutual = 0): L[t] = sum over sources s of T(c_t - c_s) M[s]
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(kThreads) m2l_kernel(
    int64_t ncells, const int32_t *__restrict__ off, const uint64_t *__restrict__ list,
    uint64_t src_mask, const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double2 *__restrict__ M, double2 *__restrict__ L, const uint8_t *__restrict__ use) {
  using S = Sizes<P>;
  __shared__ cd Ysm[kWarps][S::NY];
  __shared__ cd Msm[kWarps][S::NT];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * kWarps + wi;
  if (c >= ncells) return;
  const int e0 = off[c], e1 = off[c + 1];
  if (e1 == e0 || cnb[c] == 0) return;
  cd *Y = Ysm[wi];
  cd *Mj = Msm[wi];
  cd acc[S::R];
  int jj[S::R], kk[S::R];
#pragma unroll
  for (int r = 0; r < S::R; r++) {
    acc[r] = cd{0, 0};
    jk_of(lane + 32 * r, jj[r], kk[r]);
  }
  const double tx = ccen[3 * c], ty = ccen[3 * c + 1], tz = ccen[3 * c + 2];
  for (int e = e0; e < e1; e++) {
    const int s = (int)(list[e] & src_mask);
    if (cnb[s] == 0) continue;  // M of an empty cell is exactly zero
    if (use && !use[e]) continue;  // pair evaluated elsewhere (tensor-core classes)
    const Sph sp = sph_of(tx - ccen[3 * s], ty - ccen[3 * s + 1], tz - ccen[3 * s + 2]);
    __syncwarp();
    if (lane < P) local_column<P>(lane, sp.r, sp.x, sp.y, sp.ei, Y);
    for (int t = lane; t < S::NT; t += 32) {
      double2 v = M[(int64_t)s * S::NT + t];
      Mj[t] = cd{v.x, v.y};
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < S::R; r++) {
      if (lane + 32 * r >= S::NT) continue;
      const int j = jj[r], k = kk[r];
      const double Cnm = oddeven(j);
      for (int n = 0; n < P - j; n++) {
        const int base = (j + n) * (j + n) + j + n - k;
        for (int m = -n; m < 0; m++) {
          const int nms = n * (n + 1) / 2 - m;
          cmac(acc[r], scal(Cnm, conjd(Mj[nms])), Y[base + m]);
        }
        for (int m = 0; m <= n; m++) {
          const int nms = n * (n + 1) / 2 + m;
          const double Cnm2 = Cnm * oddeven((k - m) * (k < m) + m);
          cmac(acc[r], scal(Cnm2, Mj[nms]), Y[base + m]);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < S::R; r++) {
    const int t = lane + 32 * r;
    if (t < S::NT) L[c * S::NT + t] = make_double2(acc[r].x, acc[r].y);
  }
}

// ---------------------------------------------------------------------------
// L2L (:309-345), one level: L[c] += shifted L[parent]
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(kThreads) l2l_kernel(
    int64_t a, int64_t cnt, const int32_t *__restrict__ cnb, const int32_t *__restrict__ cparent,
    const double *__restrict__ ccen, double2 *__restrict__ L) {
  using S = Sizes<P>;
  __shared__ cd Ysm[kWarps][S::NY];
  __shared__ cd Lsm[kWarps][S::NT];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wi;
  if (w >= cnt) return;
  const int64_t c = a + w;
  if (cnb[c] == 0) return;
  const int p = cparent[c];
  cd *Y = Ysm[wi];
  cd *Lp = Lsm[wi];
  const Sph sp = sph_of(ccen[3 * c] - ccen[3 * p], ccen[3 * c + 1] - ccen[3 * p + 1],
                        ccen[3 * c + 2] - ccen[3 * p + 2]);
  if (lane < P) multipole_column<P>(lane, sp.r, sp.x, sp.y, sp.ei, Y);
  for (int t = lane; t < S::NT; t += 32) {
    double2 v = L[(int64_t)p * S::NT + t];
    Lp[t] = cd{v.x, v.y};
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < S::R; r++) {
    const int t = lane + 32 * r;
    if (t >= S::NT) continue;
    int j, k;
    jk_of(t, j, k);
    cd acc{0, 0};
    for (int n = j; n < P; n++) {
      const int base = (n - j) * (n - j) + n - j - k;
      for (int m = j + k - n; m < 0; m++) {
        const int nms = n * (n + 1) / 2 - m;
        cmac(acc, scal(oddeven(k), conjd(Lp[nms])), Y[base + m]);
      }
      for (int m = 0; m <= n; m++) {
        if (n - j >= abs(m - k)) {
          const int nms = n * (n + 1) / 2 + m;
          cmac(acc, scal(oddeven((m - k) * (m < k)), Lp[nms]), Y[base + m]);
        }
      }
    }
    double2 o = L[c * S::NT + t];
    L[c * S::NT + t] = make_double2(o.x + acc.x, o.y + acc.y);
  }
}

// ---------------------------------------------------------------------------
// L2P (:275-307): per body, trg /= q, then add the local expansion's
// potential and gradient (spherical components -> Cartesian, sph2cart :50-60).
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(kThreads) l2p_kernel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, const double2 *__restrict__ L, double *__restrict__ trg,
    int near_has_q) {
  using S = Sizes<P>;
  __shared__ cd Lsm[kWarps][S::NT];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t w = (int64_t)blockIdx.x * kWarps + wi;
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = cbeg[c], nb = cnb[c];
  cd *Lc = Lsm[wi];
  for (int t = lane; t < S::NT; t += 32) {
    double2 v = L[(int64_t)c * S::NT + t];
    Lc[t] = cd{v.x, v.y};
  }
  __syncwarp();
  const double cx = ccen[3 * c], cy = ccen[3 * c + 1], cz = ccen[3 * c + 2];
  for (int b = lane; b < nb; b += 32) {
    const int64_t bi = b0 + b;
    double r, theta, phi;
    cart2sph(sx[bi] - cx, sy[bi] - cy, sz[bi] - cz, r, theta, phi);
    const double x = cos(theta), y = sin(theta);
    const double inv_y = 1.0 / y, inv_r = 1.0 / r;
    double sp, cp;
    sincos(phi, &sp, &cp);
    const cd ei{cp, sp};
    double pot = 0, s0 = 0, s1 = 0, s2 = 0;
    double fact = 1, pn = 1, rhom = 1;
    cd eim{1.0, 0.0};
    // For each m the sums over n are taken before the common factor e^{im phi}:
    //   sa = sum ys L, sb = sum n ys L, sc = sum (yts / inv_y) L,
    // where Y_n^m = ys e^{im phi} and dY_n^m/dtheta = yts e^{im phi}.
#pragma unroll
    for (int m = 0; m < P; m++) {
      double p = pn, p1 = pn;
      double rhon = rhom;
      cd sa{0, 0}, sb{0, 0}, sc{0, 0};
#pragma unroll
      for (int n = m; n < P; n++) {
        double ys, yt;
        const double t1 = x * p1;
        if (n == m) {
          const double pnew = (2 * m + 1) * t1;
          ys = rhom * p;
          yt = rhom * (pnew - (m + 1) * t1);
          p = pnew;
          rhon = rhom * r;
        } else {
          rhon *= 1.0 / -(n + m);  // constants after unrolling
          ys = rhon * p;
          const double p2 = p1;
          p1 = p;
          const double tn = x * p1;
          p = ((2 * n + 1) * tn - (n + m) * p2) * (1.0 / (n - m + 1));
          yt = rhon * ((n - m + 1) * p - (n + 1) * tn);
          rhon *= r;
        }
        const cd Lv = Lc[n * (n + 1) / 2 + m];
        sa.x = fma(ys, Lv.x, sa.x);
        sa.y = fma(ys, Lv.y, sa.y);
        const double nys = n * ys;
        sb.x = fma(nys, Lv.x, sb.x);
        sb.y = fma(nys, Lv.y, sb.y);
        sc.x = fma(yt, Lv.x, sc.x);
        sc.y = fma(yt, Lv.y, sc.y);
      }
      const double f = (m == 0) ? 1.0 : 2.0;
      const cd za = cmul(sa, eim);
      pot += f * za.x;
      s0 += f * inv_r * (sb.x * eim.x - sb.y * eim.y);
      s1 += f * inv_y * (sc.x * eim.x - sc.y * eim.y);
      if (m > 0) s2 += 2 * (-za.y) * m;  // real(L*Y*i) = -imag(L*Y)
      rhom = rhom * r * (1.0 / (double)(-(2 * m + 2) * (2 * m + 1)));
      pn = -pn * fact * y;
      fact += 2;
      eim = cmul(eim, ei);
    }
    double *o = trg + 4 * bi;
    // The FP64 near field holds q_i * sum(q_j / r) (the reference's TRG before
    // its `ba /= b.SRC`); the mixed near field is already per unit charge.
    const double iq = near_has_q ? 1.0 / sq[bi] : 1.0;
    const double st = y, ct = x;
    const double c0 = st * cp * s0 + ct * cp * inv_r * s1 - sp * inv_r * inv_y * s2;
    const double c1 = st * sp * s0 + ct * sp * inv_r * s1 + cp * inv_r * inv_y * s2;
    const double c2 = ct * s0 - st * inv_r * s1;
    o[0] = o[0] * iq + pot;
    o[1] = o[1] * iq + c0;
    o[2] = o[2] * iq + c1;
    o[3] = o[3] * iq + c2;
  }
}

template <int P>
int upward_P(tapas_b200_ctx *ctx) {
  using S = Sizes<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->M.ensure((size_t)C * S::NT, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->M.p, 0, sizeof(double2) * (size_t)C * S::NT, s));
  {
    PhaseTimer t(ctx, &ctx->timings.p2m);
    const int64_t nl = ctx->n_nonempty_leaves;
    if (nl > 0) {
      p2m_kernel<P><<<(unsigned)((nl + kWarps - 1) / kWarps), kThreads, 0, s>>>(
          ctx->leaf_list.p, nl, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p, ctx->sx.p, ctx->sy.p,
          ctx->sz.p, ctx->sq.p, ctx->M.p);
      TB_LAUNCH_CHECK(ctx);
    }
  }
  PhaseTimer t(ctx, &ctx->timings.m2m);
  for (int lev = ctx->max_depth - 1; lev >= 0; lev--) {
    const int64_t a = ctx->level_off[lev], cnt = ctx->level_off[lev + 1] - a;
    if (cnt <= 0) continue;
    m2m_kernel<P><<<(unsigned)((cnt + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        a, cnt, ctx->cleaf.p, ctx->cnb.p, ctx->cchild.p, ctx->ccen.p, ctx->M.p);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

template <int P>
int m2l_P(tapas_b200_ctx *ctx) {
  using S = Sizes<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->L.ensure((size_t)C * S::NT, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->L.p, 0, sizeof(double2) * (size_t)C * S::NT, s));
  PhaseTimer t(ctx, &ctx->timings.m2l_fp64);
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  m2l_kernel<P><<<(unsigned)((C + kWarps - 1) / kWarps), kThreads, 0, s>>>(
      C, ctx->m2l_off.p, ctx->m2l.p, mask, ctx->cnb.p, ctx->ccen.p, ctx->M.p, ctx->L.p,
      ctx->m2l_use);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

template <int P>
int downward_P(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  {
    PhaseTimer t(ctx, &ctx->timings.l2l);
    for (int lev = 1; lev <= ctx->max_depth; lev++) {
      const int64_t a = ctx->level_off[lev], cnt = ctx->level_off[lev + 1] - a;
      if (cnt <= 0) continue;
      l2l_kernel<P><<<(unsigned)((cnt + kWarps - 1) / kWarps), kThreads, 0, s>>>(
          a, cnt, ctx->cnb.p, ctx->cparent.p, ctx->ccen.p, ctx->L.p);
      TB_LAUNCH_CHECK(ctx);
    }
  }
  PhaseTimer t(ctx, &ctx->timings.l2p);
  const int64_t nl = ctx->n_nonempty_leaves;
  if (nl > 0) {
    l2p_kernel<P><<<(unsigned)((nl + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        ctx->leaf_list.p, nl, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p, ctx->sx.p, ctx->sy.p,
        ctx->sz.p, ctx->sq.p, ctx->L.p, ctx->trg.p, ctx->near_precision == TAPAS_B200_FP64 ? 1 : 0);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

}  // namespace

#define TB_DISPATCH_P(P, FN)                                                         \
  switch (P) {                                                                       \
    case 2: return FN<2>(ctx);   case 3: return FN<3>(ctx);   case 4: return FN<4>(ctx);   \
    case 5: return FN<5>(ctx);   case 6: return FN<6>(ctx);   case 7: return FN<7>(ctx);   \
    case 8: return FN<8>(ctx);   case 9: return FN<9>(ctx);   case 10: return FN<10>(ctx); \
    case 11: return FN<11>(ctx); case 12: return FN<12>(ctx); case 13: return FN<13>(ctx); \
    case 14: return FN<14>(ctx); case 15: return FN<15>(ctx); case 16: return FN<16>(ctx); \
    default: break;                                                                  \
  }                                                                                  \
  set_error(ctx, "expansion order P=%d outside %d..%d", (P), kMinP, kMaxP);          \
  return TAPAS_B200_ERR_UNSUPPORTED;

int upward_fp64(tapas_b200_ctx *ctx, int P) { TB_DISPATCH_P(P, upward_P) }
int m2l_fp64(tapas_b200_ctx *ctx) {
  ctx->m2l_use = nullptr;
  TB_DISPATCH_P(ctx->P, m2l_P)
}

static int m2l_fp64_dispatch(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, m2l_P) }

int m2l_fp64_masked(tapas_b200_ctx *ctx, const uint8_t *use) {
  ctx->m2l_use = use;
  const int rc = m2l_fp64_dispatch(ctx);
  ctx->m2l_use = nullptr;
  return rc;
}
int downward_fp64(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, downward_P) }

}  // namespace tb
