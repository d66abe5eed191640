// Expansion kernels: P2M, M2M, M2L, L2L, L2P (ExaFMM Laplace spherical
// harmonics, ex/LaplaceSphericalCPU_tapas.h), templated on the order P.
//
// Work mapping:
//   P2M  - warp per non-empty leaf; lanes own bodies; 8 coefficients at a time
//          are summed over the warp by one reduce-scatter.
//   M2M  - per level, one FP64 GEMM of the level's precomputed translation
//          operator with the stacked multipoles of the children (below).
//   M2L  - warp per target cell over its CSR list of sources; the harmonics
//          table of each translation is built by P lanes, one Legendre
//          column per lane, into the warp's shared-memory slice.
//   L2L  - per level, one FP64 GEMM as M2M, parents to stacked children.
//   L2P  - warp per non-empty leaf; lane per body, harmonics streamed in
//          registers (no table), L of the leaf staged in shared memory.
// Mixed form only: m2l_pair_kernel (the FP64 M2L of the pairs the tensor cores
// leave, one warp per pair) and l2p32_prep/l2p32_bodies (L2P in FP32, in units
// of the leaf width, one thread per body).
#include "expansions.cuh"
#include "kernels.cuh"
#include "m2l_tc.cuh"

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
    double q = 0, dx = 0, dy = 0, dz = 0;
    if (valid) {
      q = sq[b0 + b];
      dx = sx[b0 + b] - cx;
      dy = sy[b0 + b] - cy;
      dz = sz[b0 + b] - cz;
    }
    // cart2sph (:43-47) then cos/sin of the angles, formed directly
    const Sph sp = sph_of(dx, dy, dz);
    const double rho = sp.r, x = sp.x, y = sp.y;
    const cd ei = sp.ei;
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

// warp_reduce_scatter16 for FP32 values (half the shuffles of the FP64 one).
__device__ __forceinline__ float warp_reduce_scatter16f(float (&buf)[16], int lane) {
#pragma unroll
  for (int o = 16, h = 8; o >= 2; o >>= 1, h >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; i++) {
      const float keep = up ? buf[i + h] : buf[i];
      const float send = up ? buf[i] : buf[i + h];
      buf[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return buf[0] + __shfl_xor_sync(0xffffffffu, buf[0], 1);
}

// P2M of the mixed form: each body's terms in FP32, in units of the leaf width
// w (rho' = rho / w <= ~0.87, so rho'^n stays in range at every n; M_n = w^n
// times the sum), 8 complex terms at a time summed over the warp by one
// FP32 reduce-scatter, the sums over body chunks and the output in FP64.  A
// term's rounding is ~6e-8 of itself and the warp's tree sum adds ~5 such
// roundings, so M's error stays near 1e-7 of the cell's multipoles of |q|
// (measured below 1e-6 of them per cell); where zero-mean charges cancel, that
// is more than 1e-7 of M itself (up to ~2e-5 of it measured), which the final
// potential does not feel (it sums the same terms the cancellation removed).
template <int P>
__global__ void __launch_bounds__(kThreads, 6) p2m32_kernel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ cmin, const double *__restrict__ cmax,
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
  const double width = cmax[3 * c] - cmin[3 * c], iw = 1.0 / width;
  double acc[kGroups];  // lane l: component of slot (l >> 1) & 15 of group g
#pragma unroll
  for (int g = 0; g < kGroups; g++) acc[g] = 0;
  for (int base = 0; base < nb; base += 32) {
    const int b = base + lane;
    float q = 0.f, dx = 0.f, dy = 0.f, dz = 0.f;
    if (b < nb) {
      q = (float)sq[b0 + b];
      dx = (float)((sx[b0 + b] - cx) * iw);
      dy = (float)((sy[b0 + b] - cy) * iw);
      dz = (float)((sz[b0 + b] - cz) * iw);
    }
    // cart2sph (:43-47): rho', cos/sin of alpha and e^{i beta} from the offset
    const float rxy2 = dx * dx + dy * dy;
    const float rho = sqrtf(rxy2 + dz * dz);
    float x = 1.f, y = 0.f, eix = 1.f, eiy = 0.f;
    if (rho > 0.f) {
      const float rxy = sqrtf(rxy2);
      x = dz / rho;
      y = rxy / rho;
      if (rxy > 0.f) {
        eix = dx / rxy;
        eiy = dy / rxy;
      }
    }
    float buf[16];
    int s = 0;
    float fact = 1.f, pn = 1.f, rhom = 1.f;
    float emx = 1.f, emy = 0.f;  // e^{i m beta}
#pragma unroll
    for (int m = 0; m < P; m++) {
      float p = pn, p1 = pn;
      float rhon = rhom;
#pragma unroll
      for (int n = m; n < P; n++) {
        if (n > m) rhon *= 1.f / (float)(-(n + m));  // constants after unrolling
        const float sc = q * rhon * p;
        buf[2 * (s & 7)] = sc * emx;
        buf[2 * (s & 7) + 1] = -sc * emy;
        if ((s & 7) == 7 || s == S::NT - 1) {
#pragma unroll
          for (int i = 2 * (s & 7) + 2; i < 16; i++) buf[i] = 0.f;
          acc[s >> 3] += (double)warp_reduce_scatter16f(buf, lane);
        }
        s++;
        if (n == m) {
          p = x * (float)(2 * m + 1) * p1;
          rhon = rhom * rho;
        } else {
          const float p2 = p1;
          p1 = p;
          p = (x * (float)(2 * n + 1) * p1 - (float)(n + m) * p2) * (1.f / (float)(n - m + 1));
          rhon *= rho;
        }
      }
      rhom = rhom * rho * (1.f / (float)(-(2 * m + 2) * (2 * m + 1)));
      pn = -pn * fact * y;
      fact += 2.f;
      const float ex = emx * eix - emy * eiy;
      emy = emx * eiy + emy * eix;
      emx = ex;
    }
  }
  double *Mc = reinterpret_cast<double *>(M + (int64_t)c * S::NT);
  const int d = (lane >> 1) & 15;
  if ((lane & 1) == 0) {
#pragma unroll
    for (int g = 0; g < kGroups; g++) {
      const int sp = 8 * g + (d >> 1);
      if (sp < S::NT) {
        const int t = p2m_term_index<P>(sp);
        int n, m;
        jk_of(t, n, m);
        double wn = 1.0;
        for (int k = 0; k < n; k++) wn *= width;
        Mc[2 * t + (d & 1)] = acc[g] * wn;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// M2L (:208-273, mutual = 0): L[t] = sum over sources s of T(c_t - c_s) M[s]
// ---------------------------------------------------------------------------
// One source's translation added to lane coefficients (jj[r], kk[r]): the
// source's M in Mj, the local harmonics of the offset in Y.
template <int P>
__device__ __forceinline__ void m2l_accumulate(cd (&acc)[Sizes<P>::R], const int (&jj)[Sizes<P>::R],
                                               const int (&kk)[Sizes<P>::R], int lane,
                                               const cd *Mj, const cd *Y) {
  using S = Sizes<P>;
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

template <int P>
__global__ void __launch_bounds__(kThreads) m2l_kernel(
    int64_t ncells, const int32_t *__restrict__ off, const uint64_t *__restrict__ list,
    uint64_t src_mask, const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double2 *__restrict__ M, double2 *__restrict__ L, const uint8_t *__restrict__ use,
    const uint8_t *__restrict__ own) {
  using S = Sizes<P>;
  __shared__ cd Ysm[kWarps][S::NY];
  __shared__ cd Msm[kWarps][S::NT];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * kWarps + wi;
  if (c >= ncells) return;
  const int e0 = off[c], e1 = off[c + 1];
  if (e1 == e0 || cnb[c] == 0) return;
  if (own && !(own[c] & 1)) return;  // sharded: another context's target
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
    if (use && !use[e]) continue;  // optional pair mask (null: every pair)
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

// The mixed form's FP64 remainder: one warp per listed pair (list index),
// added into L[target] with atomics, so a target with many such pairs does
// not hold one warp alone.
template <int P>
__global__ void __launch_bounds__(kThreads) m2l_pair_kernel(
    const uint32_t *__restrict__ pairs, int64_t npairs, const uint64_t *__restrict__ list,
    int shift, const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double2 *__restrict__ M, double2 *__restrict__ L) {
  using S = Sizes<P>;
  __shared__ cd Ysm[kWarps][S::NY];
  __shared__ cd Msm[kWarps][S::NT];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  cd *Y = Ysm[wi];
  cd *Mj = Msm[wi];
  int jj[S::R], kk[S::R];
#pragma unroll
  for (int r = 0; r < S::R; r++) jk_of(lane + 32 * r, jj[r], kk[r]);
  const uint64_t src_mask = (1ull << shift) - 1;
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  for (int64_t p = (int64_t)blockIdx.x * kWarps + wi; p < npairs; p += nw) {
    const uint64_t x = list[pairs[p]];
    const int c = (int)(x >> shift), s = (int)(x & src_mask);
    if (cnb[s] == 0 || cnb[c] == 0) continue;
    const Sph sp = sph_of(ccen[3 * c] - ccen[3 * s], ccen[3 * c + 1] - ccen[3 * s + 1],
                          ccen[3 * c + 2] - ccen[3 * s + 2]);
    __syncwarp();
    if (lane < P) local_column<P>(lane, sp.r, sp.x, sp.y, sp.ei, Y);
    for (int t = lane; t < S::NT; t += 32) {
      double2 v = M[(int64_t)s * S::NT + t];
      Mj[t] = cd{v.x, v.y};
    }
    __syncwarp();
    cd acc[S::R];
#pragma unroll
    for (int r = 0; r < S::R; r++) acc[r] = cd{0, 0};
    m2l_accumulate<P>(acc, jj, kk, lane, Mj, Y);
    double *Lc = reinterpret_cast<double *>(L + (int64_t)c * S::NT);
#pragma unroll
    for (int r = 0; r < S::R; r++) {
      const int t = lane + 32 * r;
      if (t < S::NT) {
        atomicAdd(Lc + 2 * t, acc[r].x);
        atomicAdd(Lc + 2 * t + 1, acc[r].y);
      }
    }
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

// L2P of the mixed form in FP32: the local expansion's terms fall off
// geometrically inside the leaf, so one FP32 evaluation of them is accurate
// to ~1e-7 of the far-field potential; the result is added into the FP64
// totals.  The evaluation runs in units of the leaf width w (L'_n = L_n w^n,
// r' = r / w: every term L Y_n^m(r) is unchanged, the gradient is scaled by
// 1/w at the end), which keeps every FP32 quantity bounded; L_n itself grows
// like 1/R^(n+1) and leaves the FP32 range at high n in small cells.
//
// One thread per body: a warp per leaf would leave 23% of its lanes idle on a
// surface tree (leaves of ~57 bodies take 2.3 passes of 32), so the leaves are
// prepared first (l2p32_prep: the width-scaled FP32 local expansion and the
// geometry, indexed by the leaf's ordinal, and each of its bodies' ordinal),
// then l2p32_bodies evaluates every body, reading its leaf's coefficients
// through L1 (the lanes of a warp share one to three leaves).
template <int P>
__global__ void __launch_bounds__(256) l2p32_prep(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ cmin, const double *__restrict__ cmax,
    const double2 *__restrict__ L, float2 *__restrict__ Lf, double4 *__restrict__ geo,
    int32_t *__restrict__ body_leaf) {
  using S = Sizes<P>;
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (w >= nleaves) return;
  const int c = leaves[w];
  const double width = cmax[3 * c] - cmin[3 * c];
  for (int t = lane; t < S::NT; t += 32) {
    int n, m;
    jk_of(t, n, m);
    double wn = 1.0;
    for (int k = 0; k < n; k++) wn *= width;
    const double2 v = L[(int64_t)c * S::NT + t];
    Lf[w * S::NT + t] = make_float2((float)(v.x * wn), (float)(v.y * wn));
  }
  if (lane == 0) geo[w] = make_double4(ccen[3 * c], ccen[3 * c + 1], ccen[3 * c + 2], width);
  const int b0 = cbeg[c], nb = cnb[c];
  for (int b = lane; b < nb; b += 32) body_leaf[b0 + b] = (int32_t)w;
}

template <int P>
__global__ void __launch_bounds__(kThreads) l2p32_bodies(
    int64_t n, const int32_t *__restrict__ body_leaf, const double4 *__restrict__ geo,
    const float2 *__restrict__ Lf, const double *__restrict__ sx,
    const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, double *__restrict__ trg, int near_has_q) {
  using S = Sizes<P>;
  for (int64_t bi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; bi < n;
       bi += (int64_t)gridDim.x * blockDim.x) {
    const int w = body_leaf[bi];
    if (w < 0) continue;  // a body another context evaluates
    const double4 g = geo[w];
    const double iw = 1.0 / g.w;
    const float2 *__restrict__ Lc = Lf + (int64_t)w * S::NT;
    const float dx = (float)((sx[bi] - g.x) * iw), dy = (float)((sy[bi] - g.y) * iw),
                dz = (float)((sz[bi] - g.z) * iw);
    const float rxy2 = dx * dx + dy * dy;
    const float r = sqrtf(rxy2 + dz * dz);
    float x = 1.f, y = 0.f, cp = 1.f, sp = 0.f;
    if (r > 0.f) {
      const float rxy = sqrtf(rxy2);
      x = dz / r;
      y = rxy / r;
      if (rxy > 0.f) {
        cp = dx / rxy;
        sp = dy / rxy;
      }
    }
    const float inv_y = 1.f / y, inv_r = 1.f / r;
    float pot = 0, s0 = 0, s1 = 0, s2 = 0;
    float fact = 1, pn = 1, rhom = 1;
    float2 eim = make_float2(1.f, 0.f);
#pragma unroll
    for (int m = 0; m < P; m++) {
      // keeps the compiler from hoisting every column's loads of the
      // coefficients ahead of the loop (register pressure)
      asm volatile("" ::: "memory");
      float p = pn, p1 = pn;
      float rhon = rhom;
      float2 sa = make_float2(0.f, 0.f), sb = sa, sc = sa;
#pragma unroll
      for (int nn = m; nn < P; nn++) {
        float ys, yt;
        const float t1 = x * p1;
        if (nn == m) {
          const float pnew = (float)(2 * m + 1) * t1;
          ys = rhom * p;
          yt = rhom * (pnew - (float)(m + 1) * t1);
          p = pnew;
          rhon = rhom * r;
        } else {
          rhon *= 1.f / (float)(-(nn + m));
          ys = rhon * p;
          const float p2 = p1;
          p1 = p;
          const float tn = x * p1;
          p = ((float)(2 * nn + 1) * tn - (float)(nn + m) * p2) * (1.f / (float)(nn - m + 1));
          yt = rhon * ((float)(nn - m + 1) * p - (float)(nn + 1) * tn);
          rhon *= r;
        }
        const float2 Lv = __ldg(Lc + nn * (nn + 1) / 2 + m);
        sa.x = fmaf(ys, Lv.x, sa.x);
        sa.y = fmaf(ys, Lv.y, sa.y);
        const float nys = (float)nn * ys;
        sb.x = fmaf(nys, Lv.x, sb.x);
        sb.y = fmaf(nys, Lv.y, sb.y);
        sc.x = fmaf(yt, Lv.x, sc.x);
        sc.y = fmaf(yt, Lv.y, sc.y);
      }
      const float f = (m == 0) ? 1.f : 2.f;
      const float zax = sa.x * eim.x - sa.y * eim.y, zay = sa.x * eim.y + sa.y * eim.x;
      pot += f * zax;
      s0 += f * inv_r * (sb.x * eim.x - sb.y * eim.y);
      s1 += f * inv_y * (sc.x * eim.x - sc.y * eim.y);
      if (m > 0) s2 += 2.f * (-zay) * (float)m;
      rhom = rhom * r * (1.f / (float)(-(2 * m + 2) * (2 * m + 1)));
      pn = -pn * fact * y;
      fact += 2.f;
      eim = make_float2(eim.x * cp - eim.y * sp, eim.x * sp + eim.y * cp);
    }
    const float st = y, ct = x;
    const float c0 = st * cp * s0 + ct * cp * inv_r * s1 - sp * inv_r * inv_y * s2;
    const float c1 = st * sp * s0 + ct * sp * inv_r * s1 + cp * inv_r * inv_y * s2;
    const float c2 = ct * s0 - st * inv_r * s1;
    double *o = trg + 4 * bi;
    const double iq = near_has_q ? 1.0 / sq[bi] : 1.0;
    o[0] = o[0] * iq + (double)pot;
    o[1] = o[1] * iq + (double)c0 * iw;
    o[2] = o[2] * iq + (double)c1 * iw;
    o[3] = o[3] * iq + (double)c2 * iw;
  }
}

// ---------------------------------------------------------------------------
// Level-batched M2M and L2L.
//
// Every cell of a level has the same width (the root cube halved per level),
// so a child's offset from its parent is one of eight per level and the
// translation of M2M (:165-206) or L2L (:309-345) is one fixed real-linear
// map per (level, octant), acting on (Re, Im) pairs.  The eight children of
// the non-leaf cells of a level are stored consecutively in parent order, so
//   M2M:  M[parent_i]          = Tup_l (2NT x 16NT) . M[children_i] (16NT)
//   L2L:  L[children_i] (16NT) += Tdn_l (16NT x 2NT) . L[parent_i]
// are one FP64 GEMM per level over the level's non-leaf cells i.  The
// operators are built from one representative parent of the level with the
// reference's formulas, one thread per (target, source) block; M2M rows of degree j read only source degrees <= j
// and L2L rows of degree j only source degrees >= j, and the GEMM skips the
// zero ranges this leaves.
// ---------------------------------------------------------------------------
constexpr int kMaxLevels = kMaxDepth + 1;
struct LevelFirstChild {
  int64_t c0[kMaxLevels];  // first cell of level l + 1 (child 0 of the level's first parent)
};

__host__ __device__ __forceinline__ int degree_of(int t) {
  int j = 0;
  while ((j + 1) * (j + 2) / 2 <= t) j++;
  return j;
}

// The real 2 x 2 block mapping a source coefficient to a target one when
// out = a * src + b * conj(src):
//   [Re out]   [a.x + b.x   b.y - a.y] [Re src]
//   [Im out] = [a.y + b.y   a.x - b.x] [Im src]
// stored transposed (operators are kept K x R, column k of the map
// contiguous): colre / colim point at the target's two rows in the source's
// real / imaginary column.
__device__ __forceinline__ void store_block(double *colre, double *colim, cd a, cd b) {
  *reinterpret_cast<double2 *>(colre) = make_double2(a.x + b.x, a.y + b.y);
  *reinterpret_cast<double2 *>(colim) = make_double2(b.y - a.y, a.x - b.x);
}

// grid (levels with children, 8 octants, 2: M2M / L2L); every entry of the
// operators is written.  Entry (target (j,k), source (j',k')) collects the
// terms of the reference's loops that read that source: M2M (:165-206) with
// n = j - j' and m = k - k' (source as is) or m = k + k' (conjugated); L2L
// (:309-345) with n = j' and m = k' (as is) or m = -k' (conjugated).
template <int P>
__global__ void __launch_bounds__(256) build_translation_ops(
    LevelFirstChild lf, const int32_t *__restrict__ cparent, const double *__restrict__ ccen,
    double *__restrict__ op_up, double *__restrict__ op_dn) {
  using S = Sizes<P>;
  constexpr int NT2 = 2 * S::NT;
  __shared__ cd Y[S::NY];
  const int l = blockIdx.x, o = blockIdx.y;
  const bool up = blockIdx.z == 0;
  const int64_t cj = lf.c0[l] + o;
  const int p = cparent[cj];
  const double dx = ccen[3 * p] - ccen[3 * cj], dy = ccen[3 * p + 1] - ccen[3 * cj + 1],
               dz = ccen[3 * p + 2] - ccen[3 * cj + 2];
  // M2M translates by parent - child, L2L by child - parent
  const Sph sp = up ? sph_of(dx, dy, dz) : sph_of(-dx, -dy, -dz);
  if (threadIdx.x < P) multipole_column<P>(threadIdx.x, sp.r, sp.x, sp.y, sp.ei, Y);
  __syncthreads();
  for (int e = threadIdx.x; e < S::NT * S::NT; e += blockDim.x) {
    const int u = e / S::NT, t = e - u * S::NT;  // consecutive threads: consecutive targets
    int j, k, jp, kp;
    jk_of(t, j, k);
    jk_of(u, jp, kp);
    cd a{0, 0}, b{0, 0};
    if (up) {
      const int n = j - jp;
      if (n >= 0) {
        if (kp >= 1) {
          const int m = k - kp;
          if (m >= -n && m <= n) {
            const double sgn = ((m >= 0) ? 1.0 : oddeven(m)) * oddeven(n);
            a = scal(sgn, Y[n * n + n - m]);
          }
        }
        const int m = k + kp;
        if (m <= n) b = scal(oddeven(k + n + m), Y[n * n + n - m]);
      }
      // K = 16 NT sources (child o's at o * 2NT), R = 2NT targets
      double *c0 = op_up + (size_t)l * NT2 * 8 * NT2 + (size_t)(o * NT2 + 2 * u) * NT2 + 2 * t;
      store_block(c0, c0 + NT2, a, b);
    } else {
      const int n = jp;
      if (n >= j) {
        const int base = (n - j) * (n - j) + n - j - k;
        if (kp >= 1 && kp <= n - j - k) b = scal(oddeven(k), Y[base - kp]);
        if (n - j >= abs(kp - k)) a = scal(oddeven((kp - k) * (kp < k)), Y[base + kp]);
      }
      // K = 2NT sources, R = 16 NT targets (child o's at o * 2NT)
      double *c0 = op_dn + (size_t)l * 8 * NT2 * NT2 + (size_t)(2 * u) * (8 * NT2) + o * NT2 + 2 * t;
      store_block(c0, c0 + 8 * NT2, a, b);
    }
  }
}

// One level's translation GEMM.  Column i is the level's i-th non-leaf cell:
// its children are cells c0 + 8i .. c0 + 8i + 7, its index cparent[c0 + 8i].
struct LevelGemm {
  const double *At; // operator, transposed: K x R, row k = the map's column k
  int R, K, nt2;    // nt2 = 2 NT
  int up;           // 1: M2M (C = A B), 0: L2L (C += A B)
  int split;        // M2M only: blockIdx.z = octant, partial products to `part`
  int64_t c0, ncols;
  const int32_t *cparent;
  double *X;        // M (up) or L (down) as doubles, nt2 per cell
  double *part;     // split: [8][ncols][R]
};

constexpr int kGM = 64, kGN = 64, kGK = 16, kGThreads = 256;  // class_gemm64 tiling
constexpr int kLThreads = 128;     // level_gemm: four warps
constexpr int kLStride = kGM + 4;  // level_gemm shared-memory row stride (doubles)

// One FP64 tensor-core MMA (m8n8k4): d (8 x 8) += a (8 x 4) b (4 x 8).  Lane l
// holds a[l / 4][l % 4], b[l % 4][l / 4] and d[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// 64 x 64 output tile per block of four warps, each warp a 32 x 32 quadrant
// as 4 x 4 FP64 MMAs (m8n8k4) per k-step of 4.  A tiles (operator rows) are
// copied as they lie (k-major), B tiles (one column per source cell) one
// column per thread; rows of both are padded to 68 doubles so that every
// fragment load of a warp is conflict-free.  The next 16-source chunk is
// loaded into registers while the current one is multiplied from shared
// memory (two buffers, one barrier per chunk).  Every output is a fixed-order
// sum, so the result does not depend on the grid.
__global__ void __launch_bounds__(kLThreads, 3) level_gemm(LevelGemm g) {
  __shared__ __align__(16) double As[2][kGK][kLStride];
  __shared__ __align__(16) double Bs[2][kGK][kLStride];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int r0 = blockIdx.y * kGM;
  const int64_t n0 = (int64_t)blockIdx.x * kGN;
  const int wm = 32 * (w & 1), wn = 32 * (w >> 1);  // the warp's quadrant
  const int fr = lane >> 2, fk = lane & 3;            // fragment row / k of this lane
  // A loads: rows r0 + 2 (tid & 31) (+1), sources (tid >> 5) + 4x, x < 4
  const int am = 2 * (tid & 31), ak = tid >> 5;
  const bool arow_ok = r0 + am < g.R;  // R even: the pair is valid together
  // B loads: column tid & 63, sources 8 (tid >> 6) .. +7
  const int bn = tid & 63, bk = 8 * (tid >> 6);
  const int64_t bcol_i = n0 + bn;
  const bool bcol_ok = bcol_i < g.ncols;
  const double *bcol = nullptr;
  if (bcol_ok) {
    const int64_t child0 = g.c0 + 8 * bcol_i;
    const int64_t cell = g.up ? child0 : (int64_t)g.cparent[child0];
    bcol = g.X + cell * g.nt2;
  }
  // source ranges holding the tile's nonzero operator columns
  int seg0, nseg, seg_len, seg_k0;
  if (g.up) {
    const int tmax = (min(r0 + kGM, g.R) - 1) / 2;
    const int jm = degree_of(tmax);
    seg0 = g.split ? (int)blockIdx.z : 0;
    nseg = g.split ? 1 : 8;
    seg_len = min(g.nt2, (jm + 1) * (jm + 2));
    seg_k0 = 0;
  } else {
    const int rs = r0 % g.nt2;
    int kstart = 0;
    if (rs + kGM <= g.nt2) {
      const int j = degree_of(rs / 2);
      kstart = j * (j + 1);
    }
    seg0 = 0;
    nseg = 1;
    seg_k0 = kstart;
    seg_len = g.nt2 - kstart;
  }
  const int cps = (seg_len + kGK - 1) / kGK;  // chunks per segment
  const int nchunks = nseg * cps;
  double2 av[4], bv[4];
  auto load_chunk = [&](int c) {
    const int sg = seg0 + c / cps, kc = (c % cps) * kGK;
    const int kseg = seg_k0 + sg * g.nt2;  // first source of the segment
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int kk = kc + ak + 4 * x;
      av[x] = (kk < seg_len && arow_ok)
                  ? *reinterpret_cast<const double2 *>(g.At + (size_t)(kseg + kk) * g.R + r0 + am)
                  : make_double2(0, 0);
      const int kb = kc + bk + 2 * x;  // even; seg_len is even
      bv[x] = (kb < seg_len && bcol_ok) ? *reinterpret_cast<const double2 *>(bcol + kseg + kb)
                                        : make_double2(0, 0);
    }
  };
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0;
  if (nchunks > 0) load_chunk(0);
  for (int c = 0; c < nchunks; c++) {
    const int buf = c & 1;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      *reinterpret_cast<double2 *>(&As[buf][ak + 4 * x][am]) = av[x];
      Bs[buf][bk + 2 * x][bn] = bv[x].x;
      Bs[buf][bk + 2 * x + 1][bn] = bv[x].y;
    }
    __syncthreads();
    if (c + 1 < nchunks) load_chunk(c + 1);
#pragma unroll
    for (int k0 = 0; k0 < kGK; k0 += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[buf][k0 + fk][wm + 8 * i + fr];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[buf][k0 + fk][wn + 8 * j + fr];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma_m8n8k4(acc[i][j], a[i], b[j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int64_t ci = n0 + wn + 8 * j + 2 * fk + e;
      if (ci >= g.ncols) continue;
      const int64_t child0 = g.c0 + 8 * ci;
      double *ccol;
      if (g.split) ccol = g.part + ((int64_t)blockIdx.z * g.ncols + ci) * g.R;
      else ccol = g.X + (g.up ? (int64_t)g.cparent[child0] : child0) * g.nt2;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int row = r0 + wm + 8 * i + fr;
        if (row >= g.R) continue;
        if (g.up) ccol[row] = acc[i][j][e];
        else ccol[row] += acc[i][j][e];
      }
    }
  }
}

// Split M2M: M[parent_i] = sum over octants o = 0..7, in that order, of part[o][i].
__global__ void sum_octant_parts(const double *__restrict__ part, int64_t ncols, int R,
                                 int64_t c0, const int32_t *__restrict__ cparent, int nt2,
                                 double *__restrict__ X) {
  const int64_t total = ncols * R;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ci = e / R;
    const int row = (int)(e - ci * R);
    double v = 0;
#pragma unroll
    for (int o = 0; o < 8; o++) v += part[(o * ncols + ci) * R + row];
    X[(int64_t)cparent[c0 + 8 * ci] * nt2 + row] = v;
  }
}

// ---------------------------------------------------------------------------
// FP64 M2L batched by offset class (plain form).  With M_n scaled by w^-n and
// L_j by w^(j+1) (w = cell width), the M2L of every pair of one offset class
// (level difference and centre offset in half-widths, m2l_tc.cu) is the same
// real K x K map (K = 2 NT), so a class is one FP64 GEMM:
//     Lt[:, targets] += T_class * Mt[:, sources].
// A target has at most one source per class, and the classes run one launch
// each in key order, so every target's sum has a fixed order (the FP64 form
// stays bit-reproducible) without atomics.
// ---------------------------------------------------------------------------

// One block per class: the map's entries from the unit-offset singular
// harmonics (evalLocal, :102-135), in FP64, stored transposed (row k = the
// map's column k, targets contiguous) like the level operators.  Entry
// (target (j,k), source (n,m)) collects the reference loop's m and -m terms
// (:229-262) times (w_s / w_t)^n = 2^(delta n).
template <int P>
__global__ void __launch_bounds__(256) build_operators64(const uint64_t *__restrict__ keys,
                                                         double *__restrict__ ops) {
  using S = Sizes<P>;
  constexpr int K = 2 * S::NT;
  __shared__ cd Y[S::NY];
  __shared__ double scale[P];
  __shared__ unsigned char deg[S::NT], ord[S::NT];
  const uint64_t key = keys[blockIdx.x];
  const int delta = (int)((key >> 42) & 63) - 32;
  const double Dx = (double)((long long)(key & 16383) - 8192);
  const double Dy = (double)((long long)((key >> 14) & 16383) - 8192);
  const double Dz = (double)((long long)((key >> 28) & 16383) - 8192);
  const double u = ldexp(1.0, min(delta, 0) - 1);  // half-widths -> target widths
  const Sph sp = sph_of(Dx * u, Dy * u, Dz * u);
  if (threadIdx.x < P) {
    local_column<P>(threadIdx.x, sp.r, sp.x, sp.y, sp.ei, Y);
    scale[threadIdx.x] = ldexp(1.0, delta * (int)threadIdx.x);
  }
  for (int t = threadIdx.x; t < S::NT; t += blockDim.x) {
    int j, k;
    jk_of(t, j, k);
    deg[t] = (unsigned char)j;
    ord[t] = (unsigned char)k;
  }
  __syncthreads();
  double *At = ops + (size_t)blockIdx.x * K * K;
  for (int idx = threadIdx.x; idx < S::NT * S::NT; idx += blockDim.x) {
    const int ti = idx / S::NT, to = idx - ti * S::NT;  // consecutive threads: targets
    double v00 = 0, v01 = 0, v10 = 0, v11 = 0;  // [out re/im][in re/im]
    const int j = deg[to], k = ord[to], n = deg[ti], ma = ord[ti];
    if (n < P - j) {
      const double Cnm = oddeven(j);
      const int base = (j + n) * (j + n) + j + n - k;
      const double C2 = Cnm * oddeven((k - ma) * (k < ma) + ma);
      const cd Yp = Y[base + ma];
      v00 = C2 * Yp.x;
      v01 = -C2 * Yp.y;
      v10 = C2 * Yp.y;
      v11 = C2 * Yp.x;
      if (ma > 0) {
        const cd Ym = Y[base - ma];
        v00 += Cnm * Ym.x;
        v01 += Cnm * Ym.y;
        v10 += Cnm * Ym.y;
        v11 += -Cnm * Ym.x;
      }
      const double sc = scale[n];
      v00 *= sc; v01 *= sc; v10 *= sc; v11 *= sc;
    }
    double *c_re = At + (size_t)(2 * ti) * K + 2 * to;
    *reinterpret_cast<double2 *>(c_re) = make_double2(v00, v10);
    *reinterpret_cast<double2 *>(c_re + K) = make_double2(v01, v11);
  }
}

// Per cell (one warp each): Mt[c][2t + re/im] = M[c][t] / w^n, 0 for an empty cell.
template <int P>
__global__ void __launch_bounds__(256) normalize_M64(int64_t ncells, const int32_t *__restrict__ cnb,
                                                     const double *__restrict__ cmin,
                                                     const double *__restrict__ cmax,
                                                     const double2 *__restrict__ M,
                                                     double *__restrict__ Mt) {
  using S = Sizes<P>;
  constexpr int K = 2 * S::NT;
  __shared__ double pw[kWarps][P];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  for (int64_t c = (int64_t)blockIdx.x * kWarps + wi; c < ncells; c += nw) {
    const bool live = cnb[c] > 0;
    __syncwarp();
    if (live && lane < P) pw[wi][lane] = pow(cmax[3 * c] - cmin[3 * c], -lane);
    __syncwarp();
    for (int kk = lane; kk < K; kk += 32) {
      double v = 0;
      if (live) {
        const double2 z = M[c * S::NT + (kk >> 1)];
        v = ((kk & 1) ? z.y : z.x) * pw[wi][degree_of(kk >> 1)];
      }
      Mt[c * K + kk] = v;
    }
  }
}

// Per cell (one warp each): L[c][t] += (sum over the slabs, in slab order,
// of Lt[c][2t, 2t+1]) / w^(j+1).
template <int P>
__global__ void __launch_bounds__(256) add_scaled_L64(int64_t ncells, const int32_t *__restrict__ cnb,
                                                      const double *__restrict__ cmin,
                                                      const double *__restrict__ cmax,
                                                      const double *__restrict__ Lt,
                                                      size_t slab, double2 *__restrict__ L) {
  using S = Sizes<P>;
  constexpr int K = 2 * S::NT;
  __shared__ double pw[kWarps][P + 1];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  for (int64_t c = (int64_t)blockIdx.x * kWarps + wi; c < ncells; c += nw) {
    if (cnb[c] == 0) continue;  // warp-uniform
    __syncwarp();
    if (lane <= P) pw[wi][lane] = pow(cmax[3 * c] - cmin[3 * c], -lane);
    __syncwarp();
    for (int t = lane; t < S::NT; t += 32) {
      const double sc = pw[wi][degree_of(t) + 1];
      double2 lt = *reinterpret_cast<const double2 *>(Lt + c * K + 2 * t);
#pragma unroll
      for (int k = 1; k < kGemmSlabs; k++) {
        const double2 v = *reinterpret_cast<const double2 *>(Lt + k * slab + c * K + 2 * t);
        lt.x += v.x;
        lt.y += v.y;
      }
      const double2 o = L[c * S::NT + t];
      L[c * S::NT + t] = make_double2(o.x + lt.x * sc, o.y + lt.y * sc);
    }
  }
}

// Streams the class GEMMs are spread over (and slabs of partial locals).
int ensure_gemm_streams(tapas_b200_ctx *ctx) {
  if (ctx->gemm_fork) return TAPAS_B200_OK;
  for (int k = 0; k < kGemmSlabs; k++) {
    TB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->gemm_streams[k], cudaStreamNonBlocking));
    TB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->gemm_join[k], cudaEventDisableTiming));
  }
  TB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->gemm_fork, cudaEventDisableTiming));
  return TAPAS_B200_OK;
}

// One class's GEMM: column p of the tile is pair vals[start + p] (source
// multipole row in, target local row updated).  Tiling as level_gemm; a row
// tile whose lowest degree is jmin reads only sources of degree < P - jmin.
struct ClassGemm64 {
  const double *At;      // K x K, row k = the map's column k
  const uint32_t *vals;  // this class's pairs (list indices)
  int len;
  int shift;
  const uint64_t *list;
  const double *Mt;
  double *Lt;
};

template <int P>
__global__ void __launch_bounds__(kGThreads, 3) class_gemm64(ClassGemm64 g) {
  constexpr int K = P * (P + 1);
  __shared__ __align__(16) double As[2][kGK][kGM];
  __shared__ __align__(16) double Bs[2][kGK][kGN];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int r0 = blockIdx.y * kGM;
  const int p0 = blockIdx.x * kGN;
  const int wr = 32 * (w & 1) + 2 * (lane & 7);
  const int tc = 16 * (w >> 1) + 4 * (lane >> 3);
  const int am = 2 * (tid & 31), ak = tid >> 5;
  const bool arow_ok = r0 + am < K;
  const int bn = tid & 63, bk = 4 * (tid >> 6);
  const uint64_t smask = (1ull << g.shift) - 1;
  const bool bcol_ok = p0 + bn < g.len;
  const double *bcol = nullptr;
  if (bcol_ok) bcol = g.Mt + (int64_t)(g.list[g.vals[p0 + bn]] & smask) * K;
  const int jmin = degree_of(r0 / 2);
  const int kmax = min(K, (P - jmin) * (P - jmin + 1));
  const int nchunks = (kmax + kGK - 1) / kGK;
  double2 av[2], bv[2];
  auto load_chunk = [&](int c) {
    const int kc = c * kGK;
#pragma unroll
    for (int x = 0; x < 2; x++) {
      const int kk = kc + ak + 8 * x;
      av[x] = (kk < kmax && arow_ok)
                  ? *reinterpret_cast<const double2 *>(g.At + (size_t)kk * K + r0 + am)
                  : make_double2(0, 0);
      const int kb = kc + bk + 2 * x;  // even; kmax is even
      bv[x] = (kb < kmax && bcol_ok) ? *reinterpret_cast<const double2 *>(bcol + kb)
                                     : make_double2(0, 0);
    }
  };
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0;
  if (nchunks > 0) load_chunk(0);
  for (int c = 0; c < nchunks; c++) {
    const int buf = c & 1;
#pragma unroll
    for (int x = 0; x < 2; x++) {
      *reinterpret_cast<double2 *>(&As[buf][ak + 8 * x][am]) = av[x];
      Bs[buf][bk + 2 * x][bn] = bv[x].x;
      Bs[buf][bk + 2 * x + 1][bn] = bv[x].y;
    }
    __syncthreads();
    if (c + 1 < nchunks) load_chunk(c + 1);
#pragma unroll
    for (int k = 0; k < kGK; k++) {
      const double2 a01 = *reinterpret_cast<const double2 *>(&As[buf][k][wr]);
      const double2 a23 = *reinterpret_cast<const double2 *>(&As[buf][k][wr + 16]);
      const double2 b01 = *reinterpret_cast<const double2 *>(&Bs[buf][k][tc]);
      const double2 b23 = *reinterpret_cast<const double2 *>(&Bs[buf][k][tc + 2]);
      const double a[4] = {a01.x, a01.y, a23.x, a23.y};
      const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int p = p0 + tc + j;
    if (p >= g.len) continue;
    double *lcol = g.Lt + (int64_t)(g.list[g.vals[p]] >> g.shift) * K;
#pragma unroll
    for (int i = 0; i < 4; i += 2) {
      const int row = r0 + wr + 8 * i;  // even; K is even
      if (row >= K) continue;
      double2 *dst = reinterpret_cast<double2 *>(lcol + row);
      const double2 o = *dst;
      *dst = make_double2(o.x + acc[i][j], o.y + acc[i + 1][j]);
    }
  }
}

__global__ void mark_list_entries(const uint32_t *__restrict__ idx, int64_t n,
                                  uint8_t *__restrict__ use) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    use[idx[i]] = 1;
}

// Builds this tree's per-level operators for order P (levels 0 .. nlev-1 have
// children).
template <int P>
int build_level_ops(tapas_b200_ctx *ctx, int &nlev, LevelFirstChild &lf) {
  using S = Sizes<P>;
  cudaStream_t s = ctx->stream;
  nlev = 0;
  for (int l = 0; l + 2 < (int)ctx->level_off.size() && l < kMaxLevels; l++) {
    if (ctx->level_off[l + 2] <= ctx->level_off[l + 1]) break;
    lf.c0[l] = ctx->level_off[l + 1];
    nlev = l + 1;
  }
  if (nlev == 0) return TAPAS_B200_OK;
  const size_t per = (size_t)(2 * S::NT) * (16 * S::NT);  // doubles per level, either op
  TB_CUDA(ctx, ctx->op_m2m.ensure(per * nlev, s));
  TB_CUDA(ctx, ctx->op_l2l.ensure(per * nlev, s));
  build_translation_ops<P><<<dim3(nlev, 8, 2), 256, 0, s>>>(lf, ctx->cparent.p, ctx->ccen.p,
                                                           ctx->op_m2m.p, ctx->op_l2l.p);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

template <int P>
int level_translate(tapas_b200_ctx *ctx, int l, const LevelFirstChild &lf, bool up) {
  using S = Sizes<P>;
  const int64_t ncols = (ctx->level_off[l + 2] - ctx->level_off[l + 1]) / 8;
  if (ncols <= 0) return TAPAS_B200_OK;
  const size_t per = (size_t)(2 * S::NT) * (16 * S::NT);
  LevelGemm g;
  g.At = (up ? ctx->op_m2m.p : ctx->op_l2l.p) + per * l;
  g.R = up ? 2 * S::NT : 16 * S::NT;
  g.K = up ? 16 * S::NT : 2 * S::NT;
  g.nt2 = 2 * S::NT;
  g.up = up ? 1 : 0;
  g.c0 = lf.c0[l];
  g.ncols = ncols;
  g.cparent = ctx->cparent.p;
  g.X = reinterpret_cast<double *>(up ? ctx->M.p : ctx->L.p);
  g.part = nullptr;
  dim3 grid((unsigned)((ncols + kGN - 1) / kGN), (unsigned)((g.R + kGM - 1) / kGM));
  // A level too small to fill the GPU splits M2M's eight octant products
  // over blocks and adds them afterwards in octant order.
  g.split = (up && (int64_t)grid.x * grid.y < 2 * ctx->num_sms) ? 1 : 0;
  if (g.split) {
    TB_CUDA(ctx, ctx->op_part.ensure((size_t)8 * ncols * g.R, ctx->stream));
    g.part = ctx->op_part.p;
    grid.z = 8;
  }
  level_gemm<<<grid, kLThreads, 0, ctx->stream>>>(g);
  TB_LAUNCH_CHECK(ctx);
  if (g.split) {
    sum_octant_parts<<<grid_for(ncols * g.R, 256), 256, 0, ctx->stream>>>(
        g.part, ncols, g.R, g.c0, g.cparent, g.nt2, g.X);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

template <int P>
int p2m_P(tapas_b200_ctx *ctx, bool p2m_f32) {
  using S = Sizes<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->M.ensure((size_t)C * S::NT, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->M.p, 0, sizeof(double2) * (size_t)C * S::NT, s));
  PhaseTimer t(ctx, &ctx->timings.p2m);
  int64_t nl = 0;
  const int32_t *leaves = work_leaves(ctx, nl);  // sharded: owned leaves only
  if (nl > 0 && p2m_f32) {
    p2m32_kernel<P><<<(unsigned)((nl + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        leaves, nl, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p, ctx->cmin.p, ctx->cmax.p, ctx->sx.p,
        ctx->sy.p, ctx->sz.p, ctx->sq.p, ctx->M.p);
    TB_LAUNCH_CHECK(ctx);
  } else if (nl > 0) {
    p2m_kernel<P><<<(unsigned)((nl + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        leaves, nl, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p, ctx->sx.p, ctx->sy.p, ctx->sz.p,
        ctx->sq.p, ctx->M.p);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

template <int P>
int m2m_P(tapas_b200_ctx *ctx) {
  PhaseTimer t(ctx, &ctx->timings.m2m);
  int nlev = 0;
  LevelFirstChild lf;
  TB_TRY(build_level_ops<P>(ctx, nlev, lf));
  ctx->level_ops_P = P;
  for (int lev = nlev - 1; lev >= 0; lev--) TB_TRY(level_translate<P>(ctx, lev, lf, true));
  return TAPAS_B200_OK;
}

// FP64 M2M level GEMMs of the parent levels max_levels - 1 .. 0 only.
template <int P>
int fp64_m2m_levels_P(tapas_b200_ctx *ctx, int max_levels) {
  int nlev = 0;
  LevelFirstChild lf;
  TB_TRY(build_level_ops<P>(ctx, nlev, lf));  // the upward pass builds them for this tree
  ctx->level_ops_P = P;
  for (int lev = std::min(nlev, max_levels) - 1; lev >= 0; lev--)
    TB_TRY(level_translate<P>(ctx, lev, lf, true));
  return TAPAS_B200_OK;
}

template <int P>
int upward_P(tapas_b200_ctx *ctx, bool p2m_f32) {
  TB_TRY(p2m_P<P>(ctx, p2m_f32));
  return m2m_P<P>(ctx);
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
      nullptr, owned_cells(ctx));
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

// The plain form's M2L: classes of >= 32 pairs as FP64 GEMMs, the others by
// the warp-per-target kernel over a pair mask (it writes L[target] first).
template <int P>
int m2l_gemm64_P(tapas_b200_ctx *ctx) {
  using S = Sizes<P>;
  constexpr int K = 2 * S::NT;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  const int64_t n = ctx->n_m2l;
  auto &T = ctx->tc;
  TB_CUDA(ctx, ctx->L.ensure((size_t)C * S::NT, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->L.p, 0, sizeof(double2) * (size_t)C * S::NT, s));
  if (n == 0) return TAPAS_B200_OK;
  M2LClassInfo ci;
  {
    PhaseTimer t(ctx, &ctx->timings.m2l_setup);
    // classes of at least 32 pairs: smaller ones cost more as one GEMM launch
    // each than on the pair kernel
    TB_TRY(m2l_classes(ctx, sizeof(double) * (size_t)K * K, 32, ci));
    if (ci.ntc > 0) {
      TB_CUDA(ctx, T.ops64.ensure((size_t)K * K * ci.ntc, s));
      build_operators64<P><<<(unsigned)ci.ntc, 256, 0, s>>>(T.tc_keys.p, T.ops64.p);
      TB_LAUNCH_CHECK(ctx);
      TB_CUDA(ctx, T.Mt64.ensure((size_t)C * K, s));
      TB_CUDA(ctx, T.Lt64.ensure((size_t)kGemmSlabs * C * K, s));
      normalize_M64<P><<<grid_for(C, kWarps, ctx->num_sms * 8), kThreads, 0, s>>>(
          C, ctx->cnb.p, ctx->cmin.p, ctx->cmax.p, ctx->M.p, T.Mt64.p);
      TB_LAUNCH_CHECK(ctx);
      TB_CUDA(ctx, cudaMemsetAsync(T.Lt64.p, 0, sizeof(double) * kGemmSlabs * (size_t)C * K, s));
    }
  }
  PhaseTimer t(ctx, &ctx->timings.m2l_fp64);
  if (ci.n64 > 0) {
    TB_CUDA(ctx, T.use64.ensure(n + 1, s));
    TB_CUDA(ctx, cudaMemsetAsync(T.use64.p, 0, (size_t)n, s));
    mark_list_entries<<<grid_for(ci.n64, 256), 256, 0, s>>>(T.pairs64.p, ci.n64, T.use64.p);
    TB_LAUNCH_CHECK(ctx);
    const uint64_t mask = (1ull << ctx->list_shift) - 1;
    m2l_kernel<P><<<(unsigned)((C + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        C, ctx->m2l_off.p, ctx->m2l.p, mask, ctx->cnb.p, ctx->ccen.p, ctx->M.p, ctx->L.p,
        T.use64.p, nullptr);
    TB_LAUNCH_CHECK(ctx);
  }
  if (ci.ntc > 0) {
    std::vector<int2> rng((size_t)ci.ntc);
    std::vector<uint64_t> keys((size_t)ci.ntc);
    TB_CUDA(ctx, cudaMemcpyAsync(rng.data(), T.cls_range.p, sizeof(int2) * ci.ntc,
                                 cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaMemcpyAsync(keys.data(), T.tc_keys.p, sizeof(uint64_t) * ci.ntc,
                                 cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    // A class runs on the helper stream of its slab and adds into that slab;
    // the slab is a hash of the class key (not of its position in this list,
    // which a sharded evaluation changes), a slab's classes run in key order
    // (a fixed order per target), the slabs concurrently, and the slabs are
    // added in slab order.
    TB_TRY(ensure_gemm_streams(ctx));
    TB_CUDA(ctx, cudaEventRecord(ctx->gemm_fork, s));
    for (int k = 0; k < kGemmSlabs; k++)
      TB_CUDA(ctx, cudaStreamWaitEvent(ctx->gemm_streams[k], ctx->gemm_fork, 0));
    ClassGemm64 g;
    g.list = ctx->m2l.p;
    g.shift = ctx->list_shift;
    g.Mt = T.Mt64.p;
    for (int64_t c = 0; c < ci.ntc; c++) {  // key order
      uint64_t hsh = keys[c] * 0x9E3779B97F4A7C15ull;
      const int k = (int)((hsh ^ (hsh >> 29)) % kGemmSlabs);
      g.Lt = T.Lt64.p + (size_t)k * C * K;
      g.At = T.ops64.p + (size_t)c * K * K;
      g.vals = T.vals.p + rng[c].x;
      g.len = rng[c].y;
      const dim3 grid((unsigned)((g.len + kGN - 1) / kGN), (unsigned)((K + kGM - 1) / kGM));
      class_gemm64<P><<<grid, kGThreads, 0, ctx->gemm_streams[k]>>>(g);
      TB_LAUNCH_CHECK(ctx);
    }
    for (int k = 0; k < kGemmSlabs; k++) {
      TB_CUDA(ctx, cudaEventRecord(ctx->gemm_join[k], ctx->gemm_streams[k]));
      TB_CUDA(ctx, cudaStreamWaitEvent(s, ctx->gemm_join[k], 0));
    }
    add_scaled_L64<P><<<grid_for(C, kWarps, ctx->num_sms * 8), kThreads, 0, s>>>(
        C, ctx->cnb.p, ctx->cmin.p, ctx->cmax.p, T.Lt64.p, (size_t)C * K, ctx->L.p);
    TB_LAUNCH_CHECK(ctx);
  }
  ctx->tc_classes = ci.ntc;
  return TAPAS_B200_OK;
}

// P < 4: every pair by the warp-per-target kernel.
template <int P>
int m2l_fp64_P(tapas_b200_ctx *ctx) {
  if constexpr (P < 4) return m2l_P<P>(ctx);
  else return m2l_gemm64_P<P>(ctx);
}

template <int P>
int m2l_pairs_P(tapas_b200_ctx *ctx) {
  using S = Sizes<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  TB_CUDA(ctx, ctx->L.ensure((size_t)C * S::NT, s));
  TB_CUDA(ctx, cudaMemsetAsync(ctx->L.p, 0, sizeof(double2) * (size_t)C * S::NT, s));
  PhaseTimer t(ctx, &ctx->timings.m2l_fp64);
  const int64_t np = ctx->m2l_npairs;
  if (np > 0) {
    m2l_pair_kernel<P><<<grid_for(np, kWarps, ctx->num_sms * 16), kThreads, 0, s>>>(
        ctx->m2l_pairs, np, ctx->m2l.p, ctx->list_shift, ctx->cnb.p, ctx->ccen.p, ctx->M.p,
        ctx->L.p);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

template <int P>
int downward_P(tapas_b200_ctx *ctx, bool l2p_f32) {
  cudaStream_t s = ctx->stream;
  {
    PhaseTimer t(ctx, &ctx->timings.l2l);
    int nlev = 0;
    LevelFirstChild lf;
    if (ctx->level_ops_P != P) {  // the operators of the upward pass are reused
      TB_TRY(build_level_ops<P>(ctx, nlev, lf));
      ctx->level_ops_P = P;
    } else {
      for (int l = 0; l + 2 < (int)ctx->level_off.size() && l < kMaxLevels; l++) {
        if (ctx->level_off[l + 2] <= ctx->level_off[l + 1]) break;
        lf.c0[l] = ctx->level_off[l + 1];
        nlev = l + 1;
      }
    }
    for (int lev = 0; lev < nlev; lev++) TB_TRY(level_translate<P>(ctx, lev, lf, false));
  }
  PhaseTimer t(ctx, &ctx->timings.l2p);
  int64_t nl = 0;
  const int32_t *leaves = work_leaves(ctx, nl);  // sharded: owned leaves only
  if (nl > 0 && l2p_f32) {
    TB_CUDA(ctx, ctx->l2p_lf.ensure((size_t)nl * Sizes<P>::NT, s));
    TB_CUDA(ctx, ctx->l2p_geo.ensure((size_t)nl, s));
    TB_CUDA(ctx, ctx->l2p_body_leaf.ensure((size_t)ctx->n, s));
    if (ctx->sharded)  // bodies of other contexts' leaves: -1
      TB_CUDA(ctx, cudaMemsetAsync(ctx->l2p_body_leaf.p, 0xff, sizeof(int32_t) * ctx->n, s));
    l2p32_prep<P><<<(unsigned)((nl + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        leaves, nl, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p, ctx->cmin.p, ctx->cmax.p, ctx->L.p,
        ctx->l2p_lf.p, ctx->l2p_geo.p, ctx->l2p_body_leaf.p);
    TB_LAUNCH_CHECK(ctx);
    l2p32_bodies<P><<<grid_for(ctx->n, kThreads, ctx->num_sms * 8), kThreads, 0, s>>>(
        ctx->n, ctx->l2p_body_leaf.p, ctx->l2p_geo.p, ctx->l2p_lf.p, ctx->sx.p, ctx->sy.p,
        ctx->sz.p, ctx->sq.p, ctx->trg.p, ctx->near_precision == TAPAS_B200_FP64 ? 1 : 0);
    TB_LAUNCH_CHECK(ctx);
  } else if (nl > 0) {
    l2p_kernel<P><<<(unsigned)((nl + kWarps - 1) / kWarps), kThreads, 0, s>>>(
        leaves, nl, ctx->cbeg.p, ctx->cnb.p, ctx->ccen.p, ctx->sx.p, ctx->sy.p,
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

template <int P>
int upward_fp64_P(tapas_b200_ctx *ctx) { return upward_P<P>(ctx, false); }
template <int P>
int upward_f32leaf_P(tapas_b200_ctx *ctx) { return upward_P<P>(ctx, true); }
int upward_fp64(tapas_b200_ctx *ctx, int P) { TB_DISPATCH_P(P, upward_fp64_P) }
int upward_fp32_p2m(tapas_b200_ctx *ctx, int P) { TB_DISPATCH_P(P, upward_f32leaf_P) }
template <int P>
int p2m_fp64_P(tapas_b200_ctx *ctx) { return p2m_P<P>(ctx, false); }
template <int P>
int p2m_f32leaf_P(tapas_b200_ctx *ctx) { return p2m_P<P>(ctx, true); }
int p2m_only(tapas_b200_ctx *ctx, int P, bool fp32) {
  if (fp32) { TB_DISPATCH_P(P, p2m_f32leaf_P) }
  TB_DISPATCH_P(P, p2m_fp64_P)
}
int m2m_only(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, m2m_P) }

int fp64_m2m_levels(tapas_b200_ctx *ctx, int max_levels) {
  switch (ctx->P) {
    case 2: return fp64_m2m_levels_P<2>(ctx, max_levels);
    case 3: return fp64_m2m_levels_P<3>(ctx, max_levels);
    case 4: return fp64_m2m_levels_P<4>(ctx, max_levels);
    case 5: return fp64_m2m_levels_P<5>(ctx, max_levels);
    case 6: return fp64_m2m_levels_P<6>(ctx, max_levels);
    case 7: return fp64_m2m_levels_P<7>(ctx, max_levels);
    case 8: return fp64_m2m_levels_P<8>(ctx, max_levels);
    case 9: return fp64_m2m_levels_P<9>(ctx, max_levels);
    case 10: return fp64_m2m_levels_P<10>(ctx, max_levels);
    case 11: return fp64_m2m_levels_P<11>(ctx, max_levels);
    case 12: return fp64_m2m_levels_P<12>(ctx, max_levels);
    case 13: return fp64_m2m_levels_P<13>(ctx, max_levels);
    case 14: return fp64_m2m_levels_P<14>(ctx, max_levels);
    case 15: return fp64_m2m_levels_P<15>(ctx, max_levels);
    case 16: return fp64_m2m_levels_P<16>(ctx, max_levels);
    default: break;
  }
  set_error(ctx, "expansion order P=%d outside %d..%d", ctx->P, kMinP, kMaxP);
  return TAPAS_B200_ERR_UNSUPPORTED;
}
int m2l_fp64(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, m2l_fp64_P) }

static int m2l_pairs_dispatch(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, m2l_pairs_P) }

int m2l_fp64_pairs(tapas_b200_ctx *ctx, const uint32_t *pairs, int64_t npairs) {
  ctx->m2l_pairs = pairs;
  ctx->m2l_npairs = npairs;
  const int rc = m2l_pairs_dispatch(ctx);
  ctx->m2l_pairs = nullptr;
  ctx->m2l_npairs = 0;
  return rc;
}
template <int P>
int downward_fp64_P(tapas_b200_ctx *ctx) { return downward_P<P>(ctx, false); }
template <int P>
int downward_f32leaf_P(tapas_b200_ctx *ctx) { return downward_P<P>(ctx, true); }
int downward_fp64(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, downward_fp64_P) }
int downward_fp32_l2p(tapas_b200_ctx *ctx) { TB_DISPATCH_P(ctx->P, downward_f32leaf_P) }

}  // namespace tb
