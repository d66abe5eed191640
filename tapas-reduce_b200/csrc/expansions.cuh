// Spherical-harmonics expansion helpers shared by the FP64 kernels.
//
// Index conventions are the reference's (ex/LaplaceSphericalCPU_tapas.h):
//   Ynm[n*n + n + m], |m| <= n < P       (full table, negative m = conjugate)
//   M[n*(n+1)/2 + m], L[...], 0 <= m <= n (NTERM = P(P+1)/2 complex values)
#pragma once
#include "common.cuh"

namespace tb {

struct cd {  // complex double
  double x, y;
};

__device__ __forceinline__ cd cmul(cd a, cd b) {
  return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__device__ __forceinline__ cd conjd(cd a) { return cd{a.x, -a.y}; }
__device__ __forceinline__ cd scal(double s, cd a) { return cd{s * a.x, s * a.y}; }
__device__ __forceinline__ void cmac(cd &acc, cd a, cd b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
__device__ __forceinline__ double oddeven(int n) { return (n & 1) ? -1.0 : 1.0; }

// 1/i for small integers 0 < i < 64: the recurrences below multiply by these
// instead of dividing (an FP64 division is a long instruction sequence); the
// results differ from exact division by at most an ulp per step.
struct RecipTable {
  double v[64];
  constexpr RecipTable() : v() {
    for (int i = 1; i < 64; i++) v[i] = 1.0 / i;
  }
};
static __constant__ RecipTable kRecip = RecipTable();
__device__ __forceinline__ double recip(int i) { return kRecip.v[i]; }

// cart2sph (ex/LaplaceSphericalCPU_tapas.h:43-47); L2P takes the angles from
// it (measured faster there than the direct form below).
__device__ __forceinline__ void cart2sph(double dx, double dy, double dz, double &r,
                                         double &theta, double &phi) {
  r = sqrt(dx * dx + dy * dy + dz * dz);
  theta = (r == 0) ? 0.0 : acos(dz / r);
  phi = atan2(dy, dx);
}

// What the other expansions need of cart2sph: r, cos(theta),
// sin(theta) and e^{i phi}, formed directly from the offset instead of through
// acos, atan2, cos and sin.  r = 0 gives theta = phi = 0 and an offset along
// the z axis phi = 0, as there.
struct Sph {
  double r, x, y;  // r, cos(theta), sin(theta)
  cd ei;           // e^{i phi}
};
__device__ __forceinline__ Sph sph_of(double dx, double dy, double dz) {
  Sph s;
  const double rxy2 = dx * dx + dy * dy;
  s.r = sqrt(rxy2 + dz * dz);
  s.x = 1.0;
  s.y = 0.0;
  s.ei = cd{1.0, 0.0};
  if (s.r > 0) {
    const double rxy = sqrt(rxy2), ir = 1.0 / s.r;
    s.x = dz * ir;
    s.y = rxy * ir;
    if (rxy > 0) {
      const double irxy = 1.0 / rxy;
      s.ei = cd{dx * irxy, dy * irxy};
    } else if (dz < 0) {
      s.y = 1.2246467991473532e-16;  // sin(acos(-1)) in FP64, as the reference gets it
    }
  }
  return s;
}

// One column m of evalMultipole (:63-99): Ynm for n = m..P-1 written to
// Y[n*n+n+m] and its conjugate to Y[n*n+n-m].  The m-recurrence prefix
// (rho^m/(2m)!, P_m^m, e^{i m beta}) is replayed for this m.
template <int P>
__device__ __forceinline__ void multipole_column(int m, double rho, double x, double y,
                                                 cd ei, cd *Y) {
  double fact = 1, pn = 1, rhom = 1;
  cd eim{1.0, 0.0};
  for (int k = 0; k < m; k++) {
    rhom *= rho;
    rhom *= -recip(2 * k + 2) * recip(2 * k + 1);
    pn = -pn * fact * y;
    fact += 2;
    eim = cmul(eim, ei);
  }
  double p = pn;
  cd v = scal(rhom * p, eim);
  Y[m * m + 2 * m] = v;
  Y[m * m] = conjd(v);
  double p1 = p;
  p = x * (2 * m + 1) * p1;
  double rhon = rhom * rho;
  for (int n = m + 1; n < P; n++) {
    rhon *= -recip(n + m);
    cd w = scal(rhon * p, eim);
    Y[n * n + n + m] = w;
    Y[n * n + n - m] = conjd(w);
    double p2 = p1;
    p1 = p;
    p = (x * (2 * n + 1) * p1 - (n + m) * p2) * recip(n - m + 1);
    rhon *= rho;
  }
}

// One column m of evalLocal (:102-135).
template <int P>
__device__ __forceinline__ void local_column(int m, double rho, double x, double y, cd ei,
                                             cd *Y) {
  const double invR = -1.0 / rho;
  double fact = 1, pn = 1, rhom = -invR;
  cd eim{1.0, 0.0};
  for (int k = 0; k < m; k++) {
    rhom *= invR;
    pn = -pn * fact * y;
    fact += 2;
    eim = cmul(eim, ei);
  }
  double p = pn;
  cd v = scal(rhom * p, eim);
  Y[m * m + 2 * m] = v;
  Y[m * m] = conjd(v);
  double p1 = p;
  p = x * (2 * m + 1) * p1;
  double rhon = rhom * invR;
  for (int n = m + 1; n < P; n++) {
    cd w = scal(rhon * p, eim);
    Y[n * n + n + m] = w;
    Y[n * n + n - m] = conjd(w);
    double p2 = p1;
    p1 = p;
    p = (x * (2 * n + 1) * p1 - (n + m) * p2) * recip(n - m + 1);
    rhon *= invR * (n - m + 1);
  }
}

// (j, k) of coefficient t = j(j+1)/2 + k.
__device__ __forceinline__ void jk_of(int t, int &j, int &k) {
  j = 0;
  while ((j + 1) * (j + 2) / 2 <= t) j++;
  k = t - j * (j + 1) / 2;
}

}  // namespace tb
