/*
 * CPU restatement of the reference Tapas/ExaFMM N-body evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see
 * fmm_oracle.h.  Parity pin: tests/test_oracle_golden.py compares this file's
 * output bit for bit with golden vectors that the unmodified reference, built
 * in oracle/_ref, produced (tests/golden/make_golden.py), and
 * tests/test_oracle_keys.py replays cpp/tests/test_morton_key.cpp.
 *
 * Build for x86-64 without FMA contraction (-ffp-contract=off, no -march):
 * that is how the reference itself is compiled, and the bit-level pins on
 * keys, cells and interaction lists depend on it.
 *
 * Reference files cited below are relative to the reference project root;
 * "ex/" abbreviates sample/exafmm-dev-13274dd4ac68/examples/.
 */
#include "fmm_oracle.h"

#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef double complex cplx;

/* ---------------------------------------------------------------------------
 * Morton keys: cpp/include/tapas/sfc_morton.h (Dim=3, uint64 keys).
 * Layout: bits 61..5 hold 19 levels of 3 bits (z,y,x from high to low within a
 * level), bits 4..0 hold the depth (DepthBits()=5, MaxDepth()=19, :154-182).
 * ------------------------------------------------------------------------- */
enum { KMAXD = 19, KDBITS = 5 };

static inline int kdepth(uint64_t k) { return (int)(k & 31u); }
static inline uint64_t kappend(uint64_t k, int d) { return (k << KDBITS) | (uint64_t)d; }
static inline uint64_t kremove(uint64_t k) { return k >> KDBITS; }

/* GetNext, sfc_morton.h:192-206 */
uint64_t oracle_key_next(uint64_t k, int n) {
  int d = kdepth(k);
  return k + ((uint64_t)n << (3 * (KMAXD - d) + KDBITS));
}
/* Child, sfc_morton.h:288-295 (IncrementDepth then OR the child digit) */
uint64_t oracle_key_child(uint64_t k, int idx) {
  k = kappend(kremove(k), kdepth(k) + 1);
  int d = kdepth(k);
  return k | ((uint64_t)idx << ((KMAXD - d) * 3 + KDBITS));
}
/* Parent, sfc_morton.h:258-271 */
uint64_t oracle_key_parent(uint64_t k) {
  int d = kdepth(k);
  if (d == 0) return k;
  k = kappend(kremove(k), d - 1);
  d = kdepth(k);
  uint64_t m = ~((((uint64_t)1 << ((KMAXD - d) * 3)) - 1) << KDBITS);
  return k & m;
}
/* IsDescendant, sfc_morton.h:248-256 */
int oracle_key_is_descendant(uint64_t asc, uint64_t dsc) {
  int depth = kdepth(asc);
  if (depth >= kdepth(dsc)) return 0;
  int s = (KMAXD - depth) * 3 + KDBITS;
  return (asc >> s) == (dsc >> s);
}
/* Includes(beg, end, c), sfc_morton.h:468-477 */
int oracle_key_includes_range(uint64_t beg, uint64_t end, uint64_t c) {
  uint64_t b = kremove(beg), e = kremove(end);
  uint64_t c1 = kremove(c), c2 = kremove(oracle_key_next(c, 1));
  return (b <= c1) && (c2 <= e);
}
/* Overlapped, sfc_morton.h:426-462 */
int oracle_key_overlapped(uint64_t x1, uint64_t x2, uint64_t y1, uint64_t y2) {
  uint64_t X1 = kremove(x1), X2 = kremove(x2), Y1 = kremove(y1), Y2 = kremove(y2);
  if (X1 <= Y1 && Y1 < X2) return 1;
  if (X1 < Y2 && Y2 <= X2) return 1;
  if (Y1 < X1 && X2 <= Y2) return 1;
  return 0;
}
/* GetDirOnDepth, sfc_morton.h:519-527 (the shifted key is truncated to int) */
int oracle_key_dir_on_depth(uint64_t k, int dim, int depth) {
  int dir = (int)(kremove(k) >> ((KMAXD - depth) * 3));
  return (dir >> dim) & 1;
}
/* GetMSBits, sfc_morton.h:240-243 */
uint64_t oracle_key_msbits(uint64_t k, int bits) { return k >> (KDBITS + 3 * KMAXD - bits); }

/* CalcFinestKey, sfc_morton.h:387-402: per level, z then y then x bit. */
uint64_t oracle_key_finest(int ax, int ay, int az) {
  int a[3] = {ax, ay, az};
  uint64_t k = 0;
  int mask = 1 << (KMAXD - 1);
  for (int i = 0; i < KMAXD; ++i) {
    for (int d = 2; d >= 0; --d) k = (k << 1) | (uint64_t)((a[d] & mask) >> (KMAXD - i - 1));
    mask >>= 1;
  }
  return kappend(k, KMAXD);
}

/* CalcRegion, sfc_morton.h:536-557: halve the root box once per level. */
void oracle_key_region(uint64_t k, const double rmin[3], const double rmax[3], double mn[3],
                       double mx[3]) {
  int depth = kdepth(k);
  for (int d = 0; d < 3; d++) { mx[d] = rmax[d]; mn[d] = rmin[d]; }
  for (int dep = 1; dep <= depth; dep++) {
    for (int dim = 0; dim < 3; dim++) {
      double c = (mx[dim] + mn[dim]) / 2;
      if (oracle_key_dir_on_depth(k, dim, dep) == 1) mn[dim] = c; else mx[dim] = c;
    }
  }
}

/* ---------------------------------------------------------------------------
 * State.
 * ------------------------------------------------------------------------- */
typedef struct {
  uint64_t key;
  int32_t leaf, depth;
  int64_t nb, bbeg;      /* body range [bbeg, bbeg+nb) in sorted order */
  int32_t parent, child0; /* children occupy 8 consecutive slots? no: see child[] */
  int32_t child[8];
  double mn[3], mx[3], center[3];
} ocell;

struct oracle_fmm {
  int64_t n;
  int P, nterm, ncrit;
  double theta;
  int mutual;                     /* the example's -m option (0 or 1) */
  uint8_t *own;                   /* sharded evaluation: per cell bit 0 = local
                                     expansion computed here, bit 1 = bodies; NULL = all */
  double *x, *y, *z, *q;          /* original order */
  double *sx, *sy, *sz, *sq;      /* sorted order */
  int64_t *perm;                  /* sorted position -> original index */
  uint64_t *skeys;
  double *trg;                    /* 4 per body, sorted order */
  double lo, hi;                  /* cube bbox [lo,hi]^3 */
  ocell *cells;
  int64_t ncells, cap;
  int max_depth;
  cplx *M, *L;                    /* ncells x nterm */
  int32_t *m2l_t, *m2l_s; int64_t nm2l, cm2l;
  int32_t *p2p_t, *p2p_s; int64_t np2p, cp2p;
  uint64_t np2p_int;
  cplx *ynm, *ynmt;               /* P*P scratch */
};

#define ODDEVEN(n) ((((n) & 1) == 1) ? -1 : 1)
#define IPOW2N(n) (((n) >= 0) ? 1 : ODDEVEN(n))

oracle_fmm *oracle_create(int64_t n, const double *x, const double *y, const double *z,
                          const double *q, int P, int ncrit, double theta) {
  if (n < 0 || P < 2 || ncrit < 1) return NULL;
  oracle_fmm *h = (oracle_fmm *)calloc(1, sizeof(oracle_fmm));
  h->n = n; h->P = P; h->nterm = P * (P + 1) / 2; h->ncrit = ncrit; h->theta = theta;
  size_t nb = (size_t)(n > 0 ? n : 1) * sizeof(double);
  h->x = malloc(nb); h->y = malloc(nb); h->z = malloc(nb); h->q = malloc(nb);
  if (n > 0) {
    memcpy(h->x, x, (size_t)n * 8); memcpy(h->y, y, (size_t)n * 8);
    memcpy(h->z, z, (size_t)n * 8); memcpy(h->q, q, (size_t)n * 8);
  }
  h->ynm = malloc(sizeof(cplx) * P * P);
  h->ynmt = malloc(sizeof(cplx) * P * P);
  return h;
}

void oracle_destroy(oracle_fmm *h) {
  if (!h) return;
  free(h->x); free(h->y); free(h->z); free(h->q);
  free(h->sx); free(h->sy); free(h->sz); free(h->sq);
  free(h->perm); free(h->skeys); free(h->trg); free(h->cells);
  free(h->M); free(h->L); free(h->m2l_t); free(h->m2l_s); free(h->p2p_t); free(h->p2p_s);
  free(h->ynm); free(h->ynmt); free(h->own);
  free(h);
}

/* ---------------------------------------------------------------------------
 * Tree build: hot/buildtree.h.
 * ------------------------------------------------------------------------- */

/* Bounding box, buildtree.h:72-87.  The reference assigns a scalar to a
 * Vec (implicit broadcast constructor, vec.h:39-43) so the box is the cube
 * [lo,hi]^3 with lo/hi the extremes over every coordinate of bodies 1..n-1
 * and the z coordinate of body 0 (std::max(a,b) = a<b ? b : a). */
static void bbox(oracle_fmm *h) {
  double lo = 0, hi = 0;
  for (int64_t i = 0; i < h->n; i++) {
    double p[3] = {h->x[i], h->y[i], h->z[i]};
    for (int d = 0; d < 3; d++) {
      if (i == 0) { hi = p[d]; lo = p[d]; }
      else {
        hi = (p[d] < hi) ? hi : p[d];
        lo = (lo < p[d]) ? lo : p[d];
      }
    }
  }
  h->lo = lo; h->hi = hi;
}

/* x86-64 cvttsd2si semantics for the reference's (int) cast of a double:
 * truncation when in range, INT_MIN otherwise (NaN and overflow). */
static inline int to_int_x86(double v) {
  if (v > -2147483649.0 && v < 2147483648.0) return (int)v;
  return (int)0x80000000u;
}

/* BodiesToKeys, buildtree.h:505-539. */
static uint64_t body_key(double lo, double hi, double px, double py, double pz) {
  const int nfc = 1 << KMAXD;
  double pitch = (hi - lo) / (double)nfc; /* identical in all 3 dims */
  double p[3] = {px, py, pz};
  int a[3];
  for (int d = 0; d < 3; d++) {
    double o = p[d] - lo;
    o = o / pitch;
    a[d] = to_int_x86(o);
    if (a[d] == nfc) a[d]--;
  }
  return oracle_key_finest(a[0], a[1], a[2]);
}

typedef struct { uint64_t k; int64_t i; } kidx;
static int cmp_kidx(const void *a, const void *b) {
  const kidx *x = a, *y = b;
  if (x->k < y->k) return -1;
  if (x->k > y->k) return 1;
  /* The reference sorts with a non-stable std::sort (common.h:249-273), so
   * the order of equal keys is unspecified; ties are broken by original
   * index here and parity is defined on keys and body sets per cell. */
  return (x->i < y->i) ? -1 : (x->i > y->i);
}

static int64_t lower_bound_u64(const uint64_t *a, int64_t lo, int64_t hi, uint64_t v) {
  while (lo < hi) {
    int64_t mid = lo + (hi - lo) / 2;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

static int32_t new_cell(oracle_fmm *h) {
  if (h->ncells == h->cap) {
    h->cap = h->cap ? 2 * h->cap : 1024;
    h->cells = realloc(h->cells, sizeof(ocell) * (size_t)h->cap);
  }
  memset(&h->cells[h->ncells], 0, sizeof(ocell));
  return (int32_t)h->ncells++;
}

/* GenerateCell, buildtree.h:388-459, on one rank (every cell is inside the
 * rank's key range, so "included" and "overlap" are always true).  A cell is a
 * leaf iff nb <= ncrit; a non-leaf always gets all 8 children, empty or not.
 * Cells at the maximum depth (19) are leaves whatever their count: the
 * reference has no defined behaviour there (its child key shift goes
 * negative), and only coincident bodies reach it. */
static int32_t gen_cell(oracle_fmm *h, uint64_t k, int64_t pbeg, int64_t pend, int32_t parent,
                        const double pmn[3], const double pmx[3], int childidx) {
  uint64_t k2 = oracle_key_next(k, 1);
  int64_t rb = lower_bound_u64(h->skeys, pbeg, pend, k);
  int64_t re = lower_bound_u64(h->skeys, pbeg, pend, k2);
  int64_t nb = re - rb;
  int depth = kdepth(k);
  int32_t ci = new_cell(h);
  ocell *c = &h->cells[ci];
  c->key = k;
  c->depth = depth;
  c->nb = nb;
  c->bbeg = rb;
  c->parent = parent;
  c->leaf = (nb <= h->ncrit) || depth >= KMAXD;
  for (int i = 0; i < 8; i++) c->child[i] = -1;
  /* Region: the parent's box halved once (same arithmetic as CalcRegion). */
  if (parent < 0) {
    for (int d = 0; d < 3; d++) { c->mn[d] = h->lo; c->mx[d] = h->hi; }
  } else {
    for (int d = 0; d < 3; d++) {
      double mid = (pmx[d] + pmn[d]) / 2;
      if ((childidx >> d) & 1) { c->mn[d] = mid; c->mx[d] = pmx[d]; }
      else { c->mn[d] = pmn[d]; c->mx[d] = mid; }
    }
  }
  for (int d = 0; d < 3; d++) c->center[d] = (c->mx[d] + c->mn[d]) / 2;
  if (depth > h->max_depth) h->max_depth = depth;
  if (!c->leaf) {
    double mn[3], mx[3];
    memcpy(mn, c->mn, sizeof mn);
    memcpy(mx, c->mx, sizeof mx);
    for (int i = 0; i < 8; i++) {
      int32_t ch = gen_cell(h, oracle_key_child(k, i), rb, re, ci, mn, mx, i);
      h->cells[ci].child[i] = ch;
    }
  }
  h->cells[ci].child0 = h->cells[ci].child[0];
  return ci;
}

int oracle_build(oracle_fmm *h) {
  int64_t n = h->n;
  if (n <= 0) return -1;
  bbox(h);
  kidx *ki = malloc(sizeof(kidx) * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    ki[i].k = body_key(h->lo, h->hi, h->x[i], h->y[i], h->z[i]);
    ki[i].i = i;
  }
  qsort(ki, (size_t)n, sizeof(kidx), cmp_kidx);
  size_t nb = (size_t)n * 8;
  h->perm = malloc((size_t)n * sizeof(int64_t));
  h->skeys = malloc((size_t)n * sizeof(uint64_t));
  h->sx = malloc(nb); h->sy = malloc(nb); h->sz = malloc(nb); h->sq = malloc(nb);
  for (int64_t s = 0; s < n; s++) {
    int64_t i = ki[s].i;
    h->perm[s] = i; h->skeys[s] = ki[s].k;
    h->sx[s] = h->x[i]; h->sy[s] = h->y[i]; h->sz[s] = h->z[i]; h->sq[s] = h->q[i];
  }
  free(ki);
  h->trg = calloc((size_t)n * 4, sizeof(double));
  h->ncells = 0; h->max_depth = 0;
  double dummy[3] = {0, 0, 0};
  gen_cell(h, 0, 0, n, -1, dummy, dummy, 0);
  h->M = calloc((size_t)h->ncells * h->nterm, sizeof(cplx));
  h->L = calloc((size_t)h->ncells * h->nterm, sizeof(cplx));
  return 0;
}

/* ---------------------------------------------------------------------------
 * Expansion kernels: ex/LaplaceSphericalCPU_tapas.h.
 * ------------------------------------------------------------------------- */

/* cart2sph, :43-47 (norm = ((0 + x^2) + y^2) + z^2, exafmm include/vec.h:166-170) */
static void cart2sph(double *r, double *theta, double *phi, const double dX[3]) {
  double s = 0;
  s += dX[0] * dX[0];
  s += dX[1] * dX[1];
  s += dX[2] * dX[2];
  *r = sqrt(s);
  *theta = (*r == 0) ? 0 : acos(dX[2] / *r);
  *phi = atan2(dX[1], dX[0]);
}

/* evalMultipole, :63-99 */
static void eval_multipole(int P, double rho, double alpha, double beta, cplx *Ynm, cplx *YnmTheta) {
  double x = cos(alpha);
  double y = sin(alpha);
  double fact = 1;
  double pn = 1;
  double rhom = 1;
  cplx ei = cexp(I * beta);
  cplx eim = 1.0;
  for (int m = 0; m < P; m++) {
    double p = pn;
    int npn = m * m + 2 * m;
    int nmn = m * m;
    Ynm[npn] = rhom * p * eim;
    Ynm[nmn] = conj(Ynm[npn]);
    double p1 = p;
    p = x * (2 * m + 1) * p1;
    YnmTheta[npn] = rhom * (p - (m + 1) * x * p1) / y * eim;
    rhom *= rho;
    double rhon = rhom;
    for (int n = m + 1; n < P; n++) {
      int npm = n * n + n + m;
      int nmm = n * n + n - m;
      rhon /= -(n + m);
      Ynm[npm] = rhon * p * eim;
      Ynm[nmm] = conj(Ynm[npm]);
      double p2 = p1;
      p1 = p;
      p = (x * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      YnmTheta[npm] = rhon * ((n - m + 1) * p - (n + 1) * x * p1) / y * eim;
      rhon *= rho;
    }
    rhom /= -(2 * m + 2) * (2 * m + 1);
    pn = -pn * fact * y;
    fact += 2;
    eim *= ei;
  }
}

/* evalLocal, :102-135 */
static void eval_local(int P, double rho, double alpha, double beta, cplx *Ynm) {
  double x = cos(alpha);
  double y = sin(alpha);
  double fact = 1;
  double pn = 1;
  double invR = -1.0 / rho;
  double rhom = -invR;
  cplx ei = cexp(I * beta);
  cplx eim = 1.0;
  for (int m = 0; m < P; m++) {
    double p = pn;
    int npn = m * m + 2 * m;
    int nmn = m * m;
    Ynm[npn] = rhom * p * eim;
    Ynm[nmn] = conj(Ynm[npn]);
    double p1 = p;
    p = x * (2 * m + 1) * p1;
    rhom *= invR;
    double rhon = rhom;
    for (int n = m + 1; n < P; n++) {
      int npm = n * n + n + m;
      int nmm = n * n + n - m;
      Ynm[npm] = rhon * p * eim;
      Ynm[nmm] = conj(Ynm[npm]);
      double p2 = p1;
      p1 = p;
      p = (x * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      rhon *= invR * (n - m + 1);
    }
    pn = -pn * fact * y;
    fact += 2;
    eim *= ei;
  }
}

/* P2M, :138-163 */
static void p2m(oracle_fmm *h, int32_t ci) {
  const ocell *c = &h->cells[ci];
  int P = h->P;
  cplx *M = h->M + (size_t)ci * h->nterm;
  for (int64_t i = 0; i < c->nb; i++) {
    int64_t b = c->bbeg + i;
    double dX[3] = {h->sx[b] - c->center[0], h->sy[b] - c->center[1], h->sz[b] - c->center[2]};
    double rho, alpha, beta;
    cart2sph(&rho, &alpha, &beta, dX);
    eval_multipole(P, rho, alpha, beta, h->ynm, h->ynmt);
    for (int n = 0; n < P; n++)
      for (int m = 0; m <= n; m++) {
        int nm = n * n + n - m;
        int nms = n * (n + 1) / 2 + m;
        M[nms] += h->sq[b] * h->ynm[nm];
      }
  }
}

/* M2M, :165-206 (all 8 children, empty ones included) */
static void m2m(oracle_fmm *h, int32_t ci) {
  const ocell *c = &h->cells[ci];
  int P = h->P;
  cplx *M = h->M + (size_t)ci * h->nterm;
  for (int i = 0; i < 8; i++) {
    int32_t cj = c->child[i];
    const ocell *C = &h->cells[cj];
    const cplx *Mj = h->M + (size_t)cj * h->nterm;
    double dX[3] = {c->center[0] - C->center[0], c->center[1] - C->center[1],
                    c->center[2] - C->center[2]};
    double rho, alpha, beta;
    cart2sph(&rho, &alpha, &beta, dX);
    eval_multipole(P, rho, alpha, beta, h->ynm, h->ynmt);
    for (int j = 0; j < P; j++) {
      for (int k = 0; k <= j; k++) {
        int jks = j * (j + 1) / 2 + k;
        cplx acc = 0;
        for (int n = 0; n <= j; n++) {
          int mlo = (-n > -j + k + n) ? -n : -j + k + n;
          int mhi = (k - 1 < n) ? k - 1 : n;
          for (int m = mlo; m <= mhi; m++) {
            int jnkms = (j - n) * (j - n + 1) / 2 + k - m;
            int nm = n * n + n - m;
            acc += Mj[jnkms] * h->ynm[nm] * (double)(IPOW2N(m) * ODDEVEN(n));
          }
          int mhi2 = (n < j + k - n) ? n : j + k - n;
          for (int m = k; m <= mhi2; m++) {
            int jnkms = (j - n) * (j - n + 1) / 2 - k + m;
            int nm = n * n + n - m;
            acc += conj(Mj[jnkms]) * h->ynm[nm] * (double)(ODDEVEN(k + n + m));
          }
        }
        M[jks] += acc;
      }
    }
  }
}

/* FMM_Upward, ex/tapas_exafmm.cxx:87-122 (children first, in index order). */
static void upward_rec(oracle_fmm *h, int32_t ci) {
  if (h->cells[ci].leaf) {
    p2m(h, ci);
  } else {
    for (int i = 0; i < 8; i++) upward_rec(h, h->cells[ci].child[i]);
    m2m(h, ci);
  }
}

int oracle_upward(oracle_fmm *h) {
  if (!h->cells) return -1;
  memset(h->M, 0, sizeof(cplx) * (size_t)h->ncells * h->nterm);
  memset(h->L, 0, sizeof(cplx) * (size_t)h->ncells * h->nterm);
  upward_rec(h, 0);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Sharded evaluation, restated for the CPU test of the multi-GPU driver
 * (tapas-reduce_b200/sharded.py): an ownership mask (bit 0: the cell's local
 * expansion is computed here, bit 1: its bodies are), the upward pass in two
 * halves with the multipoles exchanged between them, and M2L / P2P / L2L /
 * L2P restricted to owned targets.  P2M and M2M are per-cell functions of
 * their inputs, so the halves reproduce oracle_upward exactly.
 * ------------------------------------------------------------------------- */
void oracle_set_owned(oracle_fmm *h, const uint8_t *mask) {
  free(h->own);
  h->own = NULL;
  if (mask) {
    h->own = malloc((size_t)h->ncells);
    memcpy(h->own, mask, (size_t)h->ncells);
  }
}

static void m2m_rec(oracle_fmm *h, int32_t ci) {
  if (h->cells[ci].leaf) return;
  for (int i = 0; i < 8; i++) m2m_rec(h, h->cells[ci].child[i]);
  m2m(h, ci);
}

int oracle_p2m_only(oracle_fmm *h) {
  if (!h->cells) return -1;
  memset(h->M, 0, sizeof(cplx) * (size_t)h->ncells * h->nterm);
  memset(h->L, 0, sizeof(cplx) * (size_t)h->ncells * h->nterm);
  for (int64_t c = 0; c < h->ncells; c++)
    if (h->cells[c].leaf && (!h->own || (h->own[c] & 2))) p2m(h, (int32_t)c);
  return 0;
}

int oracle_m2m_only(oracle_fmm *h) {
  if (!h->cells) return -1;
  m2m_rec(h, 0);
  return 0;
}

void oracle_set_theta(oracle_fmm *h, double theta) { h->theta = theta; }

void oracle_set_multipoles(oracle_fmm *h, const double *M) {
  memcpy(h->M, M, sizeof(cplx) * (size_t)h->ncells * h->nterm);
}

/* M2L, :208-273.  With mutual the same call also translates Ci's multipole
 * into Cj's local expansion, from the harmonics at (rho, alpha + pi, beta)
 * (:222-223), accumulated in the same loop (:244-263). */
static void m2l(oracle_fmm *h, int32_t ti, int32_t si) {
  const ocell *Ci = &h->cells[ti], *Cj = &h->cells[si];
  int P = h->P;
  const int mutual = h->mutual;
  cplx *Li = h->L + (size_t)ti * h->nterm;
  cplx *Lj = h->L + (size_t)si * h->nterm;
  const cplx *Mi = h->M + (size_t)ti * h->nterm;
  const cplx *Mj = h->M + (size_t)si * h->nterm;
  double dX[3] = {Ci->center[0] - Cj->center[0], Ci->center[1] - Cj->center[1],
                  Ci->center[2] - Cj->center[2]};
  double rho, alpha, beta;
  cart2sph(&rho, &alpha, &beta, dX);
  eval_local(P, rho, alpha, beta, h->ynm);
  if (mutual) eval_local(P, rho, alpha + M_PI, beta, h->ynmt);
  for (int j = 0; j < P; j++) {
    double Cnm = ODDEVEN(j);
    for (int k = 0; k <= j; k++) {
      int jks = j * (j + 1) / 2 + k;
      cplx acc = 0, accj = 0;
      for (int n = 0; n < P - j; n++) {
        for (int m = -n; m < 0; m++) {
          int nms = n * (n + 1) / 2 - m;
          int jnkm = (j + n) * (j + n) + j + n + m - k;
          acc += conj(Mj[nms]) * Cnm * h->ynm[jnkm];
          if (mutual) accj += conj(Mi[nms]) * Cnm * h->ynmt[jnkm];
        }
        for (int m = 0; m <= n; m++) {
          int nms = n * (n + 1) / 2 + m;
          int jnkm = (j + n) * (j + n) + j + n + m - k;
          double Cnm2 = Cnm * ODDEVEN((k - m) * (k < m) + m);
          acc += Mj[nms] * Cnm2 * h->ynm[jnkm];
          if (mutual) accj += Mi[nms] * Cnm2 * h->ynmt[jnkm];
        }
      }
      Li[jks] += acc;
      if (mutual) Lj[jks] += accj;
    }
  }
}

/* P2P functor (CPU form), ex/LaplaceP2PCPU_tapas.h:48-74, over the body double
 * loop of hot/mapper.h:127-169 (targets outer). EPS2 = 0.  With mutual, a leaf
 * with itself visits j <= i only (AllowMutualInteraction, iterator.h:98-100)
 * and every pair also updates body j (`mutual && Bi.X != Bj.X`: the vec's
 * pointer conversion makes that "j is another body object"). */
static void p2p(oracle_fmm *h, int32_t ti, int32_t si) {
  const ocell *Ci = &h->cells[ti], *Cj = &h->cells[si];
  const int mutual = h->mutual;
  const int tri = mutual && ti == si;
  for (int64_t a = 0; a < Ci->nb; a++) {
    int64_t i = Ci->bbeg + a;
    double *t = h->trg + 4 * i;
    const int64_t bend = tri ? a + 1 : Cj->nb;
    for (int64_t b = 0; b < bend; b++) {
      int64_t j = Cj->bbeg + b;
      double dX[3] = {h->sx[i] - h->sx[j] - 0.0, h->sy[i] - h->sy[j] - 0.0,
                      h->sz[i] - h->sz[j] - 0.0};
      double R2 = 0;
      R2 += dX[0] * dX[0];
      R2 += dX[1] * dX[1];
      R2 += dX[2] * dX[2];
      R2 = R2 + 0.0;
      if (R2 != 0) {
        double invR2 = 1.0 / R2;
        double invR = h->sq[i] * h->sq[j] * sqrt(invR2);
        double s = invR2 * invR;
        dX[0] *= s; dX[1] *= s; dX[2] *= s;
        t[0] += invR;
        t[1] -= dX[0];
        t[2] -= dX[1];
        t[3] -= dX[2];
        if (mutual && i != j) {
          double *u = h->trg + 4 * j;
          u[0] += invR;
          u[1] += dX[0];
          u[2] += dX[1];
          u[3] += dX[2];
        }
      }
    }
  }
}

static void push_pair(int32_t **t, int32_t **s, int64_t *n, int64_t *cap, int32_t a, int32_t b) {
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 4096;
    *t = realloc(*t, sizeof(int32_t) * (size_t)*cap);
    *s = realloc(*s, sizeof(int32_t) * (size_t)*cap);
  }
  (*t)[*n] = a; (*s)[*n] = b; (*n)++;
}

static void dtt(oracle_fmm *h, int32_t ti, int32_t si);

/* ProductMapImpl (hot/mapper.h:28-121) over a cell's subcells with
 * themselves under mutual: pairs (i, j) with i <= j.  SubCellIterator spawns
 * (splits the ranges) when the parent holds >= 1000 bodies (iterator.h:203-205)
 * and runs ranges of <= 2 (kThreadSpawnThreshold, :199-201) serially; a split
 * visits (lo, lo), (hi, hi), then (lo, hi), (hi, lo), and the Serial task
 * group runs each task as it is created (threading/serial.h). */
static void self_product(oracle_fmm *h, const int32_t *ch, int spawn, int b1, int e1, int b2,
                         int e2) {
  if (!spawn || e1 - b1 == 1 || (e1 - b1 <= 2 && e2 - b2 <= 2)) {
    for (int i = b1; i < e1; i++)
      for (int j = b2; j < e2; j++)
        if (i <= j) dtt(h, ch[i], ch[j]);
  } else if (e2 - b2 == 1) {
    const int m1 = (b1 + e1) / 2;
    self_product(h, ch, spawn, b1, m1, b2, e2);
    self_product(h, ch, spawn, m1, e1, b2, e2);
  } else {
    const int m1 = (b1 + e1) / 2, m2 = (b2 + e2) / 2;
    self_product(h, ch, spawn, b1, m1, b2, m2);
    self_product(h, ch, spawn, m1, e1, m2, e2);
    self_product(h, ch, spawn, b1, m1, m2, e2);
    self_product(h, ch, spawn, m1, e1, b2, m2);
  }
}

/* FMM_DTT, ex/tapas_exafmm.cxx:209-286.  R2 is the squared centre distance
 * (geometry.h:81-83 via tapas Vec::norm, vec.h:52-58).  The lists record the
 * visited pairs (with mutual: each unordered pair once, as visited). */
static void dtt(oracle_fmm *h, int32_t ti, int32_t si) {
  const ocell *Ci = &h->cells[ti], *Cj = &h->cells[si];
  double dc[3] = {Ci->center[0] - Cj->center[0], Ci->center[1] - Cj->center[1],
                  Ci->center[2] - Cj->center[2]};
  double R2 = 0;
  R2 += dc[0] * dc[0];
  R2 += dc[1] * dc[1];
  R2 += dc[2] * dc[2];
  double Ri = 0, Rj = 0;
  for (int d = 0; d < 3; d++) {
    double wi = Ci->mx[d] - Ci->mn[d], wj = Cj->mx[d] - Cj->mn[d];
    Ri = (Ri < wi) ? wi : Ri;
    Rj = (Rj < wj) ? wj : Rj;
  }
  Ri = (Ri / 2 * 1.00001) / h->theta;
  Rj = (Rj / 2 * 1.00001) / h->theta;
  if (R2 > (Ri + Rj) * (Ri + Rj)) {
    push_pair(&h->m2l_t, &h->m2l_s, &h->nm2l, &h->cm2l, ti, si);
    if (!h->own || (h->own[ti] & 1)) m2l(h, ti, si);
  } else if (Ci->leaf && Cj->leaf) {
    /* tapas::Map over an empty body product is skipped (hot.h:1362-1369). */
    if (Ci->nb > 0 && Cj->nb > 0) {
      push_pair(&h->p2p_t, &h->p2p_s, &h->np2p, &h->cp2p, ti, si);
      /* the functor calls the reference counts (INC_P2P): j <= i within a
       * leaf under mutual */
      h->np2p_int += (h->mutual && ti == si) ? (uint64_t)(Ci->nb * (Ci->nb + 1) / 2)
                                              : (uint64_t)(Ci->nb * Cj->nb);
      if (!h->own || (h->own[ti] & 2)) p2p(h, ti, si);
    }
  } else {
    /* tapas_splitCell, :252-285 (ties split Ci). */
    int ci_leaf = Ci->leaf, cj_leaf = Cj->leaf;
    int32_t chi[8], chj[8];
    memcpy(chi, Ci->child, sizeof chi);
    memcpy(chj, Cj->child, sizeof chj);
    if (cj_leaf) {
      for (int c = 0; c < 8; c++) dtt(h, chi[c], si);
    } else if (ci_leaf) {
      for (int c = 0; c < 8; c++) dtt(h, ti, chj[c]);
    } else if (h->mutual && ti == si) {
      /* both sides split; the product of a cell's subcells with themselves
       * visits (i, j) for i <= j only, in ProductMapImpl's order */
      self_product(h, chi, Ci->nb >= 1000, 0, 8, 0, 8);
    } else if (Ri >= Rj) {
      for (int c = 0; c < 8; c++) dtt(h, chi[c], si);
    } else {
      for (int c = 0; c < 8; c++) dtt(h, ti, chj[c]);
    }
  }
}

void oracle_set_mutual(oracle_fmm *h, int mutual) { h->mutual = mutual != 0; }

int oracle_traverse(oracle_fmm *h) {
  if (!h->cells) return -1;
  h->nm2l = 0; h->np2p = 0; h->np2p_int = 0;
  memset(h->trg, 0, sizeof(double) * 4 * (size_t)h->n);
  dtt(h, 0, 0);
  return 0;
}

/* L2L, :309-345 */
static void l2l(oracle_fmm *h, int32_t ci) {
  const ocell *c = &h->cells[ci], *Cj = &h->cells[c->parent];
  int P = h->P;
  cplx *L = h->L + (size_t)ci * h->nterm;
  const cplx *Lj = h->L + (size_t)c->parent * h->nterm;
  double dX[3] = {c->center[0] - Cj->center[0], c->center[1] - Cj->center[1],
                  c->center[2] - Cj->center[2]};
  double rho, alpha, beta;
  cart2sph(&rho, &alpha, &beta, dX);
  eval_multipole(P, rho, alpha, beta, h->ynm, h->ynmt);
  for (int j = 0; j < P; j++) {
    for (int k = 0; k <= j; k++) {
      int jks = j * (j + 1) / 2 + k;
      cplx acc = 0;
      for (int n = j; n < P; n++) {
        for (int m = j + k - n; m < 0; m++) {
          int jnkm = (n - j) * (n - j) + n - j + m - k;
          int nms = n * (n + 1) / 2 - m;
          acc += conj(Lj[nms]) * h->ynm[jnkm] * (double)(ODDEVEN(k));
        }
        for (int m = 0; m <= n; m++) {
          if (n - j >= abs(m - k)) {
            int jnkm = (n - j) * (n - j) + n - j + m - k;
            int nms = n * (n + 1) / 2 + m;
            acc += Lj[nms] * h->ynm[jnkm] * (double)(ODDEVEN((m - k) * (m < k)));
          }
        }
      }
      L[jks] += acc;
    }
  }
}

/* L2P, :275-307 (first divides the P2P sum by the body's charge). */
static void l2p(oracle_fmm *h, int32_t ci) {
  const ocell *c = &h->cells[ci];
  int P = h->P;
  const cplx *L = h->L + (size_t)ci * h->nterm;
  for (int64_t a = 0; a < c->nb; a++) {
    int64_t b = c->bbeg + a;
    double *ba = h->trg + 4 * b;
    double dX[3] = {h->sx[b] - c->center[0], h->sy[b] - c->center[1], h->sz[b] - c->center[2]};
    double sph[3] = {0, 0, 0}, cart[3];
    double r, theta, phi;
    cart2sph(&r, &theta, &phi, dX);
    eval_multipole(P, r, theta, phi, h->ynm, h->ynmt);
    double qi = h->sq[b];
    ba[0] /= qi; ba[1] /= qi; ba[2] /= qi; ba[3] /= qi;
    for (int n = 0; n < P; n++) {
      int nm = n * n + n;
      int nms = n * (n + 1) / 2;
      ba[0] += creal(L[nms] * h->ynm[nm]);
      sph[0] += creal(L[nms] * h->ynm[nm]) / r * n;
      sph[1] += creal(L[nms] * h->ynmt[nm]);
      for (int m = 1; m <= n; m++) {
        nm = n * n + n + m;
        nms = n * (n + 1) / 2 + m;
        ba[0] += 2 * creal(L[nms] * h->ynm[nm]);
        sph[0] += 2 * creal(L[nms] * h->ynm[nm]) / r * n;
        sph[1] += 2 * creal(L[nms] * h->ynmt[nm]);
        sph[2] += 2 * creal(L[nms] * h->ynm[nm] * I) * m;
      }
    }
    /* sph2cart, :50-60 */
    cart[0] = sin(theta) * cos(phi) * sph[0] + cos(theta) * cos(phi) / r * sph[1] -
              sin(phi) / r / sin(theta) * sph[2];
    cart[1] = sin(theta) * sin(phi) * sph[0] + cos(theta) * sin(phi) / r * sph[1] +
              cos(phi) / r / sin(theta) * sph[2];
    cart[2] = cos(theta) * sph[0] - sin(theta) / r * sph[1];
    ba[1] += cart[0];
    ba[2] += cart[1];
    ba[3] += cart[2];
  }
}

/* FMM_Downward, ex/tapas_exafmm.cxx:124-140 */
static void downward_rec(oracle_fmm *h, int32_t ci) {
  /* sharded: a cell whose local expansion is computed elsewhere has no owned
   * descendant either (owners of bodies own all their ancestors) */
  if (h->own && !(h->own[ci] & 1)) return;
  if (ci != 0) l2l(h, ci);
  if (h->cells[ci].leaf) {
    if (h->cells[ci].nb > 0 && (!h->own || (h->own[ci] & 2))) l2p(h, ci);
  } else {
    for (int i = 0; i < 8; i++) downward_rec(h, h->cells[ci].child[i]);
  }
}

int oracle_downward(oracle_fmm *h) {
  if (!h->cells) return -1;
  downward_rec(h, 0);
  return 0;
}

int oracle_run_all(oracle_fmm *h) {
  int r = oracle_build(h);
  if (!r) r = oracle_upward(h);
  if (!r) r = oracle_traverse(h);
  if (!r) r = oracle_downward(h);
  return r;
}

/* ---------------------------------------------------------------------------
 * Accessors.
 * ------------------------------------------------------------------------- */
void oracle_bbox(const oracle_fmm *h, double lo_hi[2]) { lo_hi[0] = h->lo; lo_hi[1] = h->hi; }
int64_t oracle_ncells(const oracle_fmm *h) { return h->ncells; }
int oracle_max_depth(const oracle_fmm *h) { return h->max_depth; }

void oracle_get_cells(const oracle_fmm *h, uint64_t *key, int32_t *leaf, int32_t *nb, int64_t *bid,
                      int32_t *parent, int32_t *child0, double *center3, double *width3) {
  for (int64_t i = 0; i < h->ncells; i++) {
    const ocell *c = &h->cells[i];
    if (key) key[i] = c->key;
    if (leaf) leaf[i] = c->leaf;
    if (nb) nb[i] = (int32_t)c->nb;
    if (bid) bid[i] = c->bbeg;
    if (parent) parent[i] = c->parent;
    if (child0) child0[i] = c->child0;
    for (int d = 0; d < 3; d++) {
      if (center3) center3[3 * i + d] = c->center[d];
      if (width3) width3[3 * i + d] = c->mx[d] - c->mn[d];
    }
  }
}

void oracle_get_expansions(const oracle_fmm *h, double *M, double *L) {
  size_t t = (size_t)h->ncells * h->nterm;
  for (size_t i = 0; i < t; i++) {
    if (M) { M[2 * i] = creal(h->M[i]); M[2 * i + 1] = cimag(h->M[i]); }
    if (L) { L[2 * i] = creal(h->L[i]); L[2 * i + 1] = cimag(h->L[i]); }
  }
}

int64_t oracle_n_m2l(const oracle_fmm *h) { return h->nm2l; }
int64_t oracle_n_p2p(const oracle_fmm *h) { return h->np2p; }
uint64_t oracle_n_p2p_interactions(const oracle_fmm *h) { return h->np2p_int; }
void oracle_get_m2l(const oracle_fmm *h, int32_t *tgt, int32_t *src) {
  memcpy(tgt, h->m2l_t, sizeof(int32_t) * (size_t)h->nm2l);
  memcpy(src, h->m2l_s, sizeof(int32_t) * (size_t)h->nm2l);
}
void oracle_get_p2p(const oracle_fmm *h, int32_t *tgt, int32_t *src) {
  memcpy(tgt, h->p2p_t, sizeof(int32_t) * (size_t)h->np2p);
  memcpy(src, h->p2p_s, sizeof(int32_t) * (size_t)h->np2p);
}
void oracle_get_bodies(const oracle_fmm *h, int64_t *orig, uint64_t *keys, double *trg4) {
  if (orig) memcpy(orig, h->perm, sizeof(int64_t) * (size_t)h->n);
  if (keys) memcpy(keys, h->skeys, sizeof(uint64_t) * (size_t)h->n);
  if (trg4) memcpy(trg4, h->trg, sizeof(double) * 4 * (size_t)h->n);
}

/* ---------------------------------------------------------------------------
 * Direct sum (threaded over targets).
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t n; const double *x, *y, *z, *q;
  const int64_t *tg; double *out; int64_t t0, t1; int field;
} dargs;

static void *direct_worker(void *p) {
  dargs *a = p;
  for (int64_t t = a->t0; t < a->t1; t++) {
    int64_t i = a->tg[t];
    double o[4] = {0, 0, 0, 0};
    double qi = a->field ? 1.0 : a->q[i];
    for (int64_t j = 0; j < a->n; j++) {
      double dX[3] = {a->x[i] - a->x[j], a->y[i] - a->y[j], a->z[i] - a->z[j]};
      double R2 = 0;
      R2 += dX[0] * dX[0];
      R2 += dX[1] * dX[1];
      R2 += dX[2] * dX[2];
      if (R2 != 0) {
        double invR2 = 1.0 / R2;
        double invR = qi * a->q[j] * sqrt(invR2);
        double s = invR2 * invR;
        o[0] += invR;
        o[1] -= dX[0] * s;
        o[2] -= dX[1] * s;
        o[3] -= dX[2] * s;
      }
    }
    if (!a->field) for (int d = 0; d < 4; d++) o[d] /= a->q[i];
    for (int d = 0; d < 4; d++) a->out[4 * t + d] = o[d];
  }
  return NULL;
}

static void direct_impl(int64_t n, const double *x, const double *y, const double *z,
                        const double *q, int64_t nt, const int64_t *tg, double *out, int nth,
                        int field) {
  if (nth <= 0) nth = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (nth < 1) nth = 1;
  if (nth > 256) nth = 256;
  if (nth > nt) nth = (int)(nt > 0 ? nt : 1);
  pthread_t th[256];
  dargs a[256];
  for (int k = 0; k < nth; k++) {
    a[k] = (dargs){n, x, y, z, q, tg, out, nt * k / nth, nt * (k + 1) / nth, field};
    pthread_create(&th[k], NULL, direct_worker, &a[k]);
  }
  for (int k = 0; k < nth; k++) pthread_join(th[k], NULL);
}

void oracle_direct(int64_t n, const double *x, const double *y, const double *z, const double *q,
                   int64_t nt, const int64_t *tg, double *out, int nth) {
  direct_impl(n, x, y, z, q, nt, tg, out, nth, 0);
}

void oracle_direct_field(int64_t n, const double *x, const double *y, const double *z,
                         const double *q, int64_t nt, const int64_t *tg, double *out, int nth) {
  direct_impl(n, x, y, z, q, nt, tg, out, nth, 1);
}

/* ---------------------------------------------------------------------------
 * Barnes-Hut sample: sample/barnes-hut/bh.cc, on the same tree (q = mass).
 * ------------------------------------------------------------------------- */

/* Approximate, bh.cc:155-190: leaf with one body -> the body itself; empty
 * leaf -> zero; non-leaf -> mass and mass-weighted centre of the 8 children
 * (children summed in index order, then divided by the total mass).  Leaves
 * with more than one body (ncrit > 1; the sample asserts ncrit == 1) get the
 * same mass-weighted centre over their bodies. */
static void bh_approx_rec(oracle_fmm *h, int32_t ci, double *attr) {
  ocell *c = &h->cells[ci];
  double *a = attr + 4 * ci;
  if (c->leaf) {
    if (c->nb == 0) {
      a[0] = a[1] = a[2] = a[3] = 0;
    } else if (c->nb == 1) {
      int64_t b = c->bbeg;
      a[0] = h->sx[b]; a[1] = h->sy[b]; a[2] = h->sz[b]; a[3] = h->sq[b];
    } else {
      double w = 0, x = 0, y = 0, z = 0;
      for (int64_t i = 0; i < c->nb; i++) {
        int64_t b = c->bbeg + i;
        w += h->sq[b];
        x += h->sx[b] * h->sq[b];
        y += h->sy[b] * h->sq[b];
        z += h->sz[b] * h->sq[b];
      }
      a[0] = x / w; a[1] = y / w; a[2] = z / w; a[3] = w;
    }
    return;
  }
  double w = 0, x = 0, y = 0, z = 0;
  for (int i = 0; i < 8; i++) {
    int32_t k = c->child[i];
    bh_approx_rec(h, k, attr);
    const double *s = attr + 4 * k;
    w += s[3];
    x += s[0] * s[3];
    y += s[1] * s[3];
    z += s[2] * s[3];
  }
  a[0] = x / w; a[1] = y / w; a[2] = z / w; a[3] = w;
}

/* ComputeForce, bh.cc:135-153 */
static inline void bh_force(const double p[3], const double ap[4], double eps2, double out[4]) {
  double dx = ap[0] - p[0], dy = ap[1] - p[1], dz = ap[2] - p[2];
  double R2 = dx * dx + dy * dy + dz * dz + eps2;
  double invR = 1.0 / sqrt(R2);
  double invR3 = invR * invR * invR;
  out[0] += dx * invR3 * ap[3];
  out[1] += dy * invR3 * ap[3];
  out[2] += dz * invR3 * ap[3];
  out[3] += invR * ap[3];
}

/* interact, bh.cc:192-224, for one target body (the sample's target leaves
 * hold one body; with larger leaves every body runs its own walk). */
static void bh_walk(oracle_fmm *h, const double *attr, int32_t ci, const double p[3], double theta,
                    double eps2, double out[4], uint64_t *napprox, uint64_t *ndirect) {
  const ocell *c = &h->cells[ci];
  if (c->leaf) {
    for (int64_t i = 0; i < c->nb; i++) {
      int64_t b = c->bbeg + i;
      double ap[4] = {h->sx[b], h->sy[b], h->sz[b], h->sq[b]};
      bh_force(p, ap, eps2, out);
      (*ndirect)++;
    }
    return;
  }
  double dx = p[0] - c->center[0], dy = p[1] - c->center[1], dz = p[2] - c->center[2];
  double d = sqrt(dx * dx + dy * dy + dz * dz);
  double s = c->mx[0] - c->mn[0];
  if ((s / d) < theta) {
    bh_force(p, attr + 4 * ci, eps2, out);
    (*napprox)++;
  } else {
    for (int i = 0; i < 8; i++) bh_walk(h, attr, c->child[i], p, theta, eps2, out, napprox, ndirect);
  }
}

int oracle_bh(oracle_fmm *h, double theta, double eps2, double *out4, uint64_t *counts) {
  if (!h->cells && oracle_build(h)) return -1;
  double *attr = calloc((size_t)h->ncells * 4, sizeof(double));
  bh_approx_rec(h, 0, attr);
  uint64_t na = 0, nd = 0;
  for (int64_t b = 0; b < h->n; b++) {
    double p[3] = {h->sx[b], h->sy[b], h->sz[b]};
    double *o = out4 + 4 * b;
    o[0] = o[1] = o[2] = o[3] = 0;
    bh_walk(h, attr, 0, p, theta, eps2, o, &na, &nd);
  }
  if (counts) { counts[0] = na; counts[1] = nd; }
  free(attr);
  return 0;
}
