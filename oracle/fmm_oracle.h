/*
 * CPU restatement of the reference Tapas/ExaFMM N-body evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA library is compared
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product (tapas-reduce_b200/) never links it.
 *
 * Parity pin: its outputs are checked against the unmodified reference built
 * from its own sources (oracle/_ref, oracle/Makefile) and against the
 * reference's Morton-key known-answer tests (cpp/tests/test_morton_key.cpp).
 *
 * Every step follows the reference's operation order so that, compiled for
 * x86-64 without FMA contraction (the reference's own build), it reproduces the
 * reference's keys, cells and interaction lists bit for bit and its multipole,
 * local and body values to within a few ulps.
 */
#ifndef TAPAS_ORACLE_FMM_H_
#define TAPAS_ORACLE_FMM_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_fmm oracle_fmm;

/* Bodies are copied in (SoA, original order). P = expansion order (>=2). */
oracle_fmm *oracle_create(int64_t n, const double *x, const double *y, const double *z,
                          const double *q, int P, int ncrit, double theta);
void oracle_destroy(oracle_fmm *h);

/* Pipeline phases (return 0 on success, <0 on error). */
int oracle_build(oracle_fmm *h);     /* bbox, keys, sort, cell tree       */
int oracle_upward(oracle_fmm *h);    /* P2M + M2M                          */
int oracle_traverse(oracle_fmm *h);  /* dual-tree traversal: M2L + P2P     */
/* The example's -m option: mutual = 1 visits each unordered cell pair once
 * and applies M2L and P2P both ways (set before oracle_traverse). */
void oracle_set_mutual(oracle_fmm *h, int mutual);

/* Sharded evaluation (mutual = 0): per-cell ownership bytes in this oracle's
 * cell order (bit 0: local expansion computed here, bit 1: bodies), NULL for
 * all; the upward pass in two halves with the multipoles settable between
 * them; oracle_traverse / oracle_downward then evaluate owned targets only
 * (the other bodies' results stay 0). */
void oracle_set_owned(oracle_fmm *h, const uint8_t *mask);
int oracle_p2m_only(oracle_fmm *h);
int oracle_m2m_only(oracle_fmm *h);
void oracle_set_multipoles(oracle_fmm *h, const double *M);
void oracle_set_theta(oracle_fmm *h, double theta);
int oracle_downward(oracle_fmm *h);  /* L2L + L2P                          */
int oracle_run_all(oracle_fmm *h);

/* Results and intermediate state. */
void oracle_bbox(const oracle_fmm *h, double lo_hi[2]);
int64_t oracle_ncells(const oracle_fmm *h);
int oracle_max_depth(const oracle_fmm *h);
/* Cells in the reference's generation (depth-first) order. */
void oracle_get_cells(const oracle_fmm *h, uint64_t *key, int32_t *leaf, int32_t *nb, int64_t *bid,
                      int32_t *parent, int32_t *child0, double *center3, double *width3);
/* M, L: ncells x NTERM complex values as interleaved (re, im). */
void oracle_get_expansions(const oracle_fmm *h, double *M, double *L);
int64_t oracle_n_m2l(const oracle_fmm *h);
int64_t oracle_n_p2p(const oracle_fmm *h);            /* leaf pairs with both nb > 0 */
uint64_t oracle_n_p2p_interactions(const oracle_fmm *h);
void oracle_get_m2l(const oracle_fmm *h, int32_t *tgt, int32_t *src);
void oracle_get_p2p(const oracle_fmm *h, int32_t *tgt, int32_t *src);
/* Bodies in sorted (Morton) order: original index, key, and target values
 * (pot, ax, ay, az) as the reference leaves them (per unit charge). */
void oracle_get_bodies(const oracle_fmm *h, int64_t *orig_index, uint64_t *keys, double *trg4);

/* Key algebra (sfc_morton.h restatement), exposed for known-answer tests. */
uint64_t oracle_key_child(uint64_t k, int idx);
uint64_t oracle_key_parent(uint64_t k);
uint64_t oracle_key_next(uint64_t k, int n);
int oracle_key_is_descendant(uint64_t asc, uint64_t dsc);
int oracle_key_includes_range(uint64_t beg, uint64_t end, uint64_t c);
int oracle_key_overlapped(uint64_t x1, uint64_t x2, uint64_t y1, uint64_t y2);
int oracle_key_dir_on_depth(uint64_t k, int dim, int depth);
uint64_t oracle_key_msbits(uint64_t k, int bits);
uint64_t oracle_key_finest(int ax, int ay, int az);
void oracle_key_region(uint64_t k, const double root_min[3], const double root_max[3], double mn[3],
                       double mx[3]);

/* Barnes-Hut sample (sample/barnes-hut/bh.cc:135-224) on this handle's tree
 * (q = mass, tree built with its ncrit): out4 = (ax, ay, az, phi) per body in
 * sorted order; counts = {approximations, direct interactions}. */
int oracle_bh(oracle_fmm *h, double theta, double eps2, double *out4, uint64_t *counts);

/* FP64 direct sum (LaplaceP2PCPU_tapas.h P2P over all sources, then the
 * TRG /= SRC normalisation of tapas_exafmm.cxx:365-367) for selected targets.
 * trg4 gets 4 values per target.  nthreads <= 0 uses all cores. */
void oracle_direct(int64_t n, const double *x, const double *y, const double *z, const double *q,
                   int64_t ntargets, const int64_t *targets, double *trg4, int nthreads);
/* Field form (sum_j q_j / r, -sum_j q_j dX / r^3) that does not divide by q_i. */
void oracle_direct_field(int64_t n, const double *x, const double *y, const double *z,
                         const double *q, int64_t ntargets, const int64_t *targets, double *trg4,
                         int nthreads);

#ifdef __cplusplus
}
#endif
#endif
