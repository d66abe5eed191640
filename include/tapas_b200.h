/*
 * tapas_b200.h - C ABI of libtapas_b200.so, the sm_100a (B200) implementation
 * of the Tapas N-body evaluation path (octree build, upward pass, dual-tree
 * traversal with M2L + P2P, downward pass) for the ExaFMM Laplace
 * spherical-harmonics kernels and the Barnes-Hut monopole sample.
 *
 * Conventions
 *  - Every entry point returns an int status: 0 (TAPAS_B200_OK) or a negative
 *    tapas_b200_status.  Nothing calls exit() or abort(); the reference's
 *    CUDA_SAFE_CALL/assert error paths (cpp/include/tapas/common.h:278-287,
 *    vectormap_cuda.h:70-80) become status codes plus tapas_b200_last_error().
 *  - Plain pointers and sizes only.  `mem` arguments say whether a pointer is
 *    host memory (TAPAS_B200_HOST) or device memory (TAPAS_B200_DEVICE) on
 *    the context's GPU.
 *  - All GPU work of a context is issued on its stream (tapas_b200_set_stream);
 *    calls that return host data synchronise that stream.
 *  - Bodies are structure-of-arrays FP64 x, y, z, q.  Results are four values
 *    per body, (pot, ax, ay, az) per unit charge, exactly what the reference's
 *    TRG holds after L2P (ExaFMM kvec4, ex/LaplaceSphericalCPU_tapas.h:275-307).
 *
 * Reference paths below are relative to the reference project;
 * "ex/" = sample/exafmm-dev-13274dd4ac68/examples/.
 */
#ifndef TAPAS_B200_H_
#define TAPAS_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tapas_b200_ctx tapas_b200_ctx;

typedef enum {
  TAPAS_B200_OK = 0,
  TAPAS_B200_ERR_ARG = -1,         /* invalid argument                         */
  TAPAS_B200_ERR_CUDA = -2,        /* CUDA runtime error (see last_error)      */
  TAPAS_B200_ERR_NOMEM = -3,       /* device or host allocation failed         */
  TAPAS_B200_ERR_STATE = -4,       /* call out of order (e.g. upward before partition) */
  TAPAS_B200_ERR_CAPACITY = -5,    /* a device work queue hit its bound        */
  TAPAS_B200_ERR_UNSUPPORTED = -6, /* e.g. expansion order outside 2..16         */
  TAPAS_B200_ERR_TIMEOUT = -7      /* a bounded device wait gave up            */
} tapas_b200_status;

enum { TAPAS_B200_HOST = 0, TAPAS_B200_DEVICE = 1 };

/* Arithmetic of the expansion and near-field kernels. */
enum {
  TAPAS_B200_FP64 = 0,  /* plain FP64 everywhere (the reference's FP64 build)          */
  TAPAS_B200_MIXED = 1  /* FP32 compensated P2P; FP32 P2M and L2P in units of the leaf
                           width; split-TF32 tensor-core M2L (FP64 for rare offset
                           classes); split-TF32 tensor-core M2M at the deepest three
                           parent levels below level 3, FP64 M2M above them; FP64
                           L2L; FP64 sums and outputs                                 */
};

/* Output order of per-body results. */
enum {
  TAPAS_B200_ORDER_SORTED = 0,   /* Morton order, as CopyBackResult leaves them
                                    (ex/tapas_exafmm.cxx:388-398)                     */
  TAPAS_B200_ORDER_ORIGINAL = 1  /* the caller's input order                          */
};

typedef struct {
  int64_t n_bodies;
  int64_t n_cells;
  int64_t n_leaves;
  int32_t max_depth;
  int32_t ncrit;
  double box_lo, box_hi; /* the cube [lo,hi]^3 the keys are quantised in */
} tapas_b200_tree_stats;

typedef struct {
  int64_t n_m2l;               /* M2L translations (cell pairs)                     */
  int64_t n_p2p;               /* P2P leaf pairs with both leaves non-empty        */
  uint64_t n_p2p_interactions; /* sum over leaf pairs of nb_i * nb_j              */
  int32_t traverse_iterations;
  /* Mixed-form M2L of the last tapas_b200_m2l(MIXED) call: */
  int64_t n_m2l_tc;            /* translations evaluated on the tensor cores       */
  int64_t tc_classes;          /* offset classes run as GEMMs                      */
  int64_t tc_tiles;            /* 128-translation GEMM tiles                       */
  int64_t pairs_visited;       /* (target, source) pairs the traversal classified  */
} tapas_b200_list_stats;

/* Phase timings of the last calls, milliseconds, measured with CUDA events on
 * the context stream when profiling is on (tapas_b200_set_profiling). */
typedef struct {
  double upload, bbox_keys, sort, tree, upward, p2m, m2m, traverse, list_sort, m2l, p2p,
      downward, l2l, l2p, download;
  double m2l_fp64;  /* M2L pairs evaluated by the FP64 kernel                 */
  double m2l_tc;    /* M2L tensor-core GEMM kernel (mixed form)              */
  double m2l_setup; /* mixed-form M2L: class sort, operators, normalisation  */
} tapas_b200_timings;

/* ---- context ------------------------------------------------------------- */

/* Replaces Vectormap_CUDA_Base::Setup (cpp/include/tapas/vectormap_cuda.h:337-395):
 * binds the context to `device`, creates its stream, checks it is sm_100. */
int tapas_b200_ctx_create(int device, tapas_b200_ctx **out);
/* Replaces Vectormap_CUDA_Base::Release (vectormap_cuda.h:397-404). */
int tapas_b200_ctx_destroy(tapas_b200_ctx *ctx);
/* Use `stream` (a cudaStream_t) for all later work; NULL restores the context's own. */
int tapas_b200_set_stream(tapas_b200_ctx *ctx, void *stream);
int tapas_b200_set_profiling(tapas_b200_ctx *ctx, int on);
/* on = 1: the traversal keeps the pairs that involve empty cells, exactly as
 * the reference's FMM_DTT visits them (ex/tapas_exafmm.cxx:209-286), so the
 * lists equal the reference's; on = 0 (default): such pairs, which contribute
 * nothing, are dropped.  Results are the same either way. */
int tapas_b200_set_reference_lists(tapas_b200_ctx *ctx, int on);
int tapas_b200_get_timings(tapas_b200_ctx *ctx, tapas_b200_timings *out);
/* Bound, in GPU clock cycles, on each wait between the roles of the
 * tensor-core M2L kernel (copy ring, MMA issue, epilogue); cycles <= 0 restores
 * the default 4e9 (about 2 s).  A wait that runs out makes the kernel drain its
 * copies and MMAs, free its tensor memory and return, and the call returns
 * TAPAS_B200_ERR_TIMEOUT with the context still usable.  No counterpart in
 * the reference (its GPU path has no bounded waits); meant for tests of that
 * failure path and for callers that want a shorter watchdog. */
int tapas_b200_set_wait_limit(tapas_b200_ctx *ctx, int64_t cycles);
/* Message of the last failing call on this context ("" if none). Thread-local
 * fallback when ctx is NULL (e.g. ctx_create failure). */
const char *tapas_b200_last_error(const tapas_b200_ctx *ctx);
/* Number of kernel launches issued by this context since the last reset. */
int64_t tapas_b200_kernel_launches(tapas_b200_ctx *ctx, int reset);

/* ---- tree ---------------------------------------------------------------- */

/* Replaces tapas::Tapas<TSP>::Partition (cpp/include/tapas/hot.h:1349-1352) ->
 * Partitioner::Partition (hot.h:1241-1284) -> SamplingOctree::Build
 * (hot/buildtree.h:329-367): bounding cube, Morton keys (buildtree.h:505-539),
 * key sort (common.h:249-273), cell tree (buildtree.h:388-459; a cell is a
 * leaf iff it holds <= ncrit bodies, non-leaves always have 8 children).
 * Single rank: the MPI sampling / exchange steps reduce to the identity. */
int tapas_b200_partition(tapas_b200_ctx *ctx, const double *x, const double *y, const double *z,
                         const double *q, int64_t n, int ncrit, int mem);
int tapas_b200_tree_info(tapas_b200_ctx *ctx, tapas_b200_tree_stats *out);
/* Cells in breadth-first (level) order; any output may be NULL.  bbeg/nb are
 * the body range in sorted order; child0 = index of the first of 8 children
 * (-1 for leaves); center3/width3 = 3 doubles per cell. Host memory. */
int tapas_b200_get_cells(tapas_b200_ctx *ctx, uint64_t *key, int32_t *leaf, int32_t *nb,
                         int32_t *bbeg, int32_t *parent, int32_t *child0, double *center3,
                         double *width3);
/* Sorted bodies: original index and Morton key per sorted position. Host memory. */
int tapas_b200_get_sorted(tapas_b200_ctx *ctx, int64_t *orig_index, uint64_t *keys);
/* Number of bodies per leaf depth of the current tree (leaves deeper than
 * nbins-1 count in the last bin); nbins in 1..64; hist = nbins host int64.
 * The octree-shape feature of the learned parameter chooser (the reference
 * prints the same per-depth leaf histogram under TAPAS_DEBUG_HISTOGRAM,
 * hot/buildtree.h:89-117). */
int tapas_b200_leaf_depth_histogram(tapas_b200_ctx *ctx, int nbins, int64_t *hist);

/* ---- Barnes-Hut sample path (sample/barnes-hut/bh.cc) ---------------------- */
/* Bodies are passed to tapas_b200_partition with the mass in the q slot; the
 * sample builds its tree with ncrit = 1 (bh.cc:230). */

/* Replaces TapasBH::Map(Approximate(), *root) (bh.cc:232, Approximate :155-190):
 * per cell the mass and mass-weighted centre, children before parents. */
int tapas_b200_bh_upward(tapas_b200_ctx *ctx);
/* Replaces TapasBH::Map(interact(), tapas::Product(*root, *root), theta)
 * (bh.cc:235, interact :192-224, ComputeForce :135-153): per body a walk from
 * the root accepting cells with width / |centre - body| < theta, leaves summed
 * body by body (self included, softening eps2; the sample uses 1e-6).  Results
 * (read with tapas_b200_get_results) are the sample's float4 per body:
 * (ax, ay, az, phi).  TAPAS_B200_FP64 reproduces the sample's arithmetic;
 * TAPAS_B200_MIXED walks with FP32 positions and FP32 copies of the cells'
 * FP64 moments. */
int tapas_b200_bh_interact(tapas_b200_ctx *ctx, double theta, double eps2, int precision);
/* Cell approximations and direct body interactions of the last walk. */
int tapas_b200_bh_counts(tapas_b200_ctx *ctx, uint64_t *n_approx, uint64_t *n_direct);
/* Partition + bh_upward + bh_interact + get_results in one call (calc(),
 * bh.cc:228-245, with ncrit and theta as arguments). */
int tapas_b200_bh_evaluate(tapas_b200_ctx *ctx, const double *x, const double *y, const double *z,
                           const double *m, int64_t n, int ncrit, double theta, double eps2,
                           int precision, double *out4, int order, int mem);

/* ---- learned parameter chooser: network trained and run by own kernels ---- */
/* No counterpart in the reference (the learned part of this implementation).
 * Fully connected n_in -> n_hidden x n_layers (tanh) -> n_out (linear), FP32,
 * parameters one flat array (per layer W out x in row-major, then b). */
int tapas_b200_mlp_create(tapas_b200_ctx *ctx, int n_in, int n_hidden, int n_layers, int n_out,
                          uint64_t seed);
int64_t tapas_b200_mlp_num_params(tapas_b200_ctx *ctx);
int tapas_b200_mlp_set_params(tapas_b200_ctx *ctx, const float *params);
int tapas_b200_mlp_get_params(tapas_b200_ctx *ctx, float *params);
/* Y[n x n_out] = net(X[n x n_in]); host arrays. */
int tapas_b200_mlp_forward(tapas_b200_ctx *ctx, const float *X, int64_t n, float *Y);
/* Gradient of the mean squared error over the n samples w.r.t. all
 * parameters (flat layout) and the loss; host arrays. */
int tapas_b200_mlp_gradients(tapas_b200_ctx *ctx, const float *X, const float *Y, int64_t n,
                             float *grads, float *loss);
/* Adam training, minibatches of `batch` samples in a seeded shuffle order;
 * loss_per_epoch (may be NULL) gets the mean loss of each epoch. */
int tapas_b200_mlp_train(tapas_b200_ctx *ctx, const float *X, const float *Y, int64_t n,
                         int epochs, int batch, float lr, uint64_t seed, float *loss_per_epoch);

/* ---- evaluation ---------------------------------------------------------- */

/* Replaces TapasFMM::Map(FMM_Upward(), *root, theta) (ex/tapas_exafmm.cxx:586):
 * FMM_Upward (:87-122) -> P2M (ex/LaplaceSphericalCPU_tapas.h:138-163) per leaf
 * and M2M (:165-206) per non-leaf, children before parents.  P in 2..16. */
int tapas_b200_upward(tapas_b200_ctx *ctx, int P, int precision);

/* Replaces TapasFMM::Map(FMM_DTT(), tapas::Product(*root, *root), mutual,
 * nspawn, theta) (ex/tapas_exafmm.cxx:606) together with the GPU mapper's
 * body-pair offload (hot/mapper.h:453-690, vectormap_cuda.h:826-1005):
 * builds the M2L and P2P lists with the FMM_DTT acceptance test and split
 * rule (:209-286) and evaluates M2L (LaplaceSphericalCPU_tapas.h:208-273) and
 * P2P (LaplaceP2PCPU_tapas.h:23-74).
 * mutual = 1 is the example's -m option, which the reference's CPU build runs
 * (its CUDA build rejects it, ex/tapas_exafmm.cxx:507-515): every unordered
 * cell pair is visited once (a cell with itself splits both sides and visits
 * child pairs i <= j) and acts both ways.  The lists then hold both directions
 * of each visited pair, and the results are the reference's -m 1 results. */
int tapas_b200_traverse(tapas_b200_ctx *ctx, double theta, int mutual, int precision);
/* The same, in steps: list construction only, then each list. */
int tapas_b200_build_lists(tapas_b200_ctx *ctx, double theta, int mutual);
int tapas_b200_list_info(tapas_b200_ctx *ctx, tapas_b200_list_stats *out);
/* Copies the lists (cell indices in the get_cells order, sorted by target then
 * source) to host memory; arrays must hold list_info counts. */
int tapas_b200_get_lists(tapas_b200_ctx *ctx, int32_t *m2l_tgt, int32_t *m2l_src,
                         int32_t *p2p_tgt, int32_t *p2p_src);
int tapas_b200_m2l(tapas_b200_ctx *ctx, int precision);
int tapas_b200_p2p(tapas_b200_ctx *ctx, int precision);

/* Replaces TapasFMM::Map(FMM_Downward(), *root) (ex/tapas_exafmm.cxx:627):
 * L2L (LaplaceSphericalCPU_tapas.h:309-345) parent before child, then L2P
 * (:275-307) for every non-empty leaf. */
int tapas_b200_downward(tapas_b200_ctx *ctx, int precision);

/* ---- device views for user functors -------------------------------------- */
/* The reference offloads any __host__ __device__ body-pair functor through
 * its vectormap (cpp/include/tapas/vectormap_cuda.h:645-1005).  The templates
 * of include/tapas_b200/device.cuh do the same on this library's tree and
 * lists, compiled into the user's program by nvcc; this view gives them the
 * context's device arrays (read-only, valid until the next call that rebuilds
 * the tree or the lists).  Cells are in get_cells order; bodies in Morton
 * order; lists as build_lists left them (CSR by target cell, entries
 * target << list_shift | source, NULL before the first build_lists). */
#define TAPAS_B200_MAX_LEVELS 24
typedef struct {
  int64_t n_bodies, n_cells, n_levels;
  int64_t level_off[TAPAS_B200_MAX_LEVELS + 1]; /* host values: cells of level l are
                                                   [level_off[l], level_off[l+1]) */
  const int32_t *nb, *bbeg, *leaf, *parent, *child0, *level;
  const double *center3, *min3, *max3;          /* 3 values per cell */
  const double *x, *y, *z, *q;                  /* bodies, Morton order */
  const uint32_t *orig_index;                   /* Morton position -> caller's index */
  const int32_t *p2p_off, *m2l_off;             /* n_cells + 1 each */
  const uint64_t *p2p_list, *m2l_list;
  int64_t n_p2p, n_m2l;
  int32_t list_shift;
} tapas_b200_device_view;
int tapas_b200_get_device_view(tapas_b200_ctx *ctx, tapas_b200_device_view *out);
/* The cudaStream_t the context issues its work on (for the caller's kernels). */
int tapas_b200_get_stream(tapas_b200_ctx *ctx, void **stream);
/* Near field computed by the caller's own P2P functor (in place of
 * tapas_b200_p2p), 4 values per body in Morton order, in the reference's P2P
 * convention (sums of q_i q_j / r and q_i q_j dX / r^3, which the FP64 L2P
 * divides by q_i, ex/LaplaceSphericalCPU_tapas.h:283); host or device memory.
 * tapas_b200_downward then adds the far field to it.  No counterpart call in
 * the reference (its P2P writes the body attributes directly). */
int tapas_b200_set_near_field(tapas_b200_ctx *ctx, const double *trg4, int mem);

/* ---- sharded evaluation over several GPUs -------------------------------- */
/* The reference splits the work over MPI ranks by Morton-key ranges and builds
 * a locally essential tree per rank (cpp/include/tapas/hot/buildtree.h:
 * 162-324,461-483, hot/exact_let.h:675-1247).  Here every GPU builds the same
 * tree from all bodies (the partition is deterministic) and evaluates the
 * targets it owns; the caller's collectives do the rest (see
 * tapas-reduce_b200/sharded.py: one all-reduce of the leaves' multipoles
 * between p2m and m2m, one of the results).  No counterpart call in the
 * reference.
 * mask: one byte per cell (get_cells order) of the current tree; bit 0 = this
 * context computes the cell's local expansion (its M2L list and L2L), bit 1
 * = it evaluates the cell's bodies (P2M, P2P, L2P).  The owner of a leaf's
 * bodies must also own the local expansions of the leaf and its ancestors.
 * NULL clears the mask; a partition clears it too.  With a mask:
 *  - p2m computes the owned leaves' multipoles (the rest are zero);
 *  - m2l and p2p evaluate owned targets only; the classification of M2L
 *    pairs still sees every pair, so each target's arithmetic, and result,
 *    is the same as without a mask;
 *  - results of bodies not owned are exactly zero. */
int tapas_b200_set_owned_cells(tapas_b200_ctx *ctx, const uint8_t *mask, int mem);
/* The two halves of tapas_b200_upward: P2M of the leaves (M zeroed first),
 * then M2M of the whole tree from the leaves' multipoles. */
int tapas_b200_p2m(tapas_b200_ctx *ctx, int P, int precision);
int tapas_b200_m2m(tapas_b200_ctx *ctx);
/* Multipoles, ncells x P(P+1)/2 complex FP64 as interleaved (re, im), in host
 * or device memory (mem): read after p2m or upward, write between p2m and m2m
 * (or before traverse). */
int tapas_b200_get_multipoles(tapas_b200_ctx *ctx, double *M, int mem);
int tapas_b200_set_multipoles(tapas_b200_ctx *ctx, const double *M, int mem);

/* Multipole / local expansions, ncells x P(P+1)/2 complex FP64 values as
 * interleaved (re, im), cells in get_cells order.  Host memory; either may be NULL. */
int tapas_b200_get_expansions(tapas_b200_ctx *ctx, double *M, double *L);

/* Replaces CopyBackResult (ex/tapas_exafmm.cxx:388-398): 4 values per body. */
int tapas_b200_get_results(tapas_b200_ctx *ctx, double *trg4, int order, int mem);

/* Partition + upward + traverse + downward + get_results in one call:
 * the whole timestep of ex/tapas_exafmm.cxx:550-641 with mutual = 0. */
int tapas_b200_evaluate(tapas_b200_ctx *ctx, const double *x, const double *y, const double *z,
                        const double *q, int64_t n, int P, int ncrit, double theta, int precision,
                        double *trg4, int order, int mem);

/* FP64 direct sum on the GPU for sampled targets (the check of
 * ex/tapas_exafmm.cxx:288-383): out4 = 4 values per target, per unit charge
 * (field form: sum_j q_j/r and -sum_j q_j dX/r^3, no division by q_i).
 * Bodies are the ones of the last partition; targets are original indices. */
int tapas_b200_direct(tapas_b200_ctx *ctx, const int64_t *targets, int64_t k, double *out4,
                      int mem);

/* ---- file formats (host code; no GPU needed) ------------------------------ */

/* Body files of the reference's Dataset (exafmm include/dataset.h:313-372):
 * <dir>/source%04d.dat (rank) holds x, y, z, q of each body, one value per
 * line; <dir>/target%04d.dat holds pot, ax, ay, az.  dir NULL or "" = the
 * working directory.  Writers: digits <= 0 formats as the reference does (the
 * stream default, 6 significant digits), digits > 0 sets the precision (17
 * round-trips FP64).  Readers read n bodies starting at *position (a byte
 * offset; NULL = the file's start) and store the position after them there,
 * so successive calls continue through the file as the reference's
 * readSources/readTargets do with Dataset::filePosition.  trg4 is 4 values per
 * body.  Errors: tapas_b200_last_error(NULL). */
int tapas_b200_write_sources(const char *dir, int rank, int64_t n, const double *x,
                             const double *y, const double *z, const double *q, int digits);
int tapas_b200_write_targets(const char *dir, int rank, int64_t n, const double *trg4,
                             int digits);
int tapas_b200_read_sources(const char *dir, int rank, int64_t n, double *x, double *y,
                            double *z, double *q, int64_t *position);
int tapas_b200_read_targets(const char *dir, int rank, int64_t n, double *trg4,
                            int64_t *position);

/* The example's per-step report (ex/tapas_exafmm.cxx:651-677; RankCSV of
 * cpp/include/tapas/util.h:223-316): writes `path` with the columns Rank,
 * total, upward, traverse, downward, tree (seconds), numP2P, numM2L (the
 * -DCOUNT counters) in the reference's fixed-width layout. */
int tapas_b200_write_main_csv(const char *path, int rank, double total, double upward,
                              double traverse, double downward, double tree, uint64_t num_p2p,
                              uint64_t num_m2l);
/* Replaces the example's report of a timestep (main.csv, :651-677) and
 * Cell::Report (hot/report.h:40-152: hostnames, misc, load_balancing,
 * tree_construction, map2 .csv; the sampling, exchange and LET columns are 0
 * on one GPU) for the context's last evaluation, into files
 * <prefix><name><suffix>.csv (NULL prefix/suffix: the environment variables
 * TAPAS_REPORT_PREFIX / TAPAS_REPORT_SUFFIX, as the reference reads them).
 * Times come from the phase timings, so turn profiling on
 * (tapas_b200_set_profiling) before the evaluation; otherwise they are 0.
 * numP2P / numM2L count functor calls as the reference does: they equal the
 * reference's counters for lists built with tapas_b200_set_reference_lists(1). */
int tapas_b200_write_report(tapas_b200_ctx *ctx, const char *prefix, const char *suffix);

/* The same FP64 direct-sum check, for callers that must not allocate device
 * memory at the point where they verify accuracy: a solver loop that reserved
 * all of its device memory up front, or code sharing the GPU with other
 * streams (cudaMalloc/cudaFree synchronise the whole device).  This entry
 * point has no counterpart in the reference.
 *  - x, y, z, q (n bodies), targets (k original indices) and out4 (4*k) are
 *    caller-owned DEVICE buffers on the current device; work goes on `stream`
 *    (a cudaStream_t, NULL = default stream) and is not synchronised.
 *  - It allocates nothing: partial sums live in one fixed 2 MiB device array
 *    built into the library, present once on every GPU that loads it until
 *    the process exits.  At most 4096 targets per call; larger k returns
 *    TAPAS_B200_ERR_CAPACITY.  A target index outside [0, n) gives NaN.
 *  - Calls share that array and it keeps the last call's contents: calls
 *    that overlap on the GPU race and must be serialised by the caller.
 *  - The first call on a device looks up the array's address; make it before
 *    any stream capture.  Errors: tapas_b200_last_error(NULL). */
int tapas_b200_direct_noalloc(const double *x, const double *y, const double *z, const double *q,
                              int64_t n, const int64_t *targets, int64_t k, double *out4,
                              void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TAPAS_B200_H_ */
