// Shared definitions of libtapas_b200: context, device buffers, status
// handling, Morton key helpers and exact (contraction-free) FP64 arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tapas_b200.h"

namespace tb {

constexpr int kMaxDepth = 19;   // Morton<3, uint64_t>::MaxDepth(), sfc_morton.h:168-177
constexpr int kDepthBits = 5;   // Morton<3, uint64_t>::DepthBits(), sfc_morton.h:154-163
constexpr int kMinP = 2;
constexpr int kMaxP = 16;
constexpr int kGemmSlabs = 4;   // concurrent streams of the FP64 class GEMMs

// ---------------------------------------------------------------------------
// Error handling: every failure becomes a status code plus a message.
// ---------------------------------------------------------------------------
struct Error {
  int code;
};

void set_error(tapas_b200_ctx *ctx, const char *fmt, ...);

#define TB_CUDA(ctx, expr)                                                         \
  do {                                                                             \
    cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      ::tb::set_error((ctx), "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                      __FILE__, __LINE__);                                         \
      return e_ == cudaErrorMemoryAllocation ? TAPAS_B200_ERR_NOMEM               \
                                             : TAPAS_B200_ERR_CUDA;               \
    }                                                                              \
  } while (0)

#define TB_TRY(expr)              \
  do {                            \
    int r_ = (expr);              \
    if (r_ != TAPAS_B200_OK) return r_; \
  } while (0)

// ---------------------------------------------------------------------------
// Growable device buffer owned by a context.
// ---------------------------------------------------------------------------
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t cap = 0;
  // Ensures room for n elements; contents are NOT preserved unless keep.
  cudaError_t ensure(size_t n, cudaStream_t s, bool keep = false, size_t used = 0) {
    if (n <= cap) return cudaSuccess;
    size_t nc = cap ? cap : 1024;
    while (nc < n) nc += nc / 2 + 1024;
    T *q = nullptr;
    cudaError_t e = cudaMalloc(&q, nc * sizeof(T));
    if (e != cudaSuccess) return e;
    if (keep && p && used) {
      e = cudaMemcpyAsync(q, p, used * sizeof(T), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) { cudaFree(q); return e; }
      e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { cudaFree(q); return e; }
    }
    if (p) cudaFree(p);
    p = q;
    cap = nc;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Pinned host staging buffer.
struct HBuf {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    size_t nc = bytes + bytes / 4 + 4096;
    cudaError_t e = cudaMallocHost(&p, nc);
    cap = e == cudaSuccess ? nc : 0;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

struct Mlp;  // learned-chooser network (mlp.cu)

// Work state of the tensor-core M2L (m2l_tc.cu).
struct TcState {
  DBuf<uint64_t> keys, keys_alt, tc_keys;
  DBuf<uint32_t> vals, vals_alt;
  DBuf<uint32_t> pairs64;  // list indices of the pairs left to the FP64 kernel
  DBuf<int32_t> flag, scan, seg_start, tcflag, tcid, ntiles, tile_off;
  DBuf<int4> items, items_alt;
  DBuf<int2> cls_range;    // per selected class: first sorted pair, pair count
  DBuf<float> ops, Mt, Lt;  // per selected class its FP32 operator rows; FP32 rows of M, L
  DBuf<double> ops64, Mt64, Lt64;  // FP64 class GEMM (plain form)
  DBuf<uint8_t> use64;     // FP64 class GEMM: list entries left to the pair kernel
  DBuf<int32_t> oflag, opos;  // sharded: owned sorted pairs and their compacted positions
  DBuf<uint8_t> sel, sel2;    // sharded: class selection per sorted / compacted pair
  // tensor-core M2M of the mixed form
  DBuf<float> ops_tr;                // 8 M2M classes: octant o
  int tr_P = 0;                      // order they were built for (0: none)
  DBuf<uint64_t> tree_list;          // one level's (parent << 32 | child) pairs
  DBuf<uint32_t> iota;               // 0, 1, 2, ... (pair order of a level)
  int64_t iota_n = 0;
  DBuf<int4> tree_items;             // one level's 128-pair tiles
  bool mt_ready = false;             // Mt holds this tree's normalised split multipoles
  // class-key field ranges (largest |offset|, |level difference|) of the last
  // classification: the next one packs with them and checks that every pair fits
  bool kp_cached = false;
  int kp_bo = 0, kp_bd = 0;
  DBuf<int> err;
  void release() {
    keys.release(); keys_alt.release(); tc_keys.release(); vals.release(); vals_alt.release();
    pairs64.release(); flag.release(); scan.release(); seg_start.release(); tcflag.release();
    tcid.release(); ntiles.release(); tile_off.release(); items.release(); cls_range.release();
    ops.release(); Mt.release(); Lt.release(); ops64.release();
    Mt64.release(); Lt64.release(); use64.release(); oflag.release(); opos.release();
    sel.release(); sel2.release(); ops_tr.release(); tree_list.release();
    iota.release(); tree_items.release(); err.release();
    tr_P = 0;
    iota_n = 0;
    mt_ready = false;
  }
};

}  // namespace tb

// ---------------------------------------------------------------------------
// The context: one GPU, one stream, the current tree, lists and expansions.
// ---------------------------------------------------------------------------
struct tapas_b200_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  std::string last_error;
  int64_t launches = 0;
  bool profiling = false;
  tapas_b200_timings timings{};

  // ---- bodies (SoA FP64) ----
  int64_t n = 0;
  tb::DBuf<double> x, y, z, q;          // input order
  tb::DBuf<double4> body_pack;          // input order, (x, y, z, q) per body
  tb::DBuf<double> sx, sy, sz, sq;      // sorted order
  tb::DBuf<uint64_t> keys, keys_alt;    // sort ping-pong
  tb::DBuf<uint32_t> idx, idx_alt;      // sorted position -> original index
  tb::DBuf<double> trg;                 // 4 per body, sorted order (pot, ax, ay, az)
  tb::DBuf<double> trg_out;             // 4 per body, reorder scratch
  tb::DBuf<double> bbox;                // [lo, hi]
  tb::DBuf<double> scratch_d;           // reduction partials
  tb::DBuf<uint32_t> sort_hist;         // radix sort block histograms
  tb::DBuf<int32_t> scan_tmp;           // scan partials

  // ---- cells (SoA, breadth-first order) ----
  bool have_tree = false;
  int ncrit = 64;
  double box_lo = 0, box_hi = 0;
  int64_t ncells = 0, nleaves = 0;
  int max_depth = 0;
  std::vector<int64_t> level_off;       // cells of level L: [level_off[L], level_off[L+1])
  tb::DBuf<uint64_t> ckey;
  tb::DBuf<int32_t> cbeg, cnb, cparent, cchild, cleaf, clevel;
  tb::DBuf<double> cmin, cmax, ccen;    // 3 doubles per cell (x,y,z interleaved)
  tb::DBuf<double4> trav_geo;          // traversal: per cell {centre, MAC radius for this theta}
  tb::DBuf<int2> trav_meta;            // traversal: per cell {nb, first child or -1 for a leaf}
  tb::DBuf<int32_t> flag, flag_scan;    // per-level scratch
  tb::DBuf<int32_t> leaf_list;          // indices of non-empty leaves
  // mixed L2P, body-parallel: per evaluated leaf its FP32 local expansion and
  // (centre, width); per body its leaf's ordinal (-1: not evaluated here)
  tb::DBuf<float2> l2p_lf;
  tb::DBuf<double4> l2p_geo;
  tb::DBuf<int32_t> l2p_body_leaf;
  int64_t n_nonempty_leaves = 0;
  // Sharded evaluation (tapas_b200_set_owned_cells): per cell bit 0 = this
  // context computes the cell's local expansion, bit 1 = its bodies (P2M,
  // P2P, L2P); cleared by each partition.
  bool sharded = false;
  tb::DBuf<uint8_t> cell_own;
  tb::DBuf<int32_t> leaf_own;           // owned non-empty leaves
  int64_t n_owned_leaves = 0;

  // ---- traversal lists ----
  bool have_lists = false;
  bool sources_sorted[2] = {true, true};        // M2L, P2P: each target's sources in order
  unsigned long long longest_segment[2] = {0, 0};  // M2L, P2P: longest target segment
  double theta = 0.4;
  tb::DBuf<int2> front_a, front_b;      // (target, source) pairs
  tb::DBuf<uint64_t> m2l, p2p;          // (target << 32 | source)
  tb::DBuf<uint64_t> list_alt;
  tb::DBuf<int32_t> list_cnt;           // list ordering: per-target counts, cursors, long segments
  tb::DBuf<uint32_t> list_src;          // list ordering: sources grouped by target
  tb::DBuf<unsigned long long> counters; // [next, m2l, p2p, p2p_interactions, overflow]
  int64_t n_m2l = 0, n_p2p = 0;         // directed pairs in the lists
  int64_t n_m2l_visited = 0, n_p2p_visited = 0;  // pairs the traversal emitted (unordered if mutual)
  int mutual = 0;                       // lists of the last build_lists came from a mutual traversal
  uint64_t n_p2p_int = 0;
  int trav_iters = 0;
  int64_t trav_pairs = 0;  // (target, source) pairs the traversal classified
  int list_shift = 1;                   // packed list key = target << shift | source
  bool reference_lists = false;         // keep pairs with empty cells, as the reference visits them
  tb::DBuf<int32_t> m2l_off, p2p_off;   // CSR by target cell, ncells+1
  tb::DBuf<int32_t> m2l_tlist, p2p_tlist; // targets having list entries
  int64_t n_m2l_targets = 0, n_p2p_targets = 0;

  // ---- expansions ----
  int P = 0;
  int precision = TAPAS_B200_FP64;       // of the expansion passes (set by upward)
  int near_precision = TAPAS_B200_FP64;  // of the last P2P: FP64 sums carry q_i, mixed do not
  tb::DBuf<float4> rel4;                // mixed: hi part of (x,y,z) - c_leaf, and q, FP32
  tb::DBuf<float4> rel_lo;              // mixed: lo part of (x,y,z) - c_leaf, FP32
  tb::DBuf<uint64_t> p2p_wkey, p2p_wkey_alt;  // P2P work order: keys
  tb::DBuf<uint32_t> p2p_order, p2p_order_alt;  // target leaves by decreasing work
  tb::DBuf<int> p2p_counter;            // P2P work-queue head
  tb::DBuf<int4> p2p_items;             // P2P work items (leaf, list range, partial rows)
  tb::DBuf<int32_t> p2p_kcnt, p2p_koff, p2p_psz, p2p_poff;  // per leaf: pieces, partial rows
  tb::DBuf<double> p2p_part;            // partial sums of pieces of split leaves
  int64_t p2p_nitems = 0;
  bool p2p_split = false;
  tb::TcState tc;                       // mixed: tensor-core M2L work state
  const uint32_t *m2l_pairs = nullptr;  // FP64 M2L of listed pairs: their list indices
  int64_t m2l_npairs = 0;
  int64_t tc_classes = 0, tc_tiles = 0, tc_segments = 0, n_m2l_tc = 0;
  size_t tc_op_budget = (size_t)4 << 30;  // bytes of split-TF32 operators kept at once
  long long tc_wait_limit = 4000000000LL; // clock cycles a tensor-core M2L wait may take
  bool have_M = false, have_L = false;
  bool have_leaf_M = false;             // p2m done, m2m not yet (M holds the leaves' only)
  tb::DBuf<double2> M, L;               // ncells x nterm complex FP64
  tb::DBuf<double> op_m2m, op_l2l;      // per level: child<->parent translation operators
  int level_ops_P = 0;                  // order the operators were built for (0: none)
  tb::DBuf<double> op_part;             // M2M of small levels: per-octant partial products

  tb::Mlp *mlp = nullptr;               // learned chooser network, if created

  // ---- Barnes-Hut ----
  tb::DBuf<double4> bh_attr;            // per cell: mass-weighted centre (x,y,z) and mass
  tb::DBuf<float4> bh_attr32;           // FP32 copy for the FP32 walk
  bool have_bh_attr = false;
  uint64_t bh_napprox = 0, bh_ndirect = 0;

  tb::HBuf pinned;
  // FP64 class GEMMs: helper streams (and their fork / join events), made on first use
  cudaStream_t gemm_streams[tb::kGemmSlabs] = {};
  cudaEvent_t gemm_join[tb::kGemmSlabs] = {};
  cudaEvent_t gemm_fork = nullptr;
  // upload of the charges on a side stream while the keys are built and sorted
  cudaStream_t upload_stream = nullptr;
  cudaEvent_t q_ready = nullptr, upload_fork = nullptr;
  bool q_pending = false;  // q is being copied: pack it after waiting for q_ready
};

namespace tb {
void mlp_release(tapas_b200_ctx *ctx);
}

namespace tb {

inline int nterm_of(int P) { return P * (P + 1) / 2; }

// The non-empty leaves whose bodies this context evaluates: all of them, or
// the owned ones of a sharded evaluation.
inline const int32_t *work_leaves(const tapas_b200_ctx *ctx, int64_t &nl) {
  nl = ctx->sharded ? ctx->n_owned_leaves : ctx->n_nonempty_leaves;
  return ctx->sharded ? ctx->leaf_own.p : ctx->leaf_list.p;
}
// Per-cell ownership mask (bit 0: local expansion), or null when not sharded.
inline const uint8_t *owned_cells(const tapas_b200_ctx *ctx) {
  return ctx->sharded ? ctx->cell_own.p : nullptr;
}

inline void count_launch(tapas_b200_ctx *ctx) { ctx->launches++; }

inline cudaError_t check_launch() { return cudaGetLastError(); }

#define TB_LAUNCH_CHECK(ctx)                                                         \
  do {                                                                               \
    ::tb::count_launch(ctx);                                                         \
    cudaError_t e_ = cudaGetLastError();                                             \
    if (e_ != cudaSuccess) {                                                         \
      ::tb::set_error((ctx), "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                      __FILE__, __LINE__);                                           \
      return TAPAS_B200_ERR_CUDA;                                                    \
    }                                                                                \
  } while (0)

// Phase timer: CUDA events on the context stream, only when profiling.
struct PhaseTimer {
  tapas_b200_ctx *ctx;
  double *slot;
  cudaEvent_t a = nullptr, b = nullptr;
  PhaseTimer(tapas_b200_ctx *c, double *s) : ctx(c), slot(s) {
    if (ctx->profiling) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, ctx->stream);
    }
  }
  ~PhaseTimer() {
    if (ctx->profiling && a) {
      cudaEventRecord(b, ctx->stream);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      *slot = ms;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  }
};

inline int grid_for(int64_t n, int block, int max_blocks = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return (int)g;
}

// ---------------------------------------------------------------------------
// Device helpers.
// ---------------------------------------------------------------------------
__host__ __device__ inline int key_depth(uint64_t k) { return (int)(k & 31u); }

// GetNext (sfc_morton.h:192-206)
__host__ __device__ inline uint64_t key_next(uint64_t k) {
  int d = key_depth(k);
  return k + ((uint64_t)1 << (3 * (kMaxDepth - d) + kDepthBits));
}

// Child (sfc_morton.h:288-295)
__host__ __device__ inline uint64_t key_child(uint64_t k, int idx) {
  int d = key_depth(k) + 1;
  uint64_t kk = ((k >> kDepthBits) << kDepthBits) | (uint64_t)d;
  return kk | ((uint64_t)idx << ((kMaxDepth - d) * 3 + kDepthBits));
}

// Spread the low 19 bits of v so bit b lands at bit 3b.
__host__ __device__ inline uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x7FFFFu;
  x = (x | (x << 32)) & 0x001F00000000FFFFull;
  x = (x | (x << 16)) & 0x001F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// CalcFinestKey (sfc_morton.h:387-402): per level z, y, x from high to low,
// then AppendDepth(k, 19).  Only the low 19 bits of each anchor take part,
// exactly as the reference's `(anchor[d] & mask) >> shift` loop.
__host__ __device__ inline uint64_t finest_key(int ax, int ay, int az) {
  uint64_t k = (spread3((uint32_t)az) << 2) | (spread3((uint32_t)ay) << 1) | spread3((uint32_t)ax);
  return (k << kDepthBits) | (uint64_t)kMaxDepth;
}

// The reference's (int) conversion of a double on x86-64 (cvttsd2si):
// truncation in range, INT_MIN for NaN or out of range.
__host__ __device__ inline int to_int_x86(double v) {
  if (v > -2147483649.0 && v < 2147483648.0) return (int)v;
  return (int)0x80000000u;
}

}  // namespace tb
