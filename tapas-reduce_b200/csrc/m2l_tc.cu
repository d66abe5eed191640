// M2L on the 5th-generation tensor cores (mixed form).
//
// The spherical M2L (ex/LaplaceSphericalCPU_tapas.h:208-273) is real-linear
// in the source multipole: with M and L stored as real vectors of length
// K = 2*P(P+1)/2 (re, im per coefficient), L_t += T(c_t - c_s) M_s.  After
// scaling every cell's M_n by w^-n and L_j by w^(j+1) (w = cell width), T
// depends only on the translation's class: the level difference
// delta = depth_t - depth_s and the integer offset
// D = (c_t - c_s) / (w_min / 2) (centres of cells are odd multiples of half
// their width from the cube corner, so D is an integer vector).  Every M2L
// pair of a class is then one row of a dense GEMM
//     Lt[targets of pairs, :] += Mt[sources of pairs, :] * T_class^T (K x K).
//
// Execution:
//  1. classify: class key per M2L pair; stable radix sort of the pairs by key
//     (the target order inside a class is kept); segments = classes.
//  2. classes with >= kTcMin pairs run on the tensor cores; the rest (and
//     pairs whose offset does not fit the key) are listed for the FP64
//     kernel, which takes them one warp per pair.
//  3. per tensor-core class the real K x K operator is built in FP64 from the
//     unit-width singular harmonics and split into TF32 hi + lo parts, laid
//     out as K-major core matrices (8 rows x 16 bytes) ready for smem.
//  4. GEMM kernel, warp-specialised: a CTA takes tiles of 128 pairs of one
//     class; producer warps stream the sources' FP32 multipole rows
//     (cp.async, split into TF32 hi + lo in shared memory) and the operator's
//     K chunks (bulk copies of its hi and lo rows) through a shared-memory
//     ring; one thread issues tcgen05.mma kind::tf32 (M=128
//     pairs, N = the operator rows the chunk reaches, K=8) three times per
//     k-step (hi*hi + lo*hi + hi*lo: split-precision "3xTF32", FP32
//     accumulation in TMEM).  An output of degree j reads only sources of
//     degree n < P - j, so with outputs in degree order the rows a K-chunk
//     reaches are a prefix that shrinks along K: at P = 15 the chunks need
//     976 operator rows in all instead of 15 x 240, which divides the MMA
//     work and the operator bytes by 2.2.  Epilogue warps read a finished
//     accumulator with tcgen05.ld (one pair per TMEM lane, 32 outputs per
//     load) and add each pair's row into its target's Lt with vector
//     fire-and-forget reductions, while the next tile accumulates in the
//     second TMEM buffer.  All hand-offs are mbarriers with bounded waits.
//  5. Lt is rescaled and added into the FP64 L.
#include <algorithm>
#include <optional>

#include "expansions.cuh"
#include "kernels.cuh"
#include "m2l_tc.cuh"
#include "primitives.cuh"

namespace tb {
namespace {

constexpr int kTcMin = 16;         // pairs needed for a class to use the tensor cores
constexpr int kNTile = 128;        // pairs per tile (MMA N)
constexpr int kOffBias = 8192;

// kDense: every K-chunk reaches every operator row (the M2M operators of the
// tree translations, whose zero structure differs from M2L's).
template <int P, bool kDense = false>
struct TcShape {
  static constexpr int NT = P * (P + 1) / 2;
  static constexpr int K = 2 * NT;                    // real dimension
  static constexpr int NPAD = (K + 15) / 16 * 16;     // operator rows = MMA N (<= 2 MMAs)
  static constexpr int KC = 16;                       // K chunk per ring stage
  static constexpr int KP = ((K + KC - 1) / KC) * KC; // padded K (== NPAD)
  static constexpr int NKC = KP / KC;
  // TMEM accumulators of 128 lanes x NPAD columns: two (double-buffered
  // epilogue) at a 256-column stride when they fit in the 512 columns
  static constexpr int BSTRIDE = NPAD <= 128 ? 128 : 256;
  static constexpr int TBUF = NPAD <= 256 ? 2 : 1;
  static constexpr int TMEM_COLS = TBUF * BSTRIDE <= 256 && NPAD <= 256 ? 256 : 512;
  // one stage: multipole rows hi/lo (128 x KC) + operator rows hi/lo (NPAD x KC)
  static constexpr int STAGE_FLOATS = 2 * kNTile * KC + 2 * NPAD * KC;
  // the epilogue's transpose buffers: per epilogue warp 32 pairs x 32 outputs
  // at a row stride of 36 floats (conflict-free 16-byte accesses)
  static constexpr int EPI_STRIDE = 36;
  static constexpr int EPI_FLOATS = 8 * 32 * EPI_STRIDE;
  // stages of the copy ring: as many as the rest of ~220 KB of shared memory
  // holds (at most 6), and at most NKC + 1, so the copies run at most one
  // tile ahead
  static constexpr int NS_SMEM =
      (220 * 1024 - EPI_FLOATS * (int)sizeof(float)) / (STAGE_FLOATS * (int)sizeof(float));
  static constexpr int NS_CAP = NS_SMEM < 6 ? NS_SMEM : 6;
  static constexpr int NS = NS_CAP < NKC + 1 ? NS_CAP : NKC + 1;
  static_assert(NS >= 2, "the copy ring needs two stages");
  static constexpr size_t SMEM = ((size_t)NS * STAGE_FLOATS + EPI_FLOATS) * sizeof(float) + 1024;
  // Chunk kc holds source coefficients 8 kc .. 8 kc + 7, of degree >= nmin;
  // the outputs of degree j < P - nmin, the first (P - nmin)(P - nmin + 1)
  // real rows, are the ones it reaches (rounded up to the MMA's N step).
  static constexpr int nmin(int kc) {
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= (KC / 2) * kc) n++;
    return n;
  }
  static constexpr int nrows(int kc) {
    if (kDense) return NPAD;
    const int r = ((P - nmin(kc)) * (P - nmin(kc) + 1) + 15) / 16 * 16;
    return r < NPAD ? r : NPAD;
  }
  // An operator is stored as its chunks' reached rows only (FP32, K-major
  // core matrices): chunk kc at choff(kc), OPS_FLOATS per operator.
  static constexpr int choff(int kc) {
    int o = 0;
    for (int k = 0; k < kc; k++) o += nrows(k) * KC;
    return o;
  }
  static constexpr int OPS_FLOATS = choff(NKC);
};

// ---------------------------------------------------------------------------
// classification
// ---------------------------------------------------------------------------
// Offset class of an M2L pair: the level difference delta = depth_t - depth_s
// and D = (c_t - c_s) / (w_min / 2), an integer vector; false when a cell is
// empty (no work) or the offset is not a whole number of half-widths or too
// large for the operator's key (those pairs stay on the FP64 kernel).
__device__ __forceinline__ int pair_class(int t, int s, const int32_t *__restrict__ cnb,
                                          const int32_t *__restrict__ clevel,
                                          const double *__restrict__ cmin,
                                          const double *__restrict__ cmax,
                                          const double *__restrict__ ccen, int &delta,
                                          long long D[3]) {
  if (cnb[s] == 0 || cnb[t] == 0) return 0;  // empty
  delta = clevel[t] - clevel[s];
  const double wt = cmax[3 * t] - cmin[3 * t], ws = cmax[3 * s] - cmin[3 * s];
  const double half = 0.5 * fmin(wt, ws);
  bool ok = delta > -32 && delta < 32;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double r = (ccen[3 * t + d] - ccen[3 * s + d]) / half;
    D[d] = llrint(r);
    ok = ok && fabs(r - (double)D[d]) < 1e-3 && D[d] > -kOffBias && D[d] < kOffBias;
  }
  return ok ? 2 : 1;  // 2: a class; 1: FP64
}

// Largest |D| component and |delta| over the classed pairs (for the key width).
__global__ void class_ranges(int64_t n, const uint64_t *__restrict__ list, int shift,
                             const int32_t *__restrict__ cnb, const int32_t *__restrict__ clevel,
                             const double *__restrict__ cmin, const double *__restrict__ cmax,
                             const double *__restrict__ ccen, int *__restrict__ ranges) {
  const uint64_t mask = (1ull << shift) - 1;
  int md = 0, ml = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t v = list[e];
    int delta;
    long long D[3];
    if (pair_class((int)(v >> shift), (int)(v & mask), cnb, clevel, cmin, cmax, ccen, delta,
                   D) == 2) {
      md = max(md, (int)max(llabs(D[0]), max(llabs(D[1]), llabs(D[2]))));
      ml = max(ml, abs(delta));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    md = max(md, __shfl_xor_sync(0xffffffffu, md, o));
    ml = max(ml, __shfl_xor_sync(0xffffffffu, ml, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(ranges, md);
    atomicMax(ranges + 1, ml);
  }
}

// Sort key of a class, as narrow as the lists allow: delta + bd in the top db
// bits, then D_z, D_y, D_x + bo in cb bits each; the two largest codes of the
// (db + 3 cb + 1)-bit range mark empty and FP64 pairs.
struct KeyPack {
  int cb, db, bo, bd, bits;
  __host__ __device__ uint64_t empty() const { return (1ull << bits) - 1; }
  __host__ __device__ uint64_t rare() const { return (1ull << bits) - 2; }
  __device__ uint64_t pack(int delta, const long long D[3]) const {
    return ((uint64_t)(delta + bd) << (3 * cb)) | ((uint64_t)(D[2] + bo) << (2 * cb)) |
           ((uint64_t)(D[1] + bo) << cb) | (uint64_t)(D[0] + bo);
  }
  // the operator builder's fixed 48-bit form of a packed class
  __device__ uint64_t wide(uint64_t k) const {
    const uint64_t m = (1ull << cb) - 1;
    const long long dx = (long long)(k & m) - bo, dy = (long long)((k >> cb) & m) - bo,
                    dz = (long long)((k >> (2 * cb)) & m) - bo;
    const int delta = (int)(k >> (3 * cb)) - bd;
    return ((uint64_t)(delta + 32) << 42) | ((uint64_t)(dz + kOffBias) << 28) |
           ((uint64_t)(dy + kOffBias) << 14) | (uint64_t)(dx + kOffBias);
  }
};

// Sort key per pair.  Also the pairs' field ranges (as class_ranges) into
// ranges[0..1], and in *overflow the classed pairs outside kp's ranges (kp
// taken from an earlier list); those get the FP64 code, and a nonzero count
// means the keys must be rebuilt with the new ranges.
__global__ void classify_pairs(int64_t n, const uint64_t *__restrict__ list, int shift,
                               const int32_t *__restrict__ cnb,
                               const int32_t *__restrict__ clevel,
                               const double *__restrict__ cmin, const double *__restrict__ cmax,
                               const double *__restrict__ ccen, KeyPack kp,
                               uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                               int *__restrict__ ranges, int *__restrict__ overflow) {
  const uint64_t mask = (1ull << shift) - 1;
  int md = 0, ml = 0, over = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t v = list[e];
    int delta = 0;
    long long D[3];
    int kind =
        pair_class((int)(v >> shift), (int)(v & mask), cnb, clevel, cmin, cmax, ccen, delta, D);
    if (kind == 2) {
      const int d = (int)max(llabs(D[0]), max(llabs(D[1]), llabs(D[2])));
      md = max(md, d);
      ml = max(ml, abs(delta));
      if (d > kp.bo || abs(delta) > kp.bd) {
        kind = 1;
        over++;
      }
    }
    keys[e] = kind == 0 ? kp.empty() : (kind == 1 ? kp.rare() : kp.pack(delta, D));
    vals[e] = (uint32_t)e;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    md = max(md, __shfl_xor_sync(0xffffffffu, md, o));
    ml = max(ml, __shfl_xor_sync(0xffffffffu, ml, o));
    over += __shfl_xor_sync(0xffffffffu, over, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(ranges, md);
    atomicMax(ranges + 1, ml);
    if (over) atomicAdd(overflow, over);
  }
}

__global__ void segment_flags(const uint64_t *__restrict__ keys, int64_t n,
                              int32_t *__restrict__ flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// seg_start[c] = first sorted index of class c (c = scan value at a boundary)
__global__ void segment_starts(const int32_t *__restrict__ flag, const int32_t *__restrict__ scan,
                               int64_t n, int32_t *__restrict__ seg_start) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (flag[i]) seg_start[scan[i]] = (int32_t)i;
}

// per class: is it a tensor-core class?
__global__ void class_tc_flags(const int32_t *__restrict__ seg_start, int64_t nseg, int64_t n,
                               const uint64_t *__restrict__ keys, KeyPack kp, int64_t min_count,
                               int32_t *__restrict__ tcflag, int32_t *__restrict__ ntiles) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nseg;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = seg_start[c], e = (c + 1 < nseg) ? seg_start[c + 1] : n;
    const uint64_t k = keys[b];
    const bool tc = (k != kp.empty()) && (k != kp.rare()) && (e - b) >= min_count;
    tcflag[c] = tc ? 1 : 0;
    ntiles[c] = tc ? (int32_t)((e - b + kNTile - 1) / kNTile) : 0;
  }
}

// Pairs of non-tensor-core classes (except empty-source pairs) go to FP64.
// Appends the list index of every pair of a class left to FP64 to pairs64
// (order set by the atomics; *n64 counts them).
__global__ void mark_fp64_pairs(const int32_t *__restrict__ scan, const int32_t *__restrict__ flag,
                                const int32_t *__restrict__ tcflag,
                                const uint64_t *__restrict__ keys, KeyPack kp,
                                const uint32_t *__restrict__ vals, int64_t n,
                                uint32_t *__restrict__ pairs64, int *__restrict__ n64) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = base + threadIdx.x;
    bool fp64 = false;
    if (i < n) {
      const int cls = scan[i] + flag[i] - 1;  // inclusive scan - 1
      fp64 = keys[i] != kp.empty() && !tcflag[cls];
    }
    const unsigned mask = __ballot_sync(0xffffffffu, fp64);
    if (mask) {
      int b = 0;
      if (lane == __ffs(mask) - 1) b = atomicAdd(n64, __popc(mask));
      b = __shfl_sync(0xffffffffu, b, __ffs(mask) - 1);
      if (fp64) pairs64[b + __popc(mask & ((1u << lane) - 1))] = vals[i];
    }
  }
}

// Sharded evaluation: the sorted pairs whose target this context computes
// (ownership bit 0), each with the selection its class got over ALL pairs,
// so a pair takes the same path (GEMM or FP64 pair kernel) as in one context.
__global__ void owned_pair_flags(const uint32_t *__restrict__ vals, int64_t n,
                                 const uint64_t *__restrict__ list, int shift,
                                 const uint8_t *__restrict__ own, const int32_t *__restrict__ scan,
                                 const int32_t *__restrict__ flag,
                                 const int32_t *__restrict__ tcflag, int32_t *__restrict__ oflag,
                                 uint8_t *__restrict__ sel) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    oflag[i] = own[(int64_t)(list[vals[i]] >> shift)] & 1;
    sel[i] = (uint8_t)tcflag[scan[i] + flag[i] - 1];
  }
}

// Stable compaction of the owned sorted pairs (pos = exclusive scan of oflag).
__global__ void compact_owned_pairs(const int32_t *__restrict__ oflag,
                                    const int32_t *__restrict__ pos, int64_t n,
                                    const uint64_t *__restrict__ keys,
                                    const uint32_t *__restrict__ vals,
                                    const uint8_t *__restrict__ sel, uint64_t *__restrict__ keys2,
                                    uint32_t *__restrict__ vals2, uint8_t *__restrict__ sel2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!oflag[i]) continue;
    const int32_t p = pos[i];
    keys2[p] = keys[i];
    vals2[p] = vals[i];
    sel2[p] = sel[i];
  }
}

// Per class of the compacted pairs: its selection and tile count.
__global__ void class_flags_from_sel(const int32_t *__restrict__ seg_start, int64_t nseg,
                                     int64_t n, const uint8_t *__restrict__ sel,
                                     int32_t *__restrict__ tcflag, int32_t *__restrict__ ntiles) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nseg;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = seg_start[c], e = (c + 1 < nseg) ? seg_start[c + 1] : n;
    const bool tc = sel[b] != 0;
    tcflag[c] = tc ? 1 : 0;
    ntiles[c] = tc ? (int32_t)((e - b + kNTile - 1) / kNTile) : 0;
  }
}

struct TileItem {
  int32_t cls;    // tensor-core class index (operator slot)
  int32_t start;  // first sorted pair index
  int32_t len;    // pairs in this tile (<= kNTile)
  int32_t pad;
};

__global__ void build_tiles(const int32_t *__restrict__ seg_start, int64_t nseg, int64_t n,
                            const int32_t *__restrict__ tcflag, const int32_t *__restrict__ tcid,
                            const int32_t *__restrict__ tile_off,
                            const uint64_t *__restrict__ keys, KeyPack kp,
                            uint64_t *__restrict__ tc_keys, TileItem *__restrict__ items,
                            int2 *__restrict__ cls_range, int *__restrict__ tc_pairs) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nseg;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (!tcflag[c]) continue;
    const int64_t b = seg_start[c], e = (c + 1 < nseg) ? seg_start[c + 1] : n;
    const int id = tcid[c];
    tc_keys[id] = kp.wide(keys[b]);
    cls_range[id] = make_int2((int)b, (int)(e - b));
    atomicAdd(tc_pairs, (int)(e - b));
    int64_t o = tile_off[c];
    for (int64_t p = b; p < e; p += kNTile, o++) {
      TileItem it;
      it.cls = id;
      it.start = (int32_t)p;
      it.len = (int32_t)min((int64_t)kNTile, e - p);
      it.pad = 0;
      items[o] = it;
    }
  }
}

// Region of each tile: the octant (at tree level kRegionLevel) of its first
// pair's target, as a sort key, with the tile's index as the value.
constexpr int kRegionLevel = 2;
__global__ void tile_regions(const TileItem *__restrict__ items, int64_t nitems,
                             const uint32_t *__restrict__ sorted_vals,
                             const uint64_t *__restrict__ list, int shift,
                             const uint64_t *__restrict__ ckey, uint64_t *__restrict__ rkey,
                             uint32_t *__restrict__ rval) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nitems;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(list[sorted_vals[items[i].start]] >> shift);
    rkey[i] = (ckey[t] >> (kDepthBits + 3 * (kMaxDepth - kRegionLevel))) &
              ((1u << (3 * kRegionLevel)) - 1);
    rval[i] = (uint32_t)i;
  }
}

__global__ void gather_items(const TileItem *__restrict__ in, const uint32_t *__restrict__ order,
                             int64_t nitems, TileItem *__restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nitems;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[order[i]];
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Per-chunk tables of a shape (filled by one thread): reached rows nr[kc]
// and operator offsets co[kc] (co[NKC] = OPS_FLOATS).
template <class S>
__device__ __forceinline__ void chunk_tables(int *nr, int *co) {
  int o = 0;
  for (int kc = 0; kc < S::NKC; kc++) {
    nr[kc] = S::nrows(kc);
    co[kc] = o;
    o += nr[kc] * S::KC;
  }
  co[S::NKC] = o;
}

// Offset of operator entry (row r, column c) within an operator; the entry
// must lie in a row its chunk reaches (r < nr[c / KC]).
template <class S>
__device__ __forceinline__ int op_offset(const int *co, int r, int c) {
  return co[c / S::KC] + (r / 8) * (S::KC / 4 * 32) + ((c % S::KC) / 4) * 32 + (r % 8) * 4 +
         (c % 4);
}

// One block per tensor-core class: unit-offset singular harmonics (evalLocal,
// :102-135) in FP64, then every real operator entry the GEMM reads, rounded to
// FP32 and split into TF32 hi + lo (the class's hi rows, then its lo rows).
template <int P>
__global__ void __launch_bounds__(256) build_operators(const uint64_t *__restrict__ tc_keys,
                                                       float *__restrict__ ops) {
  using S = TcShape<P>;
  __shared__ cd Y[P * P];
  __shared__ double scale[P];                        // (w_s / w_t)^n = 2^(delta n)
  __shared__ unsigned char deg[S::NT], ord[S::NT];   // (j, k) of coefficient t
  __shared__ int nr[S::NKC], co[S::NKC + 1];
  if (threadIdx.x == 0) chunk_tables<S>(nr, co);
  const int cls = blockIdx.x;
  const uint64_t key = tc_keys[cls];
  const int delta = (int)((key >> 42) & 63) - 32;
  const double Dx = (double)((long long)(key & 16383) - kOffBias);
  const double Dy = (double)((long long)((key >> 14) & 16383) - kOffBias);
  const double Dz = (double)((long long)((key >> 28) & 16383) - kOffBias);
  // offset in units of the target width: D * 2^(min(delta,0) - 1)
  const double u = ldexp(1.0, min(delta, 0) - 1);
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
  float *op = ops + (size_t)cls * 2 * S::OPS_FLOATS;
  // one thread per complex (output, input) pair: its real 2 x 2 block
  for (int idx = threadIdx.x; idx < (S::NPAD / 2) * (S::KP / 2); idx += blockDim.x) {
    const int to = idx / (S::KP / 2), ti = idx % (S::KP / 2);  // complex output / input
    if (2 * to >= nr[(2 * ti) / S::KC]) continue;  // a row its chunk does not reach
    double v00 = 0, v01 = 0, v10 = 0, v11 = 0;  // [row re/im][column re/im]
    if (2 * to < S::K && 2 * ti < S::K) {
      const int j = deg[to], k = ord[to], n = deg[ti], ma = ord[ti];
      if (n < P - j) {
        const double Cnm = oddeven(j);
        const int base = (j + n) * (j + n) + j + n - k;
        // m = +ma term: M * Cnm2 * Y[j+n, ma-k]
        const double C2 = Cnm * oddeven((k - ma) * (k < ma) + ma);
        const cd Yp = Y[base + ma];
        v00 = C2 * Yp.x;
        v01 = -C2 * Yp.y;
        v10 = C2 * Yp.y;
        v11 = C2 * Yp.x;
        // m = -ma term (ma > 0): conj(M) * Cnm * Y[j+n, -ma-k]
        if (ma > 0) {
          const cd Ym = Y[base - ma];
          v00 += Cnm * Ym.x;
          v01 += Cnm * Ym.y;
          v10 += Cnm * Ym.y;
          v11 += -Cnm * Ym.x;
        }
        const double sc = scale[n];  // exact: a power of two in the normal range
        v00 *= sc; v01 *= sc; v10 *= sc; v11 *= sc;
      }
    }
    const double v[4] = {v00, v01, v10, v11};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int o = op_offset<S>(co, 2 * to + (e >> 1), 2 * ti + (e & 1));
      const float x = (float)v[e], hi = tf32_round(x);
      op[o] = hi;
      op[S::OPS_FLOATS + o] = tf32_round(x - hi);
    }
  }
}

// Per cell c (one warp each): Mt[c][2t + (0: re, 1: im)] = M[c][t] / w^n
// (n = degree of t, w = the cell's width) in FP32; the GEMM splits each row
// into TF32 hi + lo as it stages it.
template <int P>
__global__ void __launch_bounds__(256) normalize_M(int64_t ncells, const int32_t *__restrict__ cnb,
                                                   const double *__restrict__ cmin,
                                                   const double *__restrict__ cmax,
                                                   const double2 *__restrict__ M,
                                                   float *__restrict__ Mt) {
  using S = TcShape<P>;
  constexpr int kSlots = (S::KP + 31) / 32;
  __shared__ double pw[8][P];  // per warp: w^-n
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  int deg[kSlots];
#pragma unroll
  for (int r = 0; r < kSlots; r++) {
    const int kk = lane + 32 * r;
    int j = 0, k;
    if (kk < S::K) jk_of(kk >> 1, j, k);
    deg[r] = j;
  }
  const int64_t nw = (int64_t)gridDim.x * 8;
  for (int64_t c = (int64_t)blockIdx.x * 8 + wi; c < ncells; c += nw) {
    const bool live = cnb[c] > 0;
    __syncwarp();
    if (live && lane < P) pw[wi][lane] = pow(cmax[3 * c] - cmin[3 * c], -lane);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kSlots; r++) {
      const int kk = lane + 32 * r;
      if (kk >= S::KP) continue;
      float v = 0.f;
      if (live && kk < S::K) {
        const double2 z = M[c * S::NT + (kk >> 1)];
        v = (float)(((kk & 1) ? z.y : z.x) * pw[wi][deg[r]]);
      }
      Mt[c * S::KP + kk] = v;
    }
  }
}

// Per cell c (one warp each): L[c][t] += Lt[c][t] / w^(j+1) (j = degree of t).
template <int P>
__global__ void __launch_bounds__(256) add_scaled_L(int64_t ncells, const int32_t *__restrict__ cnb,
                                                    const double *__restrict__ cmin,
                                                    const double *__restrict__ cmax,
                                                    const float *__restrict__ Lt,
                                                    double2 *__restrict__ L) {
  using S = TcShape<P>;
  constexpr int kSlots = (S::NT + 31) / 32;
  __shared__ double pw[8][P + 1];  // per warp: w^-n, n = 0..P
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  int deg[kSlots];
#pragma unroll
  for (int r = 0; r < kSlots; r++) {
    const int t = lane + 32 * r;
    int j = 0, k;
    if (t < S::NT) jk_of(t, j, k);
    deg[r] = j;
  }
  const int64_t nw = (int64_t)gridDim.x * 8;
  for (int64_t c = (int64_t)blockIdx.x * 8 + wi; c < ncells; c += nw) {
    if (cnb[c] == 0) continue;  // warp-uniform
    __syncwarp();
    if (lane <= P) pw[wi][lane] = pow(cmax[3 * c] - cmin[3 * c], -lane);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kSlots; r++) {
      const int t = lane + 32 * r;
      if (t >= S::NT) continue;
      const double sc = pw[wi][deg[r] + 1];
      const float2 lt = *reinterpret_cast<const float2 *>(Lt + c * S::KP + 2 * t);
      const double2 o = L[c * S::NT + t];
      L[c * S::NT + t] = make_double2(o.x + (double)lt.x * sc, o.y + (double)lt.y * sc);
    }
  }
}

// ---------------------------------------------------------------------------
// tcgen05 helpers (inline PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}


__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, absolute LBO mode, SWIZZLE_NONE (layout type 0)
  return d;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z),
        "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
        "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------------------
// the GEMM kernel
// ---------------------------------------------------------------------------
// 16-byte asynchronous global -> shared copy (L2 only); with src_bytes = 0
// the destination is zero-filled and nothing is read.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}
// Arrive on `bar` once all of this thread's earlier cp.async copies have landed
// (the barrier's expected count includes this arrival).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Bulk copy of `bytes` (a multiple of 16) global -> shared, completing on `bar`.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Wait for the phase of `bar` with the given parity; gives up (false) when
// another role has raised *abort or after `limit` clock cycles (by default
// 4e9, about 2 s), then raising *abort.
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t parity, volatile int *abort,
                                           long long limit) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort) return false;
    if (clock64() - t0 > limit) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

// MMAs of one k-chunk: KC/8 k-steps of three tf32 MMAs (hi*hi, lo*hi,
// hi*lo) of the 128 multipole rows (A) against the operator rows the chunk
// reaches (B, N = nrows(kc), as two MMAs where that exceeds 256) into TMEM
// columns dcol + [0, N).  a_*: the chunk's multipole rows, b_*: its operator
// rows, both K-major core matrices.
template <int P, bool kDense = false>
__device__ __forceinline__ void issue_chunk_mmas(uint32_t dcol, uint32_t a_hi, uint32_t a_lo,
                                                 uint32_t b_hi, uint32_t b_lo, int kc, int nr) {
  using S = TcShape<P, kDense>;
  const uint32_t LBO = 128;                  // adjacent k-cores
  const uint32_t SBO = (S::KC / 4) * 128;    // adjacent 8-row groups
#pragma unroll
  for (int s = 0; s < S::KC / 8; s++) {
    const uint32_t koff = (uint32_t)s * 256u;  // two k-cores
    const uint64_t ah = umma_desc(a_hi + koff, LBO, SBO);
    const uint64_t al = umma_desc(a_lo + koff, LBO, SBO);
    const uint32_t acc = (kc > 0 || s > 0) ? 1u : 0u;
#pragma unroll
    for (int n0 = 0; n0 < S::NPAD; n0 += 256) {
      if (n0 >= nr) break;
      const int nn = nr - n0 < 256 ? nr - n0 : 256;
      // instruction descriptor: D f32, A/B tf32, K-major both, N = nn, M = 128
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(nn >> 3) << 17) |
                             ((uint32_t)(128 >> 4) << 24);
      const uint32_t boff = (uint32_t)(n0 / 8) * SBO + koff;
      const uint64_t bh = umma_desc(b_hi + boff, LBO, SBO);
      const uint64_t bl = umma_desc(b_lo + boff, LBO, SBO);
      const uint32_t d = dcol + (uint32_t)n0;
      umma_tf32(d, ah, bh, idesc, acc);
      umma_tf32(d, al, bh, idesc, 1u);
      umma_tf32(d, ah, bl, idesc, 1u);
    }
  }
}

__device__ __forceinline__ void red_add_v4(float *p, uint32_t a, uint32_t b, uint32_t c,
                                           uint32_t d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(__uint_as_float(a)),
               "f"(__uint_as_float(b)), "f"(__uint_as_float(c)), "f"(__uint_as_float(d))
               : "memory");
}

// Warp roles of the GEMM kernel.
constexpr int kProdThreads = 256;  // warps 0-7: copies into the stage ring
constexpr int kEpiWarp0 = 8;       // warps 8-15: epilogue (TMEM lane quarter warp % 4,
constexpr int kEpiWarps = 8;       //   column half (warp - 8) / 4)
constexpr int kMmaWarp = 16;       // warp 16: TMEM allocation, MMA issue (lane 0)
constexpr int kSplitWarp0 = 17;    // warps 17-24: split the staged rows into hi + lo
constexpr int kSplitThreads = 256;
constexpr int kThreadsTc = 32 * 25;

// Persistent CTA over the tiles blockIdx.x, blockIdx.x + gridDim.x, ...,
// warp-specialised; the roles meet only at mbarriers:
//  - producers (warps 0-7) walk the (tile, k-chunk) steps through an NS-stage
//    ring: every producer cp.async-copies its share of the 128 gathered
//    multipole rows (A, FP32; lanes of a warp cover whole row segments) and
//    arrives on landed[stage] when they have landed; thread 0 bulk-copies
//    the operator rows the chunk reaches (B, contiguous, split into TF32 hi
//    and lo when they were built), which complete on landed[stage] too.  A
//    stage is refilled after the MMAs that read it commit to empty[stage].
//  - the split warps (17-24) wait for landed[stage], split the multipole
//    rows into TF32 hi + lo in place and arrive on full[stage].
//  - the MMA thread (warp 16, lane 0) waits for full[stage], issues the
//    chunk's 3xTF32 MMAs into one of TBUF TMEM accumulators and commits them
//    to empty[stage]; after a tile's last chunk it commits to tfull[buffer].
//  - the epilogue warps (8-15) wait for tfull[buffer], read the accumulator
//    with tcgen05.ld (TMEM lane = pair, column = output) and add each pair's
//    outputs into its target's Lt row, then arrive on tempty[buffer], which
//    the MMA thread waits for before reusing it; with two TMEM buffers the
//    epilogue of tile i overlaps the MMAs of tile i+1.
// Every wait is bounded and also gives up when another role has aborted; the
// CTA then drains its copies and its MMAs before freeing TMEM.
template <int P, bool kDense = false>
__global__ void __launch_bounds__(kThreadsTc, 1) m2l_tc_kernel(
    const TileItem *__restrict__ items, int64_t nitems, const uint32_t *__restrict__ sorted_vals,
    const uint64_t *__restrict__ list, int shift, const float *__restrict__ ops,
    const float *__restrict__ Mt, float *__restrict__ Lt, int *__restrict__ err,
    long long wait_limit) {
  using S = TcShape<P, kDense>;
  constexpr int NS = S::NS;
  constexpr int NB = S::TBUF;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  float *base = reinterpret_cast<float *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t landed[NS], full[NS], empty[NS], tfull[2], tempty[2], fin;
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  __shared__ int nr_sh[S::NKC], co_sh[S::NKC + 1];  // reached operator rows, offsets
  volatile int *abort = &abort_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint64_t mask = (1ull << shift) - 1;
  if (tid == 0) {
    for (int i = 0; i < NS; i++) {
      mbar_init(&landed[i], kProdThreads + 1);
      mbar_init(&full[i], kSplitThreads);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], kEpiWarps);
    }
    mbar_init(&fin, 1);
    abort_sh = 0;
    chunk_tables<S>(nr_sh, co_sh);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_sh)),
                 "r"((uint32_t)S::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  const int64_t ntiles = nitems > (int64_t)blockIdx.x
                             ? (nitems - 1 - (int64_t)blockIdx.x) / gridDim.x + 1
                             : 0;
  const int64_t nsteps = ntiles * S::NKC;
  auto item_of = [&](int64_t jt) { return items[(int64_t)blockIdx.x + jt * gridDim.x]; };

  if (warp < kEpiWarp0) {
    // ---------------- producers ----------------
    // A: each row chunk is KC floats = PPR 16-byte pieces.  A warp copies 8
    // rows x PPR pieces (PPR <= 4): lane l takes row l % 8 of the warp's
    // group and piece l / 8, so its shared-memory writes fill whole core
    // matrices (8 rows x 16 bytes, no bank conflicts) and each row's chunk is
    // read as PPR x 16 contiguous bytes.  Thread t copies rows arow0 + i * RPP
    // (RPP = rows per pass of all producers, i < NRT) and fetches their
    // sources and the tile's class one tile ahead.
    constexpr int PPR = S::KC / 4;
    static_assert(PPR <= 4, "a warp covers 8 rows x PPR pieces");
    constexpr int RPW = 32 / PPR;  // rows per warp instruction
    constexpr int RPP = (kProdThreads / 32) * RPW;
    constexpr int NRT = kNTile / RPP;
    const int apiece = (tid & 31) / RPW, arow0 = (tid >> 5) * RPW + (tid & 31) % RPW;
    int cur_src[NRT], nxt_src[NRT];
    int cur_cls = 0, nxt_cls = 0;
    auto fetch = [&](int64_t jt) {
      nxt_cls = 0;
      TileItem it;
      it.len = 0;
      it.start = 0;
      if (jt < ntiles) {
        it = item_of(jt);
        nxt_cls = it.cls;
      }
#pragma unroll
      for (int i = 0; i < NRT; i++) {
        const int row = arow0 + i * RPP;
        nxt_src[i] = row < it.len ? (int)(list[sorted_vals[it.start + row]] & mask) : -1;
      }
    };
    fetch(0);
    int64_t issued = 0;
    for (int64_t step = 0; step < nsteps; step++) {
      const int st = (int)(step % NS);
      if (step >= NS &&
          !wait_phase(&empty[st], (uint32_t)((step / NS - 1) & 1), abort, wait_limit))
        break;
      const int64_t jt = step / S::NKC;
      const int kc = (int)(step % S::NKC);
      if (kc == 0) {
#pragma unroll
        for (int i = 0; i < NRT; i++) cur_src[i] = nxt_src[i];
        cur_cls = nxt_cls;
      }
      float *sA_hi = base + (size_t)st * S::STAGE_FLOATS;
      float *sB_hi = sA_hi + 2 * kNTile * S::KC;
      if (tid == 0) {
        // the chunk's operator rows (the ones it reaches), TF32 hi and lo
        const size_t boff = (size_t)cur_cls * 2 * S::OPS_FLOATS + (size_t)co_sh[kc];
        const uint32_t bbytes = (uint32_t)(nr_sh[kc] * S::KC * sizeof(float));
        mbar_expect_tx(&landed[st], 2 * bbytes);
        bulk_copy(sB_hi, ops + boff, bbytes, &landed[st]);
        bulk_copy(sB_hi + S::NPAD * S::KC, ops + boff + S::OPS_FLOATS, bbytes, &landed[st]);
      }
#pragma unroll
      for (int i = 0; i < NRT; i++) {
        const int row = arow0 + i * RPP;
        const bool have = cur_src[i] >= 0;
        const size_t aoff = (size_t)(have ? cur_src[i] : 0) * S::KP + (size_t)kc * S::KC +
                            4 * apiece;
        const int o = ((row >> 3) * PPR + apiece) * 32 + (row & 7) * 4;
        cp_async16(sA_hi + o, Mt + aoff, have ? 16u : 0u);
      }
      cp_async_arrive_noinc(&landed[st]);
      issued = step + 1;
      // the next tile's sources (a chain of dependent loads), after this
      // tile's first copies are on their way
      if (kc == 0) fetch(jt + 1);
    }
    cp_async_wait_all();
    if (tid == 0 && *abort) {
      // bulk copies of steps the MMA thread may not have consumed: let them land
      for (int64_t s = issued > NS ? issued - NS : 0; s < issued; s++) {
        const long long t0 = clock64();
        while (!mbar_try_wait(&full[s % NS], (uint32_t)((s / NS) & 1)) &&
               clock64() - t0 < 200000000LL) {
        }
      }
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      for (int64_t jt = 0; jt < ntiles && !*abort; jt++) {
        const int b = NB == 2 ? (int)(jt & 1) : 0;
        const int64_t use_b = NB == 2 ? (jt >> 1) : jt;
        if (use_b >= 1 && !wait_phase(&tempty[b], (uint32_t)((use_b - 1) & 1), abort, wait_limit)) break;
        tc_fence_after();
        const uint32_t dcol = tmem + (uint32_t)(b * S::BSTRIDE);
        bool ok = true;
        for (int kc = 0; kc < S::NKC; kc++) {
          const int64_t step = jt * S::NKC + kc;
          const int st = (int)(step % NS);
          if (!wait_phase(&full[st], (uint32_t)((step / NS) & 1), abort, wait_limit)) {
            ok = false;
            break;
          }
          fence_async_smem();  // the cp.async rows are visible to the tensor core
          tc_fence_after();
          float *sA_hi = base + (size_t)st * S::STAGE_FLOATS;
          float *sA_lo = sA_hi + kNTile * S::KC;
          float *sB_hi = sA_lo + kNTile * S::KC;
          float *sB_lo = sB_hi + S::NPAD * S::KC;
          issue_chunk_mmas<P, kDense>(dcol, smem_u32(sA_hi), smem_u32(sA_lo), smem_u32(sB_hi),
                                      smem_u32(sB_lo), kc, nr_sh[kc]);
          umma_commit(&empty[st]);
        }
        if (!ok) break;
        umma_commit(&tfull[b]);
      }
      // every MMA issued so far has completed before TMEM is freed
      umma_commit(&fin);
      const long long t0 = clock64();
      while (!mbar_try_wait(&fin, 0) && clock64() - t0 < 400000000LL) {
      }
    }
    __syncwarp();
  } else if (warp >= kSplitWarp0) {
    // ---------------- split ----------------
    // once a stage's FP32 multipole rows (and its operator rows, split when
    // they were built) have landed, the 256 threads split the multipole rows
    // into TF32 hi + lo in place (16 bytes at a time), then arrive on
    // full[stage]
    const int t = tid - kSplitWarp0 * 32;
    auto split4 = [](float *hi_p, float *lo_p) {
      const float4 x = *reinterpret_cast<const float4 *>(hi_p);
      float4 hi, lo;
      hi.x = tf32_round(x.x); lo.x = tf32_round(x.x - hi.x);
      hi.y = tf32_round(x.y); lo.y = tf32_round(x.y - hi.y);
      hi.z = tf32_round(x.z); lo.z = tf32_round(x.z - hi.z);
      hi.w = tf32_round(x.w); lo.w = tf32_round(x.w - hi.w);
      *reinterpret_cast<float4 *>(hi_p) = hi;
      *reinterpret_cast<float4 *>(lo_p) = lo;
    };
    for (int64_t step = 0; step < nsteps; step++) {
      const int st = (int)(step % NS);
      const int kc = (int)(step % S::NKC);
      if (!wait_phase(&landed[st], (uint32_t)((step / NS) & 1), abort, wait_limit)) break;
      float *sA_hi = base + (size_t)st * S::STAGE_FLOATS;
      float *sA_lo = sA_hi + kNTile * S::KC;
#pragma unroll
      for (int i = 0; i < (kNTile * S::KC) / (4 * kSplitThreads); i++) {
        const int o = 4 * (t + i * kSplitThreads);
        split4(sA_hi + o, sA_lo + o);
      }
      fence_async_smem();  // the split rows are visible to the tensor core
      mbar_arrive(&full[st]);
    }
  } else {
    // ---------------- epilogue ----------------
    // warp (q, h): TMEM lanes 32 q .. 32 q + 31 (pairs of the tile), column
    // groups of 32 outputs g = h, h + 2, ...  Each 32 x 32 block goes through
    // the warp's shared-memory buffer so that one reduction instruction adds
    // 4 pairs x 32 consecutive outputs (4 rows of Lt, 128 bytes each).
    const int q = warp & 3;
    const int h = (warp - kEpiWarp0) >> 2;
    constexpr int NG = (S::NPAD + 31) / 32;
    float *xb = base + (size_t)NS * S::STAGE_FLOATS + (warp - kEpiWarp0) * 32 * S::EPI_STRIDE;
    int tg = -1, tg_next = -1;  // target of this lane's pair, this tile and the next
    auto load_target = [&](int64_t jt) {
      TileItem it;
      it.len = 0;
      it.start = 0;
      if (jt < ntiles) it = item_of(jt);
      const int p = q * 32 + lane;
      return p < it.len ? (int)(list[sorted_vals[it.start + p]] >> shift) : -1;
    };
    tg_next = load_target(0);
    for (int64_t jt = 0; jt < ntiles; jt++) {
      const int b = NB == 2 ? (int)(jt & 1) : 0;
      const int64_t use_b = NB == 2 ? (jt >> 1) : jt;
      tg = tg_next;
      tg_next = load_target(jt + 1);
      if (!wait_phase(&tfull[b], (uint32_t)(use_b & 1), abort, wait_limit)) break;
      tc_fence_after();
#pragma unroll 1
      for (int g = h; g < NG; g += 2) {
        uint32_t v[32];
        const uint32_t taddr =
            tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * S::BSTRIDE + g * 32);
        tmem_ld32(taddr, v);
#pragma unroll
        for (int c = 0; c < 32; c += 4)
          *reinterpret_cast<uint4 *>(xb + lane * S::EPI_STRIDE + c) =
              make_uint4(v[c], v[c + 1], v[c + 2], v[c + 3]);
        __syncwarp();
        const int c4 = 4 * (lane & 7);
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int pr = 4 * k + (lane >> 3);
          const int t = __shfl_sync(0xffffffffu, tg, pr);
          const uint4 w = *reinterpret_cast<const uint4 *>(xb + pr * S::EPI_STRIDE + c4);
          if (t >= 0 && g * 32 + c4 < S::NPAD)
            red_add_v4(Lt + (size_t)t * S::KP + g * 32 + c4, w.x, w.y, w.z, w.w);
        }
        __syncwarp();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
    }
  }
  __syncthreads();
  if (tid == 0 && abort_sh) atomicExch(err, 1);
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)S::TMEM_COLS)
                 : "memory");
  }
}

}  // namespace

// Offset classes of the current M2L list (steps 1-2 and the class/tile
// tables of the header comment), for a GEMM whose operators take op_bytes per
// class: ctx->tc holds the pairs sorted by class (vals), the selected
// classes' wide keys (tc_keys), (first sorted pair, pair count) (cls_range)
// and 128-pair tiles (items), and the list indices of the pairs left to the
// FP64 pair path (pairs64).
int m2l_classes(tapas_b200_ctx *ctx, size_t op_bytes, int64_t min_pairs, M2LClassInfo &info) {
  cudaStream_t s = ctx->stream;
  info = M2LClassInfo{};
  int64_t n = ctx->n_m2l;  // pairs to evaluate here (sharded: of owned targets)
  auto &T = ctx->tc;
  // 1. classify + stable sort by class key
  TB_CUDA(ctx, T.keys.ensure(n + 1, s));
  TB_CUDA(ctx, T.keys_alt.ensure(n + 1, s));
  TB_CUDA(ctx, T.vals.ensure(n + 1, s));
  TB_CUDA(ctx, T.vals_alt.ensure(n + 1, s));
  TB_CUDA(ctx, T.pairs64.ensure(n + 1, s));
  if (n == 0) return TAPAS_B200_OK;
  // Key width from the lists' largest offsets.  The ranges of the previous
  // classification are tried first (classify_pairs reports the current ranges
  // and the pairs that do not fit); only a first call or a miss runs the
  // separate range pass.
  TB_CUDA(ctx, T.err.ensure(8, s));
  TB_CUDA(ctx, ctx->pinned.ensure(256));
  int32_t *h = reinterpret_cast<int32_t *>(ctx->pinned.p);
  KeyPack kp;
  for (bool fresh = !T.kp_cached;; fresh = true) {
    TB_CUDA(ctx, cudaMemsetAsync(T.err.p, 0, 8 * sizeof(int), s));
    if (fresh) {
      class_ranges<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(
          n, ctx->m2l.p, ctx->list_shift, ctx->cnb.p, ctx->clevel.p, ctx->cmin.p, ctx->cmax.p,
          ctx->ccen.p, T.err.p + 2);
      TB_LAUNCH_CHECK(ctx);
      TB_CUDA(ctx, cudaMemcpyAsync(h, T.err.p + 2, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   s));
      TB_CUDA(ctx, cudaStreamSynchronize(s));
      T.kp_bo = h[0];
      T.kp_bd = h[1];
      T.kp_cached = true;
    }
    auto bits_for = [](int64_t range) {  // bits holding 0..range
      int b = 1;
      while (((int64_t)1 << b) <= range) b++;
      return b;
    };
    kp.bo = T.kp_bo;
    kp.bd = T.kp_bd;
    kp.cb = bits_for(2 * (int64_t)kp.bo);
    kp.db = bits_for(2 * (int64_t)kp.bd);
    kp.bits = kp.db + 3 * kp.cb + 1;
    classify_pairs<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(
        n, ctx->m2l.p, ctx->list_shift, ctx->cnb.p, ctx->clevel.p, ctx->cmin.p, ctx->cmax.p,
        ctx->ccen.p, kp, T.keys.p, T.vals.p, T.err.p + 4, T.err.p + 6);
    TB_LAUNCH_CHECK(ctx);
    if (fresh) break;
    TB_CUDA(ctx, cudaMemcpyAsync(h, T.err.p + 4, 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    if (h[2] == 0) {
      // every pair fits; the next classification packs with this list's ranges
      T.kp_bo = h[0];
      T.kp_bd = h[1];
      break;
    }
  }
  {
    uint64_t *k = T.keys.p, *ka = T.keys_alt.p;
    uint32_t *v = T.vals.p, *va = T.vals_alt.p;
    TB_TRY(radix_sort(ctx, k, ka, v, va, n, 0, kp.bits));
    if (k != T.keys.p) { std::swap(T.keys.p, T.keys_alt.p); std::swap(T.keys.cap, T.keys_alt.cap); }
    if (v != T.vals.p) { std::swap(T.vals.p, T.vals_alt.p); std::swap(T.vals.cap, T.vals_alt.cap); }
  }
  // 2. segments = classes
  TB_CUDA(ctx, T.flag.ensure(n + 1, s));
  TB_CUDA(ctx, T.scan.ensure(n + 1, s));
  segment_flags<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(T.keys.p, n, T.flag.p);
  TB_LAUNCH_CHECK(ctx);
  TB_TRY(scan_exclusive(ctx, T.flag.p, T.scan.p, n, T.scan.p + n));
  TB_CUDA(ctx, cudaMemcpyAsync(h, T.scan.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  int64_t nseg = h[0];
  TB_CUDA(ctx, T.seg_start.ensure(nseg + 1, s));
  TB_CUDA(ctx, T.tcflag.ensure(nseg + 1, s));
  TB_CUDA(ctx, T.tcid.ensure(nseg + 1, s));
  TB_CUDA(ctx, T.ntiles.ensure(nseg + 1, s));
  TB_CUDA(ctx, T.tile_off.ensure(nseg + 1, s));
  segment_starts<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(T.flag.p, T.scan.p, n,
                                                                    T.seg_start.p);
  TB_LAUNCH_CHECK(ctx);
  // Operator memory is bounded: when more classes qualify than the budget
  // holds, only the most populated ones run on the tensor cores.
  int64_t min_count = min_pairs;
  {
    const int64_t max_classes = std::max<int64_t>(1, (int64_t)(ctx->tc_op_budget / op_bytes));
    if (nseg > max_classes) {
      std::vector<int32_t> st(nseg);
      TB_CUDA(ctx, cudaMemcpyAsync(st.data(), T.seg_start.p, sizeof(int32_t) * nseg,
                                   cudaMemcpyDeviceToHost, s));
      TB_CUDA(ctx, cudaStreamSynchronize(s));
      std::vector<int64_t> cnt(nseg);
      for (int64_t c = 0; c < nseg; c++) cnt[c] = (c + 1 < nseg ? st[c + 1] : n) - st[c];
      std::nth_element(cnt.begin(), cnt.begin() + (max_classes - 1), cnt.end(),
                       std::greater<int64_t>());
      min_count = std::max<int64_t>(min_pairs, cnt[max_classes - 1] + 1);
    }
  }
  class_tc_flags<<<grid_for(nseg, 256), 256, 0, s>>>(T.seg_start.p, nseg, n, T.keys.p, kp,
                                                      min_count, T.tcflag.p, T.ntiles.p);
  TB_LAUNCH_CHECK(ctx);
  int64_t nseg_all = nseg;
  if (ctx->sharded) {
    // keep the pairs whose target this context computes, with their classes'
    // selection; then the classes of what is left
    TB_CUDA(ctx, T.oflag.ensure(n + 1, s));
    TB_CUDA(ctx, T.opos.ensure(n + 1, s));
    TB_CUDA(ctx, T.sel.ensure(n + 1, s));
    TB_CUDA(ctx, T.sel2.ensure(n + 1, s));
    owned_pair_flags<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(
        T.vals.p, n, ctx->m2l.p, ctx->list_shift, ctx->cell_own.p, T.scan.p, T.flag.p,
        T.tcflag.p, T.oflag.p, T.sel.p);
    TB_LAUNCH_CHECK(ctx);
    TB_TRY(scan_exclusive(ctx, T.oflag.p, T.opos.p, n, T.opos.p + n));
    compact_owned_pairs<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(
        T.oflag.p, T.opos.p, n, T.keys.p, T.vals.p, T.sel.p, T.keys_alt.p, T.vals_alt.p,
        T.sel2.p);
    TB_LAUNCH_CHECK(ctx);
    TB_CUDA(ctx, cudaMemcpyAsync(h, T.opos.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    std::swap(T.keys.p, T.keys_alt.p); std::swap(T.keys.cap, T.keys_alt.cap);
    std::swap(T.vals.p, T.vals_alt.p); std::swap(T.vals.cap, T.vals_alt.cap);
    n = h[0];
    if (n == 0) {
      ctx->tc_classes = ctx->tc_tiles = 0;
      ctx->tc_segments = nseg_all;
      return TAPAS_B200_OK;
    }
    segment_flags<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(T.keys.p, n, T.flag.p);
    TB_LAUNCH_CHECK(ctx);
    TB_TRY(scan_exclusive(ctx, T.flag.p, T.scan.p, n, T.scan.p + n));
    TB_CUDA(ctx, cudaMemcpyAsync(h, T.scan.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TB_CUDA(ctx, cudaStreamSynchronize(s));
    nseg = h[0];
    segment_starts<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(T.flag.p, T.scan.p, n,
                                                                      T.seg_start.p);
    TB_LAUNCH_CHECK(ctx);
    class_flags_from_sel<<<grid_for(nseg, 256), 256, 0, s>>>(T.seg_start.p, nseg, n, T.sel2.p,
                                                              T.tcflag.p, T.ntiles.p);
    TB_LAUNCH_CHECK(ctx);
  }
  TB_TRY(scan_exclusive(ctx, T.tcflag.p, T.tcid.p, nseg, T.tcid.p + nseg));
  TB_TRY(scan_exclusive(ctx, T.ntiles.p, T.tile_off.p, nseg, T.tile_off.p + nseg));
  TB_CUDA(ctx, cudaMemsetAsync(T.err.p + 3, 0, sizeof(int), s));
  mark_fp64_pairs<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(
      T.scan.p, T.flag.p, T.tcflag.p, T.keys.p, kp, T.vals.p, n, T.pairs64.p, T.err.p + 3);
  TB_LAUNCH_CHECK(ctx);
  TB_CUDA(ctx, cudaMemcpyAsync(h, T.tcid.p + nseg, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaMemcpyAsync(h + 1, T.tile_off.p + nseg, sizeof(int32_t),
                               cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaMemcpyAsync(h + 2, T.err.p + 3, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  const int64_t ntc = h[0], nitems = h[1], n64 = h[2];
  ctx->tc_classes = ntc;
  ctx->tc_tiles = nitems;
  ctx->tc_segments = nseg_all;
  // 3. class tables
  TB_CUDA(ctx, T.tc_keys.ensure(ntc + 1, s));
  TB_CUDA(ctx, T.cls_range.ensure(ntc + 1, s));
  TB_CUDA(ctx, T.items.ensure((size_t)(nitems + 1) * sizeof(TileItem) / 16 + 1, s));
  TB_CUDA(ctx, T.err.ensure(4, s));
  TB_CUDA(ctx, cudaMemsetAsync(T.err.p, 0, 4 * sizeof(int), s));
  build_tiles<<<grid_for(nseg, 256), 256, 0, s>>>(T.seg_start.p, nseg, n, T.tcflag.p, T.tcid.p,
                                                   T.tile_off.p, T.keys.p, kp, T.tc_keys.p,
                                                   reinterpret_cast<TileItem *>(T.items.p),
                                                   T.cls_range.p, T.err.p + 1);
  TB_LAUNCH_CHECK(ctx);
  info.nseg = nseg;
  info.ntc = ntc;
  info.nitems = nitems;
  info.n64 = n64;
  return TAPAS_B200_OK;
}

namespace {

template <int P>
int m2l_tc_P(tapas_b200_ctx *ctx) {
  using S = TcShape<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  const int64_t n = ctx->n_m2l;
  auto &T = ctx->tc;
  std::optional<PhaseTimer> setup_timer;
  setup_timer.emplace(ctx, &ctx->timings.m2l_setup);
  M2LClassInfo ci;
  TB_TRY(m2l_classes(ctx, 2 * sizeof(float) * (size_t)S::OPS_FLOATS, kTcMin, ci));
  if (n == 0) {  // no M2L pair: every local expansion is zero
    TB_CUDA(ctx, ctx->L.ensure((size_t)C * S::NT, s));
    TB_CUDA(ctx, cudaMemsetAsync(ctx->L.p, 0, sizeof(double2) * (size_t)C * S::NT, s));
    return TAPAS_B200_OK;
  }
  const int64_t ntc = ci.ntc, nitems = ci.nitems, n64 = ci.n64;
  int32_t *h = reinterpret_cast<int32_t *>(ctx->pinned.p);
  if (ntc > 0) {
    TB_CUDA(ctx, T.ops.ensure((size_t)2 * S::OPS_FLOATS * ntc, s));
    build_operators<P><<<(unsigned)ntc, 256, 0, s>>>(T.tc_keys.p, T.ops.p);
    TB_LAUNCH_CHECK(ctx);
  }
  // 4. normalised multipoles, zeroed normalised locals
  TB_CUDA(ctx, T.Mt.ensure((size_t)C * S::KP, s));
  TB_CUDA(ctx, T.Lt.ensure((size_t)C * S::KP, s));
  if (!T.mt_ready) {  // the mixed upward pass leaves them ready
    normalize_M<P><<<grid_for(C, 8, ctx->num_sms * 8), 256, 0, s>>>(
        C, ctx->cnb.p, ctx->cmin.p, ctx->cmax.p, ctx->M.p, T.Mt.p);
    TB_LAUNCH_CHECK(ctx);
  }
  TB_CUDA(ctx, cudaMemsetAsync(T.Lt.p, 0, sizeof(float) * (size_t)C * S::KP, s));
  // Tiles in region order (stable, so by class inside a region): the CTAs,
  // which take consecutive tiles, then gather the multipole rows of one region
  // of the tree at a time, and those stay in L2 across its classes instead of
  // being read from HBM once per class.
  if (nitems > 1) {
    TB_CUDA(ctx, T.items_alt.ensure((size_t)(nitems + 1) * sizeof(TileItem) / 16 + 1, s));
    uint64_t *rk = T.keys.p, *rka = T.keys_alt.p;
    uint32_t *rv = reinterpret_cast<uint32_t *>(T.scan.p);
    uint32_t *rva = reinterpret_cast<uint32_t *>(T.flag.p);
    tile_regions<<<grid_for(nitems, 256), 256, 0, s>>>(
        reinterpret_cast<const TileItem *>(T.items.p), nitems, T.vals.p, ctx->m2l.p,
        ctx->list_shift, ctx->ckey.p, rk, rv);
    TB_LAUNCH_CHECK(ctx);
    TB_TRY(radix_sort(ctx, rk, rka, rv, rva, nitems, 0, 3 * kRegionLevel));
    gather_items<<<grid_for(nitems, 256), 256, 0, s>>>(
        reinterpret_cast<const TileItem *>(T.items.p), rv, nitems,
        reinterpret_cast<TileItem *>(T.items_alt.p));
    TB_LAUNCH_CHECK(ctx);
    std::swap(T.items.p, T.items_alt.p);
    std::swap(T.items.cap, T.items_alt.cap);
  }
  setup_timer.reset();
  // 5. FP64 part (rare classes) writes L; the GEMM adds into Lt
  TB_TRY(m2l_fp64_pairs(ctx, T.pairs64.p, n64));
  if (nitems > 0) {
    PhaseTimer t(ctx, &ctx->timings.m2l_tc);
    const TileItem *it = reinterpret_cast<const TileItem *>(T.items.p);
    const int grid = (int)std::min<int64_t>(nitems, ctx->num_sms);
    static_assert(S::SMEM <= 227 * 1024 - 4096, "shared memory");
    TB_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM));
    m2l_tc_kernel<P><<<grid, kThreadsTc, S::SMEM, s>>>(it, nitems, T.vals.p, ctx->m2l.p,
                                                        ctx->list_shift, T.ops.p, T.Mt.p, T.Lt.p,
                                                        T.err.p,
                                                        ctx->tc_wait_limit);
    TB_LAUNCH_CHECK(ctx);
  }
  add_scaled_L<P><<<grid_for(C, 8, ctx->num_sms * 8), 256, 0, s>>>(
      C, ctx->cnb.p, ctx->cmin.p, ctx->cmax.p, T.Lt.p, ctx->L.p);
  TB_LAUNCH_CHECK(ctx);
  TB_CUDA(ctx, cudaMemcpyAsync(h, T.err.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  ctx->n_m2l_tc = h[1];
  if (nitems > 0) {
    if (h[0]) {
      set_error(ctx, "m2l tensor-core kernel: a bounded wait on an MMA completion gave up");
      return TAPAS_B200_ERR_TIMEOUT;
    }
  }
  return TAPAS_B200_OK;
}

// ---------------------------------------------------------------------------
// M2M of the mixed form at the deepest levels, on the tensor cores.  With M_n
// scaled by w^-n, a child's offset from its parent is +-1/2 child width per
// axis at every level, so the M2M (ex/LaplaceSphericalCPU_tapas.h:165-206) has
// eight level-independent operators: Mt_parent(j) = sum 2^-j T_o Mt_child.  A
// level is then one GEMM launch over its (parent, child) pairs grouped by
// octant, the dense form of the M2L kernel.
// Only the deepest kTcUpLevels parent levels (and never levels 0 ..
// kFp64TreeLevels - 1) run on the tensor cores; the others stay FP64 (level
// GEMMs).  A split-TF32 translation keeps ~2^-22 of its input.  For the M2M
// that is harmless (the M2L reads the multipoles in the same split form; on a
// 16M-body sphere surface at P = 15 the tensor-core M2M moved the potential
// error by 0.3%), and the deepest three parent levels hold nearly all of a
// surface tree's cells.  The L2L stays FP64: it carries the whole local
// expansion of every ancestor, so a split-TF32 error there compounds down the
// chain and reaches the potential in full (tensor-core L2L on the deepest three
// parent levels raised the same case's error from 6.7e-7 to 9.2e-7, 4.7e-7 of
// it truncation).
// ---------------------------------------------------------------------------
constexpr int kFp64TreeLevels = 4;
constexpr int kTcUpLevels = 3;
constexpr int kTreeShift = 32;  // tree pair list entries: target << 32 | source

// M2M operator classes o (octant o), in FP32 in the dense GEMM's layout.  child0: the first child of any non-leaf cell; the offsets
// are its octants' centre offsets in child widths (exact: +-1/2).
template <int P>
__global__ void __launch_bounds__(256) build_tree_ops(const int32_t *__restrict__ cparent,
                                                      const double *__restrict__ ccen,
                                                      const double *__restrict__ cmin,
                                                      const double *__restrict__ cmax,
                                                      int64_t child0, float *__restrict__ ops) {
  using S = TcShape<P, true>;
  __shared__ cd Y[P * P];
  __shared__ unsigned char deg[S::NT], ord[S::NT];
  __shared__ int nr[S::NKC], co[S::NKC + 1];
  if (threadIdx.x == 0) chunk_tables<S>(nr, co);
  const int o = blockIdx.x;
  const int64_t c = child0 + o;
  const int p = cparent[c];
  const double wc = cmax[3 * c] - cmin[3 * c];
  double d[3];
  for (int k = 0; k < 3; k++) d[k] = (ccen[3 * p + k] - ccen[3 * c + k]) / wc;  // parent - child
  const Sph sp = sph_of(d[0], d[1], d[2]);
  if (threadIdx.x < P) multipole_column<P>(threadIdx.x, sp.r, sp.x, sp.y, sp.ei, Y);
  for (int t = threadIdx.x; t < S::NT; t += blockDim.x) {
    int j, k;
    jk_of(t, j, k);
    deg[t] = (unsigned char)j;
    ord[t] = (unsigned char)k;
  }
  __syncthreads();
  float *op = ops + (size_t)o * 2 * S::OPS_FLOATS;
  for (int idx = threadIdx.x; idx < (S::NPAD / 2) * (S::KP / 2); idx += blockDim.x) {
    const int to = idx / (S::KP / 2), ti = idx % (S::KP / 2);  // target / source coefficient
    cd a{0, 0}, b{0, 0};  // target += a * source + b * conj(source)
    if (2 * to < S::K && 2 * ti < S::K) {
      const int j = deg[to], k = ord[to], jp = deg[ti], kp = ord[ti];
      const int n = j - jp;
      if (n >= 0) {
        if (kp >= 1) {
          const int m = k - kp;
          if (m >= -n && m <= n)
            a = scal(((m >= 0) ? 1.0 : oddeven(m)) * oddeven(n), Y[n * n + n - m]);
        }
        const int m = k + kp;
        if (m <= n) b = scal(oddeven(k + n + m), Y[n * n + n - m]);
      }
      const double sc = ldexp(1.0, -j);
      a = scal(sc, a);
      b = scal(sc, b);
    }
    // [row re/im][column re/im] of the real 2 x 2 block
    const double v[4] = {a.x + b.x, b.y - a.y, a.y + b.y, a.x - b.x};
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int o = op_offset<S>(co, 2 * to + (e >> 1), 2 * ti + (e & 1));
      const float x = (float)v[e], hi = tf32_round(x);
      op[o] = hi;
      op[S::OPS_FLOATS + o] = tf32_round(x - hi);
    }
  }
}

// One level's 128-pair tiles: per_octant tiles of each octant's np pairs.
__global__ void tree_tiles(int64_t np, int64_t per_octant, TileItem *__restrict__ items) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 8 * per_octant;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = e / per_octant, st = (e - o * per_octant) * kNTile;
    TileItem it;
    it.cls = (int32_t)o;
    it.start = (int32_t)(o * np + st);
    it.len = (int32_t)(np - st < kNTile ? np - st : kNTile);
    it.pad = 0;
    items[e] = it;
  }
}

// The (parent, child) pairs of one level's M2M, octant-major: entry o * np + i
// is parent i's octant o.  c0: the level's first child.
__global__ void tree_pairs(int64_t c0, int64_t np, const int32_t *__restrict__ cparent,
                           uint64_t *__restrict__ list) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 8 * np;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = e / np, i = e - o * np;
    const uint64_t child = (uint64_t)(c0 + 8 * i + o), parent = (uint64_t)cparent[c0 + 8 * i];
    list[e] = parent << kTreeShift | child;
  }
}

__global__ void iota_u32(uint32_t *__restrict__ v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

// After a level's M2M: per parent (one warp each) its normalised FP32 sum A
// becomes the next GEMM's input row and its FP64 multipoles (A w^n).
template <int P>
__global__ void __launch_bounds__(256) finish_parents(int64_t c0, int64_t np,
                                                      const int32_t *__restrict__ cparent,
                                                      const double *__restrict__ cmin,
                                                      const double *__restrict__ cmax,
                                                      const float *__restrict__ acc,
                                                      float *__restrict__ Mt,
                                                      double2 *__restrict__ M) {
  using S = TcShape<P>;
  __shared__ double pw[8][P];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const int64_t nw = (int64_t)gridDim.x * 8;
  for (int64_t i = (int64_t)blockIdx.x * 8 + wi; i < np; i += nw) {
    const int64_t p = cparent[c0 + 8 * i];
    __syncwarp();
    if (lane < P) pw[wi][lane] = pow(cmax[3 * p] - cmin[3 * p], lane);
    __syncwarp();
    for (int kk = lane; kk < S::KP; kk += 32) Mt[p * S::KP + kk] = acc[p * S::KP + kk];
    for (int t = lane; t < S::NT; t += 32) {
      int j, k;
      jk_of(t, j, k);
      const float2 a = *reinterpret_cast<const float2 *>(acc + p * S::KP + 2 * t);
      M[p * S::NT + t] = make_double2((double)a.x * pw[wi][j], (double)a.y * pw[wi][j]);
    }
  }
}

// One level's M2M GEMM: the children's split rows translated into the parents'
// normalised rows of out (FP32, accumulated).
template <int P>
int tree_level_gemm(tapas_b200_ctx *ctx, int64_t c0, int64_t np, const float *rows,
                    float *out) {
  using S = TcShape<P, true>;
  cudaStream_t s = ctx->stream;
  auto &T = ctx->tc;
  tree_pairs<<<grid_for(8 * np, 256), 256, 0, s>>>(c0, np, ctx->cparent.p, T.tree_list.p);
  TB_LAUNCH_CHECK(ctx);
  const int64_t per_octant = (np + kNTile - 1) / kNTile;
  const int64_t nitems = 8 * per_octant;
  TB_CUDA(ctx, T.tree_items.ensure((size_t)nitems * sizeof(TileItem) / 16 + 1, s));
  tree_tiles<<<grid_for(nitems, 256), 256, 0, s>>>(np, per_octant,
                                                    reinterpret_cast<TileItem *>(T.tree_items.p));
  TB_LAUNCH_CHECK(ctx);
  static_assert(S::SMEM <= 227 * 1024 - 4096, "shared memory");
  TB_CUDA(ctx, cudaFuncSetAttribute(m2l_tc_kernel<P, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM));
  const int grid = (int)std::min<int64_t>(nitems, ctx->num_sms);
  m2l_tc_kernel<P, true><<<grid, kThreadsTc, S::SMEM, s>>>(
      reinterpret_cast<const TileItem *>(T.tree_items.p), nitems, T.iota.p, T.tree_list.p,
      kTreeShift, T.ops_tr.p, rows, out, T.err.p, ctx->tc_wait_limit);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

// Tree levels: parents at level l have their 8 children at
// [level_off[l + 1] + 8 i, ...); the number of levels with parents.
int tree_parent_levels(const tapas_b200_ctx *ctx) {
  int nlev = 0;
  for (int l = 0; l + 2 < (int)ctx->level_off.size(); l++) {
    if (ctx->level_off[l + 2] <= ctx->level_off[l + 1]) break;
    nlev = l + 1;
  }
  return nlev;
}

// The first parent level of the tensor-core M2M (levels above it: FP64).
int first_tc_tree_level(int nlev) { return std::max(kFp64TreeLevels, nlev - kTcUpLevels); }

// Pair lists, operators and the abort flag of the tree GEMMs; only for trees
// with parent levels from kFp64TreeLevels on (level 1 exists).
template <int P>
int tc_tree_prepare(tapas_b200_ctx *ctx) {
  using S = TcShape<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  auto &T = ctx->tc;
  TB_CUDA(ctx, T.tree_list.ensure((size_t)C + 8, s));
  if (T.iota_n < C) {
    TB_CUDA(ctx, T.iota.ensure((size_t)C + 8, s));
    iota_u32<<<grid_for(C + 8, 256), 256, 0, s>>>(T.iota.p, C + 8);
    TB_LAUNCH_CHECK(ctx);
    T.iota_n = C;
  }
  if (T.tr_P != P) {
    TB_CUDA(ctx, T.ops_tr.ensure((size_t)2 * TcShape<P, true>::OPS_FLOATS * 8, s));
    build_tree_ops<P><<<8, 256, 0, s>>>(ctx->cparent.p, ctx->ccen.p, ctx->cmin.p, ctx->cmax.p,
                                        ctx->level_off[1], T.ops_tr.p);
    TB_LAUNCH_CHECK(ctx);
    T.tr_P = P;
  }
  TB_CUDA(ctx, T.err.ensure(4, s));
  TB_CUDA(ctx, cudaMemsetAsync(T.err.p, 0, 4 * sizeof(int), s));
  return TAPAS_B200_OK;
}

int check_tc_abort(tapas_b200_ctx *ctx, const char *what) {
  int *h = reinterpret_cast<int *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemcpyAsync(h, ctx->tc.err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h[0]) {
    set_error(ctx, "%s tensor-core kernel: a bounded wait on an MMA completion gave up", what);
    return TAPAS_B200_ERR_TIMEOUT;
  }
  return TAPAS_B200_OK;
}

// Mixed upward after the FP32 P2M (leaf M in FP64): normalised split rows of
// every cell, tensor-core M2M for the deepest parent levels (from
// first_tc_tree_level, deepest first), FP64 level GEMMs above, the upper
// cells' rows.  Leaves ctx->M (FP64) and the M2L's input rows (tc.Mt) complete.
template <int P>
int tc_tree_upward_P(tapas_b200_ctx *ctx) {
  using S = TcShape<P>;
  cudaStream_t s = ctx->stream;
  const int64_t C = ctx->ncells;
  auto &T = ctx->tc;
  TB_CUDA(ctx, T.Mt.ensure((size_t)C * S::KP, s));
  TB_CUDA(ctx, T.Lt.ensure((size_t)C * S::KP, s));
  float *mt = T.Mt.p;
  normalize_M<P><<<grid_for(C, 8, ctx->num_sms * 8), 256, 0, s>>>(
      C, ctx->cnb.p, ctx->cmin.p, ctx->cmax.p, ctx->M.p, mt);
  TB_LAUNCH_CHECK(ctx);
  const int nlev = tree_parent_levels(ctx), l0 = first_tc_tree_level(nlev);
  if (nlev > l0) {
    TB_TRY(tc_tree_prepare<P>(ctx));
    TB_CUDA(ctx, cudaMemsetAsync(T.Lt.p, 0, sizeof(float) * (size_t)C * S::KP, s));
    for (int l = nlev - 1; l >= l0; l--) {
      const int64_t c0 = ctx->level_off[l + 1], np = (ctx->level_off[l + 2] - c0) / 8;
      if (np <= 0) continue;
      TB_TRY(tree_level_gemm<P>(ctx, c0, np, mt, T.Lt.p));
      finish_parents<P><<<grid_for(np, 8, ctx->num_sms * 8), 256, 0, s>>>(
          c0, np, ctx->cparent.p, ctx->cmin.p, ctx->cmax.p, T.Lt.p, mt, ctx->M.p);
      TB_LAUNCH_CHECK(ctx);
    }
    TB_TRY(check_tc_abort(ctx, "M2M"));
  }
  TB_TRY(fp64_m2m_levels(ctx, l0));
  // rows of the cells the FP64 levels produced (levels 0 .. l0 - 1)
  const int64_t ctop =
      std::min<int64_t>(C, ctx->level_off[std::min<size_t>(l0, ctx->level_off.size() - 1)]);
  if (ctop > 0) {
    normalize_M<P><<<grid_for(ctop, 8, ctx->num_sms * 8), 256, 0, s>>>(
        ctop, ctx->cnb.p, ctx->cmin.p, ctx->cmax.p, ctx->M.p, mt);
    TB_LAUNCH_CHECK(ctx);
  }
  T.mt_ready = true;
  return TAPAS_B200_OK;
}

#define TB_TC_DISPATCH(FN)                                                                   \
  switch (ctx->P) {                                                                          \
    case 4: return FN<4>(ctx);   case 5: return FN<5>(ctx);   case 6: return FN<6>(ctx);     \
    case 7: return FN<7>(ctx);   case 8: return FN<8>(ctx);   case 9: return FN<9>(ctx);     \
    case 10: return FN<10>(ctx); case 11: return FN<11>(ctx); case 12: return FN<12>(ctx);   \
    case 13: return FN<13>(ctx); case 14: return FN<14>(ctx); case 15: return FN<15>(ctx);   \
    case 16: return FN<16>(ctx);                                                             \
    default: break;                                                                          \
  }

}  // namespace

int tc_tree_upward(tapas_b200_ctx *ctx) {
  TB_TC_DISPATCH(tc_tree_upward_P)
  // P = 2, 3: the FP64 level GEMMs do every level
  ctx->tc.mt_ready = false;
  return fp64_m2m_levels(ctx, 1 << 20);
}

int m2l_tensorcore(tapas_b200_ctx *ctx) {
  switch (ctx->P) {
    case 4: return m2l_tc_P<4>(ctx);
    case 5: return m2l_tc_P<5>(ctx);
    case 6: return m2l_tc_P<6>(ctx);
    case 7: return m2l_tc_P<7>(ctx);
    case 8: return m2l_tc_P<8>(ctx);
    case 9: return m2l_tc_P<9>(ctx);
    case 10: return m2l_tc_P<10>(ctx);
    case 11: return m2l_tc_P<11>(ctx);
    case 12: return m2l_tc_P<12>(ctx);
    case 13: return m2l_tc_P<13>(ctx);
    case 14: return m2l_tc_P<14>(ctx);
    case 15: return m2l_tc_P<15>(ctx);
    case 16: return m2l_tc_P<16>(ctx);
    default: break;
  }
  // P = 2, 3: too small for the tensor-core tiles; the FP64 kernel does all.
  return m2l_fp64(ctx);
}

}  // namespace tb
