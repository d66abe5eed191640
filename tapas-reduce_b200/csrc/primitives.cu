// Device primitives of libtapas_b200: exclusive scan and LSD radix sort.
//
// Both are written for HBM bandwidth on sm_100a: one read and one write of the
// data per pass, tiles of 4096 elements per 512-thread block, block partials
// reduced by a single small kernel, and the radix scatter staged through
// shared memory so global writes are runs, not scattered words.  The radix
// sort is stable (keys with equal digits keep their input order), so equal
// Morton keys stay in input order.
#include "primitives.cuh"

namespace tb {

// ---------------------------------------------------------------------------
// Exclusive scan of int32 (block-local scan + scan of block sums + add).
// ---------------------------------------------------------------------------
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns block total.
__device__ __forceinline__ int block_excl_scan(int v, int *smem_warp, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  int incl = warp_incl_scan(v);
  if (lane == 31) smem_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nwarps ? smem_warp[lane] : 0;
    int wi = warp_incl_scan(w);
    if (lane < nwarps) smem_warp[lane] = wi - w;
    if (lane == nwarps - 1) smem_warp[32] = wi;
  }
  __syncthreads();
  total = smem_warp[32];
  int r = incl - v + smem_warp[warp];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles(const int32_t *__restrict__ in,
                                                           int32_t *__restrict__ out, int64_t n,
                                                           int32_t *__restrict__ block_sums) {
  __shared__ int sw[33];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    int64_t g = base + i;
    v[i] = g < n ? in[g] : 0;
    s += v[i];
  }
  int total;
  int off = block_excl_scan(s, sw, total);
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    int64_t g = base + i;
    if (g < n) out[g] = off;
    off += v[i];
  }
  if (threadIdx.x == 0 && block_sums) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_add(int32_t *__restrict__ out, int64_t n,
                                                         const int32_t *__restrict__ block_offs) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  const int add = block_offs[blockIdx.x];
  for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
    int64_t g = base + i;
    if (g < n) out[g] += add;
  }
}

// Sum of the last input and last output element = total.
__global__ void scan_total(const int32_t *in, const int32_t *out, int64_t n, int32_t *total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

}  // namespace

// Scan of in[0..n) into out using scratch[scratch_off..) for the block sums of
// this level and the levels below (recursive reduce-then-scan).
static int scan_level(tapas_b200_ctx *ctx, const int32_t *in, int32_t *out, int64_t n,
                      size_t scratch_off) {
  cudaStream_t s = ctx->stream;
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 1) {
    scan_tiles<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
    TB_LAUNCH_CHECK(ctx);
    return TAPAS_B200_OK;
  }
  int32_t *sums = ctx->scan_tmp.p + scratch_off;
  int32_t *offs = sums + nb + 32;
  scan_tiles<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, sums);
  TB_LAUNCH_CHECK(ctx);
  TB_TRY(scan_level(ctx, sums, offs, nb, scratch_off + 2 * (size_t)nb + 64));
  scan_add<<<(unsigned)nb, kScanThreads, 0, s>>>(out, n, offs);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

int scan_exclusive(tapas_b200_ctx *ctx, const int32_t *in, int32_t *out, int64_t n,
                   int32_t *d_total) {
  cudaStream_t s = ctx->stream;
  if (n <= 0) {
    if (d_total) TB_CUDA(ctx, cudaMemsetAsync(d_total, 0, sizeof(int32_t), s));
    return TAPAS_B200_OK;
  }
  if (n > (int64_t)0x7FFFFFFF) {
    set_error(ctx, "scan: %lld elements exceed int32 offsets", (long long)n);
    return TAPAS_B200_ERR_CAPACITY;
  }
  // scratch for every level: sum over levels of 2 * blocks + 64
  size_t need = 64;
  for (int64_t m = n; m > kScanTile;) {
    const int64_t nb = (m + kScanTile - 1) / kScanTile;
    need += 2 * (size_t)nb + 64;
    m = nb;
  }
  TB_CUDA(ctx, ctx->scan_tmp.ensure(need, s));
  TB_TRY(scan_level(ctx, in, out, n, 0));
  if (d_total) {
    scan_total<<<1, 32, 0, s>>>(in, out, n, d_total);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

// ---------------------------------------------------------------------------
// LSD radix sort of 64-bit keys with optional 32-bit values.
//
// Per pass (8-bit digit): (1) per-tile digit histogram, stored digit-major
// [256][ntiles]; (2) one block per digit scans its row over tiles, and the
// digit totals are scanned inside (3); (3) each tile ranks its elements
// stably (the lanes sharing a digit found with one warp ballot per digit
// bit), sorts them by digit in shared memory and writes them out as
// contiguous runs; its keys are loaded before the digit bases, so the two
// sets of loads overlap.
// ---------------------------------------------------------------------------
namespace {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;   // per thread
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096

__device__ __forceinline__ uint32_t digit_of(uint64_t k, int shift) {
  return (uint32_t)(k >> shift) & (kRadix - 1);
}

__global__ void __launch_bounds__(kSortThreads) radix_hist(const uint64_t *__restrict__ keys,
                                                           int64_t n, int shift,
                                                           uint32_t *__restrict__ hist,
                                                           int ntiles) {
  __shared__ uint32_t h[kRadix];
  for (int i = threadIdx.x; i < kRadix; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile;
  for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
    int64_t g = base + i;
    if (g < n) atomicAdd(&h[digit_of(keys[g], shift)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[(size_t)d * ntiles + blockIdx.x] = h[d];
}

// One block per digit: exclusive scan of hist[d][*] in place; total in totals[d].
__global__ void __launch_bounds__(1024) radix_scan_rows(uint32_t *__restrict__ hist, int ntiles,
                                                        uint32_t *__restrict__ totals) {
  __shared__ uint32_t sw[33];
  __shared__ uint32_t carry;
  const int d = blockIdx.x;
  uint32_t *row = hist + (size_t)d * ntiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int start = 0; start < ntiles; start += blockDim.x) {
    int i = start + threadIdx.x;
    uint32_t v = i < ntiles ? row[i] : 0;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) sw[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0;
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      sw[lane] = wi - w;
      if (lane == 31) sw[32] = wi;
    }
    __syncthreads();
    uint32_t c = carry;
    if (i < ntiles) row[i] = c + incl - v + sw[warp];
    __syncthreads();
    if (threadIdx.x == 0) carry = c + sw[32];
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[d] = carry;
}

template <bool kHasVals>
__global__ void __launch_bounds__(kSortThreads) radix_scatter(
    const uint64_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
    uint64_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, int64_t n, int shift,
    const uint32_t *__restrict__ hist, const uint32_t *__restrict__ totals, int ntiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // Layout: per-warp digit counters [kSortWarps][kRadix], digit start in tile
  // [kRadix], global digit base [kRadix], keys [kSortTile], vals [kSortTile].
  uint32_t *wcnt = reinterpret_cast<uint32_t *>(smem_raw);
  uint32_t *tstart = wcnt + kSortWarps * kRadix;
  uint32_t *gbase = tstart + kRadix;
  uint64_t *skeys = reinterpret_cast<uint64_t *>(gbase + kRadix);
  uint32_t *svals = reinterpret_cast<uint32_t *>(skeys + kSortTile);

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += blockDim.x) wcnt[i] = 0;
  // this thread's keys (and values), in flight during the digit-base loads
  const int64_t tile0 = (int64_t)blockIdx.x * kSortTile;
  uint64_t k[kSortItems];
  uint32_t v[kSortItems];
#pragma unroll
  for (int it = 0; it < kSortItems; it++) {
    const int64_t g = tile0 + (int64_t)warp * (32 * kSortItems) + it * 32 + lane;
    k[it] = g < n ? keys_in[g] : ~0ull;
    if (kHasVals) v[it] = g < n ? vals_in[g] : 0u;
  }

  // Global base per digit = exclusive scan of totals + this tile's row offset.
  if (threadIdx.x < 32) {
    // 256 digits scanned by one warp, 8 per lane.
    uint32_t loc[kRadix / 32];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kRadix / 32; j++) {
      loc[j] = totals[lane * (kRadix / 32) + j];
      s += loc[j];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    uint32_t run = incl - s;
#pragma unroll
    for (int j = 0; j < kRadix / 32; j++) {
      int d = lane * (kRadix / 32) + j;
      gbase[d] = run + hist[(size_t)d * ntiles + blockIdx.x];
      run += loc[j];
    }
  }
  __syncthreads();

  // Warp-striped ownership: item k of lane l in warp w is tile element
  // w*(32*kSortItems) + k*32 + l, so (warp, round, lane) is input order.
  uint32_t rank[kSortItems];
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < kSortItems; it++) {
    int64_t g = tile0 + (int64_t)warp * (32 * kSortItems) + it * 32 + lane;
    bool valid = g < n;
    uint32_t d = valid ? digit_of(k[it], shift) : 0xFFFFFFFFu;
    unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < kRadixBits; b++) {
      const bool bit = (d >> b) & 1u;
      const unsigned bb = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bb : ~bb;
    }
    if (valid) {
      uint32_t before = wcnt[warp * kRadix + d];
      rank[it] = before + __popc(peers & lt_mask);
      int leader = __ffs(peers) - 1;
      __syncwarp(peers);
      if (lane == leader) wcnt[warp * kRadix + d] = before + __popc(peers);
    } else {
      rank[it] = 0;
    }
    __syncwarp();
  }
  __syncthreads();

  // Exclusive scan over (digit, warp) of the warp counters -> tile offsets.
  // Thread t < kRadix handles digit t: prefix over warps; then digit starts
  // are scanned across digits.
  uint32_t dsum = 0;
  if (threadIdx.x < kRadix) {
    const int d = threadIdx.x;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
      uint32_t c = wcnt[w * kRadix + d];
      wcnt[w * kRadix + d] = dsum;
      dsum += c;
    }
  }
  __syncthreads();
  {
    __shared__ uint32_t ws[kRadix / 32 + 1];
    if (threadIdx.x < kRadix) {
      uint32_t incl = dsum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) ws[warp] = incl;
      __syncwarp();
      tstart[threadIdx.x] = incl - dsum;  // warp-local exclusive
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int w = 0; w < kRadix / 32; w++) {
        uint32_t t = ws[w];
        ws[w] = run;
        run += t;
      }
    }
    __syncthreads();
    if (threadIdx.x < kRadix) tstart[threadIdx.x] += ws[threadIdx.x >> 5];
    __syncthreads();
  }

  // Place elements sorted by digit in shared memory.
#pragma unroll
  for (int it = 0; it < kSortItems; it++) {
    int64_t g = tile0 + (int64_t)warp * (32 * kSortItems) + it * 32 + lane;
    if (g < n) {
      uint32_t d = digit_of(k[it], shift);
      uint32_t pos = tstart[d] + wcnt[warp * kRadix + d] + rank[it];
      skeys[pos] = k[it];
      if (kHasVals) svals[pos] = v[it];
    }
  }
  __syncthreads();

  // Write out: element i of the sorted tile goes to gbase[d] + (i - tstart[d]).
  const int64_t cnt = (n - tile0) < kSortTile ? (n - tile0) : kSortTile;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    uint64_t kk = skeys[i];
    uint32_t d = digit_of(kk, shift);
    uint64_t dst = (uint64_t)gbase[d] + (uint64_t)(i - (int)tstart[d]);
    keys_out[dst] = kk;
    if (kHasVals) vals_out[dst] = svals[i];
  }
}

size_t scatter_smem_bytes() {
  return sizeof(uint32_t) * (kSortWarps * kRadix + 2 * kRadix) + sizeof(uint64_t) * kSortTile +
         sizeof(uint32_t) * kSortTile;
}

}  // namespace

int radix_sort(tapas_b200_ctx *ctx, uint64_t *&keys, uint64_t *&keys_alt, uint32_t *&vals,
               uint32_t *&vals_alt, int64_t n, int begin_bit, int end_bit) {
  if (n <= 1) return TAPAS_B200_OK;
  if (n > (int64_t)0x7FFFFFFF) {
    set_error(ctx, "radix_sort: n=%lld exceeds 2^31-1", (long long)n);
    return TAPAS_B200_ERR_ARG;
  }
  cudaStream_t s = ctx->stream;
  const int ntiles = (int)((n + kSortTile - 1) / kSortTile);
  TB_CUDA(ctx, ctx->sort_hist.ensure((size_t)kRadix * ntiles + kRadix, s));
  uint32_t *hist = ctx->sort_hist.p;
  uint32_t *totals = hist + (size_t)kRadix * ntiles;
  const size_t smem = scatter_smem_bytes();
  const bool hv = vals != nullptr;
  // Per device and per function; cheap enough to set on every call.
  if (hv)
    TB_CUDA(ctx, cudaFuncSetAttribute(radix_scatter<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else
    TB_CUDA(ctx, cudaFuncSetAttribute(radix_scatter<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int shift = begin_bit; shift < end_bit; shift += kRadixBits) {
    radix_hist<<<ntiles, kSortThreads, 0, s>>>(keys, n, shift, hist, ntiles);
    TB_LAUNCH_CHECK(ctx);
    radix_scan_rows<<<kRadix, 1024, 0, s>>>(hist, ntiles, totals);
    TB_LAUNCH_CHECK(ctx);
    if (hv)
      radix_scatter<true><<<ntiles, kSortThreads, smem, s>>>(keys, vals, keys_alt, vals_alt, n,
                                                             shift, hist, totals, ntiles);
    else
      radix_scatter<false><<<ntiles, kSortThreads, smem, s>>>(keys, nullptr, keys_alt, nullptr, n,
                                                              shift, hist, totals, ntiles);
    TB_LAUNCH_CHECK(ctx);
    uint64_t *tk = keys; keys = keys_alt; keys_alt = tk;
    if (hv) { uint32_t *tv = vals; vals = vals_alt; vals_alt = tv; }
  }
  return TAPAS_B200_OK;
}

}  // namespace tb
