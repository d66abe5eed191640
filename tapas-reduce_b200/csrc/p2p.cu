// Near field (P2P) over the leaf-pair list, replacing the reference's
// vectormap_cuda_pack_kernel2 (cpp/include/tapas/vectormap_cuda.h:219-280)
// with the P2P functor of ex/LaplaceP2PCPU_tapas.h:23-44.
//
// The reference packs target leaves per source leaf and accumulates every
// pair with four CAS-loop atomics on the target attributes.  Here the list is
// grouped by TARGET leaf (CSR) and one warp owns a target leaf at a time:
//  - warps take target leaves from a global queue ordered by decreasing work
//    (nt * sum of source bodies), so long interaction lists start first;
//  - each lane keeps kR targets in registers (kR a template parameter, so no
//    issue slot is spent on unused target slots); FP64: kR = ceil(nt/32);
//    mixed: the targets take L = ceil(nt/kR) lanes and the warp holds
//    G = 32/L copies of them that split the sources, with kR chosen so that
//    kR/G (time per source) is least;
//  - source bodies are staged in the warp's shared-memory slice and read as
//    broadcasts; each target's sum is written once, without atomics.
//
// FP64 form: the reference's arithmetic (pot += qi qj / r, acc -= qi qj dX/r^3,
// r == 0 skipped), 1/r from rsqrt (1 ulp).
//
// Mixed form: FP32 arithmetic with results per unit charge.  Positions are
// kept as FP32 (hi, lo) offsets from the body's leaf centre; a source is moved
// into the target leaf's frame with an error-free sum (TwoSum) of its hi part
// and the FP64 centre difference, so the separation x_i - x_j is formed from
// ~47-bit operands and rounds once.  1/r is the hardware rsqrt (its error is far below
// the near field's summation error, so no Newton step).
// A source leaf whose box is far enough from the target's box skips the lo
// parts.  In the target frame a source coordinate is at most gap + tw/2 + sw
// in magnitude (gap: the boxes' separation along the farthest axis, tw, sw:
// the target and source widths) and every separation is at least gap, so one
// rounding of a coordinate is at most 2^-24 (gap + tw/2 + sw) / gap of the
// separation; with gap >= (tw/2 + sw) / 3 that is <= 4 * 2^-24 ~ 2.4e-7.
// Each source leaf is summed in plain FP32 and the partial is Kahan-added into
// the target's (sum, compensation) pair; the final near field is FP64.
#include <algorithm>
#include <cfloat>

#include "kernels.cuh"
#include "primitives.cuh"

namespace tb {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;
constexpr int kStage = 32;   // source bodies staged per warp at a time (one per lane)
constexpr int kMaxR = 3;     // FP64: targets per lane, leaves up to 96 bodies per pass
// mixed kernel: 4-warp CTAs, 4 per SM (<= 128 registers, 16 warps per SM), up to
// 3 targets per lane (leaves of more than 96 bodies take two passes)
constexpr int kMixedWarps = 4;
constexpr int kMixedMaxR = 3;  // most targets per lane of the mixed kernel
constexpr int kMixedThreads = 32 * kMixedWarps;

// ---------------------------------------------------------------------------
// work items: a target leaf with its source list, or a piece of a long list
// ---------------------------------------------------------------------------
// A target leaf whose source list holds more than kSplitSources bodies (a big
// leaf beside a dense region, e.g. the core of a Plummer sphere) is split into
// consecutive list ranges of about that many sources, so no single warp
// carries it alone.  A piece writes its partial sums to its own rows of a
// scratch array; split_reduce adds a leaf's pieces in order, so the result
// does not depend on which warp finished first.
constexpr int64_t kSplitSources = 32768;

struct WorkItem {
  int32_t leaf, e0, e1;  // target leaf (cell index) and its list range [e0, e1)
  int32_t pbase;         // -1: writes trg directly; else first row of its partials
};

// per non-empty leaf w: pieces k (>= 1) and partial rows (k * nt when split)
__global__ void leaf_pieces(const int32_t *__restrict__ leaves, int64_t nleaves,
                            const int32_t *__restrict__ off, const uint64_t *__restrict__ list,
                            uint64_t src_mask, const int32_t *__restrict__ cnb,
                            int32_t *__restrict__ kcnt, int32_t *__restrict__ psz) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nleaves;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int c = leaves[w];
    int64_t ns = 0;
    for (int e = off[c]; e < off[c + 1]; e++) ns += cnb[(int)(list[e] & src_mask)];
    const int64_t k = ns > kSplitSources ? (ns + kSplitSources - 1) / kSplitSources : 1;
    kcnt[w] = (int32_t)k;
    psz[w] = k > 1 ? (int32_t)(k * cnb[c]) : 0;
  }
}

// Items of leaf w at koff[w]..: cut its list greedily where the sources
// reach kSplitSources (at most k pieces; unused slots become empty pieces with
// zeroed partials).  Work key = nt * sources of the piece, for the queue.
__global__ void emit_items(const int32_t *__restrict__ leaves, int64_t nleaves,
                           const int32_t *__restrict__ off, const uint64_t *__restrict__ list,
                           uint64_t src_mask, const int32_t *__restrict__ cnb,
                           const int32_t *__restrict__ kcnt, const int32_t *__restrict__ koff,
                           const int32_t *__restrict__ poff, WorkItem *__restrict__ items,
                           uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                           double *__restrict__ part) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nleaves;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int c = leaves[w];
    const int e0 = off[c], e1 = off[c + 1], k = kcnt[w], nt = cnb[c];
    const int base = koff[w];
    int j = 0, ea = e0;
    int64_t acc = 0;
    for (int e = e0; e < e1; e++) {
      acc += cnb[(int)(list[e] & src_mask)];
      if ((k > 1 && acc >= kSplitSources && j < k - 1) || e == e1 - 1) {
        uint64_t work = (uint64_t)acc * (uint64_t)nt;
        if (work > 0xFFFFFFFFull) work = 0xFFFFFFFFull;
        items[base + j] = WorkItem{c, ea, e + 1, k > 1 ? poff[w] + j * nt : -1};
        keys[base + j] = 0xFFFFFFFFull - work;  // ascending sort -> decreasing work
        vals[base + j] = (uint32_t)(base + j);
        j++;
        ea = e + 1;
        acc = 0;
      }
    }
    if (e1 == e0) {  // no list: one empty item still writes the leaf's zero sums
      items[base] = WorkItem{c, e0, e0, -1};
      keys[base] = 0xFFFFFFFFull;
      vals[base] = (uint32_t)base;
      j = 1;
    }
    for (; j < k; j++) {  // unused pieces: empty, zero partials
      items[base + j] = WorkItem{c, e1, e1, poff[w] + j * nt};
      keys[base + j] = 0xFFFFFFFFull;
      vals[base + j] = (uint32_t)(base + j);
      for (int t = 0; t < 4 * nt; t++) part[4 * ((int64_t)poff[w] + (int64_t)j * nt) + t] = 0.0;
    }
  }
}

// trg rows of split leaves = sum of their pieces' partial rows, in piece order
__global__ void split_reduce(const int32_t *__restrict__ leaves, int64_t nleaves,
                             const int32_t *__restrict__ cbeg, const int32_t *__restrict__ cnb,
                             const int32_t *__restrict__ kcnt, const int32_t *__restrict__ poff,
                             const double *__restrict__ part, double *__restrict__ trg) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nleaves;
       w += (int64_t)gridDim.x * blockDim.x) {
    const int k = kcnt[w];
    if (k <= 1) continue;
    const int c = leaves[w], nt = cnb[c], b0 = cbeg[c];
    for (int t = 0; t < nt; t++) {
      double4 acc = make_double4(0, 0, 0, 0);
      for (int j = 0; j < k; j++) {
        const double4 v =
            reinterpret_cast<const double4 *>(part)[(int64_t)poff[w] + (int64_t)j * nt + t];
        acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
      }
      reinterpret_cast<double4 *>(trg)[b0 + t] = acc;
    }
  }
}

// Where a work item's sums go: trg rows of its leaf, or its partial rows.
__device__ __forceinline__ double4 *item_out(const WorkItem &it, int tb0, double *trg,
                                             double *part) {
  return it.pbase < 0 ? reinterpret_cast<double4 *>(trg) + tb0
                      : reinterpret_cast<double4 *>(part) + it.pbase;
}

__device__ __forceinline__ int next_leaf(int *counter, int lane) {
  int w = 0;
  if (lane == 0) w = atomicAdd(counter, 1);
  return __shfl_sync(0xffffffffu, w, 0);
}

// ---------------------------------------------------------------------------
// FP64
// ---------------------------------------------------------------------------
template <int kR>
__device__ __forceinline__ void fp64_tile(int lane, int wi, int tb0, int nt, int e0, int e1,
                                          const uint64_t *__restrict__ list, uint64_t mask,
                                          const int32_t *__restrict__ cbeg,
                                          const int32_t *__restrict__ cnb,
                                          const double *__restrict__ sx,
                                          const double *__restrict__ sy,
                                          const double *__restrict__ sz,
                                          const double *__restrict__ sq, double4 (*src)[32],
                                          double4 *__restrict__ out) {
  double xi[kR], yi[kR], zi[kR], qi[kR], pot[kR], ax[kR], ay[kR], az[kR];
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const int i = lane + 32 * r;
    const bool v = i < nt;
    xi[r] = v ? sx[tb0 + i] : 0.0;
    yi[r] = v ? sy[tb0 + i] : 0.0;
    zi[r] = v ? sz[tb0 + i] : 0.0;
    qi[r] = v ? sq[tb0 + i] : 0.0;
    pot[r] = ax[r] = ay[r] = az[r] = 0.0;
  }
  for (int e = e0; e < e1; e++) {
    const int s = (int)(list[e] & mask);
    const int sb0 = cbeg[s], ns = cnb[s];
    for (int chunk = 0; chunk < ns; chunk += 32) {
      const int cnt = min(32, ns - chunk);
      __syncwarp();
      if (lane < cnt) {
        const int j = sb0 + chunk + lane;
        src[wi][lane] = make_double4(sx[j], sy[j], sz[j], sq[j]);
      }
      __syncwarp();
      for (int k = 0; k < cnt; k++) {
        const double4 b = src[wi][k];
#pragma unroll
        for (int r = 0; r < kR; r++) {
          const double dx = xi[r] - b.x, dy = yi[r] - b.y, dz = zi[r] - b.z;
          const double R2 = dx * dx + dy * dy + dz * dz;
          if (R2 != 0) {
            const double invR = rsqrt(R2);
            const double qq = qi[r] * b.w * invR;
            const double s3 = invR * invR * qq;
            pot[r] += qq;
            ax[r] -= dx * s3;
            ay[r] -= dy * s3;
            az[r] -= dz * s3;
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const int i = lane + 32 * r;
    if (i < nt) out[i] = make_double4(pot[r], ax[r], ay[r], az[r]);
  }
}

// 3 CTAs of 8 warps per SM (<= 85 registers)
__global__ void __launch_bounds__(kThreads, 3) p2p_fp64_kernel(
    const uint32_t *__restrict__ order, int64_t nitems, int *__restrict__ counter,
    const WorkItem *__restrict__ items, const uint64_t *__restrict__ list, uint64_t src_mask,
    const int32_t *__restrict__ cbeg, const int32_t *__restrict__ cnb,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, double *__restrict__ trg, double *__restrict__ part) {
  __shared__ double4 src[kWarps][32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    const int w = next_leaf(counter, lane);
    if (w >= nitems) break;
    const WorkItem it = items[order[w]];
    if (it.pbase >= 0 && it.e0 == it.e1) continue;  // unused piece of a split list
    const int c = it.leaf;
    const int tb0 = cbeg[c], nt_all = cnb[c];
    const int e0 = it.e0, e1 = it.e1;
    double4 *out = item_out(it, tb0, trg, part);
    for (int tbase = 0; tbase < nt_all; tbase += 32 * kMaxR) {
      const int nt = min(nt_all - tbase, 32 * kMaxR);
      const int R = (nt + 31) / 32;
#define TB_FP64_TILE(RR)                                                                    \
  fp64_tile<RR>(lane, wi, tb0 + tbase, nt, e0, e1, list, src_mask, cbeg, cnb, sx, sy, sz, sq, \
                src, out + tbase)
      if (R == 1) TB_FP64_TILE(1);
      else if (R == 2) TB_FP64_TILE(2);
      else TB_FP64_TILE(3);
#undef TB_FP64_TILE
    }
  }
}

// ---------------------------------------------------------------------------
// mixed
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) prepare_rel(
    const int32_t *__restrict__ leaves, int64_t nleaves, const int32_t *__restrict__ cbeg,
    const int32_t *__restrict__ cnb, const double *__restrict__ ccen,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ sz,
    const double *__restrict__ sq, float4 *__restrict__ rel_hi, float4 *__restrict__ rel_lo) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (w >= nleaves) return;
  const int c = leaves[w];
  const int b0 = cbeg[c], nb = cnb[c];
  const double cx = ccen[3 * c], cy = ccen[3 * c + 1], cz = ccen[3 * c + 2];
  for (int b = lane; b < nb; b += 32) {
    const int i = b0 + b;
    const double rx = sx[i] - cx, ry = sy[i] - cy, rz = sz[i] - cz;
    const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
    rel_hi[i] = make_float4(hx, hy, hz, (float)sq[i]);
    rel_lo[i] = make_float4((float)(rx - hx), (float)(ry - hy), (float)(rz - hz), 0.f);
  }
}

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  const float y = __fsub_rn(v, comp);
  const float t = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(t, sum), y);
  sum = t;
}

// The same on a (sum, compensation) pair held in shared memory.
__device__ __forceinline__ void kahan_add_sm(float &sum_sm, float &comp_sm, float v) {
  float sum = sum_sm, comp = comp_sm;
  kahan_add(sum, comp, v);
  sum_sm = sum;
  comp_sm = comp;
}

// a + b = s + e exactly (Knuth's TwoSum)
__device__ __forceinline__ float two_sum(float a, float b, float &e) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return s;
}

// Shape of a mixed tile of nt targets: kR targets per lane, L = ceil(nt/kR)
// lanes per group, G = 32/L groups that split the sources.  Time per source
// ~ kR / G, so pick the kR in 1..kMaxRm that minimises it (ties: the larger
// kR, fewer shared loads per interaction).  nt <= 32 * kMaxRm.
template <int kMaxRm>
__device__ __forceinline__ void mixed_shape(int nt, int &R, int &L, int &G) {
  R = kMaxRm;
  L = (nt + kMaxRm - 1) / kMaxRm;
  G = 32 / L;
#pragma unroll
  for (int r = kMaxRm - 1; r >= 1; r--) {
    const int l = (nt + r - 1) / r;
    if (l > 32) break;
    const int g = 32 / l;
    if (r * G < R * g) {
      R = r;
      L = l;
      G = g;
    }
  }
}

// 1/sqrt(x) for normal x > 0 from the hardware approximation (relative error
// below 2^-22.9), without the denormal rescaling rsqrtf adds; callers treat
// x < FLT_MIN (a separation below ~1e-19) as coincident bodies.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// A staged source body in the target leaf's frame: FP32 hi part and charge,
// FP32 lo part.
struct __align__(16) SrcRec {
  float4 hi, lo;
};

// A source leaf of the current batch: body range and centre offset from the
// target leaf (FP64 difference as FP32 hi + lo).
struct __align__(16) LeafMeta {
  int b0, ns;
  int far;  // the leaf's box is far enough for plain FP32 coordinates (see above)
  float hx, hy, hz, lx, ly, lz;
};

// One tile of a target leaf: lane (g, l) = (lane / L, lane % L) holds targets
// l, l + L, ..., l + (kR-1) L and takes every G-th staged source.
//
// The source leaves of the target's list are read 32 at a time: lane j loads
// list entry j's leaf range and its centre offset (the FP64 difference split
// into FP32 hi + lo) into the warp's table in shared memory, so the dependent
// list -> cell loads are paid once per 32 source leaves.  Source bodies move
// through the warp's shared-memory slice 32 at a time; the next chunk's
// global loads are issued before the current chunk is computed.
template <int kR>
__device__ __forceinline__ void mixed_tile(
    int lane, int wi, int tb0, int nt, int L, int G, int e0, int e1, double tcx, double tcy,
    double tcz, double tw, const uint64_t *__restrict__ list, uint64_t mask,
    const int32_t *__restrict__ cbeg, const int32_t *__restrict__ cnb,
    const double *__restrict__ ccen, const double *__restrict__ cmin,
    const double *__restrict__ cmax, const float4 *__restrict__ rel_hi,
    const float4 *__restrict__ rel_lo, SrcRec (*ss)[kStage],
    LeafMeta (*mt)[32], double4 (*red)[32], float (*kc)[kMixedMaxR][8][32],
    double4 *__restrict__ out) {
  const int g = lane / L, tl = lane - g * L;
  const bool active = g < G;
  const int gs = active ? g : kStage;  // idle lanes skip the source loop
  // a source body this far from the target leaf's centre (max norm) is far;
  // the margin covers the FP32 rounding of the test itself
  const float far_body = (float)(tw * (5.0 / 6.0)) * (1.0f + 1e-6f);
  float txh[kR], tyh[kR], tzh[kR], txl[kR], tyl[kR], tzl[kR];
  float tp[kR], tx[kR], ty[kR], tz[kR];
  // the Kahan (sum, compensation) pairs of pot, ax, ay, az per target live in
  // the warp's shared-memory slice (touched once per source leaf), which keeps
  // the kernel at 6 CTAs per SM
  float(*kw)[8][32] = kc[wi];
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const int t = tl + L * r;
    const bool v = active && t < nt;
    const float4 h = v ? rel_hi[tb0 + t] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 l = v ? rel_lo[tb0 + t] : make_float4(0.f, 0.f, 0.f, 0.f);
    txh[r] = h.x; tyh[r] = h.y; tzh[r] = h.z;
    txl[r] = l.x; tyl[r] = l.y; tzl[r] = l.z;
#pragma unroll
    for (int k = 0; k < 8; k++) kw[r][k][lane] = 0.f;
    tp[r] = tx[r] = ty[r] = tz[r] = 0.f;
  }
  LeafMeta *const meta = mt[wi];
  for (int eb = e0; eb < e1; eb += 32) {
    const int nbat = min(32, e1 - eb);
    __syncwarp();
    if (lane < nbat) {
      const int s = (int)(list[eb + lane] & mask);
      LeafMeta m;
      m.b0 = cbeg[s];
      m.ns = cnb[s];
      // source frame -> target frame: FP64 centre difference as (hi, lo) floats
      const double dcx = ccen[3 * s] - tcx, dcy = ccen[3 * s + 1] - tcy,
                   dcz = ccen[3 * s + 2] - tcz;
      m.hx = (float)dcx; m.hy = (float)dcy; m.hz = (float)dcz;
      m.lx = (float)(dcx - m.hx); m.ly = (float)(dcy - m.hy); m.lz = (float)(dcz - m.hz);
      // boxes separated by gap along the farthest axis: every pair is >= gap apart
      const double sw = cmax[3 * s] - cmin[3 * s];
      const double gap = fmax(fabs(dcx), fmax(fabs(dcy), fabs(dcz))) - 0.5 * (tw + sw);
      m.far = 3.0 * gap >= 0.5 * tw + sw ? 1 : 0;
      meta[lane] = m;
    }
    __syncwarp();
    // first non-empty source leaf of the batch
    int j = 0;
    int ns_j = meta[0].ns;
    while (ns_j == 0 && ++j < nbat) ns_j = meta[j].ns;
    if (j >= nbat) continue;
    int ch = 0;
    float4 ph = make_float4(0.f, 0.f, 0.f, 0.f), pl = ph;
    {
      const int b0 = meta[j].b0;
      if (lane < min(kStage, ns_j)) {
        ph = rel_hi[b0 + lane];
        pl = rel_lo[b0 + lane];
      }
    }
    while (j < nbat) {
      const int cnt = min(kStage, ns_j - ch);
      __syncwarp();
      // Far bodies first (single floats), then near ones (hi, lo).  A body is
      // far when its whole leaf is, or when its max-norm distance from the
      // target leaf's centre is at least 5/6 of the leaf width: then every
      // target is >= D - tw/2 away while the coordinates are <= D and tw/2, so
      // one rounding is <= 2^-24 (D + tw/2) / (D - tw/2) <= 4 * 2^-24 of a
      // separation, the leaf rule's bound.
      int nfar;
      {
        const LeafMeta &m = meta[j];
        float ex = 0.f, ey = 0.f, ez = 0.f, ax = 0.f, ay = 0.f, az = 0.f, lx = 0.f, ly = 0.f,
              lz = 0.f;
        bool farb = true;
        if (lane < cnt) {
          ax = two_sum(ph.x, m.hx, ex);
          ay = two_sum(ph.y, m.hy, ey);
          az = two_sum(ph.z, m.hz, ez);
          lx = ex + (pl.x + m.lx);
          ly = ey + (pl.y + m.ly);
          lz = ez + (pl.z + m.lz);
          if (!m.far)
            farb = fmaxf(fabsf(ax + lx), fmaxf(fabsf(ay + ly), fabsf(az + lz))) >= far_body;
        }
        const unsigned valid = cnt >= 32 ? 0xffffffffu : ((1u << cnt) - 1u);
        const unsigned fm = __ballot_sync(0xffffffffu, farb) & valid;
        const unsigned below = (1u << lane) - 1u;
        nfar = __popc(fm);
        if (lane < cnt) {
          if (farb) {  // one float per coordinate, rounded once
            ss[wi][__popc(fm & below)].hi = make_float4(ax + lx, ay + ly, az + lz, ph.w);
          } else {
            const int k = nfar + __popc(~fm & valid & below);
            ss[wi][k].hi = make_float4(ax, ay, az, ph.w);
            ss[wi][k].lo = make_float4(lx, ly, lz, 0.f);
          }
        }
      }
      __syncwarp();
      // next chunk: the rest of this leaf, else the next non-empty leaf of the batch
      int j2 = j, ch2 = ch + kStage, ns2 = ns_j;
      const bool leaf_done = ch2 >= ns_j;
      if (leaf_done) {
        ch2 = 0;
        ns2 = 0;
        while (ns2 == 0 && ++j2 < nbat) ns2 = meta[j2].ns;
      }
      if (j2 < nbat) {
        const int b0 = meta[j2].b0;
        if (lane < min(kStage, ns2 - ch2)) {
          ph = rel_hi[b0 + ch2 + lane];
          pl = rel_lo[b0 + ch2 + lane];
        }
      }
      {
        // far bodies: plain FP32 coordinates in the target frame (relative
        // error of a separation <= ~2.4e-7), no r = 0 case
        auto far_src = [&](int k) {
          const float4 bh = ss[wi][k].hi;
#pragma unroll
          for (int r = 0; r < kR; r++) {
            const float dx = txh[r] - bh.x, dy = tyh[r] - bh.y, dz = tzh[r] - bh.z;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float ri = rsqrt_ftz(r2);
            const float qr = bh.w * ri;
            const float qr3 = qr * ri * ri;
            tp[r] += qr;
            tx[r] = fmaf(dx, qr3, tx[r]);
            ty[r] = fmaf(dy, qr3, ty[r]);
            tz[r] = fmaf(dz, qr3, tz[r]);
          }
        };
        if (G == 1) {
          // one group takes every source: unit stride, fixed offsets
#pragma unroll 4
          for (int k = active ? 0 : nfar; k < nfar; k++) far_src(k);
        } else {
#pragma unroll 2
          for (int k = gs; k < nfar; k += G) far_src(k);
        }
      }
      if (nfar < cnt) {
        // near bodies: separations from (hi, lo) coordinates
        // two sources in flight: their rsqrt latencies overlap
#pragma unroll 2
        for (int k = nfar + gs; k < cnt; k += G) {
          const float4 bh = ss[wi][k].hi;
          const float4 bl = ss[wi][k].lo;
#pragma unroll
          for (int r = 0; r < kR; r++) {
            const float dx = (txh[r] - bh.x) + (txl[r] - bl.x);
            const float dy = (tyh[r] - bh.y) + (tyl[r] - bl.y);
            const float dz = (tzh[r] - bh.z) + (tzl[r] - bl.z);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float ri = r2 >= FLT_MIN ? rsqrt_ftz(r2) : 0.f;
            const float qr = bh.w * ri;
            const float qr3 = qr * ri * ri;
            tp[r] += qr;
            tx[r] = fmaf(dx, qr3, tx[r]);
            ty[r] = fmaf(dy, qr3, ty[r]);
            tz[r] = fmaf(dz, qr3, tz[r]);
          }
        }
      }
      if (leaf_done) {
        // one source leaf summed in FP32: Kahan-add it into the target's sums
#pragma unroll
        for (int r = 0; r < kR; r++) {
          kahan_add_sm(kw[r][0][lane], kw[r][1][lane], tp[r]);
          kahan_add_sm(kw[r][2][lane], kw[r][3][lane], tx[r]);
          kahan_add_sm(kw[r][4][lane], kw[r][5][lane], ty[r]);
          kahan_add_sm(kw[r][6][lane], kw[r][7][lane], tz[r]);
          tp[r] = tx[r] = ty[r] = tz[r] = 0.f;
        }
      }
      j = j2;
      ch = ch2;
      ns_j = ns2;
    }
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kR; r++) {
    const float *k = &kw[r][0][lane];
    double4 v = make_double4((double)k[0] - (double)k[32], -((double)k[64] - (double)k[96]),
                             -((double)k[128] - (double)k[160]),
                             -((double)k[192] - (double)k[224]));
    if (G > 1) {
      __syncwarp();
      red[wi][lane] = v;
      __syncwarp();
      if (g == 0) {
        for (int gg = 1; gg < G; gg++) {
          const double4 o = red[wi][tl + gg * L];
          v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
        }
      }
    }
    const int t = tl + L * r;
    if (active && g == 0 && t < nt) out[t] = v;
  }
}

template <int kMaxRm, int kBlocks>
__global__ void __launch_bounds__(kMixedThreads, kBlocks) p2p_mixed_kernel(
    const uint32_t *__restrict__ order, int64_t nitems, int *__restrict__ counter,
    const WorkItem *__restrict__ items, const uint64_t *__restrict__ list, uint64_t src_mask,
    const int32_t *__restrict__ cbeg, const int32_t *__restrict__ cnb,
    const double *__restrict__ ccen, const double *__restrict__ cmin,
    const double *__restrict__ cmax, const float4 *__restrict__ rel_hi,
    const float4 *__restrict__ rel_lo, double *__restrict__ trg, double *__restrict__ part) {
  static_assert(kMaxRm <= kMixedMaxR, "targets per lane");
  __shared__ SrcRec ss[kMixedWarps][kStage];
  __shared__ LeafMeta mt[kMixedWarps][32];
  __shared__ double4 red[kMixedWarps][32];
  __shared__ float kc[kMixedWarps][kMixedMaxR][8][32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (;;) {
    const int w = next_leaf(counter, lane);
    if (w >= nitems) break;
    const WorkItem it = items[order[w]];
    if (it.pbase >= 0 && it.e0 == it.e1) continue;  // unused piece of a split list
    const int c = it.leaf;
    const int tb0 = cbeg[c], nt_all = cnb[c];
    const int e0 = it.e0, e1 = it.e1;
    double4 *out = item_out(it, tb0, trg, part);
    const double tcx = ccen[3 * c], tcy = ccen[3 * c + 1], tcz = ccen[3 * c + 2];
    const double tw = cmax[3 * c] - cmin[3 * c];
    for (int tbase = 0; tbase < nt_all; tbase += 32 * kMaxRm) {
      const int nt = min(nt_all - tbase, 32 * kMaxRm);
      int R, L, G;
      mixed_shape<kMaxRm>(nt, R, L, G);
#define TB_MIXED_TILE(RR)                                                                     \
  mixed_tile<RR>(lane, wi, tb0 + tbase, nt, L, G, e0, e1, tcx, tcy, tcz, tw, list, src_mask, \
                 cbeg, cnb, ccen, cmin, cmax, rel_hi, rel_lo, ss, mt, red, kc, out + tbase)
      if (R == 1) TB_MIXED_TILE(1);
      else if (R == 2) TB_MIXED_TILE(2);
      else if (kMaxRm == 3 || R == 3) TB_MIXED_TILE(3);
      else TB_MIXED_TILE(kMaxRm);
#undef TB_MIXED_TILE
    }
  }
}

// Builds the P2P work items of the current lists (ctx->p2p_items) and their
// queue order (ctx->p2p_order: items by decreasing work).
int p2p_items(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  int64_t nl = 0;
  const int32_t *leaves = work_leaves(ctx, nl);  // sharded: owned target leaves
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  TB_CUDA(ctx, ctx->p2p_kcnt.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_koff.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_psz.ensure(nl + 1, s));
  TB_CUDA(ctx, ctx->p2p_poff.ensure(nl + 1, s));
  leaf_pieces<<<grid_for(nl, 256), 256, 0, s>>>(leaves, nl, ctx->p2p_off.p, ctx->p2p.p,
                                                 mask, ctx->cnb.p, ctx->p2p_kcnt.p,
                                                 ctx->p2p_psz.p);
  TB_LAUNCH_CHECK(ctx);
  TB_TRY(scan_exclusive(ctx, ctx->p2p_kcnt.p, ctx->p2p_koff.p, nl, ctx->p2p_koff.p + nl));
  TB_TRY(scan_exclusive(ctx, ctx->p2p_psz.p, ctx->p2p_poff.p, nl, ctx->p2p_poff.p + nl));
  TB_CUDA(ctx, ctx->pinned.ensure(256));
  int32_t *h = reinterpret_cast<int32_t *>(ctx->pinned.p);
  TB_CUDA(ctx, cudaMemcpyAsync(h, ctx->p2p_koff.p + nl, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaMemcpyAsync(h + 1, ctx->p2p_poff.p + nl, sizeof(int32_t),
                               cudaMemcpyDeviceToHost, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  const int64_t ni = h[0], npart = h[1];
  if (ni < nl || npart < 0) {
    set_error(ctx, "p2p: work item count overflow");
    return TAPAS_B200_ERR_CAPACITY;
  }
  ctx->p2p_nitems = ni;
  ctx->p2p_split = npart > 0;
  TB_CUDA(ctx, ctx->p2p_items.ensure((size_t)ni * sizeof(WorkItem) / sizeof(int4) + 1, s));
  TB_CUDA(ctx, ctx->p2p_part.ensure(4 * (size_t)npart + 4, s));
  TB_CUDA(ctx, ctx->p2p_wkey.ensure(ni + 1, s));
  TB_CUDA(ctx, ctx->p2p_wkey_alt.ensure(ni + 1, s));
  TB_CUDA(ctx, ctx->p2p_order.ensure(ni + 1, s));
  TB_CUDA(ctx, ctx->p2p_order_alt.ensure(ni + 1, s));
  TB_CUDA(ctx, ctx->p2p_counter.ensure(4, s));
  emit_items<<<grid_for(nl, 256), 256, 0, s>>>(
      leaves, nl, ctx->p2p_off.p, ctx->p2p.p, mask, ctx->cnb.p, ctx->p2p_kcnt.p,
      ctx->p2p_koff.p, ctx->p2p_poff.p, reinterpret_cast<WorkItem *>(ctx->p2p_items.p),
      ctx->p2p_wkey.p, ctx->p2p_order.p, ctx->p2p_part.p);
  TB_LAUNCH_CHECK(ctx);
  uint64_t *k = ctx->p2p_wkey.p, *ka = ctx->p2p_wkey_alt.p;
  uint32_t *v = ctx->p2p_order.p, *va = ctx->p2p_order_alt.p;
  TB_TRY(radix_sort(ctx, k, ka, v, va, ni, 0, 32));
  if (v != ctx->p2p_order.p) {
    std::swap(ctx->p2p_order.p, ctx->p2p_order_alt.p);
    std::swap(ctx->p2p_order.cap, ctx->p2p_order_alt.cap);
  }
  if (k != ctx->p2p_wkey.p) {
    std::swap(ctx->p2p_wkey.p, ctx->p2p_wkey_alt.p);
    std::swap(ctx->p2p_wkey.cap, ctx->p2p_wkey_alt.cap);
  }
  TB_CUDA(ctx, cudaMemsetAsync(ctx->p2p_counter.p, 0, sizeof(int), s));
  return TAPAS_B200_OK;
}

// Adds the pieces of split leaves into trg (after a P2P kernel).
int p2p_finish(tapas_b200_ctx *ctx) {
  if (!ctx->p2p_split) return TAPAS_B200_OK;
  int64_t nl = 0;
  const int32_t *leaves = work_leaves(ctx, nl);
  split_reduce<<<grid_for(nl, 256), 256, 0, ctx->stream>>>(
      leaves, nl, ctx->cbeg.p, ctx->cnb.p, ctx->p2p_kcnt.p, ctx->p2p_poff.p,
      ctx->p2p_part.p, ctx->trg.p);
  TB_LAUNCH_CHECK(ctx);
  return TAPAS_B200_OK;
}

int p2p_grid(tapas_b200_ctx *ctx, int warps_per_block) {
  // persistent: enough warps to fill the GPU, never more than the work items
  const int64_t ni = ctx->p2p_nitems;
  int64_t g = (int64_t)ctx->num_sms * (64 / warps_per_block);
  const int64_t need = (ni + warps_per_block - 1) / warps_per_block;
  return (int)std::max<int64_t>(1, std::min(g, need));
}

}  // namespace

// Sharded: the rows of bodies another context evaluates are exactly zero, so
// the contexts' results add up without changing a bit.
static int zero_results_if_sharded(tapas_b200_ctx *ctx) {
  if (ctx->sharded)
    TB_CUDA(ctx, cudaMemsetAsync(ctx->trg.p, 0, sizeof(double) * 4 * (size_t)ctx->n, ctx->stream));
  return TAPAS_B200_OK;
}

int p2p_fp64(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  TB_TRY(zero_results_if_sharded(ctx));
  int64_t nl = 0;
  work_leaves(ctx, nl);
  if (nl == 0) return TAPAS_B200_OK;
  TB_TRY(p2p_items(ctx));
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  p2p_fp64_kernel<<<p2p_grid(ctx, kWarps), kThreads, 0, s>>>(
      ctx->p2p_order.p, ctx->p2p_nitems, ctx->p2p_counter.p,
      reinterpret_cast<const WorkItem *>(ctx->p2p_items.p), ctx->p2p.p, mask, ctx->cbeg.p,
      ctx->cnb.p, ctx->sx.p, ctx->sy.p, ctx->sz.p, ctx->sq.p, ctx->trg.p, ctx->p2p_part.p);
  TB_LAUNCH_CHECK(ctx);
  return p2p_finish(ctx);
}

int p2p_mixed(tapas_b200_ctx *ctx) {
  cudaStream_t s = ctx->stream;
  TB_TRY(zero_results_if_sharded(ctx));
  int64_t nw = 0;
  work_leaves(ctx, nw);
  if (nw == 0) return TAPAS_B200_OK;
  const int64_t nl = ctx->n_nonempty_leaves;  // every source leaf needs its offsets
  TB_CUDA(ctx, ctx->rel4.ensure(ctx->n, s));
  TB_CUDA(ctx, ctx->rel_lo.ensure(ctx->n, s));
  prepare_rel<<<(unsigned)((nl + 7) / 8), 256, 0, s>>>(ctx->leaf_list.p, nl, ctx->cbeg.p,
                                                      ctx->cnb.p, ctx->ccen.p, ctx->sx.p,
                                                      ctx->sy.p, ctx->sz.p, ctx->sq.p,
                                                      ctx->rel4.p, ctx->rel_lo.p);
  TB_LAUNCH_CHECK(ctx);
  TB_TRY(p2p_items(ctx));
  const uint64_t mask = (1ull << ctx->list_shift) - 1;
  // up to 3 targets per lane; the Kahan pairs in shared memory keep the kernel
  // at 80 registers, 24 warps per SM
  p2p_mixed_kernel<3, 6><<<p2p_grid(ctx, kMixedWarps), kMixedThreads, 0, s>>>(
      ctx->p2p_order.p, ctx->p2p_nitems, ctx->p2p_counter.p,
      reinterpret_cast<const WorkItem *>(ctx->p2p_items.p), ctx->p2p.p, mask, ctx->cbeg.p,
      ctx->cnb.p, ctx->ccen.p, ctx->cmin.p, ctx->cmax.p, ctx->rel4.p, ctx->rel_lo.p,
      ctx->trg.p, ctx->p2p_part.p);
  TB_LAUNCH_CHECK(ctx);
  return p2p_finish(ctx);
}

}  // namespace tb
