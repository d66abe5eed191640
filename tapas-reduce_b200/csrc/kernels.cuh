// Host-side launchers of the evaluation kernels (all on ctx->stream).
#pragma once
#include "common.cuh"

namespace tb {
// FP64 expansion passes (expansions.cu); P in [kMinP, kMaxP].
int upward_fp64(tapas_b200_ctx *ctx, int P);
// P2M in FP32 (FP64 sums and output), then FP64 M2M.
int upward_fp32_p2m(tapas_b200_ctx *ctx, int P);
// The two halves of the upward pass: P2M of the leaves this context
// evaluates (M zeroed first; fp32: the mixed form's P2M), and the FP64 M2M of
// the whole tree from the leaves' M (order ctx->P).
int p2m_only(tapas_b200_ctx *ctx, int P, bool fp32);
int m2m_only(tapas_b200_ctx *ctx);
// FP64 M2M level GEMMs of parent levels max_levels - 1 .. 0 only (deepest
// first), order ctx->P; builds the level operators for the current tree.
int fp64_m2m_levels(tapas_b200_ctx *ctx, int max_levels);
// The plain FP64 form's M2L: one FP64 GEMM per offset class (classes in key
// order, so every target's sum has a fixed order), the rare classes' pairs by
// the warp-per-target FP64 kernel.
int m2l_fp64(tapas_b200_ctx *ctx);
// L zeroed, then the FP64 M2L of the pairs at list indices pairs[0..npairs)
// added into it (atomics: the order of a target's sums is not fixed).
int m2l_fp64_pairs(tapas_b200_ctx *ctx, const uint32_t *pairs, int64_t npairs);
int downward_fp64(tapas_b200_ctx *ctx);
// FP64 L2L, then L2P in FP32 added to the near field.
int downward_fp32_l2p(tapas_b200_ctx *ctx);
// Near field (p2p.cu).
int p2p_fp64(tapas_b200_ctx *ctx);
int p2p_mixed(tapas_b200_ctx *ctx);
}  // namespace tb
