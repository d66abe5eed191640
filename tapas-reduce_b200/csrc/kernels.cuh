// Host-side launchers of the evaluation kernels (all on ctx->stream).
#pragma once
#include "common.cuh"

namespace tb {
// FP64 expansion passes (expansions.cu); P in [kMinP, kMaxP].
int upward_fp64(tapas_b200_ctx *ctx, int P);
int m2l_fp64(tapas_b200_ctx *ctx);
// FP64 M2L over the pairs e with use[e] != 0 only (L is zeroed first).
int m2l_fp64_masked(tapas_b200_ctx *ctx, const uint8_t *use);
int downward_fp64(tapas_b200_ctx *ctx);
// Near field (p2p.cu).
int p2p_fp64(tapas_b200_ctx *ctx);
int p2p_mixed(tapas_b200_ctx *ctx);
}  // namespace tb
