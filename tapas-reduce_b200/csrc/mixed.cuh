// Mixed-precision evaluation path (TAPAS_B200_MIXED) on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
int upward_mixed(tapas_b200_ctx *ctx, int P);
int m2l_mixed(tapas_b200_ctx *ctx);
int downward_mixed(tapas_b200_ctx *ctx);
// Makes ctx->M / ctx->L hold FP64 values of the last evaluation (no-op when
// the path already keeps them in FP64).
int mixed_sync_fp64_view(tapas_b200_ctx *ctx);
void mixed_release(tapas_b200_ctx *ctx);
}  // namespace tb
