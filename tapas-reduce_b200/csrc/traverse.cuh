// Dual-tree traversal: M2L / P2P list construction on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
int build_lists(tapas_b200_ctx *ctx, double theta);
}  // namespace tb
