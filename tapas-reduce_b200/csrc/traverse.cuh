// Dual-tree traversal: M2L / P2P list construction on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
// mutual = 1: the reference's mutual traversal (every unordered cell pair
// visited once); the lists are expanded to directed (target, source) pairs.
int build_lists(tapas_b200_ctx *ctx, double theta, int mutual);
}  // namespace tb
