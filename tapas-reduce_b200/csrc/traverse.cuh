// Dual-tree traversal: M2L / P2P list construction on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
// mutual = 1: the reference's mutual traversal (every unordered cell pair
// visited once); the lists are expanded to directed (target, source) pairs.
// sort_sources = false (the mixed form): both lists are grouped by target,
// each target's sources left in scatter order (the mixed M2L regroups its
// pairs by offset class, and the FP32 near field sums in any order);
// sort_list_sources() sorts them where the order matters (the FP64 M2L's and
// P2P's summation order, the list and device-view accessors).
int build_lists(tapas_b200_ctx *ctx, double theta, int mutual, bool sort_sources = true);
int sort_list_sources(tapas_b200_ctx *ctx, int w);  // w = 0: M2L, 1: P2P
int sort_list_sources(tapas_b200_ctx *ctx);         // both
}  // namespace tb
