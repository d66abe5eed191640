// Dual-tree traversal: M2L / P2P list construction on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
// mutual = 1: the reference's mutual traversal (every unordered cell pair
// visited once); the lists are expanded to directed (target, source) pairs.
// sort_m2l_sources = false (the mixed form, whose M2L regroups the pairs by
// offset class): the M2L list is grouped by target, its sources not sorted
// inside a target; sort_m2l_sources() sorts them where the order matters
// (the FP64 M2L's summation order, the list and device-view accessors).
int build_lists(tapas_b200_ctx *ctx, double theta, int mutual, bool sort_m2l_sources = true);
int sort_m2l_sources(tapas_b200_ctx *ctx);
}  // namespace tb
