// Octree construction (bbox, keys, sort, cells) on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
int ensure_cells(tapas_b200_ctx *ctx, int64_t need, int64_t used);
// Builds the tree of the bodies already in ctx->x/y/z/q (ctx->n of them).
int build_tree(tapas_b200_ctx *ctx, int ncrit);
// Bodies per leaf depth (deeper leaves in the last bin), nbins <= 64, host out.
int leaf_depth_histogram(tapas_b200_ctx *ctx, int nbins, int64_t *out);
// Barnes-Hut sample path (bh.cu).
int bh_upward(tapas_b200_ctx *ctx);
int bh_interact(tapas_b200_ctx *ctx, double theta, double eps2, int precision);
}  // namespace tb
