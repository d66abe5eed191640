// M2L batched by offset class: the tensor-core (tcgen05, split TF32) GEMM of
// the mixed form and the FP64 GEMM of the plain form, on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
// Evaluates the M2L list into ctx->L (FP64 storage): offset classes with
// enough pairs on the tensor cores, the remainder with the FP64 kernel.
int m2l_tensorcore(tapas_b200_ctx *ctx);

// The mixed form's M2M, after its FP32 P2M: tensor-core GEMMs per level over
// (parent, child) pairs grouped by octant with level-independent,
// width-normalised operators at the deepest three parent levels below level
// 3, FP64 level GEMMs above them.  Completes ctx->M and the M2L's input rows.
// (The mixed form's L2L is the FP64 one.)
int tc_tree_upward(tapas_b200_ctx *ctx);

// Result of the offset classification of the current M2L list.
struct M2LClassInfo {
  int64_t nseg = 0;    // classes, including the empty-pair and unclassed groups
  int64_t ntc = 0;     // classes selected for a GEMM (tables in ctx->tc)
  int64_t nitems = 0;  // 128-pair tiles of the selected classes
  int64_t n64 = 0;     // pairs left to the FP64 pair path (list indices in ctx->tc.pairs64)
};
// Classifies and sorts the M2L pairs by offset class and selects the classes
// with at least min_pairs pairs, at most as many as ctx->tc_op_budget bytes of
// operators of op_bytes each hold (the most populated first).  Fills
// ctx->tc: vals (list indices sorted by class), tc_keys (selected classes'
// keys: delta + 32 in bits 42-47, D_z, D_y, D_x + 8192 in 14 bits each),
// cls_range (first sorted pair, pair count), items (128-pair tiles) and
// pairs64; err[1] = pairs in selected classes.
int m2l_classes(tapas_b200_ctx *ctx, size_t op_bytes, int64_t min_pairs, M2LClassInfo &info);
}  // namespace tb
