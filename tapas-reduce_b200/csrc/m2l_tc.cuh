// Tensor-core (tcgen05, split TF32) M2L of the mixed path, on ctx->stream.
#pragma once
#include "common.cuh"

namespace tb {
// Evaluates the M2L list into ctx->L (FP64 storage): offset classes with
// enough pairs on the tensor cores, the remainder with the FP64 kernel.
int m2l_tensorcore(tapas_b200_ctx *ctx);
}  // namespace tb
