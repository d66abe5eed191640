// Mixed-precision evaluation path (TAPAS_B200_MIXED).
//
// Near field: FP32 compensated P2P (p2p.cu, p2p_mixed).  M2L: offset-class
// batched split-TF32 GEMMs on the tensor cores (m2l_tc.cu).  P2M and L2P run
// in FP32 in units of the leaf width (FP64 sums and outputs); M2M and L2L stay
// FP64.  L2P adds to the near-field result, which is per unit charge (so
// without the reference's division by q_i).
#include "kernels.cuh"
#include "m2l_tc.cuh"
#include "mixed.cuh"

namespace tb {

int upward_mixed(tapas_b200_ctx *ctx, int P) { return upward_fp32_p2m(ctx, P); }

int m2l_mixed(tapas_b200_ctx *ctx) { return m2l_tensorcore(ctx); }

int downward_mixed(tapas_b200_ctx *ctx) { return downward_fp32_l2p(ctx); }

int mixed_sync_fp64_view(tapas_b200_ctx *ctx) {
  (void)ctx;
  return TAPAS_B200_OK;
}

void mixed_release(tapas_b200_ctx *ctx) {
  ctx->rel4.release();
  ctx->rel_lo.release();
  ctx->p2p_wkey.release();
  ctx->p2p_wkey_alt.release();
  ctx->p2p_order.release();
  ctx->p2p_order_alt.release();
  ctx->p2p_counter.release();
  ctx->p2p_items.release();
  ctx->p2p_kcnt.release();
  ctx->p2p_koff.release();
  ctx->p2p_psz.release();
  ctx->p2p_poff.release();
  ctx->p2p_part.release();
  ctx->tc.release();
}

}  // namespace tb
