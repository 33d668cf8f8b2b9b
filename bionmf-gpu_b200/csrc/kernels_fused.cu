// kernels_fused.cu -- fused half-iteration arm (placeholder until the tcgen05 kernel lands).
#include "nmfb_internal.cuh"

int nmfb_fused_prepare(nmfb_ctx *ctx) { (void)ctx; return NMFB_OK; }
int nmfb_fused_release(nmfb_ctx *ctx) { (void)ctx; return NMFB_OK; }
int nmfb_fused_update_H(nmfb_ctx *ctx, int adjust) { (void)adjust; return nmfb_fail(ctx, NMFB_ENODEV, "fused arm not built"); }
int nmfb_fused_update_W(nmfb_ctx *ctx, int adjust) { (void)adjust; return nmfb_fail(ctx, NMFB_ENODEV, "fused arm not built"); }
