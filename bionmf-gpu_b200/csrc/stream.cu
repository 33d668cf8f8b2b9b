// stream.cu -- out-of-core V: the input matrix stays in host memory and is
// streamed through the GPU in row blocks, for matrices larger than device
// memory (the reference's blockwise mode: block plan in src/GPU_setup.c:
// 902-1270, partial uploads in src/matrix_operations.c:1712-1905).
//
// The host matrix is page-locked in place (cudaHostRegister, read-only) and
// copied block by block with cudaMemcpy2DAsync on a copy stream into two
// device block buffers (double buffering): the copy of block b+1 overlaps the
// kernels of block b, ordered by events (copied[slot] before the kernels that
// read the slot, consumed[slot] before the next copy into it).  W, H and all
// other state stay resident.
//
//   update_H: acc = colsum(W); for every row block b:
//               WH_b = W_b H^T, Q_b = V_b ./ WH_b, Aux += Q_b^T W_b
//             (per-block split partials summed into Aux in block order, so
//             the result does not depend on timing); H = H .* Aux ./ acc.
//   update_W: acc = colsum(H); for every row block b (independent rows):
//               WH_b = W_b H^T, Q_b = V_b ./ WH_b, W_b = W_b .* (Q_b H) ./ acc.
//
// Single pass over V per iteration: inside nmfb_run, an update_W that is not
// the last of a convergence-test block also computes, while V_b is on the
// device, the next update_H's block term with the block's new W rows and the
// unchanged H (WH'_b = W'_b H^T, Q'_b = V_b ./ WH'_b, Aux += Q'_b^T W'_b); the
// next update_H then only applies H = H .* Aux ./ colsum(W').  The kernels,
// operands and block order are those of the separate pass, so the results are
// identical; V crosses the link once per iteration instead of twice (11 passes
// per test block of 10 iterations: the block's first update_H still reads V,
// because the test's EPS adjust rewrites H after the block's last update_W).
// The kernels are the plain FP32 arm's (kernels_plain.cu) on row blocks: the
// path is bound by the host link, two orders of magnitude below HBM.
#include "nmfb_internal.cuh"

#include <stdlib.h>

namespace {

struct StreamPlan {
    const float *hV;        // host V (registered), n x hldv
    size_t hldv;
    int registered;
    uint32_t rows;          // rows per block
    float *dVb[2];          // device block buffers, rows x ldv
    float *dWHb;            // quotient block, rows x ldv
    float *dAux;            // m x kp: update_H partial sums over the blocks
    cudaStream_t cs;        // copy stream
    cudaEvent_t copied[2], consumed[2];
    int used[2];
    int haux_ready;         // dAux holds the next update_H's sum (from update_W's pass)
};

__global__ void k_accum(float *__restrict__ aux, const float *__restrict__ part, uint32_t nsplit, size_t stride,
                        size_t total, int first, const nmfb::ConvState *st)
{
    if (st && *(volatile const uint32_t *)&st->converged) return;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        float s = first ? 0.0f : aux[e];
        for (uint32_t q = 0; q < nsplit; q++) s += part[q * stride + e];
        aux[e] = s;
    }
}

// Queue the H2D copy of block b into its slot on the copy stream.
int issue_copy(nmfb_ctx *ctx, StreamPlan *p, uint32_t b)
{
    uint32_t const slot = b & 1, i0 = b * p->rows;
    uint32_t const nb = (ctx->n - i0) < p->rows ? (ctx->n - i0) : p->rows;
    if (p->used[slot]) NMFB_CUDA_TRY(ctx, cudaStreamWaitEvent(p->cs, p->consumed[slot], 0));
    NMFB_CUDA_TRY(ctx, cudaMemcpy2DAsync(p->dVb[slot], ctx->ldv * sizeof(float), p->hV + (size_t)i0 * p->hldv,
                                         p->hldv * sizeof(float), ctx->m * sizeof(float), nb, cudaMemcpyHostToDevice,
                                         p->cs));
    NMFB_CUDA_TRY(ctx, cudaEventRecord(p->copied[slot], p->cs));
    return NMFB_OK;
}

// Run body(b, i0, rows, V_block) for every block on the compute stream, with
// the copy of the next block in flight.
template <class Body>
int for_blocks(nmfb_ctx *ctx, StreamPlan *p, Body body)
{
    uint32_t const nblocks = (ctx->n + p->rows - 1) / p->rows;
    int rc = issue_copy(ctx, p, 0);
    if (rc) return rc;
    for (uint32_t b = 0; b < nblocks; b++) {
        if (b + 1 < nblocks && (rc = issue_copy(ctx, p, b + 1))) return rc;
        uint32_t const slot = b & 1, i0 = b * p->rows;
        uint32_t const nb = (ctx->n - i0) < p->rows ? (ctx->n - i0) : p->rows;
        NMFB_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, p->copied[slot], 0));
        if ((rc = body(b, i0, nb, p->dVb[slot]))) return rc;
        NMFB_CUDA_TRY(ctx, cudaEventRecord(p->consumed[slot], ctx->stream));
        p->used[slot] = 1;
    }
    return NMFB_OK;
}

StreamPlan *plan_of(nmfb_ctx *ctx) { return (StreamPlan *)ctx->splan; }

}  // namespace

int nmfb_stream_prepare(nmfb_ctx *ctx, uint32_t block_rows)
{
    if (ctx->splan) return NMFB_OK;
    StreamPlan *p = (StreamPlan *)calloc(1, sizeof(StreamPlan));
    if (!p) return nmfb_fail(ctx, NMFB_ENOMEM, "stream plan");
    ctx->splan = p;
    if (block_rows == 0) {
        // about 256 MB per block buffer
        size_t const want = ((size_t)256 << 20) / (ctx->ldv * sizeof(float));
        block_rows = (uint32_t)(want < 64 ? 64 : want);
    }
    if (block_rows > ctx->n) block_rows = ctx->n;
    p->rows = block_rows;
    size_t const blk = (size_t)block_rows * ctx->ldv * sizeof(float);
    cudaError_t e = nmfb_malloc(ctx, (void **)&p->dVb[0], blk);
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&p->dVb[1], blk);
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&p->dWHb, blk);
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&p->dAux, (size_t)ctx->m * ctx->kp * sizeof(float));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nmfb_fail(ctx, NMFB_ENOMEM, "streamed-V block buffers (%u rows): %s", block_rows, cudaGetErrorString(e));
    }
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(p->dVb[0], 0, blk, ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(p->dVb[1], 0, blk, ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&p->cs, cudaStreamNonBlocking));
    for (int s = 0; s < 2; s++) {
        NMFB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&p->copied[s], cudaEventDisableTiming));
        NMFB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&p->consumed[s], cudaEventDisableTiming));
    }
    return NMFB_OK;
}

int nmfb_stream_release(nmfb_ctx *ctx)
{
    StreamPlan *p = plan_of(ctx);
    if (!p) return NMFB_OK;
    if (p->cs) cudaStreamSynchronize(p->cs);
    if (p->registered) cudaHostUnregister((void *)p->hV);
    for (int s = 0; s < 2; s++) {
        if (p->dVb[s]) nmfb_free(ctx, p->dVb[s]);
        if (p->copied[s]) cudaEventDestroy(p->copied[s]);
        if (p->consumed[s]) cudaEventDestroy(p->consumed[s]);
    }
    if (p->dWHb) nmfb_free(ctx, p->dWHb);
    if (p->dAux) nmfb_free(ctx, p->dAux);
    if (p->cs) cudaStreamDestroy(p->cs);
    free(p);
    ctx->splan = nullptr;
    return NMFB_OK;
}

int nmfb_stream_set_V(nmfb_ctx *ctx, const float *V, size_t ldv)
{
    StreamPlan *p = plan_of(ctx);
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(p->cs));
    if (p->registered) {
        cudaHostUnregister((void *)p->hV);
        p->registered = 0;
    }
    size_t const bytes = ((size_t)(ctx->n - 1) * ldv + ctx->m) * sizeof(float);
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, V) == cudaSuccess && attr.type == cudaMemoryTypeHost) {
        p->hV = V;            // already page-locked by the caller (cudaHostAlloc / registered)
        p->hldv = ldv;
        p->used[0] = p->used[1] = 0;
        return NMFB_OK;
    }
    cudaGetLastError();
    cudaError_t e = cudaHostRegister((void *)V, bytes, cudaHostRegisterPortable | cudaHostRegisterReadOnly);
    if (e != cudaSuccess && e != cudaErrorHostMemoryAlreadyRegistered) {
        cudaGetLastError();   // read-only registration unsupported here: register read-write
        e = cudaHostRegister((void *)V, bytes, cudaHostRegisterPortable);
    }
    if (e == cudaSuccess) {
        p->registered = 1;
    } else if (e == cudaErrorHostMemoryAlreadyRegistered) {
        cudaGetLastError();   // the caller's memory is already page-locked
    } else {
        cudaGetLastError();
        return nmfb_fail(ctx, NMFB_ECUDA, "page-locking the host matrix (%zu bytes) failed: %s", bytes,
                         cudaGetErrorString(e));
    }
    p->hV = V;
    p->hldv = ldv;
    p->used[0] = p->used[1] = 0;
    return NMFB_OK;
}

int nmfb_stream_update_H(nmfb_ctx *ctx, int adjust)
{
    StreamPlan *p = plan_of(ctx);
    int rc = nmfb_prof_begin(ctx, 2);
    if (rc) return rc;
    if ((rc = nmfb_colsum(ctx, ctx->dW, ctx->n, ctx->dAccW, 0))) return rc;
    size_t const total = (size_t)ctx->m * ctx->kp;
    if (p->haux_ready) {
        // the sum was formed during the previous update_W's pass over V
        p->haux_ready = 0;
        if ((rc = nmfb_muldiv(ctx, ctx->dH, ctx->m, p->dAux, 1, total, ctx->dAccW, adjust))) return rc;
        return nmfb_prof_end(ctx, 2);
    }
    unsigned grid = (unsigned)((total + 255) / 256);
    if (grid > 8u * (unsigned)ctx->sm_count) grid = 8u * (unsigned)ctx->sm_count;
    rc = for_blocks(ctx, p, [&](uint32_t b, uint32_t i0, uint32_t nb, const float *Vb) -> int {
        const float *Wb = ctx->dW + (size_t)i0 * ctx->kp;
        int r = nmfb_plain_wh(ctx, Wb, nb, p->dWHb);
        if (!r) r = nmfb_plain_div(ctx, Vb, p->dWHb, nb);
        uint32_t ns = 0;
        if (!r) r = nmfb_plain_red(ctx, p->dWHb, 1, Wb, ctx->m, nb, &ns);
        if (r) return r;
        k_accum<<<grid, 256, 0, ctx->stream>>>(p->dAux, ctx->dPart, ns, total, total, b == 0, ctx->dState);
        NMFB_LAUNCH_CHECK(ctx);
        return NMFB_OK;
    });
    if (rc) return rc;
    if ((rc = nmfb_muldiv(ctx, ctx->dH, ctx->m, p->dAux, 1, total, ctx->dAccW, adjust))) return rc;
    return nmfb_prof_end(ctx, 2);
}

int nmfb_stream_update_W(nmfb_ctx *ctx, int adjust)
{
    StreamPlan *p = plan_of(ctx);
    int rc = nmfb_prof_begin(ctx, 3);
    if (rc) return rc;
    if ((rc = nmfb_colsum(ctx, ctx->dH, ctx->m, ctx->dAccH, 1))) return rc;
    // fold the next update_H's pass into this one (see the file comment)
    bool const fold = ctx->in_run && !adjust;
    size_t const total = (size_t)ctx->m * ctx->kp;
    unsigned grid = (unsigned)((total + 255) / 256);
    if (grid > 8u * (unsigned)ctx->sm_count) grid = 8u * (unsigned)ctx->sm_count;
    p->haux_ready = 0;
    rc = for_blocks(ctx, p, [&](uint32_t b, uint32_t i0, uint32_t nb, const float *Vb) -> int {
        float *Wb = ctx->dW + (size_t)i0 * ctx->kp;
        int r = nmfb_plain_wh(ctx, Wb, nb, p->dWHb);
        if (!r) r = nmfb_plain_div(ctx, Vb, p->dWHb, nb);
        uint32_t ns = 0;
        if (!r) r = nmfb_plain_red(ctx, p->dWHb, 0, ctx->dH, nb, ctx->m, &ns);
        if (!r) r = nmfb_muldiv(ctx, Wb, nb, ctx->dPart, ns, (size_t)nb * ctx->kp, ctx->dAccH, adjust);
        if (r || !fold) return r;
        // next update_H's term of this block, with the new W rows
        r = nmfb_plain_wh(ctx, Wb, nb, p->dWHb);
        if (!r) r = nmfb_plain_div(ctx, Vb, p->dWHb, nb);
        if (!r) r = nmfb_plain_red(ctx, p->dWHb, 1, Wb, ctx->m, nb, &ns);
        if (r) return r;
        k_accum<<<grid, 256, 0, ctx->stream>>>(p->dAux, ctx->dPart, ns, total, total, b == 0, ctx->dState);
        NMFB_LAUNCH_CHECK(ctx);
        return NMFB_OK;
    });
    if (rc) return rc;
    p->haux_ready = fold ? 1 : 0;
    return nmfb_prof_end(ctx, 3);
}

// End of nmfb_run: a sum formed by the run's last update_W is not used.
void nmfb_stream_end_run(nmfb_ctx *ctx)
{
    StreamPlan *p = plan_of(ctx);
    if (p) p->haux_ready = 0;
}

int nmfb_stream_objectives(nmfb_ctx *ctx, double out[3])
{
    StreamPlan *p = plan_of(ctx);
    out[0] = out[1] = out[2] = 0.0;
    return for_blocks(ctx, p, [&](uint32_t, uint32_t i0, uint32_t nb, const float *Vb) -> int {
        double part[3];
        int r = nmfb_objectives_rows(ctx, Vb, ctx->dW + (size_t)i0 * ctx->kp, nb, part);
        if (r) return r;
        for (int q = 0; q < 3; q++) out[q] += part[q];   // block order: deterministic
        return NMFB_OK;
    });
}
