// kernels_plain.cu -- the unfused FP32 SIMT arm (NMFB_ARM_PLAIN).
//
// It keeps the reference's five-step structure of a half-iteration
// (src/NMF_routines.c:376-525 / 1014-1164), with the n x m quotient
// materialised in HBM, but with hand-written kernels instead of cuBLAS:
//   1. acc  = colsum(W or H)                 (k_colsum, kernels_common.cu)
//   2. WH   = W * H^T        -> n x m         (k_gemm_nt)
//   3. WH   = V ./ WH                         (k_div)
//   4. Xaux = reduce(WH, other factor)        (k_gemm_red, split over the reduction)
//   5. X    = X .* Xaux ./ acc                (k_muldiv, kernels_common.cu)
// It is the measured "plain" baseline that the fused arm is compared against.
#include "nmfb_internal.cuh"

using nmfb::ConvState;

namespace {

__device__ __forceinline__ bool halted(const ConvState *st) { return st && *(volatile const uint32_t *)&st->converged; }

// C[i][j] = sum_c A[i][c] * B[j][c]; A: ra x kp, B: rb x kp (row-major), C: ra x ldc.
// 64 x 64 output tile per block, 256 threads, 4 x 4 outputs per thread.
__global__ void __launch_bounds__(256) k_gemm_nt(const float *__restrict__ A, const float *__restrict__ B,
                                                 float *__restrict__ Cm, uint32_t ra, uint32_t rb, uint32_t kp,
                                                 size_t ldc, const ConvState *st)
{
    if (halted(st)) return;
    __shared__ float As[16][64 + 4];
    __shared__ float Bs[16][64 + 4];
    uint32_t const tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    uint32_t const i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (uint32_t c0 = 0; c0 < kp; c0 += 16) {
        for (uint32_t e = threadIdx.x; e < 64 * 16; e += 256) {
            uint32_t const r = e / 16, c = e % 16;
            uint32_t const ia = i0 + r, jb = j0 + r;
            As[c][r] = (ia < ra) ? A[(size_t)ia * kp + c0 + c] : 0.0f;
            Bs[c][r] = (jb < rb) ? B[(size_t)jb * kp + c0 + c] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (uint32_t c = 0; c < 16; c++) {
            float a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) { a[q] = As[c][ty * 4 + q]; b[q] = Bs[c][tx * 4 + q]; }
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] = fmaf(a[p], b[q], acc[p][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 4; p++) {
        uint32_t const i = i0 + ty * 4 + p;
        if (i >= ra) continue;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint32_t const j = j0 + tx * 4 + q;
            if (j < rb) Cm[(size_t)i * ldc + j] = acc[p][q];
        }
    }
}

// WH = V ./ WH over the n x m region (matrix_div_sub in division mode; the
// reference uses fdividef, src/GPU_kernels.cu:1687-1695).  Rows over
// blockIdx.y, columns in float4 chunks over blockIdx.x (rows start on
// 128-byte boundaries: ld is a multiple of 32); a ragged tail of m % 4 columns
// element by element.  Padding columns are neither read nor written.
__global__ void k_div(const float *__restrict__ V, float *__restrict__ WH, uint32_t n, uint32_t m, size_t ld,
                      const ConvState *st)
{
    if (halted(st)) return;
    uint32_t const m4 = m / 4;
    for (uint32_t i = blockIdx.y; i < n; i += gridDim.y) {
        const float4 *v4 = reinterpret_cast<const float4 *>(V + (size_t)i * ld);
        float4 *w4 = reinterpret_cast<float4 *>(WH + (size_t)i * ld);
        for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < m4; q += gridDim.x * blockDim.x) {
            float4 const a = v4[q];
            float4 b = w4[q];
            b.x = __fdividef(a.x, b.x);
            b.y = __fdividef(a.y, b.y);
            b.z = __fdividef(a.z, b.z);
            b.w = __fdividef(a.w, b.w);
            w4[q] = b;
        }
        if (blockIdx.x == 0)
            for (uint32_t j = 4 * m4 + threadIdx.x; j < m; j += blockDim.x) {
                size_t const o = (size_t)i * ld + j;
                WH[o] = __fdividef(V[o], WH[o]);
            }
    }
}

// Launch shape of k_div for `rows` rows: enough column threads for a row's
// float4 chunks, rows spread over blockIdx.y up to 64K and ~16 CTAs per SM.
dim3 div_grid(const nmfb_ctx *ctx, uint32_t rows)
{
    uint32_t const gx = (ctx->m / 4 + 255) / 256 > 0 ? (ctx->m / 4 + 255) / 256 : 1;
    uint32_t gy = (16u * (uint32_t)ctx->sm_count + gx - 1) / gx;
    if (gy > rows) gy = rows;
    if (gy > 65535u) gy = 65535u;
    if (gy == 0) gy = 1;
    return dim3(gx, gy);
}

// Out[o][c] = sum_r Q(o, r) * F[r][c] for r in this block's reduction chunk.
// Q(o, r) = Qm[o][r] when !transQ, Qm[r][o] when transQ (Qm has leading dim ldq).
// F: nred x kp.  Partial results go to part[chunk][o][c] (o < nout, c < kp).
// Block: 64 outputs x up to 64 columns per pass; 256 threads, 4 x 4 per thread.
__global__ void __launch_bounds__(256) k_gemm_red(const float *__restrict__ Qm, size_t ldq, int transQ,
                                                  const float *__restrict__ F, uint32_t nout, uint32_t nred,
                                                  uint32_t kp, uint32_t chunk, float *__restrict__ part,
                                                  const ConvState *st)
{
    if (halted(st)) return;
    __shared__ float Qs[32][64 + 1];
    __shared__ float Fs[32][64 + 1];
    uint32_t const o0 = blockIdx.x * 64;
    uint32_t const r_begin = blockIdx.y * chunk;
    uint32_t const r_end = min(nred, r_begin + chunk);
    uint32_t const osub = threadIdx.x / 16, csub = threadIdx.x % 16;
    float *outp = part + (size_t)blockIdx.y * nout * kp;
    for (uint32_t cg = 0; cg < kp; cg += 64) {
        uint32_t const kc = min(64u, kp - cg);
        float acc[4][4] = {};
        for (uint32_t r0 = r_begin; r0 < r_end; r0 += 32) {
            for (uint32_t e = threadIdx.x; e < 32 * 64; e += 256) {
                uint32_t r, o;
                if (transQ) { r = e / 64; o = e % 64; }  // contiguous along o
                else { o = e / 32; r = e % 32; }        // contiguous along r
                uint32_t const gr = r0 + r, go = o0 + o;
                float q = 0.0f;
                if (gr < r_end && go < nout)
                    q = transQ ? Qm[(size_t)gr * ldq + go] : Qm[(size_t)go * ldq + gr];
                Qs[r][o] = q;
            }
            for (uint32_t e = threadIdx.x; e < 32 * 64; e += 256) {
                uint32_t const r = e / 64, c = e % 64;
                uint32_t const gr = r0 + r;
                Fs[r][c] = (gr < r_end && c < kc) ? F[(size_t)gr * kp + cg + c] : 0.0f;
            }
            __syncthreads();
#pragma unroll 8
            for (uint32_t r = 0; r < 32; r++) {
                float q[4], f[4];
#pragma unroll
                for (int p = 0; p < 4; p++) q[p] = Qs[r][osub * 4 + p];
#pragma unroll
                for (int s = 0; s < 4; s++) f[s] = Fs[r][csub + 16 * s];
#pragma unroll
                for (int p = 0; p < 4; p++)
#pragma unroll
                    for (int s = 0; s < 4; s++) acc[p][s] = fmaf(q[p], f[s], acc[p][s]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int p = 0; p < 4; p++) {
            uint32_t const o = o0 + osub * 4 + p;
            if (o >= nout) continue;
#pragma unroll
            for (int s = 0; s < 4; s++) {
                uint32_t const c = csub + 16 * s;
                if (c < kc) outp[(size_t)o * kp + cg + c] = acc[p][s];
            }
        }
    }
}

struct RedPlan {
    uint32_t nsplit, chunk;
};

RedPlan plan_split(nmfb_ctx *ctx, uint32_t nout, uint32_t nred)
{
    uint32_t const oblocks = (nout + 63) / 64;
    uint32_t want = (8u * (uint32_t)ctx->sm_count + oblocks - 1) / oblocks;   // ~8 CTAs per SM of work
    if (want < 1) want = 1;
    if (want > NMFB_MAX_SPLIT) want = NMFB_MAX_SPLIT;
    uint32_t chunk = (nred + want - 1) / want;
    chunk = ((chunk + 31) / 32) * 32;
    if (chunk == 0) chunk = 32;
    uint32_t const nsplit = (nred + chunk - 1) / chunk;
    return {nsplit, chunk};
}

int plain_half(nmfb_ctx *ctx, bool is_H, int adjust)
{
    // 1. column sums of the factor that is NOT being updated.
    float *X = is_H ? ctx->dH : ctx->dW;           // updated factor
    const float *Y = is_H ? ctx->dW : ctx->dH;     // other factor
    uint32_t const xrows = is_H ? ctx->m : ctx->n;
    uint32_t const yrows = is_H ? ctx->n : ctx->m;
    float *acc = is_H ? ctx->dAccW : ctx->dAccH;
    int const whole = is_H ? 2 : 3, main = is_H ? 0 : 1;
    int rc = nmfb_prof_begin(ctx, whole);
    if (rc) return rc;
    if ((rc = nmfb_colsum(ctx, Y, yrows, acc, is_H ? 0 : 1))) return rc;
    // 2. WH = W * H^T (n x m)
    dim3 g((ctx->m + 63) / 64, (ctx->n + 63) / 64);
    k_gemm_nt<<<g, 256, 0, ctx->stream>>>(ctx->dW, ctx->dH, ctx->dWH, ctx->n, ctx->m, ctx->kp, ctx->ldv, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    // 3. WH = V ./ WH
    k_div<<<div_grid(ctx, ctx->n), 256, 0, ctx->stream>>>(ctx->dV, ctx->dWH, ctx->n, ctx->m, ctx->ldv, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    // 4. Xaux = Q^T Y (update_H) or Q Y (update_W), split over the reduction.
    RedPlan const p = plan_split(ctx, xrows, yrows);
    if ((size_t)p.nsplit * xrows * ctx->kp > ctx->part_items)
        return nmfb_fail(ctx, NMFB_EINVAL, "partial buffer too small (%u splits of %u rows)", p.nsplit, xrows);
    dim3 rg((xrows + 63) / 64, p.nsplit);
    if ((rc = nmfb_prof_begin(ctx, main))) return rc;
    k_gemm_red<<<rg, 256, 0, ctx->stream>>>(ctx->dWH, ctx->ldv, is_H ? 1 : 0, Y, xrows, yrows, ctx->kp, p.chunk,
                                           ctx->dPart, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    if ((rc = nmfb_prof_end(ctx, main))) return rc;
    // 5. X = X .* Xaux ./ acc  (+ EPS adjust on test iterations)
    rc = nmfb_muldiv(ctx, X, xrows, ctx->dPart, p.nsplit, (size_t)xrows * ctx->kp, acc, adjust);
    if (rc) return rc;
    return nmfb_prof_end(ctx, whole);
}

}  // namespace

// Row-block building blocks for the streamed mode (stream.cu): the same
// kernels on `rows` rows of W and a rows x ldv block of V / WH.
int nmfb_plain_wh(nmfb_ctx *ctx, const float *W, uint32_t rows, float *WH)
{
    dim3 g((ctx->m + 63) / 64, (rows + 63) / 64);
    k_gemm_nt<<<g, 256, 0, ctx->stream>>>(W, ctx->dH, WH, rows, ctx->m, ctx->kp, ctx->ldv, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

int nmfb_plain_div(nmfb_ctx *ctx, const float *V, float *WH, uint32_t rows)
{
    k_div<<<div_grid(ctx, rows), 256, 0, ctx->stream>>>(V, WH, rows, ctx->m, ctx->ldv, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

int nmfb_plain_red(nmfb_ctx *ctx, const float *Q, int transQ, const float *F, uint32_t nout, uint32_t nred,
                   uint32_t *nsplit)
{
    RedPlan const p = plan_split(ctx, nout, nred);
    if ((size_t)p.nsplit * nout * ctx->kp > ctx->part_items)
        return nmfb_fail(ctx, NMFB_EINVAL, "partial buffer too small (%u splits of %u rows)", p.nsplit, nout);
    dim3 rg((nout + 63) / 64, p.nsplit);
    k_gemm_red<<<rg, 256, 0, ctx->stream>>>(Q, ctx->ldv, transQ, F, nout, nred, ctx->kp, p.chunk, ctx->dPart,
                                           ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    *nsplit = p.nsplit;
    return NMFB_OK;
}

int nmfb_plain_update_H(nmfb_ctx *ctx, int adjust) { return plain_half(ctx, true, adjust); }
int nmfb_plain_update_W(nmfb_ctx *ctx, int adjust) { return plain_half(ctx, false, adjust); }
