// finish.cuh -- the second launch of a fused half-iteration (both fused arms):
// the multiplicative update of X from the fused kernel's split partials, the EPS
// adjust, X's split copies for the next half-iteration and its column sums.
#pragma once

#include <cuda_bf16.h>
#include <float.h>
#include <stdint.h>

#include "nmfb_internal.cuh"
#include "fused_common.cuh"

namespace {

using nmfb::ConvState;
using nmfb_tc::BO;
using nmfb_tc::tf32_rna;

constexpr uint32_t FIN_ECH = 32;   // row blocks per chunk of k_finish's column sums
constexpr uint32_t FIN_RB = 32;    // rows of X per k_finish CTA

// k_finish's launch shape for a factor of `rows` rows: KP / 4 threads per row
// of a 32-row set, RPT row sets per CTA (each thread takes one row of each),
// and enough CTAs to cover every 64-row block of the split copies (rows past
// the end get zeros there).  RPT > 1 when there are few splits: more loads in
// flight per thread, fewer waves of CTAs.
template <int KP>
constexpr int fin_threads() { return (int)FIN_RB * (KP / 4); }
inline uint32_t fin_rpt(uint32_t nsplit) { return nsplit <= 2 ? 4u : nsplit <= 4 ? 2u : 1u; }
inline uint32_t fin_blocks(uint32_t rows, uint32_t rpt)
{
    uint32_t const rows64 = (rows + 63u) / 64u * 64u;
    return (rows64 + FIN_RB * rpt - 1) / (FIN_RB * rpt);
}

// Two floats to a BF16 pair (round to nearest even), `first` in the low half.
__device__ __forceinline__ uint32_t fin_bf16x2(float first, float second)
{
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(second), "f"(first));
    return r;
}

// Finish of a half-iteration, one CTA per FIN_RB = 32 rows of X, KP / 4 threads
// per row (four consecutive columns each), right after the fused kernel
// (k_fused_half, LAYOUT 0, or k_fused_bf16, LAYOUT 1):
//   Xaux = the split partials summed in split order; X = X * Xaux / accY
//   (matrix_mul_div, src/GPU_kernels.cu:1885-2058: product first, then the
//   division, correctly rounded) with the EPS adjust when asked (kernel_adjust,
//   :2338-2345); then X's split copies in the arm's layout (LAYOUT 0:
//   k_split_factor's, LAYOUT 1: k_split_bf16's) and its column
//   sums (matrix_to_row, src/GPU_kernels.cu:871-1066) in FP64: a shuffle tree over
//   each warp's rows, the warps in order, row blocks in chunks of FIN_ECH in block
//   order, the chunks in order -- fixed orders throughout, so the result does not
//   depend on scheduling.  It replaces the reference's mul_div + adjust and, for the
//   next half-iteration, its column sums, in one launch.  Small blocks and the
//   partials of up to eight splits in flight per thread keep each CTA's chain of
//   dependent memory round trips short: the kernel is latency-bound, its traffic
//   (the partials, X and its copies) small.
struct FinishArgs {
    uint32_t O, nsplit, k;
    int adjust;
    const float *part;    // [split][O][KP]
    float *X;
    const float *accY;    // column sums of Y (KP)
    float *xhi, *xT;      // LAYOUT 0: X's split copies (the FP32 arm's SplitLayout of X's rows)
    __nv_bfloat16 *xBl, *xB, *xBT;
    uint32_t xnblk32, xnblkbr;
    __nv_bfloat16 *bhi, *blo, *bT;   // LAYOUT 1: bf16 hi, lo (rows x KP) and per 64 rows [hi^T ; lo^T]
    uint32_t bnblk64;
    double *cs;           // [row block][KP] FP64 column-sum partials, then from row csoff [chunk][KP]
    uint32_t csoff;
    float *accX;          // column sums of the new X (KP)
    uint32_t *tick;       // [chunks + 1] retirement counters (left at 0)
    const ConvState *st;
};

template <int KP, int BR, int LAYOUT, int RPT>
__global__ void __launch_bounds__(FIN_RB * KP / 4, 128 / KP) k_finish(const FinishArgs a)   // <= 64 registers
{
    constexpr int TPR = KP / 4;                  // threads per row
    constexpr int NT = (int)FIN_RB * TPR;        // 128 / 256 / 512 threads for KP = 16 / 32 / 64
    constexpr int NW = NT / 32;                  // warps
    constexpr int QB = 8 / RPT;                  // splits per row in flight (8 loads per thread)
    static_assert(32 % TPR == 0 && NT % KP == 0 && QB >= 1, "k_finish shape");
    if (a.st && *(volatile const uint32_t *)&a.st->converged) return;
    __shared__ double ws[NW * KP + NT];
    __shared__ float sx[KP * 33];                // x of one 32-row set, column-major (padded)
    __shared__ uint32_t eflag;
    uint32_t const tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    uint32_t const row = tid / TPR, c0 = (tid % TPR) * 4;
    uint32_t const blk = blockIdx.x, nob = gridDim.x;
    size_t const qs = (size_t)a.O * KP;
    // this thread's rows: one in each 32-row set of the CTA's block
    uint32_t o[RPT];
    bool in[RPT];
    float x[RPT][4];
    float4 xv[RPT];
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        o[r] = (blk * RPT + r) * FIN_RB + row;
        in[r] = o[r] < a.O;
#pragma unroll
        for (int i = 0; i < 4; i++) x[r][i] = 0.0f;
        xv[r] = in[r] ? *reinterpret_cast<const float4 *>(a.X + (size_t)o[r] * KP + c0)   // independent of the partials
                      : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    // Xaux: each row's split partials in split order, QB splits of every row in flight
    for (uint32_t q = 0; q < a.nsplit; q += QB) {
        float4 v[RPT][QB];
#pragma unroll
        for (int r = 0; r < RPT; r++)
#pragma unroll
            for (int j = 0; j < QB; j++)
                v[r][j] = (in[r] && q + j < a.nsplit)
                              ? __ldcg(reinterpret_cast<const float4 *>(a.part + (size_t)o[r] * KP + c0 + (q + j) * qs))
                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int r = 0; r < RPT; r++)
#pragma unroll
            for (int j = 0; j < QB; j++)
                if (q + j < a.nsplit) {
                    x[r][0] += v[r][j].x;
                    x[r][1] += v[r][j].y;
                    x[r][2] += v[r][j].z;
                    x[r][3] += v[r][j].w;
                }
    }
    double csum[4] = {0.0, 0.0, 0.0, 0.0};   // this thread's rows of its columns, in row-set order
#pragma unroll
    for (int r = 0; r < RPT; r++) {
        if (in[r]) {
            float const xs[4] = {xv[r].x, xv[r].y, xv[r].z, xv[r].w};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                uint32_t const cc = c0 + i;
                float v = 0.0f;
                if (cc < a.k) {
                    v = __fdiv_rn(xs[i] * x[r][i], __ldg(a.accY + cc));
                    if (a.adjust) v = fmaxf(v, FLT_MIN);
                }
                x[r][i] = v;
            }
            *reinterpret_cast<float4 *>(a.X + (size_t)o[r] * KP + c0) = make_float4(x[r][0], x[r][1], x[r][2], x[r][3]);
        }
#pragma unroll
        for (int i = 0; i < 4; i++) csum[i] += (double)x[r][i];
        // split copies: the row-major ones straight from registers; the transposed
        // blocks through shared memory (x of the 32-row set, column-major), so that
        // every store below covers 64-128 contiguous bytes.  Rows past the end are
        // zero in the transposed blocks that exist.
        if (LAYOUT == 0) {
            if (in[r]) {
                float h[4], l[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    h[i] = tf32_rna(x[r][i]);
                    l[i] = x[r][i] - h[i];
                }
                size_t const e = (size_t)o[r] * KP + c0;
                *reinterpret_cast<float4 *>(a.xhi + e) = make_float4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint2 *>(a.xBl + e) = make_uint2(fin_bf16x2(l[0], l[1]), fin_bf16x2(l[2], l[3]));
                *reinterpret_cast<uint2 *>(a.xB + e) =
                    make_uint2(fin_bf16x2(x[r][0], x[r][1]), fin_bf16x2(x[r][2], x[r][3]));
            }
        } else if (in[r]) {
            // hi = bf16(x), lo = bf16(x - hi), both rounded to nearest (k_split_bf16)
            size_t const e = (size_t)o[r] * KP + c0;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                __nv_bfloat16 const h = __float2bfloat16_rn(x[r][i]);
                a.bhi[e + i] = h;
                a.blo[e + i] = __float2bfloat16_rn(x[r][i] - __bfloat162float(h));
            }
        }
        __syncthreads();   // the previous row set's readers of sx are done
#pragma unroll
        for (int i = 0; i < 4; i++) sx[(c0 + i) * 33 + row] = x[r][i];
        __syncthreads();
        uint32_t const set0 = (blk * RPT + r) * FIN_RB;   // first row of this set
        if (LAYOUT == 0) {
            uint32_t const b32 = set0 / 32, bbr = set0 / BR;
            float *T32 = a.xT + (size_t)b32 * 2 * KP * 32;
            __nv_bfloat16 *BT = a.xBT + (size_t)bbr * KP * BR + set0 % BR;
            for (uint32_t e = tid; e < (uint32_t)KP * 32; e += NT) {
                uint32_t const c = e / 32, t = e % 32;
                float const v = sx[c * 33 + t];
                float const h = tf32_rna(v);
                if (b32 < a.xnblk32) {
                    T32[c * 32 + t] = h;
                    T32[(KP + c) * 32 + t] = v - h;
                }
                if (bbr < a.xnblkbr) BT[(size_t)c * BR + t] = __float2bfloat16_rn(v);
            }
        } else {
            uint32_t const b64 = set0 / 64;
            __nv_bfloat16 *T64 = a.bT + (size_t)b64 * 2 * KP * 64 + set0 % 64;
            if (b64 < a.bnblk64)
                for (uint32_t e = tid; e < (uint32_t)KP * 32; e += NT) {
                    uint32_t const c = e / 32, t = e % 32;
                    float const v = sx[c * 33 + t];
                    __nv_bfloat16 const h = __float2bfloat16_rn(v);
                    T64[(size_t)c * 64 + t] = h;
                    T64[(size_t)(KP + c) * 64 + t] = __float2bfloat16_rn(v - __bfloat162float(h));
                }
        }
    }
    // column sums of this row block: each thread's rows (above), the warp's lanes
    // of each column by a shuffle tree (lane TPR r + g holds row r, column group
    // g), then the warps in order
#pragma unroll
    for (int c = 0; c < 4; c++) {
        double v = csum[c];
#pragma unroll
        for (int off = 16; off >= TPR; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane < (uint32_t)TPR) ws[warp * KP + c0 + c] = v;
    }
    __syncthreads();
    if (tid < (uint32_t)KP) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < NW; w++) t += ws[w * KP + tid];
        a.cs[(size_t)blk * KP + tid] = t;
    }
    __threadfence();
    __syncthreads();
    uint32_t const nch = (nob + FIN_ECH - 1) / FIN_ECH, ch = blk / FIN_ECH;
    uint32_t const b0 = ch * FIN_ECH, bn = min(nob - b0, FIN_ECH);
    if (tid == 0) eflag = (atomicAdd(&a.tick[ch], 1u) == bn - 1) ? 1u : 0u;
    __syncthreads();
    if (!eflag) return;
    // last row block of its chunk: the chunk's partials in block order
    __threadfence();
    constexpr int GRP = NT / KP;
    uint32_t const g = tid / KP, c = tid % KP;
    double t = 0.0;
    for (uint32_t b = g; b < bn; b += GRP) t += __ldcg(a.cs + (size_t)(b0 + b) * KP + c);
    ws[NW * KP + tid] = t;
    __syncthreads();
    if (tid < (uint32_t)KP) {
        double u = 0.0;
        for (int gg = 0; gg < GRP; gg++) u += ws[NW * KP + gg * KP + tid];
        a.cs[((size_t)a.csoff + ch) * KP + tid] = u;
    }
    if (tid == 0) a.tick[ch] = 0u;
    __threadfence();
    __syncthreads();
    if (tid == 0) eflag = (atomicAdd(&a.tick[nch], 1u) == nch - 1) ? 1u : 0u;
    __syncthreads();
    if (!eflag) return;
    // last chunk: the chunk sums in order
    __threadfence();
    double v = 0.0;
    for (uint32_t q = g; q < nch; q += GRP) v += __ldcg(a.cs + ((size_t)a.csoff + q) * KP + c);
    __syncthreads();
    ws[NW * KP + tid] = v;
    __syncthreads();
    if (tid < (uint32_t)KP) {
        double u = 0.0;
        for (int gg = 0; gg < GRP; gg++) u += ws[NW * KP + gg * KP + tid];
        a.accX[tid] = (float)u;
    }
    if (tid == 0) a.tick[nch] = 0u;
}

// k_finish for the factor of a.O rows, with the row sets per thread that its
// split count calls for (the block count is fin_blocks(a.O, fin_rpt(a.nsplit))).
template <int KP, int BR, int LAYOUT>
void fin_launch(const FinishArgs &a, cudaStream_t s)
{
    uint32_t const rpt = fin_rpt(a.nsplit), nb = fin_blocks(a.O, rpt);
    if (rpt == 4)
        k_finish<KP, BR, LAYOUT, 4><<<nb, fin_threads<KP>(), 0, s>>>(a);
    else if (rpt == 2)
        k_finish<KP, BR, LAYOUT, 2><<<nb, fin_threads<KP>(), 0, s>>>(a);
    else
        k_finish<KP, BR, LAYOUT, 1><<<nb, fin_threads<KP>(), 0, s>>>(a);
}

}  // namespace
