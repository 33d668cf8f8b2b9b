// kernels_common.cu -- small kernels shared by every update arm:
//   * deterministic column sums of W / H            (reference: matrix_to_row)
//   * mul-div update with fused EPS adjust       (reference: matrix_mul_div + matrix_adjust)
//   * classification (argmax) + device-side connectivity test and stop rule
//                                                   (reference: get_classification + get_difference)
//   * FP64 objective reductions (||V||^2, ||V-WH||^2, KL divergence)
//
// All reductions use fixed-order trees so results do not depend on timing.
#include "nmfb_internal.cuh"

#include <float.h>
#include <stdarg.h>

using nmfb::ConvState;

int nmfb_fail(nmfb_ctx *ctx, int code, const char *fmt, ...)
{
    if (ctx) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

namespace {

__device__ __forceinline__ bool halted(const ConvState *st) { return st && *(volatile const uint32_t *)&st->converged; }

// EPS adjust of the reference (src/GPU_kernels.cu:2338-2345): fmaxf(x, FLT_MIN),
// which also maps NaN to FLT_MIN.
__device__ __forceinline__ float adjust_value(float v) { return fmaxf(v, FLT_MIN); }

// ---------------------------------------------------------------------------
// Column sums: block b reduces rows [r0, r1) of X (rows x kp) into part[b][*];
// the last block to retire sums the block partials (FP64) in a fixed order:
// thread group g (of blockDim / kp) sums blocks g, g + groups, ... in order,
// then the groups are added in order.  Many short blocks with four loads in
// flight per thread keep the reads bandwidth-bound rather than latency-bound.
__global__ void k_colsum(const float *__restrict__ X, uint32_t rows, uint32_t kp, double *__restrict__ part,
                         float *__restrict__ acc, uint32_t *__restrict__ ticket, const ConvState *st)
{
    if (halted(st)) return;
    __shared__ double red[256];
    __shared__ bool is_last;
    uint32_t const lanes = blockDim.x / kp;  // row lanes per block
    uint32_t const c = threadIdx.x % kp;
    uint32_t const rl = threadIdx.x / kp;
    uint32_t const per = (rows + gridDim.x - 1) / gridDim.x;
    uint32_t const r0 = blockIdx.x * per;
    uint32_t const r1 = min(rows, r0 + per);
    double s = 0.0;
    if (rl < lanes) {
        uint32_t r = r0 + rl;
        for (; r + 3 * lanes < r1; r += 4 * lanes) {
            float const a0 = X[(size_t)r * kp + c], a1 = X[(size_t)(r + lanes) * kp + c];
            float const a2 = X[(size_t)(r + 2 * lanes) * kp + c], a3 = X[(size_t)(r + 3 * lanes) * kp + c];
            s += (double)a0;
            s += (double)a1;
            s += (double)a2;
            s += (double)a3;
        }
        for (; r < r1; r += lanes) s += (double)X[(size_t)r * kp + c];
    }
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < kp) {
        double t = 0.0;
        for (uint32_t l = 0; l < lanes; l++)
            t += red[l * kp + threadIdx.x];
        part[(size_t)blockIdx.x * kp + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    uint32_t const groups = lanes;
    double t = 0.0;
    if (rl < groups)
        for (uint32_t b = rl; b < gridDim.x; b += groups) t += __ldcg(&part[(size_t)b * kp + c]);
    red[threadIdx.x] = t;
    __syncthreads();
    if (threadIdx.x < kp) {
        double u = 0.0;
        for (uint32_t g = 0; g < groups; g++) u += red[g * kp + threadIdx.x];
        acc[threadIdx.x] = (float)u;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// ---------------------------------------------------------------------------
// Factor update, one thread per entry of X (rows x kp):
//   mode FU_MULDIV: v = (X[r][c] * sum_s part[s][r][c]) / acc[c]  (matrix_mul_div,
//                   src/GPU_kernels.cu:2013-2019: product first, then the division),
//                   followed by the EPS adjust when `adjust` is set;
//   mode FU_ADJUST: v = fmaxf(X[r][c], FLT_MIN)                   (matrix_adjust).
// Padding columns c >= k are kept at 0.  The split partials are summed in
// split order, so the result does not depend on scheduling.
enum { FU_MULDIV = 1, FU_ADJUST = 2 };

__global__ void __launch_bounds__(256) k_factor(int mode, float *__restrict__ X, uint32_t rows, uint32_t kp, uint32_t k,
                                                const float *__restrict__ part, uint32_t nsplit, size_t split_stride,
                                                const float *__restrict__ acc, int adjust, const ConvState *st)
{
    if (halted(st)) return;
    size_t const total = (size_t)rows * kp;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        uint32_t const c = (uint32_t)(idx % kp);
        float v = 0.0f;
        if (c < k) {
            if (mode == FU_MULDIV) {
                float s = 0.0f;
                for (uint32_t q = 0; q < nsplit; q++) s += part[q * split_stride + idx];
                v = __fdiv_rn(X[idx] * s, acc[c]);
                if (adjust) v = adjust_value(v);
            } else {
                v = adjust_value(X[idx]);
            }
        }
        X[idx] = v;
    }
}

// ---------------------------------------------------------------------------
// Classification with the reference's lane-exact tie rule (kernel_idx_max,
// src/GPU_kernels.cu:2508-2656, 2880-3110, 3177-3267):
//   group width bdx = 32 for k <= 96, else next_pow2(ceil(ceil32(k)/3));
//   thread t scans columns t, t+bdx, t+2*bdx (< k), keeping the first strict max;
//   idle threads hold (-1, 0); shared-memory tree for half = bdx/2 .. 32 and a
//   xor butterfly for half = 16 .. 1, each lane keeping its own value on ties;
//   lane 0 holds the result.
// Optionally applies the test's EPS adjust to H first (adjust(H) happens right
// before get_classification in the reference, src/NMF_GPU.c:611-655).
// Also records first[label] = min sample index per label (canonical partition).
__global__ void k_classify(float *__restrict__ H, uint32_t m, uint32_t kp, uint32_t k, uint32_t bdx,
                           int adjust, uint32_t *__restrict__ labels, uint32_t *__restrict__ first,
                           const ConvState *st)
{
    if (halted(st)) return;
    extern __shared__ unsigned char smem_raw[];
    float *sval = reinterpret_cast<float *>(smem_raw);
    uint32_t *sidx = reinterpret_cast<uint32_t *>(sval + blockDim.x);
    uint32_t const groups = blockDim.x / bdx;
    uint32_t const g = threadIdx.x / bdx;
    uint32_t const t = threadIdx.x % bdx;
    uint32_t const j = blockIdx.x * groups + g;
    bool const valid = j < m;
    float *row = H + (size_t)(valid ? j : 0) * kp;

    if (adjust && valid) {
        for (uint32_t c = t; c < kp; c += bdx) {
            if (c >= k) continue;
            row[c] = adjust_value(row[c]);
        }
        __syncwarp();
    }
    float v = -1.0f;
    uint32_t id = 0;
    if (valid && t < k) {
        v = row[t];
        id = t;
        for (uint32_t it = 1; it < 3; it++) {
            uint32_t const c = t + it * bdx;
            if (c < k) {
                float const x = row[c];
                if (x > v) { v = x; id = c; }
            }
        }
    }
    if (bdx > 32) {
        sval[threadIdx.x] = v;
        sidx[threadIdx.x] = id;
        for (uint32_t half = bdx / 2; half >= 32; half >>= 1) {
            __syncthreads();
            if (t < half) {
                float const ov = sval[threadIdx.x + half];
                uint32_t const oi = sidx[threadIdx.x + half];
                if (v < ov) { v = ov; id = oi; }
            }
            __syncthreads();
            if (t < half) { sval[threadIdx.x] = v; sidx[threadIdx.x] = id; }
        }
        __syncthreads();
    }
    if (t < 32) {
        unsigned const mask = 0xffffffffu;
        for (uint32_t half = 16; half > 0; half >>= 1) {
            float const ov = __shfl_xor_sync(mask, v, half);
            uint32_t const oi = __shfl_xor_sync(mask, id, half);
            if (v < ov) { v = ov; id = oi; }
        }
        if (t == 0 && valid) {
            labels[j] = id;
            atomicMin(&first[id], j);
        }
    }
}

// Connectivity comparison and stop rule.  Two classification vectors define
// the same partition (get_difference == 0, src/common.c:1195-1209) iff every
// sample maps to the same first-occurrence representative in both.  The last
// block applies the reference's counter rule (src/NMF_GPU.c:695-709).
__global__ void k_conv_compare(const uint32_t *__restrict__ labels, uint32_t *__restrict__ first,
                               uint32_t *__restrict__ lastrep, uint32_t m, uint32_t nfirst, ConvState *st)
{
    if (halted(st)) return;
    __shared__ bool is_last;
    uint32_t local_diff = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        uint32_t const rep = first[labels[j]];
        if (rep != lastrep[j]) local_diff = 1;
        lastrep[j] = rep;
    }
    if (__syncthreads_or(local_diff) && threadIdx.x == 0)
        atomicOr(&st->diff, 1u);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        is_last = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    for (uint32_t c = threadIdx.x; c < nfirst; c += blockDim.x)
        first[c] = 0xffffffffu;
    if (threadIdx.x == 0) {
        uint32_t const diff = atomicAdd(&st->diff, 0u);
        st->tests_done += 1;
        if (diff)
            st->inc = 0;
        else if (st->inc < st->stop_threshold)
            st->inc += 1;
        else {
            st->converged = 1;
            st->conv_tests = st->tests_done;
        }
        st->diff = 0;
        st->ticket = 0;
    }
}

// ---------------------------------------------------------------------------
// FP64 objectives over V (n x m, ld ldv) and W (n x kp), H (m x kp):
// out[0] = ||V||^2, out[1] = ||V - WH||^2, out[2] = KL(V || WH).
__global__ void k_objective(const float *__restrict__ V, size_t ldv, const float *__restrict__ W,
                            const float *__restrict__ H, uint32_t n, uint32_t m, uint32_t kp, uint32_t k,
                            double *__restrict__ part, double *__restrict__ out, uint32_t *__restrict__ ticket)
{
    __shared__ double red[3][256];
    __shared__ bool is_last;
    double sv = 0.0, sd = 0.0, kl = 0.0;
    size_t const total = (size_t)n * m;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        uint32_t const i = (uint32_t)(e / m), j = (uint32_t)(e % m);
        const float *w = W + (size_t)i * kp;
        const float *h = H + (size_t)j * kp;
        double wh = 0.0;
        for (uint32_t c = 0; c < k; c++)
            wh += (double)w[c] * (double)h[c];
        double const v = V[(size_t)i * ldv + j];
        sv += v * v;
        sd += (v - wh) * (v - wh);
        kl += (v > 0.0 ? v * log(v / wh) : 0.0) - v + wh;
    }
    red[0][threadIdx.x] = sv;
    red[1][threadIdx.x] = sd;
    red[2][threadIdx.x] = kl;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 3) part[(size_t)blockIdx.x * 3 + threadIdx.x] = red[threadIdx.x][0];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (uint32_t b = 0; b < gridDim.x; b++) t += __ldcg(&part[(size_t)b * 3 + threadIdx.x]);
        out[threadIdx.x] = t;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

inline unsigned grid_for(size_t items, unsigned block, unsigned cap)
{
    size_t g = (items + block - 1) / block;
    if (g > cap) g = cap;
    if (g == 0) g = 1;
    return (unsigned)g;
}

}  // namespace

// ---------------------------------------------------------------------------
int nmfb_colsum(nmfb_ctx *ctx, const float *X, uint32_t rows, float *acc, int which)
{
    unsigned const block = 256;
    unsigned grid = (rows + 31) / 32;        // ~32 rows per block; at most 1024 block partials
    if (grid > 1024u) grid = 1024u;
    if (grid < 1) grid = 1;
    k_colsum<<<grid, block, 0, ctx->stream>>>(X, rows, ctx->kp, ctx->dColPart + (size_t)which * 1024 * ctx->kp, acc,
                                             ctx->dTickets + which, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

static int launch_factor(nmfb_ctx *ctx, int mode, float *X, uint32_t rows, const float *part, uint32_t nsplit,
                         size_t split_stride, const float *acc, int adjust, const ConvState *st)
{
    size_t const total = (size_t)rows * ctx->kp;
    unsigned const grid = grid_for(total, 256, 8u * (unsigned)ctx->sm_count);
    k_factor<<<grid, 256, 0, ctx->stream>>>(mode, X, rows, ctx->kp, ctx->k, part, nsplit, split_stride, acc, adjust, st);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

int nmfb_muldiv(nmfb_ctx *ctx, float *X, uint32_t rows, const float *part, uint32_t nsplit, size_t split_stride,
                const float *acc, int adjust)
{
    return launch_factor(ctx, FU_MULDIV, X, rows, part, nsplit, split_stride, acc, adjust, ctx->dState);
}

int nmfb_adjust_rows(nmfb_ctx *ctx, float *X, uint32_t rows)
{
    return launch_factor(ctx, FU_ADJUST, X, rows, nullptr, 0, 0, nullptr, 0, nullptr);
}

static uint32_t classify_width(uint32_t k)
{
    uint32_t const kp32 = ((k + 31u) / 32u) * 32u;
    if (kp32 <= 96u) return 32u;
    uint32_t b = (kp32 + 2u) / 3u, p = 1;
    while (p < b) p <<= 1;
    return p > 1024u ? 1024u : p;
}

static int launch_classify(nmfb_ctx *ctx, int adjust, const ConvState *st)
{
    uint32_t const bdx = classify_width(ctx->k);
    uint32_t const block = bdx >= 256 ? bdx : 256;
    uint32_t const groups = block / bdx;
    uint32_t const grid = (ctx->m + groups - 1) / groups;
    size_t const smem = (size_t)block * (sizeof(float) + sizeof(uint32_t));
    k_classify<<<grid, block, smem, ctx->stream>>>(ctx->dH, ctx->m, ctx->kp, ctx->k, bdx, adjust, ctx->dLabels,
                                                  ctx->dFirst, st);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

int nmfb_classify_and_test(nmfb_ctx *ctx, uint32_t niter_test_conv)
{
    (void)niter_test_conv;
    int rc = launch_classify(ctx, 1, ctx->dState);
    if (rc) return rc;
    unsigned const grid = grid_for(ctx->m, 256, 2u * (unsigned)ctx->sm_count);
    k_conv_compare<<<grid, 256, 0, ctx->stream>>>(ctx->dLabels, ctx->dFirst, ctx->dLastRep, ctx->m, ctx->kp,
                                                 ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

int nmfb_classify_only(nmfb_ctx *ctx)
{
    int rc = launch_classify(ctx, 0, nullptr);
    if (rc) return rc;
    // first[] was consumed only as scratch here; restore it for the next test.
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dFirst, 0xff, ctx->kp * sizeof(uint32_t), ctx->stream));
    return NMFB_OK;
}

int nmfb_reset_conv(nmfb_ctx *ctx, uint32_t stop_threshold)
{
    ConvState s;
    memset(&s, 0, sizeof(s));
    s.stop_threshold = stop_threshold;
    *ctx->hState = s;
    NMFB_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dState, ctx->hState, sizeof(ConvState), cudaMemcpyHostToDevice,
                                       ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dLastRep, 0, ctx->m * sizeof(uint32_t), ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dFirst, 0xff, ctx->kp * sizeof(uint32_t), ctx->stream));
    // The host mirror is overwritten by the copy above only after it executes;
    // wait so that a later read of hState cannot see a stale value.
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return NMFB_OK;
}

int nmfb_objectives_rows(nmfb_ctx *ctx, const float *V, const float *W, uint32_t rows, double out[3])
{
    unsigned const grid = 4u * (unsigned)ctx->sm_count;
    k_objective<<<grid, 256, 0, ctx->stream>>>(V, ctx->ldv, W, ctx->dH, rows, ctx->m, ctx->kp, ctx->k, ctx->dObj,
                                              ctx->dObj + 3 * 1024, ctx->dObjTicket);
    NMFB_LAUNCH_CHECK(ctx);
    NMFB_CUDA_TRY(ctx, cudaMemcpyAsync(out, ctx->dObj + 3 * 1024, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return NMFB_OK;
}

int nmfb_objectives(nmfb_ctx *ctx, double *dot_V, double *dot_VWH, double *kl)
{
    double host[3];
    int const rc = ctx->splan ? nmfb_stream_objectives(ctx, host) : nmfb_objectives_rows(ctx, ctx->dV, ctx->dW, ctx->n, host);
    if (rc) return rc;
    if (dot_V) *dot_V = host[0];
    if (dot_VWH) *dot_VWH = host[1];
    if (kl) *kl = host[2];
    return NMFB_OK;
}
