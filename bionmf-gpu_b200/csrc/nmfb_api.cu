// nmfb_api.cu -- the C ABI of include/nmfb200.h: context life cycle, data
// movement, the nmf() iteration loop with device-side convergence test.
#include "nmfb_internal.cuh"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <mutex>
#include <new>
#include <vector>

using nmfb::ConvState;

#define NMFB_VERSION "nmfb200 0.1 (sm_100a)"

// One library-owned stream-ordered memory pool per device; freed blocks stay
// in the pool for the next context (no device-wide synchronisation and no new
// mappings when contexts come and go) until nmfb_release_cached trims it.
static std::mutex g_pool_mutex;
static cudaMemPool_t g_pools[64];

static cudaError_t device_pool(int device, cudaMemPool_t *out)
{
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[device]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
        g_pools[device] = pool;
    }
    *out = g_pools[device];
    return cudaSuccess;
}

cudaError_t nmfb_malloc(nmfb_ctx *ctx, void **p, size_t bytes)
{
    cudaMemPool_t pool;
    cudaError_t e = device_pool(ctx->device, &pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes, pool, ctx->own_stream);
}

// Page-locked host staging buffers, shared by every context of the process.
// Allocating or freeing page-locked memory is ordered against the work of all
// streams of the device, so a context that did either for each upload or
// download would stall the kernels of every other context in flight (many
// solves served side by side); buffers taken from here are allocated once,
// in power-of-two sizes, and reused.
namespace {
struct StageBuf {
    void *p;
    size_t bytes;
    bool busy;
};
std::mutex g_stage_mutex;
std::vector<StageBuf> g_stage;

}  // namespace

void *nmfb_stage_get(size_t bytes)
{
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    StageBuf *best = nullptr;
    for (StageBuf &b : g_stage)
        if (!b.busy && b.bytes >= bytes && (!best || b.bytes < best->bytes)) best = &b;
    if (best) {
        best->busy = true;
        return best->p;
    }
    size_t sz = 4096;
    while (sz < bytes) sz <<= 1;
    void *p = nullptr;
    if (cudaHostAlloc(&p, sz, cudaHostAllocPortable) != cudaSuccess) {   // usable by every device's context
        cudaGetLastError();
        return nullptr;
    }
    g_stage.push_back({p, sz, true});
    return p;
}

void nmfb_stage_put(void *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    for (StageBuf &b : g_stage)
        if (b.p == p) {
            b.busy = false;
            return;
        }
}

namespace {
// Free the staging buffers no context holds.
void stage_trim()
{
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    std::vector<StageBuf> keep;
    for (StageBuf &b : g_stage) {
        if (b.busy)
            keep.push_back(b);
        else
            cudaFreeHost(b.p);
    }
    g_stage.swap(keep);
}
}  // namespace

int nmfb_release_cached(int device)
{
    stage_trim();
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        if (device >= 0 && device < 64) pool = g_pools[device];
    }
    if (!pool) return NMFB_OK;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return NMFB_ECUDA;
    if (cudaSetDevice(device) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemPoolTrimTo(pool, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaSetDevice(prev);
        return NMFB_ECUDA;
    }
    cudaSetDevice(prev);
    return NMFB_OK;
}

void nmfb_free(nmfb_ctx *ctx, void *p)
{
    if (p) cudaFreeAsync(p, ctx->own_stream);
}

namespace {

uint32_t padded_rank(uint32_t k)
{
    if (k <= 16) return 16;
    return ((k + 31u) / 32u) * 32u;
}

int check_ctx(nmfb_ctx *ctx)
{
    if (!ctx) return NMFB_EINVAL;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return nmfb_fail(ctx, NMFB_ECUDA, "cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
    return NMFB_OK;
}

template <class T>
int dev_alloc(nmfb_ctx *ctx, T **p, size_t items, const char *what)
{
    *p = nullptr;
    if (items == 0) items = 1;
    cudaError_t e = nmfb_malloc(ctx, (void **)p, items * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return nmfb_fail(ctx, NMFB_ENOMEM, "cudaMalloc(%s, %zu bytes): %s", what, items * sizeof(T),
                         cudaGetErrorString(e));
    }
    return NMFB_OK;
}

void free_all(nmfb_ctx *ctx)
{
    void *bufs[] = {ctx->dV,       ctx->dW,       ctx->dH,    ctx->dAccW,       ctx->dAccH,   ctx->dWH,
                    ctx->dPart,    ctx->dColPart, ctx->dTickets, ctx->dObj, ctx->dObjTicket, ctx->dLabels,
                    ctx->dFirst,   ctx->dLastRep, ctx->dState};
    for (void *b : bufs)
        if (b) nmfb_free(ctx, b);
    nmfb_stage_put(ctx->hState);
    nmfb_stream_release(ctx);
    nmfb_bf16_release(ctx);
    nmfb_fused_release(ctx);
    for (int c = 0; c < 4; c++) {
        if (!ctx->prof_ev[c]) continue;
        for (int i = 0; i < 2 * NMFB_PROF_POOL; i++) cudaEventDestroy(ctx->prof_ev[c][i]);
        free(ctx->prof_ev[c]);
    }
    if (ctx->blk_exec) cudaGraphExecDestroy(ctx->blk_exec);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
}

// Upload a host (rows x cols, ld) float matrix into a device rows x kp buffer
// with zero padding, through a pinned staging buffer.
int upload_factor(nmfb_ctx *ctx, float *dst, const float *src, uint32_t rows, uint32_t cols, size_t ld)
{
    size_t const bytes = (size_t)rows * ctx->kp * sizeof(float);
    float *stage = (float *)nmfb_stage_get(bytes);
    if (!stage) return nmfb_fail(ctx, NMFB_ENOMEM, "page-locked staging buffer of %zu bytes", bytes);
    for (uint32_t r = 0; r < rows; r++) {
        float *d = stage + (size_t)r * ctx->kp;
        memcpy(d, src + (size_t)r * ld, cols * sizeof(float));
        for (uint32_t c = cols; c < ctx->kp; c++) d[c] = 0.0f;
    }
    cudaError_t e = cudaMemcpyAsync(dst, stage, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    nmfb_stage_put(stage);
    if (e != cudaSuccess) return nmfb_fail(ctx, NMFB_ECUDA, "upload: %s", cudaGetErrorString(e));
    return NMFB_OK;
}

int download_factor(nmfb_ctx *ctx, float *dst, const float *src, uint32_t rows, size_t ld)
{
    size_t const bytes = (size_t)rows * ctx->kp * sizeof(float);
    float *stage = (float *)nmfb_stage_get(bytes);
    if (!stage) return nmfb_fail(ctx, NMFB_ENOMEM, "page-locked staging buffer of %zu bytes", bytes);
    cudaError_t e = cudaMemcpyAsync(stage, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess)
        for (uint32_t r = 0; r < rows; r++) memcpy(dst + (size_t)r * ld, stage + (size_t)r * ctx->kp, ctx->k * sizeof(float));
    nmfb_stage_put(stage);
    if (e != cudaSuccess) return nmfb_fail(ctx, NMFB_ECUDA, "download: %s", cudaGetErrorString(e));
    return NMFB_OK;
}

// Upload the host matrix V (n x m, ld) into the device's n x ldv layout.  From
// page-locked memory: one pitched DMA.  From pageable memory: rows are packed
// at the device pitch (padding zero) into two page-locked staging buffers of
// at most 8 MB in turn, each copied with one DMA while the next is filled (a
// pitched copy straight from pageable memory moves one short row at a time).
int upload_V(nmfb_ctx *ctx, const float *V, size_t ld)
{
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, V) == cudaSuccess && pa.type == cudaMemoryTypeHost) {
        NMFB_CUDA_TRY(ctx, cudaMemcpy2DAsync(ctx->dV, ctx->ldv * sizeof(float), V, ld * sizeof(float),
                                             ctx->m * sizeof(float), ctx->n, cudaMemcpyHostToDevice, ctx->stream));
        NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        return NMFB_OK;
    }
    cudaGetLastError();
    size_t const row_bytes = ctx->ldv * sizeof(float);
    uint32_t const per = (uint32_t)((size_t)(8u << 20) / row_bytes > 0 ? (size_t)(8u << 20) / row_bytes : 1);
    uint32_t const rows = per < ctx->n ? per : ctx->n;
    float *stage[2] = {(float *)nmfb_stage_get(rows * row_bytes), (float *)nmfb_stage_get(rows * row_bytes)};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t e = (stage[0] && stage[1]) ? cudaSuccess : cudaErrorMemoryAllocation;
    for (int b = 0; b < 2 && e == cudaSuccess; b++) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
    uint32_t c = 0;
    for (uint32_t r0 = 0; r0 < ctx->n && e == cudaSuccess; r0 += rows, c++) {
        uint32_t const nr = ctx->n - r0 < rows ? ctx->n - r0 : rows;
        float *const st = stage[c & 1];
        if (c >= 2) e = cudaEventSynchronize(ev[c & 1]);   // the DMA of chunk c - 2 has read this buffer
        if (e != cudaSuccess) break;
        for (uint32_t r = 0; r < nr; r++) {
            float *d = st + (size_t)r * ctx->ldv;
            memcpy(d, V + (size_t)(r0 + r) * ld, ctx->m * sizeof(float));
            memset(d + ctx->m, 0, (ctx->ldv - ctx->m) * sizeof(float));
        }
        e = cudaMemcpyAsync(ctx->dV + (size_t)r0 * ctx->ldv, st, nr * row_bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[c & 1], ctx->stream);
    }
    cudaError_t const es = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = es;
    for (int b = 0; b < 2; b++) {
        if (ev[b]) cudaEventDestroy(ev[b]);
        nmfb_stage_put(stage[b]);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nmfb_fail(ctx, e == cudaErrorMemoryAllocation ? NMFB_ENOMEM : NMFB_ECUDA, "upload of V: %s",
                         cudaGetErrorString(e));
    }
    return NMFB_OK;
}

int do_update_H(nmfb_ctx *ctx, int adjust)
{
    if (ctx->splan) return nmfb_stream_update_H(ctx, adjust);
    if (ctx->arm == NMFB_ARM_PLAIN) return nmfb_plain_update_H(ctx, adjust);
    if (ctx->arm >= NMFB_ARM_BF16) return nmfb_bf16_update_H(ctx, adjust);
    return nmfb_fused_update_H(ctx, adjust);
}

int do_update_W(nmfb_ctx *ctx, int adjust)
{
    if (ctx->splan) return nmfb_stream_update_W(ctx, adjust);
    if (ctx->arm == NMFB_ARM_PLAIN) return nmfb_plain_update_W(ctx, adjust);
    if (ctx->arm >= NMFB_ARM_BF16) return nmfb_bf16_update_W(ctx, adjust);
    return nmfb_fused_update_W(ctx, adjust);
}

int ready(nmfb_ctx *ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!ctx->v_set) return nmfb_fail(ctx, NMFB_ESTATE, "V has not been set (nmfb_set_V)");
    if (!ctx->wh_set) return nmfb_fail(ctx, NMFB_ESTATE, "W/H have not been initialised");
    return NMFB_OK;
}

}  // namespace

extern "C" {

const char *nmfb_version(void) { return NMFB_VERSION; }

int nmfb_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int usable = 0;
    for (int d = 0; d < n; d++) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) == cudaSuccess && major == 10) usable++;
    }
    return usable;
}

static int create_impl(nmfb_ctx **out, int device, uint32_t n, uint32_t m, uint32_t k, int arm, int streamed,
                       uint32_t block_rows)
{
    if (!out) return NMFB_EINVAL;
    *out = nullptr;
    nmfb_ctx *ctx = new (std::nothrow) nmfb_ctx;
    if (!ctx) return NMFB_ENOMEM;
    memset(ctx, 0, sizeof(*ctx));
    ctx->device = device;
    ctx->arm = arm;
    *out = ctx;  // returned even on failure so that nmfb_last_error works; caller destroys it
    if (n < 2 || m < 2) return nmfb_fail(ctx, NMFB_EINVAL, "both matrix dimensions must be greater than 1 (n=%u, m=%u)", n, m);
    if (k < 2) return nmfb_fail(ctx, NMFB_EINVAL, "invalid factorization rank: K=%u (must be >= 2)", k);
    if (k > (n < m ? n : m))
        return nmfb_fail(ctx, NMFB_EINVAL,
                         "invalid factorization rank: K=%u. It must not be greater than any of matrix dimensions.", k);
    if (k > 256) return nmfb_fail(ctx, NMFB_EINVAL, "factorization rank K=%u exceeds the supported maximum of 256", k);
    if (arm < NMFB_ARM_FUSED || arm > NMFB_ARM_BF16X3)
        return nmfb_fail(ctx, NMFB_EINVAL, "unknown arm %d", arm);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return nmfb_fail(ctx, NMFB_ENODEV, "no CUDA device %d (devices: %d)", device, ndev);
    }
    int major = 0, minor = 0, sms = 0;
    NMFB_CUDA_TRY(ctx, cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    NMFB_CUDA_TRY(ctx, cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
    NMFB_CUDA_TRY(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (major != 10)
        return nmfb_fail(ctx, NMFB_ENODEV, "device %d is sm_%d%d; this engine is built for sm_100a only", device,
                         major, minor);
    NMFB_CUDA_TRY(ctx, cudaSetDevice(device));
    ctx->sm_count = sms;
    NMFB_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
    ctx->stream = ctx->own_stream;
    ctx->n = n;
    ctx->m = m;
    ctx->k = k;
    ctx->kp = padded_rank(k);
    ctx->ldv = ((size_t)m + 31) / 32 * 32;
    size_t const kp = ctx->kp;
    size_t const maxr = n > m ? n : m;
    int rc;
    if (!streamed && (rc = dev_alloc(ctx, &ctx->dV, (size_t)n * ctx->ldv, "V"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dW, (size_t)n * kp, "W"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dH, (size_t)m * kp, "H"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dAccW, kp, "accW"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dAccH, kp, "accH"))) return rc;
    // Split-reduction partials: both arms size their splits so that
    // nsplit * rows <= 4*SMs*128 + 2*rows + 128 (see the split planners).
    ctx->part_items = ((size_t)512 * ctx->sm_count + 4 * maxr + 256) * kp;
    if ((rc = dev_alloc(ctx, &ctx->dPart, ctx->part_items, "partials"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dColPart, (size_t)2 * 1024 * kp, "colsum partials"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dTickets, 16, "tickets"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dObj, (size_t)3 * 1024 + 8, "objective"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dObjTicket, 4, "objective ticket"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dLabels, m, "labels"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dFirst, kp, "first"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dLastRep, m, "last rep"))) return rc;
    if ((rc = dev_alloc(ctx, &ctx->dState, 1, "state"))) return rc;
    ctx->hState = (ConvState *)nmfb_stage_get(2 * sizeof(ConvState));
    if (!ctx->hState) return nmfb_fail(ctx, NMFB_ENOMEM, "page-locked convergence state");
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dTickets, 0, 16 * sizeof(uint32_t), ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dObjTicket, 0, 4 * sizeof(uint32_t), ctx->stream));
    if (ctx->dV) NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dV, 0, (size_t)n * ctx->ldv * sizeof(float), ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dW, 0, (size_t)n * kp * sizeof(float), ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dH, 0, (size_t)m * kp * sizeof(float), ctx->stream));
    if ((rc = nmfb_reset_conv(ctx, 40))) return rc;
    if (streamed) {
        if ((rc = nmfb_stream_prepare(ctx, block_rows))) return rc;
        ctx->arm = NMFB_ARM_PLAIN;
    } else if ((rc = nmfb_set_arm(ctx, arm))) {
        return rc;
    }
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->own_stream));   // allocations usable from any stream
    return NMFB_OK;
}

uint64_t nmfb_context_bytes(int device, uint32_t n, uint32_t m, uint32_t k, int arm, uint32_t stream_rows)
{
    if (n < 2 || m < 2 || k < 2) return 0;
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    uint64_t const kp = padded_rank(k), ldv = ((uint64_t)m + 31) / 32 * 32, maxr = n > m ? n : m;
    uint64_t b = 0;
    uint64_t const nv = (uint64_t)n * ldv * 4;
    b += stream_rows ? 0 : nv;                                         // V
    b += ((uint64_t)n + m + 2) * kp * 4;                               // W, H, colsums
    b += ((uint64_t)512 * sms + 4 * maxr + 256) * kp * 4;               // split partials
    b += 2 * 1024 * kp * 8 + 64 + (3 * 1024 + 8) * 8 + 16 + (2ull * m + kp) * 4 + 64;   // test / objective state
    if (stream_rows) {
        uint64_t const rows = stream_rows < n ? stream_rows : n;
        b += 3 * rows * ldv * 4 + (uint64_t)m * kp * 4;               // block buffers, Aux
    } else if (arm == NMFB_ARM_PLAIN) {
        b += nv;                                                       // WH
    } else {
        b += 4 + (2 * ((uint64_t)n + m) + ((n + 31) / 32 + (m + 31) / 32) * 64) * kp * 4;   // TF32 splits
        if (arm >= NMFB_ARM_BF16)
            b += (2 * ((uint64_t)n + m) + ((n + 63) / 64 + (m + 63) / 64) * 128) * kp * 2;  // BF16 splits
    }
    return b + 32ull * (2u << 20);   // allocation granularity slack for ~32 buffers
}

int nmfb_create(nmfb_ctx **out, int device, uint32_t n, uint32_t m, uint32_t k, int arm)
{
    return create_impl(out, device, n, m, k, arm, 0, 0);
}

int nmfb_create_streamed(nmfb_ctx **out, int device, uint32_t n, uint32_t m, uint32_t k, uint32_t block_rows)
{
    return create_impl(out, device, n, m, k, NMFB_ARM_PLAIN, 1, block_rows);
}

int nmfb_set_arm(nmfb_ctx *ctx, int arm)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (arm < NMFB_ARM_FUSED || arm > NMFB_ARM_BF16X3)
        return nmfb_fail(ctx, NMFB_EINVAL, "unknown arm %d", arm);
    if (ctx->splan) {
        if (arm != NMFB_ARM_PLAIN)
            return nmfb_fail(ctx, NMFB_EINVAL, "a streamed-V context runs the plain FP32 arm on row blocks only");
        return NMFB_OK;
    }
    if (arm == NMFB_ARM_PLAIN) {
        if (!ctx->dWH && (rc = dev_alloc(ctx, &ctx->dWH, (size_t)ctx->n * ctx->ldv, "WH"))) return rc;
        if (ctx->stream != ctx->own_stream) NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->own_stream));
        ctx->arm = arm;
        return NMFB_OK;
    }
    if (ctx->kp > 64)
        return nmfb_fail(ctx, NMFB_EINVAL, "the fused arms support ranks up to 64 (k=%u); use NMFB_ARM_PLAIN", ctx->k);
    if ((rc = nmfb_fused_prepare(ctx))) return rc;
    if (arm >= NMFB_ARM_BF16 && (rc = nmfb_bf16_prepare(ctx))) return rc;
    if (ctx->stream != ctx->own_stream) NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->own_stream));
    ctx->arm = arm;
    return NMFB_OK;
}

int nmfb_destroy(nmfb_ctx *ctx)
{
    if (!ctx) return NMFB_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    delete ctx;
    return NMFB_OK;
}

const char *nmfb_last_error(const nmfb_ctx *ctx)
{
    if (!ctx) return "null context";
    return ctx->err;
}

int nmfb_set_V(nmfb_ctx *ctx, const float *V, size_t ldv)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!V || ldv < ctx->m) return nmfb_fail(ctx, NMFB_EINVAL, "nmfb_set_V: null V or ldv (%zu) < m (%u)", ldv, ctx->m);
    if (ctx->splan) {
        if ((rc = nmfb_stream_set_V(ctx, V, ldv))) return rc;
        ctx->v_set = 1;
        return NMFB_OK;
    }
    if ((rc = upload_V(ctx, V, ldv))) return rc;
    ctx->v_set = 1;
    return NMFB_OK;
}

int nmfb_set_V_device(nmfb_ctx *ctx, const float *dV, size_t ldv)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!dV || ldv < ctx->m) return nmfb_fail(ctx, NMFB_EINVAL, "nmfb_set_V_device: null V or ldv < m");
    if (ctx->splan) return nmfb_fail(ctx, NMFB_ESTATE, "a streamed-V context reads V from host memory (nmfb_set_V)");
    NMFB_CUDA_TRY(ctx, cudaMemcpy2DAsync(ctx->dV, ctx->ldv * sizeof(float), dV, ldv * sizeof(float),
                                         ctx->m * sizeof(float), ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
    ctx->v_set = 1;
    return NMFB_OK;
}

int nmfb_init_random(nmfb_ctx *ctx, uint32_t seed)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    uint32_t const n = ctx->n, m = ctx->m, k = ctx->k;
    float *W = (float *)malloc((size_t)n * k * sizeof(float));
    float *H = (float *)malloc((size_t)m * k * sizeof(float));
    if (!W || !H) {
        free(W);
        free(H);
        return nmfb_fail(ctx, NMFB_ENOMEM, "host allocation for the initial factors");
    }
    // src/NMF_routines.c:206-233 and 299-307: srandom(seed); W first, then H;
    // (float)random()/(float)RAND_MAX + FLT_MIN per factor entry.  The same
    // glibc generator through a private state (initstate_r / random_r with the
    // default 128-byte state gives srandom/random's sequence), so contexts on
    // different host threads do not share the process-wide generator.
    char rstate[128];
    struct random_data rd;
    memset(&rd, 0, sizeof(rd));
    initstate_r(seed, rstate, sizeof(rstate), &rd);
    auto next = [&]() -> float {
        int32_t r;
        random_r(&rd, &r);
        return ((float)r) / ((float)RAND_MAX) + FLT_MIN;
    };
    for (size_t e = 0; e < (size_t)n * k; e++) W[e] = next();
    for (size_t e = 0; e < (size_t)m * k; e++) H[e] = next();
    rc = nmfb_set_WH(ctx, W, k, H, k);
    free(W);
    free(H);
    return rc;
}

int nmfb_set_WH(nmfb_ctx *ctx, const float *W, size_t ldw, const float *H, size_t ldh)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!W || !H || ldw < ctx->k || ldh < ctx->k) return nmfb_fail(ctx, NMFB_EINVAL, "nmfb_set_WH: bad arguments");
    if ((rc = upload_factor(ctx, ctx->dW, W, ctx->n, ctx->k, ldw))) return rc;
    if ((rc = upload_factor(ctx, ctx->dH, H, ctx->m, ctx->k, ldh))) return rc;
    ctx->wh_set = 1;
    return NMFB_OK;
}

int nmfb_update_H(nmfb_ctx *ctx)
{
    int rc = ready(ctx);
    if (rc) return rc;
    ctx->fz_ok[0] = ctx->fz_ok[1] = 0;   // the caller may have changed W or H since
    return do_update_H(ctx, 0);
}

int nmfb_update_W(nmfb_ctx *ctx)
{
    int rc = ready(ctx);
    if (rc) return rc;
    ctx->fz_ok[0] = ctx->fz_ok[1] = 0;
    return do_update_W(ctx, 0);
}

int nmfb_adjust(nmfb_ctx *ctx)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if ((rc = nmfb_adjust_rows(ctx, ctx->dH, ctx->m))) return rc;
    return nmfb_adjust_rows(ctx, ctx->dW, ctx->n);
}

int nmfb_get_classification(nmfb_ctx *ctx, uint32_t *labels)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if (!labels) return nmfb_fail(ctx, NMFB_EINVAL, "null labels");
    if ((rc = nmfb_classify_only(ctx))) return rc;
    NMFB_CUDA_TRY(ctx, cudaMemcpyAsync(labels, ctx->dLabels, ctx->m * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                       ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return NMFB_OK;
}

// One convergence-test block: J iterations (EPS adjust of W in the last
// update_W) and the classification / connectivity test.
static int enqueue_block(nmfb_ctx *ctx, uint32_t J)
{
    int rc = 0;
    for (uint32_t i = 0; i < J && rc == 0; i++) {
        rc = do_update_H(ctx, 0);
        if (!rc) rc = do_update_W(ctx, i + 1 == J);
    }
    if (!rc) rc = nmfb_classify_and_test(ctx, J);
    ctx->fz_ok[1] = 0;   // the test's EPS adjust rewrote H
    return rc;
}

// Queue one test block, through a CUDA graph captured once per (J, arm,
// stream) when profiling is off and V is resident; kernel launches otherwise.
static int launch_block(nmfb_ctx *ctx, uint32_t J)
{
    static int const use_graphs = getenv("NMFB_NO_GRAPHS") == nullptr;
    if (!use_graphs || ctx->prof_on || ctx->splan) return enqueue_block(ctx, J);
    // the graph holds no preparation launch: make W's split copies current first
    int const rc0 = (ctx->arm == NMFB_ARM_FUSED || ctx->arm == NMFB_ARM_FUSED_TF32) ? nmfb_fused_ready_W(ctx)
                    : ctx->arm >= NMFB_ARM_BF16                                    ? nmfb_bf16_ready_W(ctx)
                                                                                   : NMFB_OK;
    if (rc0) return rc0;
    if (!ctx->blk_exec || ctx->blk_J != J || ctx->blk_arm != ctx->arm || ctx->blk_stream != ctx->stream ||
        ctx->blk_wait != ctx->wait_ns) {
        if (ctx->blk_exec) {
            NMFB_CUDA_TRY(ctx, cudaGraphExecDestroy(ctx->blk_exec));
            ctx->blk_exec = nullptr;
        }
        uint64_t const l0 = ctx->launches;
        NMFB_CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int const rc = enqueue_block(ctx, J);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ctx->blk_exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            ctx->blk_exec = nullptr;
            return nmfb_fail(ctx, NMFB_ECUDA, "capturing the test block: %s", cudaGetErrorString(e));
        }
        ctx->blk_kernels = ctx->launches - l0;
        ctx->launches = l0;
        ctx->blk_J = J;
        ctx->blk_arm = ctx->arm;
        ctx->blk_stream = ctx->stream;
        ctx->blk_wait = ctx->wait_ns;
    }
    NMFB_CUDA_TRY(ctx, cudaGraphLaunch(ctx->blk_exec, ctx->stream));
    ctx->launches += ctx->blk_kernels;
    ctx->fz_ok[0] = 1;   // the block ends with update_W's epilogue and the test's adjust of H
    ctx->fz_ok[1] = 0;
    return NMFB_OK;
}

int nmfb_run(nmfb_ctx *ctx, uint32_t n_iters, uint32_t niter_test_conv, uint32_t stop_threshold, uint32_t *iterations,
             int *converged)
{
    int rc = ready(ctx);
    if (rc) return rc;
    if (n_iters == 0 || niter_test_conv == 0 || stop_threshold == 0)
        return nmfb_fail(ctx, NMFB_EINVAL, "nIters, niter_test_conv and stop_threshold must be positive");
    if ((rc = nmfb_reset_conv(ctx, stop_threshold))) return rc;
    ctx->fz_ok[0] = ctx->fz_ok[1] = 0;
    uint32_t const niter_conv = n_iters / niter_test_conv;
    uint32_t const niter_rem = n_iters % niter_test_conv;
    // Test blocks are queued in batches; the host looks at the device state of
    // the previous batch (already finished or nearly so) before queueing more.
    // Kernels queued after the stop rule fired return immediately.
    uint32_t const batch = 4;
    cudaEvent_t ev[2];
    NMFB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    NMFB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    ctx->in_run = 1;
    int stopped = 0;
    uint32_t b = 0, q = 0;
    while (b < niter_conv && !stopped) {
        uint32_t const end = (b + batch < niter_conv) ? b + batch : niter_conv;
        for (; b < end; b++) {
            rc = launch_block(ctx, niter_test_conv);
            if (rc) break;
        }
        if (rc) break;
        ConvState *slot = ctx->hState + (q & 1);
        cudaError_t e = cudaMemcpyAsync(slot, ctx->dState, sizeof(ConvState), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev[q & 1], ctx->stream);
        if (e != cudaSuccess) {
            rc = nmfb_fail(ctx, NMFB_ECUDA, "state copy: %s", cudaGetErrorString(e));
            break;
        }
        if (q > 0) {
            e = cudaEventSynchronize(ev[(q - 1) & 1]);
            if (e != cudaSuccess) {
                rc = nmfb_fail(ctx, NMFB_ECUDA, "event wait: %s", cudaGetErrorString(e));
                break;
            }
            if (ctx->hState[(q - 1) & 1].converged) stopped = 1;
        }
        q++;
    }
    if (!rc && !stopped && niter_rem) {
        // Remaining iterations without adjust; skipped on the device if converged.
        for (uint32_t i = 0; i < niter_rem && rc == 0; i++) {
            rc = do_update_H(ctx, 0);
            if (!rc) rc = do_update_W(ctx, 0);
        }
    }
    ConvState fin;
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(ctx->hState, ctx->dState, sizeof(ConvState), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = nmfb_fail(ctx, NMFB_ECUDA, "final state: %s", cudaGetErrorString(e));
        fin = ctx->hState[0];
        // Re-arm the kernels for single-step calls made after this run.
        if (!rc) {
            e = cudaMemsetAsync(&ctx->dState->converged, 0, sizeof(uint32_t), ctx->stream);
            if (e != cudaSuccess) rc = nmfb_fail(ctx, NMFB_ECUDA, "re-arm: %s", cudaGetErrorString(e));
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    ctx->fz_ok[0] = ctx->fz_ok[1] = 0;
    ctx->in_run = 0;
    if (ctx->splan) nmfb_stream_end_run(ctx);
    if (rc) return rc;
    {
        uint32_t code = 0;
        if ((rc = nmfb_fused_error(ctx, &code))) return rc;
        if (code) return nmfb_fail(ctx, NMFB_ETIMEOUT, "fused kernel: bounded wait expired (site %u)", code);
    }
    if (converged) *converged = fin.converged ? 1 : 0;
    if (iterations) *iterations = fin.converged ? fin.conv_tests * niter_test_conv : n_iters;
    return NMFB_OK;
}

int nmfb_get_W(nmfb_ctx *ctx, float *W, size_t ldw)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!W || ldw < ctx->k) return nmfb_fail(ctx, NMFB_EINVAL, "nmfb_get_W: bad arguments");
    return download_factor(ctx, W, ctx->dW, ctx->n, ldw);
}

int nmfb_get_H(nmfb_ctx *ctx, float *H, size_t ldh)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!H || ldh < ctx->k) return nmfb_fail(ctx, NMFB_EINVAL, "nmfb_get_H: bad arguments");
    return download_factor(ctx, H, ctx->dH, ctx->m, ldh);
}

int nmfb_dot_product_VWH(nmfb_ctx *ctx, double *dot_V, double *dot_VWH)
{
    int rc = ready(ctx);
    if (rc) return rc;
    return nmfb_objectives(ctx, dot_V, dot_VWH, nullptr);
}

int nmfb_kl_divergence(nmfb_ctx *ctx, double *kl)
{
    int rc = ready(ctx);
    if (rc) return rc;
    return nmfb_objectives(ctx, nullptr, nullptr, kl);
}

int nmfb_device_factors(nmfb_ctx *ctx, float **dW, float **dH, uint32_t *ldk)
{
    if (!ctx) return NMFB_EINVAL;
    if (dW) *dW = ctx->dW;
    if (dH) *dH = ctx->dH;
    if (ldk) *ldk = ctx->kp;
    return NMFB_OK;
}

int nmfb_device_V(nmfb_ctx *ctx, float **dV, size_t *ldv)
{
    if (!ctx) return NMFB_EINVAL;
    if (ctx->splan) return nmfb_fail(ctx, NMFB_ESTATE, "a streamed-V context holds no device copy of V");
    if (dV) *dV = ctx->dV;
    if (ldv) *ldv = ctx->ldv;
    return NMFB_OK;
}

int nmfb_set_stream(nmfb_ctx *ctx, void *stream)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return NMFB_OK;
}

static int prof_harvest(nmfb_ctx *ctx, int cls)
{
    uint32_t const n = ctx->prof_n[cls];
    if (n == 0) return NMFB_OK;
    cudaEvent_t *ev = ctx->prof_ev[cls];
    NMFB_CUDA_TRY(ctx, cudaEventSynchronize(ev[2 * n - 1]));
    double s = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        float ms = 0.0f;
        NMFB_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]));
        s += ms;
    }
    ctx->prof_ms[cls] += s;
    ctx->prof_cnt[cls] += n;
    ctx->prof_n[cls] = 0;
    return NMFB_OK;
}

int nmfb_prof_begin(nmfb_ctx *ctx, int cls)
{
    if (!ctx->prof_on) return NMFB_OK;
    if (ctx->prof_n[cls] == NMFB_PROF_POOL) {
        int rc = prof_harvest(ctx, cls);
        if (rc) return rc;
    }
    NMFB_CUDA_TRY(ctx, cudaEventRecord(ctx->prof_ev[cls][2 * ctx->prof_n[cls]], ctx->stream));
    return NMFB_OK;
}

int nmfb_prof_end(nmfb_ctx *ctx, int cls)
{
    if (!ctx->prof_on) return NMFB_OK;
    NMFB_CUDA_TRY(ctx, cudaEventRecord(ctx->prof_ev[cls][2 * ctx->prof_n[cls] + 1], ctx->stream));
    ctx->prof_n[cls]++;
    return NMFB_OK;
}

int nmfb_profile(nmfb_ctx *ctx, int enable)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    for (int c = 0; c < 4; c++) {
        if (enable && !ctx->prof_ev[c]) {
            ctx->prof_ev[c] = (cudaEvent_t *)calloc(2 * NMFB_PROF_POOL, sizeof(cudaEvent_t));
            if (!ctx->prof_ev[c]) return nmfb_fail(ctx, NMFB_ENOMEM, "profile events");
            for (int i = 0; i < 2 * NMFB_PROF_POOL; i++)
                NMFB_CUDA_TRY(ctx, cudaEventCreate(&ctx->prof_ev[c][i]));
        }
        ctx->prof_n[c] = 0;
        ctx->prof_ms[c] = 0.0;
        ctx->prof_cnt[c] = 0;
    }
    ctx->prof_on = enable ? 1 : 0;
    return NMFB_OK;
}

int nmfb_profile_read(nmfb_ctx *ctx, int cls, double *total_ms, uint32_t *count)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (cls < 0 || cls > 3) return nmfb_fail(ctx, NMFB_EINVAL, "profile class %d", cls);
    if (ctx->prof_ev[cls] && (rc = prof_harvest(ctx, cls))) return rc;
    if (total_ms) *total_ms = ctx->prof_ms[cls];
    if (count) *count = ctx->prof_cnt[cls];
    return NMFB_OK;
}

int nmfb_synchronize(nmfb_ctx *ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    uint32_t code = 0;
    if ((rc = nmfb_fused_error(ctx, &code))) return rc;
    if (code) return nmfb_fail(ctx, NMFB_ETIMEOUT, "fused kernel: bounded wait expired (site %u)", code);
    return NMFB_OK;
}

uint64_t nmfb_launch_count(const nmfb_ctx *ctx) { return ctx ? ctx->launches : 0; }

int nmfb_set_wait_limit(nmfb_ctx *ctx, uint64_t ns)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    ctx->wait_ns = (unsigned long long)ns;
    return NMFB_OK;
}

int nmfb_set_sm_limit(nmfb_ctx *ctx, uint32_t sms)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    int dev_sms = 0;
    NMFB_CUDA_TRY(ctx, cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device));
    // The partials were sized for the device's SM count; fewer SMs need fewer.
    ctx->sm_count = (sms == 0 || sms > (uint32_t)dev_sms) ? dev_sms : (int)sms;
    if (ctx->blk_exec) {   // the captured block holds launch shapes of the old count
        NMFB_CUDA_TRY(ctx, cudaGraphExecDestroy(ctx->blk_exec));
        ctx->blk_exec = nullptr;
    }
    return NMFB_OK;
}

}  // extern "C"
