// noalloc.cu -- nmfb_update_H_noalloc: the update_H half-iteration for callers
// that must not allocate device memory.
//
// Who needs it: a host framework that owns the whole device-memory budget
// (a caching allocator that has already reserved the HBM, or a plugin host
// that hands out every device buffer itself) cannot let a library call
// cudaMalloc behind its back, and a latency-sensitive loop cannot afford the
// device-wide synchronisation that cudaFree implies.  Such a caller keeps V, W
// and H in its own device buffers and calls this one function; everything
// else the update needs lives in a fixed, file-scope device array.
//
// Scratch: g_noalloc_scratch, NMFB_NOALLOC_SCRATCH_BYTES (16 MiB) per device,
// part of the library's device image: every GPU that loads the library holds
// it until the process exits.  Layout (offsets in bytes from the 256-aligned
// base):
//   [0, 32 KiB)            colpart: NA_MAX_SPLITS x 64 doubles, per-split column
//                          sums of W
//   [32 KiB, 16 MiB)       part:    nsplit x m x k floats, per-split partial
//                          sums of Q^T W (Q = V ./ (W H^T))
// Every scratch word a call reads is written earlier in the same call (each
// (split, row, factor) slot by exactly one CTA), so nothing carries over from
// the previous call and nothing has to be cleared.  All calls share the one
// array: two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it and both results are undefined.
//
// Host code sees g_noalloc_scratch only as a host-side stand-in symbol; the
// device address comes from cudaGetSymbolAddress, taken on the first call made
// while a device is current and cached with that device's current context (a
// call under a different context -- after cudaDeviceReset, say -- takes it
// again).  Make the first call on a device before any stream capture.
//
// The arithmetic follows the reference's update_H (src/NMF_routines.c:704-1000
// with kernel_mul_div, src/GPU_kernels.cu:1886-2058): colsum(W) in FP64 summed in split order,
// Haux = Q^T W with Q = V ./ (W H^T), then H = (H .* Haux) ./ colsum(W),
// product first, then a correctly-rounded division.  It is an FP32 SIMT
// variant of the engine's own update_H; results agree with nmfb_update_H to
// FP32 rounding, not bit for bit.
#include "../../include/nmfb200.h"

#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>

namespace {

constexpr size_t NA_SCRATCH_BYTES = (size_t)NMFB_NOALLOC_SCRATCH_BYTES;
constexpr uint32_t NA_MAX_SPLITS = 64;
constexpr uint32_t NA_KMAX = 64;
constexpr size_t NA_COLPART_BYTES = (size_t)NA_MAX_SPLITS * NA_KMAX * sizeof(double);   // 32 KiB
constexpr size_t NA_PART_FLOATS = (NA_SCRATCH_BYTES - NA_COLPART_BYTES) / sizeof(float);
static_assert(NA_PART_FLOATS == (size_t)NMFB_NOALLOC_MAX_MK, "header limit and scratch layout disagree");

constexpr int NA_THREADS = 256;   // one column j of V (one sample) per thread
constexpr int NA_WT = 32;         // rows of W staged in shared memory per step
constexpr int NA_MAX_DEV = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

// CTA (x, s) covers samples j in [256x, 256x+256) and rows i of split s.
// part[s][j][c] = sum_{i in split s} V[i][j] / (W_i . H_j) * W[i][c];
// CTAs with x == 0 also write colpart[s][c] = sum_{i in split s} W[i][c] (FP64).
template <int KB>
__global__ void __launch_bounds__(NA_THREADS) k_na_partials(const float *__restrict__ V, size_t ldv,
                                                            const float *__restrict__ W, size_t ldw,
                                                            const float *__restrict__ H, size_t ldh, uint32_t n,
                                                            uint32_t m, uint32_t k, uint32_t rows_per_split,
                                                            float *__restrict__ part, double *__restrict__ colpart)
{
    __shared__ float sW[NA_WT][KB];
    uint32_t const tid = threadIdx.x;
    uint32_t const j = blockIdx.x * NA_THREADS + tid;
    uint32_t const s = blockIdx.y;
    bool const active = j < m;
    bool const colsum_cta = blockIdx.x == 0;
    uint64_t const r0_wide = (uint64_t)s * rows_per_split;
    uint32_t const r0 = r0_wide < n ? (uint32_t)r0_wide : n;
    uint32_t const r1 = (uint64_t)r0 + rows_per_split < n ? r0 + rows_per_split : n;

    float h[KB], acc[KB];
#pragma unroll
    for (int c = 0; c < KB; c++) {
        h[c] = (active && (uint32_t)c < k) ? H[(size_t)j * ldh + c] : 0.0f;
        acc[c] = 0.0f;
    }
    double cs = 0.0;
    for (uint32_t i0 = r0; i0 < r1; i0 += NA_WT) {
        uint32_t const rows = min((uint32_t)NA_WT, r1 - i0);
        __syncthreads();
        for (uint32_t e = tid; e < (uint32_t)(NA_WT * KB); e += NA_THREADS) {
            uint32_t const r = e / KB, c = e % KB;
            sW[r][c] = (r < rows && c < k) ? W[(size_t)(i0 + r) * ldw + c] : 0.0f;
        }
        __syncthreads();
        if (colsum_cta && tid < (uint32_t)KB)
            for (uint32_t r = 0; r < rows; r++) cs += (double)sW[r][tid];
        if (active) {
            for (uint32_t r = 0; r < rows; r++) {
                float wh = 0.0f;
#pragma unroll
                for (int c = 0; c < KB; c++) wh = fmaf(sW[r][c], h[c], wh);
                float const q = V[(size_t)(i0 + r) * ldv + j] / wh;
#pragma unroll
                for (int c = 0; c < KB; c++) acc[c] = fmaf(q, sW[r][c], acc[c]);
            }
        }
    }
    if (active) {
        float *dst = part + ((size_t)s * m + j) * k;
#pragma unroll
        for (int c = 0; c < KB; c++)
            if ((uint32_t)c < k) dst[c] = acc[c];
    }
    if (colsum_cta && tid < k) colpart[(size_t)s * NA_KMAX + tid] = cs;
}

// H[j][c] = (H[j][c] * sum_s part[s][j][c]) / (float)sum_s colpart[s][c],
// both sums in split order.
__global__ void __launch_bounds__(NA_THREADS) k_na_finish(float *__restrict__ H, size_t ldh, uint32_t m, uint32_t k,
                                                          uint32_t nsplit, const float *__restrict__ part,
                                                          const double *__restrict__ colpart)
{
    size_t const total = (size_t)m * k;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        uint32_t const j = (uint32_t)(idx / k), c = (uint32_t)(idx % k);
        float s = 0.0f;
        double a = 0.0;
        for (uint32_t q = 0; q < nsplit; q++) {
            s += part[(size_t)q * total + idx];
            a += colpart[(size_t)q * NA_KMAX + c];
        }
        float *hp = H + (size_t)j * ldh + c;
        *hp = __fdiv_rn(*hp * s, (float)a);
    }
}

struct DeviceSlot {
    bool ready;
    void *cu_ctx;             // CUDA context the address below belongs to
    unsigned char *scratch;   // device address of g_noalloc_scratch in that context
    int sm_count;
};

std::mutex g_slot_mutex;
DeviceSlot g_slots[NA_MAX_DEV];

// The calling thread's current CUDA context (driver cuCtxGetCurrent, found
// through the runtime's entry-point query so the library links only cudart).
void *current_cu_ctx()
{
    typedef int (*GetCurrent)(void **);
    static GetCurrent fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<GetCurrent>(p);
    }
    void *c = nullptr;
    if (!fn || fn(&c) != 0) return nullptr;
    return c;
}

// With the device current: resolve the scratch array's device address and the
// SM count, once per device and context.  The address is cached with the
// context it was taken in: after cudaDeviceReset, or under another context of
// the same device, the module is loaded anew at another address, so a changed
// context resolves it again.  Allocates nothing.
int device_slot(int dev, DeviceSlot *out)
{
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    DeviceSlot &slot = g_slots[dev];
    void *const cu_ctx = current_cu_ctx();
    if (!slot.ready || slot.cu_ctx != cu_ctx) {
        slot.ready = false;
        int major = 0, sms = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            return NMFB_ECUDA;
        }
        if (major != 10) return NMFB_ENODEV;
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) {
            cudaGetLastError();
            return NMFB_ECUDA;
        }
        slot.scratch = static_cast<unsigned char *>(ptr);
        slot.sm_count = sms;
        slot.cu_ctx = cu_ctx;
        slot.ready = true;
    }
    *out = slot;
    return NMFB_OK;
}

template <int KB>
cudaError_t launch_partials(dim3 grid, cudaStream_t st, const float *V, size_t ldv, const float *W, size_t ldw,
                            const float *H, size_t ldh, uint32_t n, uint32_t m, uint32_t k, uint32_t rps,
                            float *part, double *colpart)
{
    k_na_partials<KB><<<grid, NA_THREADS, 0, st>>>(V, ldv, W, ldw, H, ldh, n, m, k, rps, part, colpart);
    return cudaGetLastError();
}

}  // namespace

extern "C" int nmfb_update_H_noalloc(const float *V, size_t ldv, const float *W, size_t ldw, float *H, size_t ldh,
                                     uint32_t n, uint32_t m, uint32_t k, void *stream)
{
    if (!V || !W || !H || n == 0 || m == 0 || k == 0 || k > NA_KMAX || ldv < m || ldw < k || ldh < k)
        return NMFB_EINVAL;
    if ((uint64_t)m * k > (uint64_t)NA_PART_FLOATS) return NMFB_ETOOBIG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return NMFB_ENODEV;
    }
    if (dev < 0 || dev >= NA_MAX_DEV) return NMFB_ENODEV;
    DeviceSlot slot;
    int const rc = device_slot(dev, &slot);
    if (rc != NMFB_OK) return rc;

    double *colpart = reinterpret_cast<double *>(slot.scratch);
    float *part = reinterpret_cast<float *>(slot.scratch + NA_COLPART_BYTES);
    cudaStream_t const st = static_cast<cudaStream_t>(stream);

    // Splits over the rows of V: enough CTAs for ~4 per SM, limited by the
    // scratch (nsplit * m * k floats), by NA_MAX_SPLITS and by n.
    uint32_t const xblocks = (m + NA_THREADS - 1) / NA_THREADS;
    uint64_t want = ((uint64_t)4 * slot.sm_count + xblocks - 1) / xblocks;
    uint64_t const fit = (uint64_t)NA_PART_FLOATS / ((uint64_t)m * k);
    if (want > fit) want = fit;
    if (want > NA_MAX_SPLITS) want = NA_MAX_SPLITS;
    if (want > n) want = n;
    if (want < 1) want = 1;
    uint32_t const rps = (uint32_t)((n + want - 1) / want);
    uint32_t const nsplit = (uint32_t)((n + rps - 1) / rps);

    dim3 const grid(xblocks, nsplit);
    cudaError_t e;
    if (k <= 16)
        e = launch_partials<16>(grid, st, V, ldv, W, ldw, H, ldh, n, m, k, rps, part, colpart);
    else if (k <= 32)
        e = launch_partials<32>(grid, st, V, ldv, W, ldw, H, ldh, n, m, k, rps, part, colpart);
    else
        e = launch_partials<64>(grid, st, V, ldv, W, ldw, H, ldh, n, m, k, rps, part, colpart);
    if (e != cudaSuccess) return NMFB_ECUDA;

    uint64_t const total = (uint64_t)m * k;
    uint64_t blocks = (total + NA_THREADS - 1) / NA_THREADS;
    uint64_t const cap = (uint64_t)8 * slot.sm_count;
    if (blocks > cap) blocks = cap;
    k_na_finish<<<(unsigned)blocks, NA_THREADS, 0, st>>>(H, ldh, m, k, nsplit, part, colpart);
    if (cudaGetLastError() != cudaSuccess) return NMFB_ECUDA;
    return NMFB_OK;
}
