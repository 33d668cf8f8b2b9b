/*
 * nmfb200.h -- C ABI of the B200-native KL-NMF engine (drop-in for the
 * single-GPU path of NMF-mGPU / bioinfo-cnb/bionmf-gpu).
 *
 * The reference keeps all device state in globals (src/GPU_setup.c:191-285)
 * and exposes its loop through the entry points cited below.  This library
 * holds that state in an opaque context instead; one context = one
 * factorisation V (n x m) ~ W (n x k) * H (k x m) on one device.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, integers.  No CUDA or torch types.
 *  - Host matrices are row-major with an explicit leading dimension in items.
 *    H is exchanged as the reference stores it, "transposed": m rows of k
 *    factors (src/NMF_GPU.c:70-76), unless a function says otherwise.
 *  - Every function returns 0 (NMFB_OK) on success or a negative NMFB_E* code;
 *    nmfb_last_error() describes the last failure of a context.  There is no
 *    CPU fallback: without a usable sm_100 device nmfb_create() fails.
 *  - A context is not thread-safe; use one host thread per context.
 *  - Work is queued on the context's CUDA stream; functions that return host
 *    data synchronise that stream.
 */
#ifndef NMFB200_H
#define NMFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NMFB_OK 0
#define NMFB_EINVAL (-1)   /* invalid argument (sizes, rank, null pointer) */
#define NMFB_ECUDA (-2)    /* CUDA runtime error (message in nmfb_last_error) */
#define NMFB_ENOMEM (-3)   /* device or pinned memory allocation failed */
#define NMFB_ENODEV (-4)   /* no sm_100 device / extension not usable */
#define NMFB_ESTATE (-5)   /* call out of order (e.g. update before V is set) */
#define NMFB_ETIMEOUT (-6) /* a bounded device wait ran out */
#define NMFB_ETOOBIG (-7)  /* problem larger than nmfb_update_H_noalloc's fixed scratch */

/* Update kernels ("arms").  All arms run the same method; they differ only
 * in how the two n x m x k contractions of a half-iteration are evaluated. */
#define NMFB_ARM_FUSED 0  /* fused half-iteration (one launch): TF32 hi x (hi + lo) products plus the
                           * lo x y term as a BF16 product, FP32 accumulation (FP32-accurate, ~2^-20 per product) */
#define NMFB_ARM_PLAIN 1  /* unfused FP32 SIMT kernels mirroring the reference's 5 steps */
#define NMFB_ARM_FUSED_TF32 2 /* fused, 1xTF32 denominator (reduced precision) */
#define NMFB_ARM_BF16 3       /* fused, BF16 operands, FP32 accumulation (reduced precision) */
#define NMFB_ARM_SPLIT_BF16 4 /* fused, split-BF16 WH denominator (3 products), one BF16 product in the second contraction */
#define NMFB_ARM_BF16X3 5     /* fused, split-BF16 (3 products) in both contractions (FP32-class) */

typedef struct nmfb_ctx nmfb_ctx;

/* Library version string. */
const char *nmfb_version(void);

/* Number of CUDA devices usable by the engine (sm_100 class); 0 if none. */
int nmfb_device_count(void);

/*
 * initialize_GPU + setup_GPU (src/GPU_setup.c:569-868, 2105-2239).
 * Creates a context for an n x m input and rank k on `device`, allocating all
 * device buffers.  Fails with NMFB_EINVAL if k < 2, k > min(n, m) (as
 * src/NMF_GPU.c:1121-1128) or k > 256, and with NMFB_ENOMEM if the matrices
 * do not fit the device.
 */
int nmfb_create(nmfb_ctx **ctx, int device, uint32_t n, uint32_t m, uint32_t k, int arm);

/* Blockwise (out-of-core) mode, for V larger than device memory: the
 * reference's block plan and partial uploads (src/GPU_setup.c:902-1270,
 * src/matrix_operations.c:1712-1905).  V is not copied to the device;
 * nmfb_set_V page-locks the caller's host matrix in place (it must stay valid
 * and unchanged until the context is destroyed or given another V) and every
 * half-iteration streams it in blocks of `block_rows` rows (0 = about 256 MB
 * per block) through two device buffers, the copy of the next block
 * overlapping the kernels of the current one.  Runs the plain FP32 arm on row
 * blocks; results equal the resident plain arm's up to FP32 summation order.
 * nmfb_set_V_device and nmfb_device_V fail with NMFB_ESTATE on such a context. */
int nmfb_create_streamed(nmfb_ctx **ctx, int device, uint32_t n, uint32_t m, uint32_t k, uint32_t block_rows);

/* Device memory a context of these sizes and arm will allocate (bytes, an
 * upper bound including allocation granularity; stream_rows > 0 for the
 * blockwise mode), for admission control by a memory budget.  No counterpart
 * in the reference, which sizes its blocks from the free memory instead
 * (src/GPU_setup.c:902-1210).  Returns 0 for invalid sizes. */
uint64_t nmfb_context_bytes(int device, uint32_t n, uint32_t m, uint32_t k, int arm, uint32_t stream_rows);

/* Context device memory comes from a library-owned stream-ordered pool per
 * device (cudaMallocFromPoolAsync), and page-locked host staging buffers (for
 * uploads and downloads, up to 8 MB each, one or two per call in flight) from
 * a process-wide pool, so contexts can be created, fed and destroyed while
 * others compute without synchronising the device.  Freed memory stays
 * cached in the pools for the next context; this returns the device pool's
 * memory to the driver (after synchronising the device) and frees the
 * staging buffers no call holds.  No counterpart in the reference. */
int nmfb_release_cached(int device);

/* finalize_GPU_device (src/GPU_setup.c:2291): frees everything. NULL is a no-op. */
int nmfb_destroy(nmfb_ctx *ctx);

/* Last error message of this context (never NULL). */
const char *nmfb_last_error(const nmfb_ctx *ctx);

/* Select the update arm (NMFB_ARM_*) of an existing context. */
int nmfb_set_arm(nmfb_ctx *ctx, int arm);

/*
 * init_V's upload (src/NMF_GPU.c:212-303 + upload_matrix_partial,
 * src/matrix_operations.c:1712-1905): copies V (n x m, host, row-major,
 * leading dimension ldv >= m) to the device.  Values must be finite and >= 0.
 */
int nmfb_set_V(nmfb_ctx *ctx, const float *V, size_t ldv);

/* Same, from a device pointer (device-to-device copy on the context stream). */
int nmfb_set_V_device(nmfb_ctx *ctx, const float *dV, size_t ldv);

/*
 * init_random + set_random_values in the reference's CPU_RANDOM mode
 * (src/NMF_routines.c:206-233, 271-362): srandom(seed), then W row by row and
 * H row by row, each value (float)random()/(float)RAND_MAX + FLT_MIN.
 * Bit-identical to the reference's host initialisation for the same seed.
 */
int nmfb_init_random(nmfb_ctx *ctx, uint32_t seed);

/* Upload explicit initial factors: W (n x k, ldw >= k), H (m x k, ldh >= k). */
int nmfb_set_WH(nmfb_ctx *ctx, const float *W, size_t ldw, const float *H, size_t ldh);

/* update_H (src/NMF_routines.c:704-1000): H = H .* (W' (V ./ (W H))) ./ colsum(W). */
int nmfb_update_H(nmfb_ctx *ctx);

/* update_W (src/NMF_routines.c:1344-1636): W = W .* ((V ./ (W H)) H') ./ colsum(H). */
int nmfb_update_W(nmfb_ctx *ctx);

/* matrix_adjust on H then W (src/NMF_GPU.c:611-638; src/GPU_kernels.cu:2220-2370). */
int nmfb_adjust(nmfb_ctx *ctx);

/*
 * get_classification (src/NMF_routines.c:1646-1744): for each of the m
 * samples, the index of its largest factor in H, with the reference's tie
 * rule (kernel_idx_max, src/GPU_kernels.cu:3177-3267).  `labels` is a host
 * array of m entries.  Synchronises the stream.
 */
int nmfb_get_classification(nmfb_ctx *ctx, uint32_t *labels);

/*
 * nmf() (src/NMF_GPU.c:312-924, loop :522-795): runs up to n_iters
 * iterations, testing convergence every niter_test_conv iterations (adjust H
 * and W, classify, compare connectivity with the previous test) and stopping
 * once the classification has not changed for stop_threshold more tests.
 * The stable-count and stop flag live on the device; the host does not read
 * them after every test.  Outputs the iterations performed (iter * J on
 * convergence, else n_iters) and whether it converged.
 */
int nmfb_run(nmfb_ctx *ctx, uint32_t n_iters, uint32_t niter_test_conv, uint32_t stop_threshold,
             uint32_t *iterations, int *converged);

/* Download W (n x k into ldw >= k) and H (m x k into ldh >= k). */
int nmfb_get_W(nmfb_ctx *ctx, float *W, size_t ldw);
int nmfb_get_H(nmfb_ctx *ctx, float *H, size_t ldh);

/*
 * dot_product_VWH (src/NMF_routines.c:2680-2794), FP64 accumulation:
 * dot_V = ||V||^2, dot_VWH = ||V - W H||^2.  The reference prints
 * sqrt(dot_VWH)/sqrt(dot_V) as "Distance between V and W*H".
 */
int nmfb_dot_product_VWH(nmfb_ctx *ctx, double *dot_V, double *dot_VWH);

/* Generalised KL divergence sum(V log(V/WH) - V + WH) in FP64 (0 log 0 = 0).
 * The reference has no counterpart; it is the objective the updates descend. */
int nmfb_kl_divergence(nmfb_ctx *ctx, double *kl);

/* Raw device pointers of the factors (for zero-copy callers): W is n x ldk,
 * H is m x ldk, row-major, float, padding columns zero. */
int nmfb_device_factors(nmfb_ctx *ctx, float **dW, float **dH, uint32_t *ldk);

/* Device pointer and leading dimension of V inside the context. */
int nmfb_device_V(nmfb_ctx *ctx, float **dV, size_t *ldv);

/* Queue the context's work on `stream` (a cudaStream_t passed as void*; NULL
 * restores the context's own stream).  The caller keeps ownership. */
int nmfb_set_stream(nmfb_ctx *ctx, void *stream);

/* Device-time profiling of the update kernels with CUDA events recorded on the
 * context stream around each launch.  enable=1 starts (and clears) the record;
 * nmfb_profile_read() synchronises and returns, for kernel class `cls`
 * (0: update_H main kernel, 1: update_W main kernel, 2: whole update_H,
 * 3: whole update_W), the summed milliseconds and the number of launches. */
int nmfb_profile(nmfb_ctx *ctx, int enable);
int nmfb_profile_read(nmfb_ctx *ctx, int cls, double *total_ms, uint32_t *count);

/* Block the host until all queued work of the context is done. */
int nmfb_synchronize(nmfb_ctx *ctx);

/* Kernel launches issued by this context since creation (for accounting). */
uint64_t nmfb_launch_count(const nmfb_ctx *ctx);

/* Limit, in nanoseconds, of every bounded device-side wait of the fused
 * kernels (0 restores the default, 1 s).  A wait that runs out makes its CTA
 * stop, drain the copies and tensor-core work it has in flight and exit; the
 * next nmfb_run / nmfb_synchronize returns NMFB_ETIMEOUT once (the factors are
 * then undefined; the context stays usable after nmfb_init_random or
 * nmfb_set_WH).  No counterpart in the reference, whose kernels do not wait
 * on one another. */
int nmfb_set_wait_limit(nmfb_ctx *ctx, uint64_t ns);

/* Number of SMs this context sizes its launches for (0: all of the device's).
 * The fused arms split each half-iteration's reduction so that one wave of
 * CTAs fills that many SMs; a smaller figure leaves room for the kernels of
 * other contexts on other streams (many small solves served side by side)
 * and gives each CTA a longer run of tiles.  The split count, and with it the
 * summation order, depends on this figure and the sizes only.  No counterpart
 * in the reference, which runs one factorisation per process. */
int nmfb_set_sm_limit(nmfb_ctx *ctx, uint32_t sms);

/* ---------------------------------------------------------------------------
 * Batched solves: rank-selection and restart sweeps.  The reference runs one
 * factorisation per process (nmf(), src/NMF_GPU.c:522-795; its user guide,
 * doc/user_guide.txt.md:367, points to repeated runs and the consensus method
 * of Brunet et al. for choosing k).  A batch runs nprob independent copies of
 * that loop on one V (n x m), problem p with rank ranks[p] in [2, 20], all in
 * one persistent launch, and then summarises each rank's restarts as an exact
 * integer consensus matrix and its cophenetic correlation (FP64).
 */
typedef struct nmfb_batch nmfb_batch;

int nmfb_batch_create(nmfb_batch **b, int device, uint32_t n, uint32_t m, uint32_t nprob, const uint32_t *ranks);
int nmfb_batch_destroy(nmfb_batch *b);
const char *nmfb_batch_last_error(const nmfb_batch *b);

/* V: host or device pointer, n x m, leading dimension ldv >= m. */
int nmfb_batch_set_V(nmfb_batch *b, const float *V, size_t ldv);

/* CPU_RANDOM initialisation of every problem (src/NMF_routines.c:299-307),
 * problem p from srandom(seeds[p]): the same W, H as nmfb_init_random. */
int nmfb_batch_init_random(nmfb_batch *b, const uint32_t *seeds);

/* Explicit initial factors of problem p: W (n x k), H (m x k). */
int nmfb_batch_set_WH(nmfb_batch *b, uint32_t p, const float *W, size_t ldw, const float *H, size_t ldh);

/* Tile shape of problem p: wt rows of W per update_H tile (multiple of 8,
 * 8..512), jt columns of V per update_W tile (a power of two, 4..64). */
int nmfb_batch_set_tiles(nmfb_batch *b, uint32_t p, uint32_t wt, uint32_t jt);

/* CTAs that share each problem (a thread-block cluster; no counterpart in the
 * reference, which runs one problem per process): 1, 2, 4 or 8, or 0 for the
 * automatic choice (8 when nprob * 8 fits the CTA slots of the device, else 4).
 * The CTAs split W's rows and add their partial sums in a fixed order, so a
 * result depends on this value but is the same on every run with it; 1 keeps
 * the single-CTA summation order.  nmfb_batch_get_cluster reports the value
 * the last nmfb_batch_run used. */
int nmfb_batch_set_cluster(nmfb_batch *b, uint32_t ctas);
int nmfb_batch_get_cluster(const nmfb_batch *b, uint32_t *ctas);

/* Run every problem to convergence or n_iters with the reference's rules
 * (-i n_iters, -j niter_test_conv, -t stop_threshold).  iterations[p] and
 * converged[p] (either may be NULL) as nmfb_run reports them. */
int nmfb_batch_run(nmfb_batch *b, uint32_t n_iters, uint32_t niter_test_conv, uint32_t stop_threshold,
                   uint32_t *iterations, int *converged);

/* Device time of the last nmfb_batch_run launch (CUDA events), milliseconds. */
int nmfb_batch_last_ms(const nmfb_batch *b, double *ms);

/* Classification of every problem's final H (nprob x m, row p = problem p). */
int nmfb_batch_get_classification(nmfb_batch *b, uint32_t *labels);
int nmfb_batch_get_WH(nmfb_batch *b, uint32_t p, float *W, size_t ldw, float *H, size_t ldh);

/* Consensus of the problems of rank k: counts (m x m, may be NULL) = number of
 * those runs that co-cluster each sample pair; *nruns = their number;
 * *cophenetic (may be NULL) = cophenetic correlation of average-linkage
 * clustering of 1 - counts / nruns. */
int nmfb_batch_consensus(nmfb_batch *b, uint32_t k, uint32_t *counts, uint32_t *nruns, double *cophenetic);

/* ---------------------------------------------------------------------------
 * Serving (no counterpart in the reference, which solves one matrix per
 * process): requests with their own V (n x m, m <= max_m), rank k (2..max_k,
 * at most 20), seed and -i/-j/-t are queued on the device while a persistent
 * kernel runs; clusters of `ctas` CTAs take them in submission order as they
 * free up, so a request that arrives while others run starts as soon as a
 * cluster is free, and runs the reference's loop exactly as the batched
 * engine does (a request's result does not depend on what else is queued).
 * The kernel leaves after idle_ms without work and is launched again by the
 * next submit or poll.  Device memory per request: nmfb_serve_request_bytes,
 * taken from a pool owned by the server when the request is submitted and
 * returned by nmfb_serve_fetch.  One thread may submit while others poll,
 * wait and fetch; each ticket is polled and fetched by one thread.
 */
typedef struct nmfb_serve nmfb_serve;

int nmfb_serve_create(nmfb_serve **s, int device, uint32_t max_m, uint32_t max_k, uint32_t capacity, uint32_t ctas,
                      uint32_t idle_ms);
int nmfb_serve_destroy(nmfb_serve *s);
const char *nmfb_serve_last_error(const nmfb_serve *s);
uint64_t nmfb_serve_request_bytes(uint32_t n, uint32_t m, uint32_t k);

/* Uploads V (host or device pointer, leading dimension ldv), initialises W and
 * H as nmfb_init_random(seed) does, and queues the request; *ticket identifies
 * it.  NMFB_ESTATE when `capacity` requests are already queued or unfetched. */
int nmfb_serve_submit(nmfb_serve *s, const float *V, size_t ldv, uint32_t n, uint32_t m, uint32_t k, uint32_t seed,
                      uint32_t n_iters, uint32_t niter_test_conv, uint32_t stop_threshold, uint32_t *ticket);
int nmfb_serve_poll(nmfb_serve *s, uint32_t ticket, int *done);
int nmfb_serve_wait(nmfb_serve *s, uint32_t ticket, double timeout_s);   /* NMFB_ETIMEOUT after timeout_s */

/* Copies a finished request's W (n x k), H (m x k) and labels (m); any may be
 * NULL.  Frees the request's device memory and its ticket. */
int nmfb_serve_fetch(nmfb_serve *s, uint32_t ticket, float *W, size_t ldw, float *H, size_t ldh, uint32_t *labels,
                     uint32_t *iterations, int *converged);

/* ---------------------------------------------------------------------------
 * update_H without any allocation.  No counterpart in the reference: it is an
 * addition of this library for callers that must not allocate device memory,
 * such as a host framework whose caching allocator already owns the HBM, a
 * plugin host that hands out every device buffer itself, or a latency-bound
 * loop that cannot take the device-wide synchronisation of cudaFree.
 *
 * Computes H = H .* (W' (V ./ (W H))) ./ colsum(W), the same update as
 * nmfb_update_H (results agree to FP32 rounding), on caller-owned DEVICE
 * buffers of the calling thread's current device: V (n x m, ldv >= m),
 * W (n x k, ldw >= k) and H (m x k, ldh >= k, updated in place).  The work is
 * queued on `stream` (a cudaStream_t as void*, NULL = default stream) and the
 * call returns without waiting for it.
 *
 * It calls no cudaMalloc, cudaFree or allocating library routine.  Its scratch
 * is one file-scope device array of NMFB_NOALLOC_SCRATCH_BYTES (16 MiB) that
 * every GPU which loads this library holds until the process exits.  Limits:
 * 1 <= k <= 64 and m * k <= NMFB_NOALLOC_MAX_MK; larger problems are rejected
 * with NMFB_ETOOBIG before any work is queued (invalid pointers, ranks or
 * leading dimensions give NMFB_EINVAL).
 *
 * The first call on a device looks up the scratch array's device address
 * (cudaGetSymbolAddress) and caches it; make that first call before any stream
 * capture.  All calls share the one array and no state carries over between
 * them, but calls whose work overlaps on the GPU (other streams, other host
 * threads) race on it: serialise them.
 */
#define NMFB_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
#define NMFB_NOALLOC_MAX_MK 4186112u /* (16 MiB - 32 KiB of column sums) / 4 bytes */
int nmfb_update_H_noalloc(const float *V, size_t ldv, const float *W, size_t ldw, float *H, size_t ldh,
                          uint32_t n, uint32_t m, uint32_t k, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* NMFB200_H */
