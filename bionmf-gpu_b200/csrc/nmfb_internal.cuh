// nmfb_internal.cuh -- engine-private declarations shared by the .cu files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include "../../include/nmfb200.h"

namespace nmfb {

// Device-side state of the convergence test (src/NMF_GPU.c:544-709).
struct ConvState {
    uint32_t inc;          // tests without change (reference `inc`)
    uint32_t converged;    // 1 once the stop rule fired; later kernels are no-ops
    uint32_t tests_done;   // convergence tests performed
    uint32_t conv_tests;   // value of `iter` (tests counted) at convergence
    uint32_t diff;         // any connectivity difference found by the current test
    uint32_t ticket;       // block retirement counter of the compare kernel
    uint32_t stop_threshold;
    uint32_t pad;
};

}  // namespace nmfb

struct nmfb_ctx {
    int device;
    int arm;
    cudaStream_t stream;
    uint32_t n, m, k, kp;  // kp: internal padded rank (16, 32, or a multiple of 32)
    size_t ldv;            // leading dimension of V on the device (items, multiple of 32)
    int v_set, wh_set;

    float *dV;             // n x ldv
    float *dW, *dH;        // n x kp, m x kp (padding columns zero)
    float *dAccW, *dAccH;  // kp each: column sums of W and of H
    float *dWH;            // plain arm: n x ldv quotient buffer
    float *dPart;          // split-reduction partials (max(n, m) x kp x nsplit)
    size_t part_items;
    double *dColPart;      // colsum partials
    uint32_t *dTickets;    // [0]: colsum W, [1]: colsum H, [2..]: misc
    double *dObj;          // objective partials + results
    uint32_t *dObjTicket;

    int sm_count;
    void *tmaps;           // fused-arm tensor maps (host copy), see kernels_fused.cu
    void *bplan;           // bf16-arm plan, see kernels_bf16.cu
    void *splan;           // streamed-V plan (V stays in host memory), see stream.cu

    // Convergence test state.
    uint32_t *dLabels;     // m
    uint32_t *dFirst;      // kp: first sample index of every label
    uint32_t *dLastRep;    // m: canonical partition of the previous test
    nmfb::ConvState *dState;
    nmfb::ConvState *hState;  // pinned host mirror

    // Fused arms: the split copies and column sums of W ([0]) and of H ([1]) match
    // the factor (written by the previous half-iteration's epilogue).  Trusted
    // only inside one nmfb_run or step call; every entry point starts from 0.
    int fz_ok[2];
    // Inside nmfb_run: the blockwise mode may fold the next update_H's pass over
    // V into update_W's pass (the factors change only through the run's own
    // updates there).
    int in_run;

    uint64_t launches;
    unsigned long long wait_ns;  // bounded-wait limit of the fused kernels (0: the 1 s default)
    // CUDA graph of one convergence-test block (nmfb_run): replayed instead of
    // re-launching its ~12 kernels per iteration; rebuilt when J, the arm or
    // the stream change.
    cudaGraphExec_t blk_exec;
    uint32_t blk_J;
    int blk_arm;
    cudaStream_t blk_stream;
    unsigned long long blk_wait;
    uint64_t blk_kernels;
    cudaStream_t own_stream;

    // Event profiling (nmfb_profile): per class a pool of (start, stop) pairs.
    int prof_on;
    cudaEvent_t *prof_ev[4];
    uint32_t prof_n[4];
    double prof_ms[4];
    uint32_t prof_cnt[4];
    char err[512];
};

// ---- device memory -------------------------------------------------------
// Stream-ordered allocation on the context's own stream (cudaMallocAsync /
// cudaFreeAsync): creating and destroying contexts while others compute does
// not synchronise the device, as cudaFree would.
cudaError_t nmfb_malloc(nmfb_ctx *ctx, void **p, size_t bytes);
void nmfb_free(nmfb_ctx *ctx, void *p);

// Page-locked host staging buffers shared by the whole process (nmfb_api.cu):
// allocating or freeing page-locked memory is ordered against every stream of
// the device, so uploads and downloads take buffers from this pool instead.
// nmfb_stage_get returns a buffer of at least `bytes` (nullptr if none can be
// allocated); nmfb_stage_put hands it back once the copies reading or writing
// it have completed.
void *nmfb_stage_get(size_t bytes);
void nmfb_stage_put(void *p);

// ---- error helpers -------------------------------------------------------
int nmfb_fail(nmfb_ctx *ctx, int code, const char *fmt, ...);

#define NMFB_CUDA_TRY(ctx, call)                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return nmfb_fail((ctx), NMFB_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                            \
    } while (0)

#define NMFB_LAUNCH_CHECK(ctx)                                                               \
    do {                                                                                     \
        (ctx)->launches++;                                                                   \
        cudaError_t e_ = cudaGetLastError();                                                 \
        if (e_ != cudaSuccess)                                                               \
            return nmfb_fail((ctx), NMFB_ECUDA, "kernel launch: %s (%s:%d)",                 \
                             cudaGetErrorString(e_), __FILE__, __LINE__);                    \
    } while (0)

// ---- profiling (nmfb_api.cu) ---------------------------------------------------
#define NMFB_PROF_POOL 512
extern "C" int nmfb_prof_begin(nmfb_ctx *ctx, int cls);
extern "C" int nmfb_prof_end(nmfb_ctx *ctx, int cls);

// ---- kernels_common.cu ----------------------------------------------------
int nmfb_colsum(nmfb_ctx *ctx, const float *X, uint32_t rows, float *acc, int which);
int nmfb_muldiv(nmfb_ctx *ctx, float *X, uint32_t rows, const float *part, uint32_t nsplit,
                size_t split_stride, const float *acc, int adjust);
int nmfb_adjust_rows(nmfb_ctx *ctx, float *X, uint32_t rows);
int nmfb_classify_and_test(nmfb_ctx *ctx, uint32_t niter_test_conv);
int nmfb_classify_only(nmfb_ctx *ctx);
int nmfb_reset_conv(nmfb_ctx *ctx, uint32_t stop_threshold);
int nmfb_objectives(nmfb_ctx *ctx, double *dot_V, double *dot_VWH, double *kl);
int nmfb_objectives_rows(nmfb_ctx *ctx, const float *V, const float *W, uint32_t rows, double out[3]);

// ---- kernels_plain.cu -----------------------------------------------------
int nmfb_plain_update_H(nmfb_ctx *ctx, int adjust);
int nmfb_plain_update_W(nmfb_ctx *ctx, int adjust);
int nmfb_plain_wh(nmfb_ctx *ctx, const float *W, uint32_t rows, float *WH);
int nmfb_plain_div(nmfb_ctx *ctx, const float *V, float *WH, uint32_t rows);
int nmfb_plain_red(nmfb_ctx *ctx, const float *Q, int transQ, const float *F, uint32_t nout, uint32_t nred,
                   uint32_t *nsplit);

// ---- stream.cu --------------------------------------------------------------
int nmfb_stream_prepare(nmfb_ctx *ctx, uint32_t block_rows);
int nmfb_stream_release(nmfb_ctx *ctx);
int nmfb_stream_set_V(nmfb_ctx *ctx, const float *V, size_t ldv);
int nmfb_stream_update_H(nmfb_ctx *ctx, int adjust);
int nmfb_stream_update_W(nmfb_ctx *ctx, int adjust);
int nmfb_stream_objectives(nmfb_ctx *ctx, double out[3]);
void nmfb_stream_end_run(nmfb_ctx *ctx);

// ---- kernels_fused.cu -----------------------------------------------------
int nmfb_fused_prepare(nmfb_ctx *ctx);
int nmfb_fused_release(nmfb_ctx *ctx);
int nmfb_fused_update_H(nmfb_ctx *ctx, int adjust);
int nmfb_fused_update_W(nmfb_ctx *ctx, int adjust);
int nmfb_fused_error(nmfb_ctx *ctx, uint32_t *code);
int nmfb_fused_ready_W(nmfb_ctx *ctx);
uint32_t *nmfb_fused_err_word(nmfb_ctx *ctx);

// ---- kernels_bf16.cu ------------------------------------------------------
int nmfb_bf16_prepare(nmfb_ctx *ctx);
int nmfb_bf16_release(nmfb_ctx *ctx);
int nmfb_bf16_update_H(nmfb_ctx *ctx, int adjust);
int nmfb_bf16_update_W(nmfb_ctx *ctx, int adjust);
int nmfb_bf16_ready_W(nmfb_ctx *ctx);

// Max number of reduction splits used by any arm (sizes dPart).
#define NMFB_MAX_SPLIT 64
