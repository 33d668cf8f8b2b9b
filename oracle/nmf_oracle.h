/*
 * nmf_oracle.h -- CPU restatement of the NMF-mGPU single-GPU KL-NMF loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA engine and the timed CPU baseline ("port") of the benchmark.  The
 * product path never links, loads or calls it.
 *
 * Parity pin: the oracle is checked against outputs of the reference's own
 * CUDA build (compiled from the reference sources by oracle/Makefile into
 * oracle/_ref/, run on a B200 in CPU_RANDOM + FIXED_INIT mode); the committed
 * fixtures live in tests/golden/.
 *
 * Layout conventions (same as the reference, src/NMF_GPU.c:70-90):
 *   V : n x m, row-major, leading dimension ldv (items)
 *   W : n x k, row-major, leading dimension ldw
 *   H : m x k, row-major, leading dimension ldh   ("H transposed", as the
 *       reference stores it: row j of H holds the k factors of sample j)
 */
#ifndef NMF_ORACLE_H
#define NMF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CPU_RANDOM initialisation (src/NMF_routines.c:299-307, src/NMF_GPU.c:364-436):
 * srandom(seed); W row by row, then H row by row, each value
 * (float)random()/(float)RAND_MAX + FLT_MIN.  Padding columns (k..ld) = 1.0. */
void oracle_init_random(uint32_t seed, uint32_t n, uint32_t m, uint32_t k,
                        float *W, size_t ldw, float *H, size_t ldh);

/* One multiplicative half-update (src/NMF_routines.c:376-525 and 1014-1164). */
void oracle_update_H_f32(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                         const float *W, size_t ldw, float *H, size_t ldh);
void oracle_update_W_f32(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                         float *W, size_t ldw, const float *H, size_t ldh);
void oracle_update_H_f64(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                         const double *W, size_t ldw, double *H, size_t ldh);
void oracle_update_W_f64(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                         double *W, size_t ldw, const double *H, size_t ldh);

/* matrix_adjust (src/GPU_kernels.cu:2338-2345): x = fmax(x, FLT_MIN), NaN -> FLT_MIN. */
void oracle_adjust_f32(float *A, uint32_t rows, uint32_t k, size_t ld);
void oracle_adjust_f64(double *A, uint32_t rows, uint32_t k, size_t ld);

/* get_classification -> kernel_idx_max (src/GPU_kernels.cu:2508-2656, 2880-3110,
 * 3177-3267) with the reference's exact tie behaviour.  kp = padded rank used by
 * the reference to size the thread block (ceil(k/32)*32). */
void oracle_classify_f32(const float *H, uint32_t m, uint32_t k, size_t ldh, uint32_t *labels);
void oracle_classify_f64(const double *H, uint32_t m, uint32_t k, size_t ldh, uint32_t *labels);

/* get_difference (src/common.c:1195-1209): number of sample pairs whose
 * co-membership differs between the two classification vectors. */
uint64_t oracle_difference(const uint32_t *cls, const uint32_t *last, uint32_t m);

/* The whole nmf() loop (src/NMF_GPU.c:522-795) from the given W, H.
 * Returns the number of iterations performed; *converged set accordingly. */
uint32_t oracle_nmf_f32(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                        float *W, size_t ldw, float *H, size_t ldh,
                        uint32_t nIters, uint32_t niter_test_conv, uint32_t stop_threshold,
                        int *converged);
uint32_t oracle_nmf_f64(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                        double *W, size_t ldw, double *H, size_t ldh,
                        uint32_t nIters, uint32_t niter_test_conv, uint32_t stop_threshold,
                        int *converged);

/* dot_product_VWH (src/NMF_routines.c:2680-2794) in FP64: ||V||^2 and ||V-WH||^2. */
void oracle_dot_VWH(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                    const float *W, size_t ldw, const float *H, size_t ldh,
                    double *dot_V, double *dot_VWH);

/* Generalised KL divergence D(V||WH) = sum V log(V/WH) - V + WH, FP64, 0 log 0 = 0.
 * Not computed by the reference (it only prints the Frobenius ratio). */
double oracle_kl_divergence(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                            const float *W, size_t ldw, const float *H, size_t ldh);

/* Consensus of a restart sweep (Brunet et al., PNAS 2004; cited by the
 * reference's doc/user_guide.txt.md:367): C[a][b] = number of the nruns
 * classification vectors (labels, nruns x m) that put samples a and b in the
 * same class.  Exact integer counts. */
void oracle_consensus(const uint32_t *labels, uint32_t nruns, uint32_t m, uint32_t *C);

/* Cophenetic correlation of average-linkage (UPGMA) clustering of the m x m
 * distance matrix D (symmetric, zero diagonal), FP64: merge the two active
 * clusters at the smallest distance (lowest (a, b) slot pair on ties, a < b),
 * the merged cluster keeps slot a with distance (|a| D[a][x] + |b| D[b][x]) /
 * (|a| + |b|) to every other cluster x; the cophenetic distance of two samples
 * is the merge height that joins them; result = Pearson correlation of D and
 * the cophenetic distances over all pairs a < b. */
double oracle_cophenetic_dist(const double *D, uint32_t m);

/* The same on the consensus counts: D = 1 - C / nruns off the diagonal. */
double oracle_cophenetic(const uint32_t *C, uint32_t m, uint32_t nruns);

/* Number of OpenMP threads the oracle will use (for the benchmark record). */
int oracle_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
