// batch.cu -- many independent KL-NMF solves in one persistent launch
// (rank-selection and restart sweeps), with exact integer consensus matrices
// and the FP64 cophenetic correlation of each rank's restarts.
//
// Every problem runs the reference's complete loop (src/NMF_GPU.c:522-795):
// update_H, update_W; after every niter_test_conv iterations the EPS adjust of
// W (fused into the block's last update_W) and of H (fused into the
// classification), the argmax classification with the reference's lane-exact
// tie rule (src/GPU_kernels.cu:2508-2656, 3177-3267) and the connectivity test
// (src/common.c:1195-1209) with the stop rule of src/NMF_GPU.c:695-709; the
// remaining n_iters % niter_test_conv iterations run without adjust.
//
// Work distribution: persistent thread-block clusters of C CTAs (C = 1, 2, 4
// or 8; as many clusters as fit on the GPU, at most one per problem) take
// problems from an atomic work queue in the order the host gives (largest rank
// first), and one cluster runs one problem to its end.  Within a cluster, CTA r
// owns a contiguous slice of W's rows and every CTA holds the whole of H: the
// update_H partial sums over W's rows and the partial column sums of W are
// added across the cluster in rank order through distributed shared memory, so
// every CTA computes the same H, the same classification and the same stop
// decision.  Convergence iteration counts are data dependent (a sweep's
// problems stop after 430 to 2000 iterations), so with one CTA per problem the
// few longest problems set the launch time; splitting each problem over C SMs
// divides that tail by about C.  C = 1 keeps the single-CTA summation order.
//
// Per problem, in one CTA of NT = 256 threads:
//   shared memory: H (m x ks, ks = k rounded up to 4), a staging tile (rows of
//                  W for update_H, or an NT x (jt+1) tile of V for update_W),
//                  colsum vectors, labels and the previous partition;
//   global memory: V (n x ldv, shared by all problems of a sweep, L2-resident
//                  at sweep sizes) and W (n x ks, padding columns zero).
//   update_H: thread j owns sample j: h_j in registers, WH_ij = W_i . h_j with
//             W_i broadcast from the staged tile, Haux_j += (V_ij / WH_ij) W_i,
//             summed per tile of wt rows and then across tiles;
//             H_j = (H_j .* Haux_j) ./ colsum(W)   (product first, then a
//             correctly-rounded division, as kernel_mul_div);
//   update_W: thread i owns row i: W_i in registers, V staged through shared
//             memory in NT x jt tiles (coalesced loads, conflict-free reads),
//             H_j broadcast from shared memory; same formulas mirrored.
//   colsum(W) and colsum(H) are reduced from the rows each thread just wrote,
//   in a fixed order (warp shuffles, then warps in order).
// Ranks 2..20 are compiled as exact-rank instantiations (no padded flops).
// Problem inputs (V, W, H) are read through L2 only (cp.async.cg, ld.global.cg):
// the serving kernel outlives the requests whose buffers the host frees and
// reuses, and an SM's L1 is not coherent with copies the host makes meanwhile.
// Tile shapes (wt, jt) are per-problem values (nmfb_batch_set_tiles; the
// Python layer's autotuner picks them per (k, m) bucket).
#include "nmfb_internal.cuh"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace {

constexpr int NT = 256;
constexpr int NW = NT / 32;
constexpr uint32_t KMIN = 2, KMAX = 20;

struct Problem {
    const float *V;      // n x ldv
    float *W;            // n x ks
    float *H;            // m x ks
    uint32_t *labels;    // m: classification of the final H
    uint64_t ldv;
    uint32_t n, m, k, ks;
    uint32_t wt, jt;     // tile shapes
    uint32_t n_iters, niter_test_conv, stop_threshold;   // the problem's -i, -j, -t
    uint32_t iterations; // out
    uint32_t converged;  // out
    uint32_t tests;      // out: convergence tests performed
};

__host__ __device__ constexpr uint32_t ks_of(uint32_t k) { return (k + 3u) & ~3u; }

// Shared-memory layout of one problem (offsets in floats).  The staging region
// holds two buffers (double buffering) of either phase:
//   update_H: V rows [i0, i0+wt) x columns [j0, j0+cs) (cs = min(NT, ldv)) and
//             W rows [i0, i0+wt) (wt x ks);
//   update_W: V rows [i0, i0+NT) x columns [j0, j0+jt), row stride jt + 4
//             (16-byte aligned rows; float4 reads of 8 consecutive rows hit
//             8 distinct bank groups).
struct SmemLayout {
    uint32_t h, stage, red, accw, acch, lab, rep, first, part, partw, total;
    uint32_t cs, hbuf, wbuf, vst;   // update_H column span and buffer sizes; update_W row stride
};
__host__ __device__ inline SmemLayout smem_layout(uint32_t m, uint32_t ks, uint32_t wt, uint32_t jt, uint64_t ldv)
{
    SmemLayout L;
    L.cs = ldv < (uint64_t)NT ? (uint32_t)ldv : (uint32_t)NT;
    L.hbuf = wt * (L.cs + ks);
    L.vst = jt + 4;
    L.wbuf = NT * L.vst;
    uint32_t const stage = 2u * (L.hbuf > L.wbuf ? L.hbuf : L.wbuf);
    L.h = 0;
    L.stage = (m * ks + 3u) & ~3u;
    L.red = L.stage + stage;
    L.accw = L.red + NW * ks;
    L.acch = L.accw + ks;
    L.lab = L.acch + ks;
    L.rep = L.lab + m;
    L.first = L.rep + m;
    L.part = L.first + 32;                 // this CTA's update_H partials (m x ks), read by the cluster
    L.partw = L.part + ((m * ks + 3u) & ~3u);   // this CTA's partial column sums of W (ks)
    L.total = L.partw + ks;
    return L;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    uint32_t const s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// 1/x with rcp.approx.ftz.f32 (PTX: at most 1 ulp of error); the quotient is
// v * (1/wh).  Every element the loops visit is a real one (no zero padding),
// so a zero denominator behaves as in the reference's division (v / 0 = inf,
// 0 / 0 = NaN).
__device__ __forceinline__ float quotient(float v, float wh)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(wh));
    return v * r;
}

// Load the first K of a 16-byte aligned row of KS floats with float4 loads.
template <int K>
__device__ __forceinline__ void load_row(const float *p, float (&x)[K])
{
    constexpr int KS = (int)ks_of(K);
#pragma unroll
    for (int q = 0; q < KS / 4; q++) {
        float4 const f = reinterpret_cast<const float4 *>(p)[q];
        if (4 * q + 0 < K) x[4 * q + 0] = f.x;
        if (4 * q + 1 < K) x[4 * q + 1] = f.y;
        if (4 * q + 2 < K) x[4 * q + 2] = f.z;
        if (4 * q + 3 < K) x[4 * q + 3] = f.w;
    }
}

// One element of a contraction: wh = a . b, q = v / wh, acc += q * b.
template <int K>
__device__ __forceinline__ void element(float v, const float (&a)[K], const float (&b)[K], float (&acc)[K])
{
    float wh = 0.0f;
#pragma unroll
    for (int c = 0; c < K; c++) wh = fmaf(a[c], b[c], wh);
    float const q = quotient(v, wh);
#pragma unroll
    for (int c = 0; c < K; c++) acc[c] = fmaf(q, b[c], acc[c]);
}

// Sum v[0..K) over the CTA in a fixed order; thread c < K writes out[c].
template <int K>
__device__ __forceinline__ void block_sum(float (&v)[K], float *red, float *out, uint32_t ks)
{
    uint32_t const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < K; c++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], off);
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < K; c++) red[warp * ks + c] = v[c];
    __syncthreads();
    if (threadIdx.x < (uint32_t)K) {
        float s = 0.0f;
        for (int w = 0; w < NW; w++) s += red[w * ks + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// This CTA's place in its problem's cluster: rank, cluster size and the rows
// [r0, r1) of W it owns.
struct Slice {
    uint32_t rank, size, r0, r1;
};

// Sum over the cluster, in rank order, of the float at offset `off` of every
// CTA's shared memory (this CTA's own included).
__device__ __forceinline__ float cluster_sum(float *sm, uint32_t off, uint32_t csize)
{
    cg::cluster_group cl = cg::this_cluster();
    float s = 0.0f;
    for (uint32_t q = 0; q < csize; q++) s += cl.map_shared_rank(sm, q)[off];
    return s;
}

// colsum(W) into accw: this CTA's rows (wsum, per thread), then for a cluster
// the partials of every CTA added in rank order.
template <int K>
__device__ void colsum_W(float (&wsum)[K], float *sm, const SmemLayout &L, const Slice &X)
{
    constexpr uint32_t KS = ks_of(K);
    if (X.size == 1) {
        block_sum<K>(wsum, sm + L.red, sm + L.accw, KS);
        return;
    }
    block_sum<K>(wsum, sm + L.red, sm + L.partw, KS);
    cg::this_cluster().sync();   // every CTA's partial column sums are written
    if (threadIdx.x < (uint32_t)K) sm[L.accw + threadIdx.x] = cluster_sum(sm, L.partw + threadIdx.x, X.size);
    __syncthreads();
}

// update_H: stage tile t (rows of V for columns [j0, j0+cs) and rows of W) into buffer b.
template <uint32_t KS>
__device__ __forceinline__ void stage_H(const Problem &P, float *buf, const SmemLayout &L, uint32_t j0, uint32_t i0,
                                        uint32_t rows)
{
    uint32_t const q4 = L.cs / 4;
    float *sV = buf, *sW = buf + P.wt * L.cs;
    // chunk e = r * q4 + q walks in steps of NT without a division per chunk
    uint32_t const dr = NT / q4, dq = NT - dr * q4;
    uint32_t r = threadIdx.x / q4, q = threadIdx.x - r * q4;
    const float *src_v = P.V + (size_t)i0 * P.ldv + j0;
    while (r < rows) {
        if (j0 + 4 * q < P.ldv) cp_async16(sV + r * L.cs + 4 * q, src_v + (size_t)r * P.ldv + 4 * q);
        r += dr;
        q += dq;
        if (q >= q4) {
            q -= q4;
            r += 1;
        }
    }
    const float *src = P.W + (size_t)i0 * KS;
    for (uint32_t e = threadIdx.x; e < rows * (KS / 4); e += NT) cp_async16(sW + 4 * e, src + 4 * e);
}

// With a cluster, each CTA sums over its own rows of W into `part`; after a
// cluster barrier every CTA adds the partials of all CTAs in rank order and
// updates its copy of H (the same values in every CTA).  The next write of
// `part` comes after the cluster barrier of the following colsum_W, so no CTA
// overwrites partials that another may still read.
template <int K>
__device__ void update_H(const Problem &P, float *sm, const SmemLayout &L, const Slice &X)
{
    constexpr uint32_t KS = ks_of(K);
    float *sH = sm + L.h;
    float *stage = sm + L.stage;
    uint32_t const half = (L.hbuf > L.wbuf ? L.hbuf : L.wbuf);
    const float *accW = sm + L.accw;
    uint32_t const tid = threadIdx.x, m = P.m, wt = P.wt;
    uint32_t const ntiles = (X.r1 - X.r0 + wt - 1) / wt;
    float hsum[K];
#pragma unroll
    for (int c = 0; c < K; c++) hsum[c] = 0.0f;
    for (uint32_t j0 = 0; j0 < m; j0 += NT) {
        uint32_t const j = j0 + tid;
        bool const active = j < m;
        float h[K], acc[K];
#pragma unroll
        for (int c = 0; c < K; c++) {
            h[c] = active ? sH[j * KS + c] : 0.0f;
            acc[c] = 0.0f;
        }
        __syncthreads();   // the staging region may still be read by the previous phase
        if (ntiles) stage_H<KS>(P, stage, L, j0, X.r0, min(wt, X.r1 - X.r0));
        cp_async_commit();
        for (uint32_t t = 0; t < ntiles; t++) {
            uint32_t const i0 = X.r0 + t * wt;
            uint32_t const rows = min(wt, X.r1 - i0);
            if (t + 1 < ntiles) stage_H<KS>(P, stage + ((t + 1) & 1) * half, L, j0, i0 + wt, min(wt, X.r1 - i0 - wt));
            cp_async_commit();
            cp_async_wait1();
            __syncthreads();
            const float *sV = stage + (t & 1) * half;
            const float *sW = sV + wt * L.cs;
            if (active) {
                float tl[K];
#pragma unroll
                for (int c = 0; c < K; c++) tl[c] = 0.0f;
#pragma unroll 4
                for (uint32_t r = 0; r < rows; r++) {
                    float w[K];
                    load_row<K>(sW + r * KS, w);
                    element<K>(sV[r * L.cs + tid], h, w, tl);
                }
#pragma unroll
                for (int c = 0; c < K; c++) acc[c] += tl[c];
            }
            __syncthreads();
        }
        if (active) {
            if (X.size == 1) {
#pragma unroll
                for (int c = 0; c < K; c++) {
                    float const hn = __fdiv_rn(h[c] * acc[c], accW[c]);
                    sH[j * KS + c] = hn;
                    hsum[c] += hn;
                }
            } else {
#pragma unroll
                for (int c = 0; c < K; c++) sm[L.part + j * KS + c] = acc[c];
            }
        }
    }
    if (X.size > 1) {
        cg::this_cluster().sync();   // every CTA's partials are written
        for (uint32_t j = tid; j < m; j += NT)
#pragma unroll
            for (int c = 0; c < K; c++) {
                float const tot = cluster_sum(sm, L.part + j * KS + c, X.size);
                float const hn = __fdiv_rn(sH[j * KS + c] * tot, accW[c]);
                sH[j * KS + c] = hn;
                hsum[c] += hn;
            }
    }
    block_sum<K>(hsum, sm + L.red, sm + L.acch, KS);
}

// update_W: stage V rows [i0, i0+rows) x columns [j0, j0+jt) into buffer b (row stride vst).
__device__ __forceinline__ void stage_W(const Problem &P, float *buf, const SmemLayout &L, uint32_t i0, uint32_t rows,
                                        uint32_t j0)
{
    // jt is a power of two (4..64), so q4 = jt / 4 divides NT: every thread keeps
    // one chunk column q and walks the rows in steps of NT / q4.
    uint32_t const q4 = P.jt / 4, dr = NT / q4;
    uint32_t const q = threadIdx.x & (q4 - 1);
    const float *src = P.V + (size_t)i0 * P.ldv + j0 + 4 * q;
    if (j0 + 4 * q < P.ldv)
        for (uint32_t r = threadIdx.x / q4; r < rows; r += dr) cp_async16(buf + r * L.vst + 4 * q, src + (size_t)r * P.ldv);
}

template <int K>
__device__ void update_W(const Problem &P, float *sm, const SmemLayout &L, bool adjust, const Slice &X)
{
    constexpr uint32_t KS = ks_of(K);
    const float *sH = sm + L.h;
    float *stage = sm + L.stage;
    uint32_t const half = (L.hbuf > L.wbuf ? L.hbuf : L.wbuf);
    const float *accH = sm + L.acch;
    uint32_t const tid = threadIdx.x, m = P.m, jt = P.jt;
    uint32_t const ntiles = (m + jt - 1) / jt;
    float wsum[K];
#pragma unroll
    for (int c = 0; c < K; c++) wsum[c] = 0.0f;
    for (uint32_t i0 = X.r0; i0 < X.r1; i0 += NT) {
        uint32_t const i = i0 + tid;
        bool const active = i < X.r1;
        uint32_t const rows = min((uint32_t)NT, X.r1 - i0);
        float w[K], aux[K];
#pragma unroll
        for (int c = 0; c < K; c++) {
            w[c] = active ? __ldcg(P.W + (size_t)i * KS + c) : 0.0f;
            aux[c] = 0.0f;
        }
        __syncthreads();   // the staging region may still be read by the previous phase
        stage_W(P, stage, L, i0, rows, 0);
        cp_async_commit();
        for (uint32_t t = 0; t < ntiles; t++) {
            uint32_t const j0 = t * jt;
            uint32_t const cols = min(jt, m - j0);
            if (t + 1 < ntiles) stage_W(P, stage + ((t + 1) & 1) * half, L, i0, rows, j0 + jt);
            cp_async_commit();
            cp_async_wait1();
            __syncthreads();
            if (active) {
                const float *vrow = stage + (t & 1) * half + tid * L.vst;
                float tl[K];
#pragma unroll
                for (int c = 0; c < K; c++) tl[c] = 0.0f;
                uint32_t const cols4 = cols & ~3u;
                const float *hrow = sH + j0 * KS;
                for (uint32_t jj = 0; jj < cols4; jj += 4) {
                    float4 const v4 = *reinterpret_cast<const float4 *>(vrow + jj);
                    float hj[K];
                    load_row<K>(hrow + (jj + 0) * KS, hj);
                    element<K>(v4.x, w, hj, tl);
                    load_row<K>(hrow + (jj + 1) * KS, hj);
                    element<K>(v4.y, w, hj, tl);
                    load_row<K>(hrow + (jj + 2) * KS, hj);
                    element<K>(v4.z, w, hj, tl);
                    load_row<K>(hrow + (jj + 3) * KS, hj);
                    element<K>(v4.w, w, hj, tl);
                }
                for (uint32_t jj = cols4; jj < cols; jj++) {
                    float hj[K];
                    load_row<K>(hrow + jj * KS, hj);
                    element<K>(vrow[jj], w, hj, tl);
                }
#pragma unroll
                for (int c = 0; c < K; c++) aux[c] += tl[c];
            }
            __syncthreads();
        }
        if (active) {
#pragma unroll
            for (int c = 0; c < K; c++) {
                float wn = __fdiv_rn(w[c] * aux[c], accH[c]);
                if (adjust) wn = fmaxf(wn, FLT_MIN);
                P.W[(size_t)i * KS + c] = wn;
                wsum[c] += wn;
            }
        }
    }
    colsum_W<K>(wsum, sm, L, X);
}

// Warp-per-sample classification of H with the reference's tie rule (k <= 32:
// lane t holds column t, idle lanes hold (-1, 0); xor butterfly 16..1, a lane
// takes the other value only if it is strictly larger).  With `adjust`, H is
// first clamped to FLT_MIN (the test's matrix_adjust).  Records first[label].
template <int K>
__device__ void classify(float *sm, const SmemLayout &L, uint32_t m, bool adjust)
{
    constexpr uint32_t KS = ks_of(K);
    float *sH = sm + L.h;
    uint32_t *lab = reinterpret_cast<uint32_t *>(sm + L.lab);
    uint32_t *first = reinterpret_cast<uint32_t *>(sm + L.first);
    uint32_t const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t j = warp; j < m; j += NW) {
        float v = -1.0f;
        uint32_t id = 0;
        if (lane < (uint32_t)K) {
            float x = sH[j * KS + lane];
            if (adjust) {
                x = fmaxf(x, FLT_MIN);
                sH[j * KS + lane] = x;
            }
            v = x;
            id = lane;
        }
#pragma unroll
        for (uint32_t half = 16; half > 0; half >>= 1) {
            float const ov = __shfl_xor_sync(0xffffffffu, v, half);
            uint32_t const oi = __shfl_xor_sync(0xffffffffu, id, half);
            if (v < ov) {
                v = ov;
                id = oi;
            }
        }
        if (lane == 0) {
            lab[j] = id;
            atomicMin(&first[id], j);
        }
    }
    __syncthreads();
}

template <int K>
__device__ void run_problem(Problem &P, float *sm, uint32_t *s_ctl, const Slice &X)
{
    constexpr uint32_t KS = ks_of(K);
    SmemLayout const L = smem_layout(P.m, KS, P.wt, P.jt, P.ldv);
    uint32_t const tid = threadIdx.x, m = P.m;
    uint32_t *lab = reinterpret_cast<uint32_t *>(sm + L.lab);
    uint32_t *rep = reinterpret_cast<uint32_t *>(sm + L.rep);
    uint32_t *first = reinterpret_cast<uint32_t *>(sm + L.first);
    // s_ctl[0] = inc, [1] = converged, [2] = tests

    {
        const float4 *src = reinterpret_cast<const float4 *>(P.H);
        float4 *dst = reinterpret_cast<float4 *>(sm + L.h);
        for (uint32_t e = tid; e < m * KS / 4; e += NT) dst[e] = __ldcg(src + e);
    }
    for (uint32_t j = tid; j < m; j += NT) rep[j] = 0u;   // the first test compares with an all-zero vector
    if (tid < 32) first[tid] = 0xffffffffu;
    if (tid == 0) {
        s_ctl[0] = 0;
        s_ctl[1] = 0;
        s_ctl[2] = 0;
    }
    {   // colsum(W) of the initial W
        float ws[K];
#pragma unroll
        for (int c = 0; c < K; c++) ws[c] = 0.0f;
        for (uint32_t i = X.r0 + tid; i < X.r1; i += NT)
#pragma unroll
            for (int c = 0; c < K; c++) ws[c] += __ldcg(P.W + (size_t)i * KS + c);
        __syncthreads();
        colsum_W<K>(ws, sm, L, X);
    }

    uint32_t const J = P.niter_test_conv;
    uint32_t const nblocks = P.n_iters / J, rem = P.n_iters % J;
    for (uint32_t b = 0; b < nblocks; b++) {
        for (uint32_t it = 0; it < J; it++) {
            update_H<K>(P, sm, L, X);
            update_W<K>(P, sm, L, it + 1 == J, X);
        }
        classify<K>(sm, L, m, true);
        uint32_t local = 0;
        for (uint32_t j = tid; j < m; j += NT) {
            uint32_t const r = first[lab[j]];
            local |= (r != rep[j]) ? 1u : 0u;
            rep[j] = r;
        }
        int const any = __syncthreads_or((int)local);
        if (tid < 32) first[tid] = 0xffffffffu;
        if (tid == 0) {
            s_ctl[2] += 1;
            if (any)
                s_ctl[0] = 0;
            else if (s_ctl[0] < P.stop_threshold)
                s_ctl[0] += 1;
            else
                s_ctl[1] = 1;
        }
        __syncthreads();
        if (X.size > 1) {
            // Every CTA of the cluster holds the same H and labels, so their stop
            // decisions agree; still, take rank 0's, so that the cluster barriers
            // of the next iteration are reached by all CTAs or by none.  The
            // second barrier keeps rank 0 from changing s_ctl before the others
            // have read it.
            cg::cluster_group const cl = cg::this_cluster();
            cl.sync();
            uint32_t const stop0 = *cl.map_shared_rank(&s_ctl[1], 0u);
            cl.sync();
            if (tid == 0) s_ctl[1] = stop0;
            __syncthreads();
        }
        if (s_ctl[1]) break;
    }
    if (!s_ctl[1])
        for (uint32_t it = 0; it < rem; it++) {
            update_H<K>(P, sm, L, X);
            update_W<K>(P, sm, L, false, X);
        }
    // final classification (no adjust) and write-back (every CTA of a cluster
    // holds the same H and labels; rank 0 writes them)
    classify<K>(sm, L, m, false);
    if (X.rank == 0) {
        for (uint32_t j = tid; j < m; j += NT) P.labels[j] = lab[j];
        const float4 *src = reinterpret_cast<const float4 *>(sm + L.h);
        float4 *dst = reinterpret_cast<float4 *>(P.H);
        for (uint32_t e = tid; e < m * KS / 4; e += NT) dst[e] = src[e];
    }
    if (tid == 0) {
        P.converged = s_ctl[1];
        P.tests = s_ctl[2];
        P.iterations = s_ctl[1] ? s_ctl[2] * J : P.n_iters;
    }
    __syncthreads();
}

// KMAX: the largest rank the instantiation handles (10 or 20).  A batch whose
// ranks are all <= 10 (a rank sweep) runs the 10-rank variant: without the
// k = 11..20 paths in the kernel, its registers are allocated for k <= 10.
template <int KMAX>
__global__ void __launch_bounds__(NT, 2) k_batch(Problem *__restrict__ probs, const uint32_t *__restrict__ order,
                                                 uint32_t nprob, uint32_t *__restrict__ queue)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    __shared__ uint32_t s_next;
    __shared__ uint32_t s_ctl[4];
    cg::cluster_group const cl = cg::this_cluster();
    uint32_t const crank = cl.block_rank(), csize = cl.num_blocks();
    for (;;) {
        __syncthreads();
        if (crank == 0 && threadIdx.x == 0) s_next = atomicAdd(queue, 1u);
        uint32_t q;
        if (csize > 1) {
            cl.sync();
            q = *cl.map_shared_rank(&s_next, 0u);
            // rank 0 rewrites s_next, and any CTA may leave the kernel, only after
            // every CTA has read it (and, earlier, every partial it needed)
            cl.sync();
        } else {
            __syncthreads();
            q = s_next;
        }
        if (q >= nprob) break;
        Problem P = probs[order[q]];
        uint32_t const chunk = (P.n + csize - 1) / csize;
        Slice const X{crank, csize, min(P.n, crank * chunk), min(P.n, crank * chunk + chunk)};
        switch (P.k) {
#define NMFB_BATCH_CASE(KK) \
    case KK: run_problem<KK>(P, sm, s_ctl, X); break;
            NMFB_BATCH_CASE(2) NMFB_BATCH_CASE(3) NMFB_BATCH_CASE(4) NMFB_BATCH_CASE(5) NMFB_BATCH_CASE(6)
            NMFB_BATCH_CASE(7) NMFB_BATCH_CASE(8) NMFB_BATCH_CASE(9) NMFB_BATCH_CASE(10)
#undef NMFB_BATCH_CASE
            default:
                if (KMAX > 10) {
                    switch (P.k) {
#define NMFB_BATCH_CASE(KK) \
    case KK: run_problem<(KMAX > 10 ? KK : 2)>(P, sm, s_ctl, X); break;
                        NMFB_BATCH_CASE(11) NMFB_BATCH_CASE(12) NMFB_BATCH_CASE(13) NMFB_BATCH_CASE(14)
                        NMFB_BATCH_CASE(15) NMFB_BATCH_CASE(16) NMFB_BATCH_CASE(17) NMFB_BATCH_CASE(18)
                        NMFB_BATCH_CASE(19) NMFB_BATCH_CASE(20)
#undef NMFB_BATCH_CASE
                        default: break;
                    }
                }
                break;
        }
        if (crank == 0 && threadIdx.x == 0) {
            Problem *dst = probs + order[q];
            dst->iterations = P.iterations;
            dst->converged = P.converged;
            dst->tests = P.tests;
        }
    }
}

__device__ __forceinline__ unsigned long long device_clock_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr uint32_t NO_TICKET = 0xffffffffu;

// Serving: requests are published one at a time into a ring of `capacity`
// descriptors while the kernel runs (the host copies a request's data and
// descriptor, then the new published count, in that order on one stream).
// A cluster's rank 0 claims the next published ticket with a compare-and-swap
// on `taken`, waiting at most idle_ns for one; after that, or once `closing`
// is set, the cluster leaves, and the host launches the kernel again when
// more work is published.  Every wait is bounded by idle_ns.  A finished
// problem's W, H and labels are in device memory before its completion record
// (host-mapped memory) is written: iterations, converged, tests, then the
// ticket + 1 after a system-scope fence.
__global__ void __launch_bounds__(NT, 2) k_serve(const Problem *__restrict__ ring, uint32_t capacity,
                                                 uint32_t *taken, const volatile uint32_t *published,
                                                 const volatile uint32_t *closing, volatile uint32_t *done,
                                                 unsigned long long idle_ns)
{
    extern __shared__ float4 smem4[];
    float *sm = reinterpret_cast<float *>(smem4);
    __shared__ uint32_t s_next;
    __shared__ uint32_t s_ctl[4];
    cg::cluster_group const cl = cg::this_cluster();
    uint32_t const crank = cl.block_rank(), csize = cl.num_blocks();
    for (;;) {
        __syncthreads();
        if (crank == 0 && threadIdx.x == 0) {
            uint32_t got = NO_TICKET;
            unsigned long long const t0 = device_clock_ns();
            for (;;) {
                uint32_t const t = *(volatile uint32_t *)taken;
                if (t < *published) {
                    if (atomicCAS(taken, t, t + 1u) == t) {
                        got = t;
                        break;
                    }
                    continue;
                }
                if (*closing || device_clock_ns() - t0 > idle_ns) break;
                __nanosleep(2000);
            }
            s_next = got;
        }
        uint32_t q;
        if (csize > 1) {
            cl.sync();
            q = *cl.map_shared_rank(&s_next, 0u);
            cl.sync();
        } else {
            __syncthreads();
            q = s_next;
        }
        if (q == NO_TICKET) break;
        uint32_t const slot = q % capacity;
        // the descriptor was written by a host copy: read it through L2
        Problem P;
        {
            const uint2 *src = reinterpret_cast<const uint2 *>(ring + slot);
            uint2 *dst = reinterpret_cast<uint2 *>(&P);
#pragma unroll
            for (uint32_t w = 0; w < sizeof(Problem) / sizeof(uint2); w++) dst[w] = __ldcg(src + w);
        }
        uint32_t const chunk = (P.n + csize - 1) / csize;
        Slice const X{crank, csize, min(P.n, crank * chunk), min(P.n, crank * chunk + chunk)};
        switch (P.k) {
#define NMFB_SERVE_CASE(KK) \
    case KK: run_problem<KK>(P, sm, s_ctl, X); break;
            NMFB_SERVE_CASE(2) NMFB_SERVE_CASE(3) NMFB_SERVE_CASE(4) NMFB_SERVE_CASE(5) NMFB_SERVE_CASE(6)
            NMFB_SERVE_CASE(7) NMFB_SERVE_CASE(8) NMFB_SERVE_CASE(9) NMFB_SERVE_CASE(10) NMFB_SERVE_CASE(11)
            NMFB_SERVE_CASE(12) NMFB_SERVE_CASE(13) NMFB_SERVE_CASE(14) NMFB_SERVE_CASE(15) NMFB_SERVE_CASE(16)
            NMFB_SERVE_CASE(17) NMFB_SERVE_CASE(18) NMFB_SERVE_CASE(19) NMFB_SERVE_CASE(20)
#undef NMFB_SERVE_CASE
            default: break;
        }
        // every CTA's stores of W (and rank 0's of H and the labels) are done
        __threadfence();
        if (csize > 1)
            cl.sync();
        else
            __syncthreads();
        if (crank == 0 && threadIdx.x == 0) {
            volatile uint32_t *rec = done + 4 * (size_t)slot;
            rec[1] = P.iterations;
            rec[2] = P.converged;
            rec[3] = P.tests;
            __threadfence_system();
            rec[0] = q + 1u;
        }
    }
}

// ---------------------------------------------------------------------------
// Consensus: C[a][b] = number of runs r in `sel` with labels_r[a] == labels_r[b]
// (exact integer co-clustering counts).  One CTA per row a.
__global__ void k_consensus(const uint32_t *const *__restrict__ labels, const uint32_t *__restrict__ sel, uint32_t nsel,
                            uint32_t m, uint32_t *__restrict__ C)
{
    uint32_t const a = blockIdx.x;
    for (uint32_t b = threadIdx.x; b < m; b += blockDim.x) {
        uint32_t cnt = 0;
        for (uint32_t s = 0; s < nsel; s++) {
            const uint32_t *l = labels[sel[s]];
            cnt += (l[a] == l[b]) ? 1u : 0u;
        }
        C[(size_t)a * m + b] = cnt;
    }
}

__device__ __forceinline__ double consensus_distance(uint32_t c, double runs)
{
    return __dsub_rn(1.0, __ddiv_rn((double)c, runs));
}

// Cophenetic correlation (Brunet et al., PNAS 2004) of the consensus C over
// nruns runs, in FP64, one CTA of 1024 threads:
//   D = 1 - C / nruns (zero diagonal);
//   average-linkage (UPGMA) agglomeration: repeatedly merge the two active
//   clusters at the smallest distance, the lowest (a, b) slot pair first on
//   ties; the merged cluster keeps slot a and its distance to x becomes
//   (|a| D[a][x] + |b| D[b][x]) / (|a| + |b|); the cophenetic distance of two
//   samples is the height at which their clusters merge;
//   result = Pearson correlation of D and the cophenetic distances over all
//   pairs a < b (means first, then centred sums).
// Work buffers (global): Dw (m*m), coph (m*m); cid, csize (m each).
__global__ void __launch_bounds__(1024) k_cophenetic(const uint32_t *__restrict__ C, uint32_t m, uint32_t nruns,
                                                     double *__restrict__ Dw, double *__restrict__ coph,
                                                     uint32_t *__restrict__ cid, uint32_t *__restrict__ csize,
                                                     double *__restrict__ out)
{
    __shared__ double s_d[1024];
    __shared__ uint32_t s_a[1024], s_b[1024];
    __shared__ double s_r[3][1024];
    uint32_t const tid = threadIdx.x, nt = blockDim.x;
    double const runs = (double)nruns;
    size_t const mm = (size_t)m * m;
    for (size_t e = tid; e < mm; e += nt) {
        uint32_t const a = (uint32_t)(e / m), b = (uint32_t)(e % m);
        Dw[e] = (a == b) ? 0.0 : consensus_distance(C[e], runs);
        coph[e] = 0.0;
    }
    for (uint32_t a = tid; a < m; a += nt) {
        cid[a] = a;
        csize[a] = 1;
    }
    __syncthreads();
    for (uint32_t step = 0; step + 1 < m; step++) {
        double best = INFINITY;
        uint32_t ba = 0xffffffffu, bb = 0xffffffffu;
        for (size_t e = tid; e < mm; e += nt) {
            uint32_t const a = (uint32_t)(e / m), b = (uint32_t)(e % m);
            if (a < b && csize[a] && csize[b]) {
                double const d = Dw[e];
                if (d < best) {   // e grows with (a, b): the first strict minimum is the lowest pair
                    best = d;
                    ba = a;
                    bb = b;
                }
            }
        }
        s_d[tid] = best;
        s_a[tid] = ba;
        s_b[tid] = bb;
        __syncthreads();
        for (uint32_t s = nt / 2; s > 0; s >>= 1) {
            if (tid < s) {
                double const od = s_d[tid + s];
                uint32_t const oa = s_a[tid + s], ob = s_b[tid + s];
                if (od < s_d[tid] || (od == s_d[tid] && (oa < s_a[tid] || (oa == s_a[tid] && ob < s_b[tid])))) {
                    s_d[tid] = od;
                    s_a[tid] = oa;
                    s_b[tid] = ob;
                }
            }
            __syncthreads();
        }
        uint32_t const A = s_a[0], B = s_b[0];
        double const h = s_d[0];
        double const na = (double)csize[A], nb = (double)csize[B];
        __syncthreads();
        for (size_t e = tid; e < mm; e += nt) {
            uint32_t const a = (uint32_t)(e / m), b = (uint32_t)(e % m);
            uint32_t const ca = cid[a], cb = cid[b];
            if ((ca == A && cb == B) || (ca == B && cb == A)) coph[e] = h;
        }
        __syncthreads();
        for (uint32_t x = tid; x < m; x += nt) {
            if (x != A && x != B && csize[x]) {
                double const d = __ddiv_rn(__dadd_rn(__dmul_rn(na, Dw[(size_t)A * m + x]), __dmul_rn(nb, Dw[(size_t)B * m + x])),
                                           __dadd_rn(na, nb));
                Dw[(size_t)A * m + x] = d;
                Dw[(size_t)x * m + A] = d;
            }
        }
        __syncthreads();
        for (uint32_t x = tid; x < m; x += nt)
            if (cid[x] == B) cid[x] = A;
        if (tid == 0) {
            csize[A] += csize[B];
            csize[B] = 0;
        }
        __syncthreads();
    }
    // Pearson correlation over a < b: means, then centred sums.
    double const np = (double)m * (double)(m - 1) / 2.0;
    double sx = 0.0, sy = 0.0;
    for (size_t e = tid; e < mm; e += nt) {
        uint32_t const a = (uint32_t)(e / m), b = (uint32_t)(e % m);
        if (a < b) {
            sx += consensus_distance(C[e], runs);
            sy += coph[e];
        }
    }
    s_r[0][tid] = sx;
    s_r[1][tid] = sy;
    __syncthreads();
    for (uint32_t s = nt / 2; s > 0; s >>= 1) {
        if (tid < s) {
            s_r[0][tid] += s_r[0][tid + s];
            s_r[1][tid] += s_r[1][tid + s];
        }
        __syncthreads();
    }
    double const mx = s_r[0][0] / np, my = s_r[1][0] / np;
    __syncthreads();
    double cxy = 0.0, cxx = 0.0, cyy = 0.0;
    for (size_t e = tid; e < mm; e += nt) {
        uint32_t const a = (uint32_t)(e / m), b = (uint32_t)(e % m);
        if (a < b) {
            double const x = consensus_distance(C[e], runs) - mx;
            double const y = coph[e] - my;
            cxy += x * y;
            cxx += x * x;
            cyy += y * y;
        }
    }
    s_r[0][tid] = cxy;
    s_r[1][tid] = cxx;
    s_r[2][tid] = cyy;
    __syncthreads();
    for (uint32_t s = nt / 2; s > 0; s >>= 1) {
        if (tid < s)
            for (int q = 0; q < 3; q++) s_r[q][tid] += s_r[q][tid + s];
        __syncthreads();
    }
    if (tid == 0) out[0] = (s_r[1][0] > 0.0 && s_r[2][0] > 0.0) ? s_r[0][0] / sqrt(s_r[1][0] * s_r[2][0]) : 0.0;
}

}  // namespace

// ---------------------------------------------------------------------------
struct nmfb_batch {
    int device;
    cudaStream_t stream;
    uint32_t n, m, nprob;
    size_t ldv;
    int sm_count;
    size_t smem_optin;
    std::vector<uint32_t> ranks;
    std::vector<uint32_t> wt, jt;        // per-problem tile shapes
    uint32_t cluster;                     // CTAs per problem (0 = automatic)
    uint32_t last_cluster;                // the value the last run used
    float *dV;
    float *dW, *dH;                       // per-problem slices (n x ks, m x ks)
    std::vector<size_t> woff, hoff;       // float offsets of each problem's slices
    uint32_t *dLabels;                    // nprob x m
    Problem *dProbs;
    uint32_t *dOrder, *dQueue;
    uint32_t **dLabelPtrs;
    int v_set, wh_set;
    cudaEvent_t ev0, ev1;
    float last_ms;
    char err[512];
};

static int bfail(nmfb_batch *b, int code, const char *fmt, ...)
{
    if (b) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(b->err, sizeof(b->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define BTRY(b, call)                                                                                      \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return bfail((b), NMFB_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));     \
    } while (0)

static size_t problem_smem_bytes(uint32_t m, uint32_t k, uint32_t wt, uint32_t jt)
{
    uint64_t const ldv = ((uint64_t)m + 31) / 32 * 32;
    return (size_t)smem_layout(m, ks_of(k), wt, jt, ldv).total * sizeof(float);
}

// Default tile shapes: wt rows of W per update_H tile, jt columns of V per update_W tile.
static void default_tiles(uint32_t k, uint32_t m, uint32_t *wt, uint32_t *jt)
{
    (void)k;
    *wt = 32;
    *jt = m >= 64 ? 32 : 16;
}

static Problem make_problem(const nmfb_batch *b, uint32_t p)
{
    Problem P;
    memset(&P, 0, sizeof(P));
    uint32_t const k = b->ranks[p];
    P.V = b->dV;
    P.W = b->dW + b->woff[p];
    P.H = b->dH + b->hoff[p];
    P.labels = b->dLabels + (size_t)p * b->m;
    P.ldv = b->ldv;
    P.n = b->n;
    P.m = b->m;
    P.k = k;
    P.ks = ks_of(k);
    P.wt = b->wt[p];
    P.jt = b->jt[p];
    return P;
}

extern "C" {

int nmfb_batch_create(nmfb_batch **out, int device, uint32_t n, uint32_t m, uint32_t nprob, const uint32_t *ranks)
{
    if (!out) return NMFB_EINVAL;
    *out = nullptr;
    nmfb_batch *b = new (std::nothrow) nmfb_batch();
    if (!b) return NMFB_ENOMEM;
    *out = b;
    b->device = device;
    if (n < 2 || m < 2 || nprob == 0 || !ranks) return bfail(b, NMFB_EINVAL, "invalid batch dimensions");
    for (uint32_t p = 0; p < nprob; p++)
        if (ranks[p] < KMIN || ranks[p] > KMAX || ranks[p] > (n < m ? n : m))
            return bfail(b, NMFB_EINVAL, "problem %u: factorization rank %u must be in [2, min(%u, n, m)]", p, ranks[p],
                         KMAX);
    b->n = n;
    b->m = m;
    b->nprob = nprob;
    b->ldv = ((size_t)m + 31) / 32 * 32;
    b->ranks.assign(ranks, ranks + nprob);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return bfail(b, NMFB_ENODEV, "no CUDA device %d", device);
    }
    cudaDeviceProp prop;
    BTRY(b, cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return bfail(b, NMFB_ENODEV, "device %d is sm_%d%d; this engine is built for sm_100a", device, prop.major, prop.minor);
    BTRY(b, cudaSetDevice(device));
    b->sm_count = prop.multiProcessorCount;
    b->smem_optin = prop.sharedMemPerBlockOptin;
    b->wt.resize(nprob);
    b->jt.resize(nprob);
    b->woff.resize(nprob);
    b->hoff.resize(nprob);
    size_t wtot = 0, htot = 0;
    for (uint32_t p = 0; p < nprob; p++) {
        default_tiles(ranks[p], m, &b->wt[p], &b->jt[p]);
        if (problem_smem_bytes(m, ranks[p], b->wt[p], b->jt[p]) + 64 > b->smem_optin)
            return bfail(b, NMFB_EINVAL, "m = %u with k = %u does not fit the batched engine's shared memory", m, ranks[p]);
        b->woff[p] = wtot;
        b->hoff[p] = htot;
        wtot += (size_t)n * ks_of(ranks[p]);
        htot += (size_t)m * ks_of(ranks[p]);
    }
    BTRY(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BTRY(b, cudaEventCreate(&b->ev0));
    BTRY(b, cudaEventCreate(&b->ev1));
    if (cudaMalloc(&b->dV, (size_t)n * b->ldv * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&b->dW, wtot * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&b->dH, htot * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&b->dLabels, (size_t)nprob * m * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&b->dProbs, nprob * sizeof(Problem)) != cudaSuccess ||
        cudaMalloc(&b->dOrder, nprob * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&b->dQueue, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&b->dLabelPtrs, nprob * sizeof(uint32_t *)) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, NMFB_ENOMEM, "device allocation for the batch failed");
    }
    BTRY(b, cudaMemsetAsync(b->dV, 0, (size_t)n * b->ldv * sizeof(float), b->stream));
    BTRY(b, cudaMemsetAsync(b->dW, 0, wtot * sizeof(float), b->stream));
    BTRY(b, cudaMemsetAsync(b->dH, 0, htot * sizeof(float), b->stream));
    std::vector<uint32_t *> lp(nprob);
    for (uint32_t p = 0; p < nprob; p++) lp[p] = b->dLabels + (size_t)p * m;
    BTRY(b, cudaMemcpyAsync(b->dLabelPtrs, lp.data(), nprob * sizeof(uint32_t *), cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    return NMFB_OK;
}

int nmfb_batch_destroy(nmfb_batch *b)
{
    if (!b) return NMFB_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    void *bufs[] = {b->dV, b->dW, b->dH, b->dLabels, b->dProbs, b->dOrder, b->dQueue, b->dLabelPtrs};
    for (void *p : bufs)
        if (p) cudaFree(p);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return NMFB_OK;
}

const char *nmfb_batch_last_error(const nmfb_batch *b) { return b ? b->err : "null batch"; }

int nmfb_batch_set_V(nmfb_batch *b, const float *V, size_t ldv)
{
    if (!b || !V || ldv < b->m) return bfail(b, NMFB_EINVAL, "nmfb_batch_set_V: bad arguments");
    BTRY(b, cudaSetDevice(b->device));
    BTRY(b, cudaMemcpy2DAsync(b->dV, b->ldv * sizeof(float), V, ldv * sizeof(float), b->m * sizeof(float), b->n,
                              cudaMemcpyDefault, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    b->v_set = 1;
    return NMFB_OK;
}

int nmfb_batch_init_random(nmfb_batch *b, const uint32_t *seeds)
{
    if (!b || !seeds) return bfail(b, NMFB_EINVAL, "nmfb_batch_init_random: bad arguments");
    BTRY(b, cudaSetDevice(b->device));
    uint32_t const n = b->n, m = b->m;
    size_t wmax = 0, hmax = 0;
    for (uint32_t p = 0; p < b->nprob; p++) {
        wmax = std::max(wmax, (size_t)n * ks_of(b->ranks[p]));
        hmax = std::max(hmax, (size_t)m * ks_of(b->ranks[p]));
    }
    float *stage = nullptr;
    BTRY(b, cudaMallocHost(&stage, 2 * (wmax + hmax) * sizeof(float)));
    cudaError_t e = cudaSuccess;
    for (uint32_t p = 0; p < b->nprob && e == cudaSuccess; p++) {
        float *W = stage + (p & 1) * (wmax + hmax);
        float *H = W + wmax;
        uint32_t const k = b->ranks[p], ks = ks_of(k);
        if (p >= 2) e = cudaStreamSynchronize(b->stream);   // the staging half of problem p-2 is free again
        if (e != cudaSuccess) break;
        // CPU_RANDOM initialisation (src/NMF_routines.c:206-233, 299-307):
        // srandom(seed); W (n x k) then H (m x k), random()/RAND_MAX + FLT_MIN.
        // (the generator through a private state: initstate_r / random_r
        // reproduce srandom / random's sequence without the process-wide one)
        char rstate[128];
        struct random_data rd;
        memset(&rd, 0, sizeof(rd));
        initstate_r(seeds[p], rstate, sizeof(rstate), &rd);
        auto next = [&]() -> float {
            int32_t r;
            random_r(&rd, &r);
            return ((float)r) / ((float)RAND_MAX) + FLT_MIN;
        };
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t c = 0; c < ks; c++) W[(size_t)i * ks + c] = (c < k) ? next() : 0.0f;
        for (uint32_t j = 0; j < m; j++)
            for (uint32_t c = 0; c < ks; c++) H[(size_t)j * ks + c] = (c < k) ? next() : 0.0f;
        e = cudaMemcpyAsync(b->dW + b->woff[p], W, (size_t)n * ks * sizeof(float), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->dH + b->hoff[p], H, (size_t)m * ks * sizeof(float), cudaMemcpyHostToDevice, b->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFreeHost(stage);
    if (e != cudaSuccess) return bfail(b, NMFB_ECUDA, "init_random: %s", cudaGetErrorString(e));
    b->wh_set = 1;
    return NMFB_OK;
}

int nmfb_batch_set_WH(nmfb_batch *b, uint32_t p, const float *W, size_t ldw, const float *H, size_t ldh)
{
    if (!b || p >= b->nprob || !W || !H) return bfail(b, NMFB_EINVAL, "nmfb_batch_set_WH: bad arguments");
    uint32_t const k = b->ranks[p], ks = ks_of(k);
    if (ldw < k || ldh < k) return bfail(b, NMFB_EINVAL, "nmfb_batch_set_WH: leading dimension below k");
    BTRY(b, cudaSetDevice(b->device));
    BTRY(b, cudaMemcpy2DAsync(b->dW + b->woff[p], ks * sizeof(float), W, ldw * sizeof(float), k * sizeof(float), b->n,
                              cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaMemcpy2DAsync(b->dH + b->hoff[p], ks * sizeof(float), H, ldh * sizeof(float), k * sizeof(float), b->m,
                              cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    b->wh_set = 1;
    return NMFB_OK;
}

int nmfb_batch_set_tiles(nmfb_batch *b, uint32_t p, uint32_t wt, uint32_t jt)
{
    if (!b || p >= b->nprob) return bfail(b, NMFB_EINVAL, "nmfb_batch_set_tiles: bad problem");
    if (wt < 8 || wt > 512 || (wt & 7) || jt < 4 || jt > 64 || (jt & (jt - 1)))
        return bfail(b, NMFB_EINVAL, "tile shape out of range (wt in [8, 512], multiple of 8; jt a power of two in [4, 64])");
    if (problem_smem_bytes(b->m, b->ranks[p], wt, jt) + 64 > b->smem_optin)
        return bfail(b, NMFB_EINVAL, "tile shape does not fit shared memory");
    b->wt[p] = wt;
    b->jt[p] = jt;
    return NMFB_OK;
}

int nmfb_batch_set_cluster(nmfb_batch *b, uint32_t ctas)
{
    if (!b) return NMFB_EINVAL;
    if (ctas != 0 && ctas != 1 && ctas != 2 && ctas != 4 && ctas != 8)
        return bfail(b, NMFB_EINVAL, "CTAs per problem must be 0 (automatic), 1, 2, 4 or 8");
    b->cluster = ctas;
    return NMFB_OK;
}

int nmfb_batch_get_cluster(const nmfb_batch *b, uint32_t *ctas)
{
    if (!b || !ctas) return NMFB_EINVAL;
    *ctas = b->last_cluster;
    return NMFB_OK;
}

int nmfb_batch_run(nmfb_batch *b, uint32_t n_iters, uint32_t niter_test_conv, uint32_t stop_threshold,
                   uint32_t *iterations, int *converged)
{
    if (!b) return NMFB_EINVAL;
    if (n_iters == 0 || niter_test_conv == 0 || stop_threshold == 0)
        return bfail(b, NMFB_EINVAL, "nIters, niter_test_conv and stop_threshold must be positive");
    if (!b->v_set || !b->wh_set) return bfail(b, NMFB_ESTATE, "set V and the initial factors first");
    BTRY(b, cudaSetDevice(b->device));
    std::vector<Problem> P(b->nprob);
    std::vector<uint32_t> order(b->nprob);
    size_t smem = 0;
    for (uint32_t p = 0; p < b->nprob; p++) {
        P[p] = make_problem(b, p);
        P[p].n_iters = n_iters;
        P[p].niter_test_conv = niter_test_conv;
        P[p].stop_threshold = stop_threshold;
        order[p] = p;
        smem = std::max(smem, problem_smem_bytes(b->m, b->ranks[p], b->wt[p], b->jt[p]));
    }
    // largest rank first (all problems of a sweep share n and m), stable on the index
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return b->ranks[x] > b->ranks[y]; });
    BTRY(b, cudaMemcpyAsync(b->dProbs, P.data(), b->nprob * sizeof(Problem), cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaMemcpyAsync(b->dOrder, order.data(), b->nprob * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    BTRY(b, cudaMemsetAsync(b->dQueue, 0, sizeof(uint32_t), b->stream));
    uint32_t kmax = 0;
    for (uint32_t p = 0; p < b->nprob; p++) kmax = std::max(kmax, b->ranks[p]);
    auto const kern = kmax <= 10 ? k_batch<10> : k_batch<20>;
    BTRY(b, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    BTRY(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) return bfail(b, NMFB_EINVAL, "batched kernel does not fit on an SM with %zu B shared memory", smem);
    // CTAs per problem: automatic = 8 when the batch leaves most CTA slots idle
    // at one problem per 8 CTAs, else 4 (a problem's time shrinks about C-fold,
    // so the few problems that run to the iteration cap no longer set the
    // launch time).
    uint32_t const slots = (uint32_t)per_sm * (uint32_t)b->sm_count;
    uint32_t C = b->cluster ? b->cluster : ((uint64_t)b->nprob * 8 <= slots ? 8u : 4u);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C * (uint32_t)b->sm_count, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = b->stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    BTRY(b, cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg));
    if (nclusters < 1) return bfail(b, NMFB_EINVAL, "no cluster of %u batched CTAs fits on the device", C);
    uint32_t ncl = (uint32_t)nclusters < b->nprob ? (uint32_t)nclusters : b->nprob;
    cfg.gridDim = dim3(ncl * C, 1, 1);
    b->last_cluster = C;
    BTRY(b, cudaEventRecord(b->ev0, b->stream));
    BTRY(b, cudaLaunchKernelEx(&cfg, kern, b->dProbs, (const uint32_t *)b->dOrder, b->nprob, b->dQueue));
    BTRY(b, cudaEventRecord(b->ev1, b->stream));
    BTRY(b, cudaMemcpyAsync(P.data(), b->dProbs, b->nprob * sizeof(Problem), cudaMemcpyDeviceToHost, b->stream));
    BTRY(b, cudaStreamSynchronize(b->stream));
    BTRY(b, cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
    for (uint32_t p = 0; p < b->nprob; p++) {
        if (iterations) iterations[p] = P[p].iterations;
        if (converged) converged[p] = (int)P[p].converged;
    }
    return NMFB_OK;
}

int nmfb_batch_last_ms(const nmfb_batch *b, double *ms)
{
    if (!b || !ms) return NMFB_EINVAL;
    *ms = b->last_ms;
    return NMFB_OK;
}

int nmfb_batch_get_classification(nmfb_batch *b, uint32_t *labels)
{
    if (!b || !labels) return bfail(b, NMFB_EINVAL, "null labels");
    BTRY(b, cudaSetDevice(b->device));
    BTRY(b, cudaMemcpy(labels, b->dLabels, (size_t)b->nprob * b->m * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return NMFB_OK;
}

int nmfb_batch_get_WH(nmfb_batch *b, uint32_t p, float *W, size_t ldw, float *H, size_t ldh)
{
    if (!b || p >= b->nprob) return bfail(b, NMFB_EINVAL, "bad problem index");
    uint32_t const k = b->ranks[p], ks = ks_of(k);
    if ((W && ldw < k) || (H && ldh < k)) return bfail(b, NMFB_EINVAL, "leading dimension below k");
    BTRY(b, cudaSetDevice(b->device));
    if (W)
        BTRY(b, cudaMemcpy2D(W, ldw * sizeof(float), b->dW + b->woff[p], ks * sizeof(float), k * sizeof(float), b->n,
                             cudaMemcpyDeviceToHost));
    if (H)
        BTRY(b, cudaMemcpy2D(H, ldh * sizeof(float), b->dH + b->hoff[p], ks * sizeof(float), k * sizeof(float), b->m,
                             cudaMemcpyDeviceToHost));
    return NMFB_OK;
}

int nmfb_batch_consensus(nmfb_batch *b, uint32_t k, uint32_t *counts, uint32_t *nruns, double *cophenetic)
{
    if (!b) return NMFB_EINVAL;
    std::vector<uint32_t> sel;
    for (uint32_t p = 0; p < b->nprob; p++)
        if (b->ranks[p] == k) sel.push_back(p);
    if (nruns) *nruns = (uint32_t)sel.size();
    if (sel.empty()) return bfail(b, NMFB_EINVAL, "no problem of rank %u in the batch", k);
    BTRY(b, cudaSetDevice(b->device));
    uint32_t const m = b->m;
    size_t const mm = (size_t)m * m;
    uint32_t *dSel = nullptr, *dC = nullptr, *dCid = nullptr;
    double *dWork = nullptr;
    cudaError_t e = cudaMalloc(&dSel, sel.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dC, mm * sizeof(uint32_t));
    if (e == cudaSuccess && cophenetic) e = cudaMalloc(&dWork, (2 * mm + 1) * sizeof(double));
    if (e == cudaSuccess && cophenetic) e = cudaMalloc(&dCid, 2 * (size_t)m * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dSel, sel.data(), sel.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) {
        k_consensus<<<m, 256, 0, b->stream>>>(b->dLabelPtrs, dSel, (uint32_t)sel.size(), m, dC);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && cophenetic) {
        k_cophenetic<<<1, 1024, 0, b->stream>>>(dC, m, (uint32_t)sel.size(), dWork, dWork + mm, dCid, dCid + m,
                                                dWork + 2 * mm);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && counts) e = cudaMemcpyAsync(counts, dC, mm * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess && cophenetic)
        e = cudaMemcpyAsync(cophenetic, dWork + 2 * mm, sizeof(double), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(dSel);
    cudaFree(dC);
    cudaFree(dWork);
    cudaFree(dCid);
    if (e != cudaSuccess) return bfail(b, NMFB_ECUDA, "consensus: %s", cudaGetErrorString(e));
    return NMFB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving: a persistent k_serve launch fed with requests as they arrive.
namespace {

constexpr uint32_t SERVE_WT = 16, SERVE_JT = 16;   // tile shapes that size the launch's shared memory

// Tile shapes of a served problem: within the staging buffer the launch
// reserves for (max_m, max_k), the tallest update_H tile (narrow problems
// get many rows per tile: their per-tile work is small next to the staging
// latency) and the widest update_W tile.
void serve_tiles(uint32_t max_m, uint32_t max_k, uint32_t m, uint32_t k, uint32_t *wt, uint32_t *jt)
{
    uint64_t const ldmax = ((uint64_t)max_m + 31) / 32 * 32, ld = ((uint64_t)m + 31) / 32 * 32;
    SmemLayout const Lmax = smem_layout(max_m, ks_of(max_k), SERVE_WT, SERVE_JT, ldmax);
    uint32_t const cap = Lmax.hbuf > Lmax.wbuf ? Lmax.hbuf : Lmax.wbuf;
    uint32_t const cs = ld < (uint64_t)NT ? (uint32_t)ld : (uint32_t)NT;
    uint32_t w = cap / (cs + ks_of(k));
    w = w > 512 ? 512 : (w & ~7u);
    *wt = w < 8 ? 8 : w;
    uint32_t j = 64;
    while (j > 4 && (uint32_t)NT * (j + 4) > cap) j >>= 1;
    *jt = j;
}

struct ServeSlot {
    uint32_t ticket;      // ticket + 1 while occupied, 0 when free
    uint32_t n, m, k;
    float *V, *W, *H;
    uint32_t *labels;
};

uint64_t serve_bytes(uint32_t n, uint32_t m, uint32_t k)
{
    uint64_t const ldv = ((uint64_t)m + 31) / 32 * 32, ks = ks_of(k);
    return ((uint64_t)n * ldv + (uint64_t)n * ks + (uint64_t)m * ks + m) * 4u + 4 * 256u;
}

}  // namespace

struct nmfb_serve {
    int device;
    uint32_t max_m, max_k, capacity, ctas, nclusters;
    unsigned long long idle_ns;
    size_t smem;
    cudaStream_t kstream, cstream, rstream;   // kernel, uploads, results
    cudaMemPool_t pool;
    Problem *dRing, *hRing;                   // descriptors (device) and their pinned host copies
    uint32_t *dCtl;                           // [0] taken, [32] published
    uint32_t *hPub;                           // pinned: published value per slot (ticket + 1)
    volatile uint32_t *hClosing;              // mapped: set by destroy
    volatile uint32_t *hDone;                 // mapped: completion records, 4 words per slot
    uint32_t *dClosingAlias, *dDoneAlias;
    cudaEvent_t kdone;
    bool running;
    uint32_t next_ticket, published;
    std::vector<ServeSlot> slots;
    std::mutex mu;
    char err[512];
};

static int sfail(nmfb_serve *s, int code, const char *fmt, ...)
{
    if (s) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(s->err, sizeof(s->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define STRY(s, call)                                                                                      \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return sfail((s), NMFB_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));     \
    } while (0)

// Launch k_serve if it is not running and published work is untaken (caller holds mu).
static int serve_ensure_running(nmfb_serve *s)
{
    if (s->running) {
        cudaError_t const q = cudaEventQuery(s->kdone);
        if (q == cudaErrorNotReady) return NMFB_OK;
        if (q != cudaSuccess) return sfail(s, NMFB_ECUDA, "serving kernel: %s", cudaGetErrorString(q));
        s->running = false;
    }
    uint32_t taken = 0;
    STRY(s, cudaMemcpyAsync(&taken, s->dCtl, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->kstream));
    STRY(s, cudaStreamSynchronize(s->kstream));
    if (taken >= s->published) return NMFB_OK;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = s->ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(s->nclusters * s->ctas, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = s->smem;
    cfg.stream = s->kstream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    STRY(s, cudaLaunchKernelEx(&cfg, k_serve, (const Problem *)s->dRing, s->capacity, s->dCtl,
                               (const volatile uint32_t *)(s->dCtl + 32), (const volatile uint32_t *)s->dClosingAlias,
                               (volatile uint32_t *)s->dDoneAlias, s->idle_ns));
    STRY(s, cudaEventRecord(s->kdone, s->kstream));
    s->running = true;
    return NMFB_OK;
}

extern "C" {

uint64_t nmfb_serve_request_bytes(uint32_t n, uint32_t m, uint32_t k) { return serve_bytes(n, m, k); }

int nmfb_serve_create(nmfb_serve **out, int device, uint32_t max_m, uint32_t max_k, uint32_t capacity,
                      uint32_t ctas, uint32_t idle_ms)
{
    if (!out) return NMFB_EINVAL;
    *out = nullptr;
    nmfb_serve *s = new (std::nothrow) nmfb_serve();
    if (!s) return NMFB_ENOMEM;
    *out = s;
    s->device = device;
    if (max_m < 2 || max_k < KMIN || max_k > KMAX || capacity == 0 || capacity > (1u << 20) ||
        (ctas != 1 && ctas != 2 && ctas != 4 && ctas != 8) || idle_ms == 0)
        return sfail(s, NMFB_EINVAL, "serve: max_m >= 2, max_k in [2, 20], capacity in [1, 2^20], ctas 1/2/4/8, idle > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return sfail(s, NMFB_ENODEV, "no CUDA device %d", device);
    }
    int major = 0, sms = 0, optin = 0;
    STRY(s, cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10) return sfail(s, NMFB_ENODEV, "device %d is not sm_100a", device);
    STRY(s, cudaSetDevice(device));
    STRY(s, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    STRY(s, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    s->max_m = max_m;
    s->max_k = max_k;
    s->capacity = capacity;
    s->ctas = ctas;
    s->idle_ns = (unsigned long long)idle_ms * 1000000ull;
    s->smem = problem_smem_bytes(max_m, max_k, SERVE_WT, SERVE_JT);
    if (s->smem + 64 > (size_t)optin)
        return sfail(s, NMFB_EINVAL, "serve: max_m = %u with max_k = %u does not fit shared memory", max_m, max_k);
    STRY(s, cudaFuncSetAttribute(k_serve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s->smem));
    {
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ctas * (uint32_t)sms, 1, 1);
        cfg.blockDim = dim3(NT, 1, 1);
        cfg.dynamicSmemBytes = s->smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int ncl = 0;
        STRY(s, cudaOccupancyMaxActiveClusters(&ncl, k_serve, &cfg));
        if (ncl < 1) return sfail(s, NMFB_EINVAL, "serve: no cluster of %u CTAs fits", ctas);
        s->nclusters = (uint32_t)ncl;
    }
    STRY(s, cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking));
    STRY(s, cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking));
    STRY(s, cudaStreamCreateWithFlags(&s->rstream, cudaStreamNonBlocking));
    STRY(s, cudaEventCreateWithFlags(&s->kdone, cudaEventDisableTiming));
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    STRY(s, cudaMemPoolCreate(&s->pool, &props));
    uint64_t keep = UINT64_MAX;
    STRY(s, cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    STRY(s, cudaMalloc(&s->dRing, (size_t)capacity * sizeof(Problem)));
    STRY(s, cudaMalloc(&s->dCtl, 64 * sizeof(uint32_t)));
    STRY(s, cudaMemset(s->dCtl, 0, 64 * sizeof(uint32_t)));
    STRY(s, cudaMallocHost(&s->hRing, (size_t)capacity * sizeof(Problem)));
    STRY(s, cudaMallocHost(&s->hPub, (size_t)capacity * sizeof(uint32_t)));
    void *p = nullptr;
    STRY(s, cudaHostAlloc(&p, sizeof(uint32_t), cudaHostAllocMapped));
    s->hClosing = (volatile uint32_t *)p;
    *s->hClosing = 0;
    STRY(s, cudaHostGetDevicePointer((void **)&s->dClosingAlias, p, 0));
    STRY(s, cudaHostAlloc(&p, (size_t)capacity * 4 * sizeof(uint32_t), cudaHostAllocMapped));
    memset(p, 0, (size_t)capacity * 4 * sizeof(uint32_t));
    s->hDone = (volatile uint32_t *)p;
    STRY(s, cudaHostGetDevicePointer((void **)&s->dDoneAlias, p, 0));
    s->slots.assign(capacity, ServeSlot{});
    return NMFB_OK;
}

int nmfb_serve_destroy(nmfb_serve *s)
{
    if (!s) return NMFB_OK;
    cudaSetDevice(s->device);
    if (s->hClosing) *s->hClosing = 1;
    if (s->kstream) cudaStreamSynchronize(s->kstream);
    if (s->cstream) cudaStreamSynchronize(s->cstream);
    if (s->rstream) cudaStreamSynchronize(s->rstream);
    for (ServeSlot &sl : s->slots)
        if (sl.ticket) {
            cudaFree(sl.V);
            cudaFree(sl.W);
            cudaFree(sl.H);
            cudaFree(sl.labels);
        }
    if (s->dRing) cudaFree(s->dRing);
    if (s->dCtl) cudaFree(s->dCtl);
    if (s->hRing) cudaFreeHost(s->hRing);
    if (s->hPub) cudaFreeHost(s->hPub);
    if (s->hClosing) cudaFreeHost((void *)s->hClosing);
    if (s->hDone) cudaFreeHost((void *)s->hDone);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->kdone) cudaEventDestroy(s->kdone);
    if (s->kstream) cudaStreamDestroy(s->kstream);
    if (s->cstream) cudaStreamDestroy(s->cstream);
    if (s->rstream) cudaStreamDestroy(s->rstream);
    delete s;
    return NMFB_OK;
}

const char *nmfb_serve_last_error(const nmfb_serve *s) { return s ? s->err : "null server"; }

int nmfb_serve_submit(nmfb_serve *s, const float *V, size_t ldv, uint32_t n, uint32_t m, uint32_t k, uint32_t seed,
                      uint32_t n_iters, uint32_t niter_test_conv, uint32_t stop_threshold, uint32_t *ticket)
{
    if (!s || !V || !ticket) return sfail(s, NMFB_EINVAL, "nmfb_serve_submit: null argument");
    if (n < 2 || m < 2 || m > s->max_m || ldv < m || k < KMIN || k > s->max_k || k > (n < m ? n : m))
        return sfail(s, NMFB_EINVAL, "request %u x %u, k = %u outside the server's limits (m <= %u, 2 <= k <= min(%u, n, m))",
                     n, m, k, s->max_m, s->max_k);
    if (n_iters == 0 || niter_test_conv == 0 || stop_threshold == 0)
        return sfail(s, NMFB_EINVAL, "nIters, niter_test_conv and stop_threshold must be positive");
    {
        uint32_t wt, jt;
        serve_tiles(s->max_m, s->max_k, m, k, &wt, &jt);
        if (problem_smem_bytes(m, k, wt, jt) > s->smem)
            return sfail(s, NMFB_EINVAL, "request %u x %u, k = %u: tiles exceed the server's shared memory", n, m, k);
    }
    std::lock_guard<std::mutex> lock(s->mu);
    STRY(s, cudaSetDevice(s->device));
    uint32_t const t = s->next_ticket, slot = t % s->capacity;
    ServeSlot &sl = s->slots[slot];
    if (sl.ticket) return sfail(s, NMFB_ESTATE, "all %u request slots are in use (fetch finished requests first)", s->capacity);
    uint32_t const ks = ks_of(k);
    uint64_t const ldp = ((uint64_t)m + 31) / 32 * 32;
    // CPU_RANDOM initialisation (src/NMF_routines.c:299-307), as nmfb_init_random
    std::vector<float> W((size_t)n * ks), H((size_t)m * ks);
    {
        char rstate[128];
        struct random_data rd;
        memset(&rd, 0, sizeof(rd));
        initstate_r(seed, rstate, sizeof(rstate), &rd);
        auto next = [&]() -> float {
            int32_t r;
            random_r(&rd, &r);
            return ((float)r) / ((float)RAND_MAX) + FLT_MIN;
        };
        for (uint32_t i = 0; i < n; i++)
            for (uint32_t c = 0; c < ks; c++) W[(size_t)i * ks + c] = (c < k) ? next() : 0.0f;
        for (uint32_t j = 0; j < m; j++)
            for (uint32_t c = 0; c < ks; c++) H[(size_t)j * ks + c] = (c < k) ? next() : 0.0f;
    }
    ServeSlot ns{};
    cudaError_t e = cudaMallocFromPoolAsync((void **)&ns.V, (size_t)n * ldp * sizeof(float), s->pool, s->cstream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&ns.W, W.size() * sizeof(float), s->pool, s->cstream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&ns.H, H.size() * sizeof(float), s->pool, s->cstream);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)&ns.labels, (size_t)m * sizeof(uint32_t), s->pool, s->cstream);
    if (e != cudaSuccess) {
        if (ns.V) cudaFreeAsync(ns.V, s->cstream);
        if (ns.W) cudaFreeAsync(ns.W, s->cstream);
        if (ns.H) cudaFreeAsync(ns.H, s->cstream);
        cudaGetLastError();
        return sfail(s, NMFB_ENOMEM, "request memory: %s", cudaGetErrorString(e));
    }
    // The request's V, W and H into its device buffers.  From pageable host memory
    // V's rows are packed at the device pitch (padding zero) into one of the
    // library's page-locked staging buffers, W and H behind them, and copied with
    // one DMA each (a pitched copy from pageable memory moves one short row at a
    // time); device or page-locked V is copied directly.  The staging buffer is
    // handed back once the copies are done (end of this call).
    cudaPointerAttributes pa;
    bool const pageable = !(cudaPointerGetAttributes(&pa, V) == cudaSuccess &&
                            (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeHost ||
                             pa.type == cudaMemoryTypeManaged));
    cudaGetLastError();
    size_t const vfl = (size_t)n * ldp;
    struct StageGuard {
        float *p;
        cudaStream_t st;
        ~StageGuard()
        {
            if (p) {
                cudaStreamSynchronize(st);   // the copies reading it are done
                nmfb_stage_put(p);
            }
        }
    } stage{pageable ? (float *)nmfb_stage_get((vfl + W.size() + H.size()) * sizeof(float)) : nullptr, s->cstream};
    if (stage.p) {
        for (uint32_t i = 0; i < n; i++) {
            float *d = stage.p + (size_t)i * ldp;
            memcpy(d, V + (size_t)i * ldv, m * sizeof(float));
            memset(d + m, 0, (ldp - m) * sizeof(float));
        }
        memcpy(stage.p + vfl, W.data(), W.size() * sizeof(float));
        memcpy(stage.p + vfl + W.size(), H.data(), H.size() * sizeof(float));
        STRY(s, cudaMemcpyAsync(ns.V, stage.p, vfl * sizeof(float), cudaMemcpyHostToDevice, s->cstream));
        STRY(s, cudaMemcpyAsync(ns.W, stage.p + vfl, W.size() * sizeof(float), cudaMemcpyHostToDevice, s->cstream));
        STRY(s, cudaMemcpyAsync(ns.H, stage.p + vfl + W.size(), H.size() * sizeof(float), cudaMemcpyHostToDevice,
                                s->cstream));
    } else {
        STRY(s, cudaMemsetAsync(ns.V, 0, vfl * sizeof(float), s->cstream));
        STRY(s, cudaMemcpy2DAsync(ns.V, ldp * sizeof(float), V, ldv * sizeof(float), m * sizeof(float), n,
                                  cudaMemcpyDefault, s->cstream));
        STRY(s, cudaMemcpyAsync(ns.W, W.data(), W.size() * sizeof(float), cudaMemcpyHostToDevice, s->cstream));
        STRY(s, cudaMemcpyAsync(ns.H, H.data(), H.size() * sizeof(float), cudaMemcpyHostToDevice, s->cstream));
    }
    Problem &P = s->hRing[slot];
    memset(&P, 0, sizeof(P));
    P.V = ns.V;
    P.W = ns.W;
    P.H = ns.H;
    P.labels = ns.labels;
    P.ldv = ldp;
    P.n = n;
    P.m = m;
    P.k = k;
    P.ks = ks;
    serve_tiles(s->max_m, s->max_k, m, k, &P.wt, &P.jt);
    P.n_iters = n_iters;
    P.niter_test_conv = niter_test_conv;
    P.stop_threshold = stop_threshold;
    STRY(s, cudaMemcpyAsync(s->dRing + slot, &P, sizeof(Problem), cudaMemcpyHostToDevice, s->cstream));
    s->hDone[4 * (size_t)slot] = 0;
    // the new published count follows the request's data on the same stream
    s->hPub[slot] = t + 1u;
    STRY(s, cudaMemcpyAsync(s->dCtl + 32, &s->hPub[slot], sizeof(uint32_t), cudaMemcpyHostToDevice, s->cstream));
    // the W / H vectors have been copied (into the staging buffer, or by the
    // pageable copies, which return once staged) and may go
    ns.ticket = t + 1u;
    ns.n = n;
    ns.m = m;
    ns.k = k;
    sl = ns;
    s->next_ticket = t + 1u;
    s->published = t + 1u;
    *ticket = t;
    return serve_ensure_running(s);
}

int nmfb_serve_poll(nmfb_serve *s, uint32_t ticket, int *done)
{
    if (!s || !done) return NMFB_EINVAL;
    uint32_t const slot = ticket % s->capacity;
    // The slot is rewritten by submit and fetch under the lock; read it under
    // the lock too, so a poll from one host thread never races them.
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->slots[slot].ticket != ticket + 1u) return sfail(s, NMFB_EINVAL, "ticket %u is not pending", ticket);
    *done = (s->hDone[4 * (size_t)slot] == ticket + 1u) ? 1 : 0;
    if (*done) {
        std::atomic_thread_fence(std::memory_order_acquire);
        return NMFB_OK;
    }
    STRY(s, cudaSetDevice(s->device));
    return serve_ensure_running(s);
}

int nmfb_serve_wait(nmfb_serve *s, uint32_t ticket, double timeout_s)
{
    auto const t0 = std::chrono::steady_clock::now();
    for (;;) {
        int done = 0;
        int const rc = nmfb_serve_poll(s, ticket, &done);
        if (rc != NMFB_OK || done) return rc;
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s)
            return sfail(s, NMFB_ETIMEOUT, "request %u not finished after %.1f s", ticket, timeout_s);
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

int nmfb_serve_fetch(nmfb_serve *s, uint32_t ticket, float *W, size_t ldw, float *H, size_t ldh, uint32_t *labels,
                     uint32_t *iterations, int *converged)
{
    if (!s) return NMFB_EINVAL;
    int done = 0;
    int rc = nmfb_serve_poll(s, ticket, &done);
    if (rc) return rc;
    if (!done) return sfail(s, NMFB_ESTATE, "request %u has not finished", ticket);
    uint32_t const slot = ticket % s->capacity;
    std::lock_guard<std::mutex> lock(s->mu);
    STRY(s, cudaSetDevice(s->device));
    ServeSlot &sl = s->slots[slot];
    uint32_t const ks = ks_of(sl.k);
    if ((W && ldw < sl.k) || (H && ldh < sl.k)) return sfail(s, NMFB_EINVAL, "leading dimension below k");
    if (W)
        STRY(s, cudaMemcpy2DAsync(W, ldw * sizeof(float), sl.W, ks * sizeof(float), sl.k * sizeof(float), sl.n,
                                  cudaMemcpyDeviceToHost, s->rstream));
    if (H)
        STRY(s, cudaMemcpy2DAsync(H, ldh * sizeof(float), sl.H, ks * sizeof(float), sl.k * sizeof(float), sl.m,
                                  cudaMemcpyDeviceToHost, s->rstream));
    if (labels)
        STRY(s, cudaMemcpyAsync(labels, sl.labels, (size_t)sl.m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->rstream));
    STRY(s, cudaStreamSynchronize(s->rstream));
    if (iterations) *iterations = s->hDone[4 * (size_t)slot + 1];
    if (converged) *converged = (int)s->hDone[4 * (size_t)slot + 2];
    STRY(s, cudaFreeAsync(sl.V, s->rstream));
    STRY(s, cudaFreeAsync(sl.W, s->rstream));
    STRY(s, cudaFreeAsync(sl.H, s->rstream));
    STRY(s, cudaFreeAsync(sl.labels, s->rstream));
    sl = ServeSlot{};
    return NMFB_OK;
}

}  // extern "C"
