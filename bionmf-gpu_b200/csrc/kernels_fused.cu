// kernels_fused.cu -- the fused half-iteration arm (NMFB_ARM_FUSED / _FUSED_TF32).
//
// One kernel computes, for a block of 128 rows of the factor being updated
// (X = W for update_W, X = H for update_H) and a range of the reduction
// dimension, the partial  Xaux = sum_r  (V ./ (X Y^T))[o][r] * Y[r][:]
// without ever materialising the n x m quotient:
//
//   TMA      : V tile (128 x BR, FP32) into a VST-deep ring; the Y tile
//              operands into a YST-deep ring.
//   split    : k_split_factor, once per half-iteration, writes the other
//              factor Y as TF32 hi (round to nearest) and the transposed hi/lo
//              blocks that MMA2 reads K-major (lo = y - hi, exact; an MN-major
//              read of a TF32 operand returns zeros on sm_100a), plus BF16
//              copies bf16(lo), bf16(y) and bf16(y) transposed per tile; the Y
//              producer TMA-loads them per tile.  X (128 rows per CTA) is split
//              once per CTA by the accumulator warps.
//   MMA1     : D (TMEM, 128 x BR) = Xh Yh^T                    (kind::tf32, k-steps of 8)
//              + [bf16(Xh) | bf16(Xl)] [bf16(Yl) ; bf16(Y)]^T (kind::f16, K = 2 KP, k-steps of 16).
//   epilogue : R = V / D in FP32 registers (V times an approximate reciprocal,
//              <= 1.5 ulp; the reference uses fdividef);  R = Rh + Rl with
//              Rh = TF32(R) written back over D and bf16(Rl) packed into a
//              separate TMEM region.
//   MMA2     : Acc[tile] (TMEM, 128 x 2 KP) = Rh [Yh | Yl]   (kind::tf32, N = 2 KP)
//              + bf16(Rl) bf16(Y) into Acc[0:KP]               (kind::f16, K = 16).
//   epilogue : adds Acc[tile] into FP32 registers (per-tile accumulation keeps
//              the tensor core's FP32 sums short) and writes the split's
//              partial; k_finish (one CTA per 32 rows) sums the splits, applies
//              X = X .* Xaux ./ colsum(Y) (and the EPS adjust when asked), and
//              writes X's split copies and column sums for the next
//              half-iteration: two launches per half-iteration.
//
// Precision of the two contractions: x y = xh yh + xh yl + xl y with xh, yh
// TF32.  The large term xh yh (and, in MMA2, rh yl) is an exact TF32 product
// with FP32 accumulation; the small terms, each at most 2^-12 of the whole,
// are BF16 products (relative rounding 2^-9 of the term), so every product is
// accurate to about 2^-20 relative.  Against the 3 x TF32 form (12 + 16 MMAs
// per 64-column tile at k = 32, all at the tensor pipe's per-instruction floor
// of N <= 64) this issues 8 + 12, and the R warps' epilogue stays one TMEM load
// and one reciprocal per element.
//
// Reference equivalent: get_H_BLM / get_W_BLN (src/NMF_routines.c:376-525,
// 1014-1164): two cuBLAS SGEMMs around matrix_div_sub with WH in HBM.
//
// Warp roles: warp 0 = V producer (TMA), warp 1 = MMA issuer and TMEM owner,
// warp 2 = Y producer (TMA), warps 4-11 (or 4-19) = R warps in two teams that
// take alternate tiles (warp w reads TMEM lanes 32*(w%4)..+31), last 4 warps =
// accumulator and split warps.
// V stages are released as soon as the epilogue has read them, Y stages when
// MMA2 (the last reader) has completed.
// Every mbarrier wait is bounded (1 s of %globaltimer); on expiry the kernel
// records an error word that the host turns into NMFB_ETIMEOUT.
// No TMA multicast is used anywhere.
#include "nmfb_internal.cuh"
#include "fused_common.cuh"
#include "finish.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <float.h>
#include <cudaTypedefs.h>

using nmfb::ConvState;
using namespace nmfb_tc;

namespace {

// kind::f16 instruction descriptor with BF16 A and B (K-major) and FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16xf32(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// kind::f16 MMA with A from tensor memory (two BF16 per 32-bit column, the
// lower K index in the low half) and B from shared memory.
__device__ __forceinline__ void mma_ts_bf16(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                            uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// Two floats to a BF16 pair (round to nearest even), `first` in the low half.
__device__ __forceinline__ uint32_t bf16x2_rn(float first, float second)
{
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(second), "f"(first));
    return r;
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t *r)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}

// Swizzle of a K-major operand whose rows are `bytes` long: the UMMA layout code
// and the tensor-map mode (rows of 32 / 64 / 128 bytes).
__host__ __device__ constexpr uint32_t umma_layout(int bytes) { return bytes == 32 ? 6u : bytes == 64 ? 4u : 2u; }

struct FusedMaps {
    CUtensorMap v;       // V, box [128 x BR] (H side, no swizzle) or [32 x 128] (W side, 128B swizzle)
    CUtensorMap y;       // TF32 hi part of the other factor (rows x KP), box rows = BR
    CUtensorMap yt;      // its transposed split: per 32 rows, [hi^T (KP x 32) ; lo^T (KP x 32)]
    CUtensorMap ylb;     // BF16 copy of its lo part (rows x KP), box [KP x BR]
    CUtensorMap yb;      // BF16 copy (rows x KP), box [KP x BR]
    CUtensorMap ybt;     // BF16 transposed tiles: per BR rows, KP rows of BR values; box [BR x KP]
};

struct FusedArgs {
    uint32_t O, R;        // output rows, reduction length
    uint32_t tiles_per_split, nsplit;
    float *part;          // [split][O][KP]
    uint32_t *err;        // device error word
    const ConvState *st;
    const float *X;       // factor being updated (O x KP), read once per CTA into TMEM
    unsigned long long wait_ns;  // limit of every bounded wait (%globaltimer ns)
#ifdef NMFB_FUSED_DEBUG
    float *dbg;           // block 0, tile 0: D | V | Rh | Acc (debug builds only; 128 x 64 each)
#endif
};

// ---------------------------------------------------------------------------
template <int KP>
struct Geo {
    static constexpr int BR = (KP >= 64) ? 32 : 64;       // reduction rows per tile
    static constexpr int CB = (KP == 16) ? 16 : 32;       // floats per swizzle column block
    static constexpr int NB = KP / CB;                     // column blocks
    static constexpr int ROWB = CB * 4;                    // bytes per row of a block
    static constexpr uint32_t LAYOUT = (KP == 16) ? 4u : 2u;  // SW64 : SW128
    static constexpr int YBLK = BR * ROWB;                 // bytes of one Yh column block
    static constexpr int YTBLK = KP * 128;                 // bytes of one Y^T part (32 reduction rows)
    static constexpr int YTPAIR = 2 * YTBLK;               // Y^T hi part followed by its lo part
    static constexpr int YBYTES = BR * KP * 4;
    static constexpr int VBYTES = BO * BR * 4;
    static constexpr int YSTAGE = YBYTES;                  // Yh (TF32), NB column blocks
    static constexpr int YTSTAGE = 2 * YBYTES;             // YTh | YTl (per 32 rows)
    static constexpr int YBB = BR * KP * 2;                // one BF16 tile of BR rows of 2 KP bytes
    static constexpr int YBTB = KP * BR * 2;               // bf16(Y)^T tile, KP rows of 2 BR bytes
    static constexpr int YBSTAGE = 2 * YBB + YBTB;         // bf16(Yl) | bf16(Y) | bf16(Y)^T
    static constexpr uint32_t BLAYOUT = umma_layout(2 * KP);
    static constexpr uint32_t BTLAYOUT = umma_layout(2 * BR);
    static constexpr int YST = 3;
    static constexpr int FIXED = 1024 + 512;
    static constexpr int YALL = YST * (YSTAGE + YTSTAGE + YBSTAGE);
    static constexpr int VAVAIL = (SMEM_LIMIT - FIXED - YALL) / VBYTES;
    static constexpr int VST = VAVAIL > 6 ? 6 : VAVAIL;    // V ring depth (HBM stream)
    static constexpr int SMEM = FIXED + YALL + VST * VBYTES;
    static_assert(VST >= 3, "shared-memory ring too small");
    static_assert(YBB % 1024 == 0 && YBSTAGE % 1024 == 0 && YSTAGE % 1024 == 0, "1024-byte stage alignment");
    static constexpr int NR = (KP >= 64) ? 8 : 16;        // R warps
    static constexpr int NTHR = (4 + NR + 4) * 32;
    static constexpr uint32_t ACC = 2 * KP;                // TMEM columns of one per-tile accumulator
    static constexpr uint32_t NDB = (KP == 16) ? 4 : (KP == 32) ? 3 : 2;   // D buffers (MMA1 runs NDB tiles ahead)
    static constexpr uint32_t DA0 = 2 * ACC;               // D[b] (then Rh[b]) at DA0 + b BR
    static constexpr uint32_t RL0 = DA0 + NDB * BR;        // bf16(Rl)[b] at RL0 + b BR/2
    static constexpr uint32_t XC0 = RL0 + NDB * BR / 2;    // X hi (TF32), KP columns
    static constexpr uint32_t XB0 = XC0 + KP;              // bf16(X hi) | bf16(X lo), KP/2 columns each
    static_assert(XB0 + KP <= 512, "TMEM columns exceeded");
};

// TMEM columns: per-tile accumulators Acc[b] at b*2KP (2KP columns: the Rh Yh +
// bf16(Rl) bf16(Y) sum and the Rh Yl part side by side); D[b] (BR columns, then
// Rh[b]) at DA0 + b*BR and bf16(Rl)[b] (BR/2 columns, column group g of 16 in
// its 8 columns RL0 + b*BR/2 + 8g), b < NDB; then the CTA's 128 rows of X as
// TF32 hi (KP columns) and bf16(X hi) | bf16(X lo) (KP/2 columns each), the A
// operands of MMA1 for every tile (so MMA1 reads only Y from shared memory).

// Split a factor Y (rows x kp, FP32, padding columns zero) for the fused
// kernel's TMA loads, one CTA per block of `br` rows (br = the kernel's tile):
//   hi = TF32(y) (round to nearest), rows x kp;
//   T: per 32 rows, the transposed hi block (kp rows of 32 floats) followed by
//      the transposed lo block (lo = y - hi, exact), rows past the end zero;
//   Bl = bf16(lo), B = bf16(y): rows x kp each;
//   BT: per br rows, the transposed bf16(y) block (kp rows of br values), rows
//      past the end zero.
// The transposes go through shared memory.
__global__ void __launch_bounds__(256) k_split_factor(const float *__restrict__ Y, uint32_t rows, uint32_t kp,
                                                      uint32_t br, float *__restrict__ hi, float *__restrict__ T,
                                                      __nv_bfloat16 *__restrict__ Bl, __nv_bfloat16 *__restrict__ B,
                                                      __nv_bfloat16 *__restrict__ BT, const ConvState *st)
{
    if (st && *(volatile const uint32_t *)&st->converged) return;
    __shared__ float th[64][65], tl[64][65];
    __shared__ __nv_bfloat16 tb[64][66];
    uint32_t const r0 = blockIdx.x * br;
    for (uint32_t e = threadIdx.x; e < br * kp; e += blockDim.x) {
        uint32_t const r = e / kp, c = e % kp;
        bool const in = r0 + r < rows;
        float const y = in ? Y[(size_t)(r0 + r) * kp + c] : 0.0f;
        float const h = tf32_rna(y), l = y - h;
        __nv_bfloat16 const yb = __float2bfloat16_rn(y);
        if (in) {
            hi[(size_t)(r0 + r) * kp + c] = h;
            Bl[(size_t)(r0 + r) * kp + c] = __float2bfloat16_rn(l);
            B[(size_t)(r0 + r) * kp + c] = yb;
        }
        th[r][c] = h;
        tl[r][c] = l;
        tb[r][c] = yb;
    }
    __syncthreads();
    uint32_t const nblk32 = (rows + 31) / 32;
    for (uint32_t sub = 0; sub < br / 32; sub++) {
        uint32_t const blk = r0 / 32 + sub;
        if (blk >= nblk32) break;
        float *dst = T + (size_t)blk * 2 * kp * 32;
        for (uint32_t e = threadIdx.x; e < 2 * kp * 32; e += blockDim.x) {
            uint32_t const row = e / 32, rr = sub * 32 + e % 32;
            dst[e] = row < kp ? th[rr][row] : tl[rr][row - kp];
        }
    }
    __nv_bfloat16 *bt = BT + (size_t)blockIdx.x * kp * br;
    for (uint32_t e = threadIdx.x; e < kp * br; e += blockDim.x) bt[e] = tb[e % br][e / br];
}

// Warp roles: 0 = V producer (TMA), 1 = MMA issuer + TMEM owner, 2 = X and Y
// producer (TMA), 3 = idle, 4..11 = R warps (V / D, feed MMA2), 12..15 =
// accumulator warps (sum the per-tile MMA2 results in FP32 registers; split X
// and, YST tiles ahead, each Y tile into TF32 hi/lo and its transpose).
template <bool HSIDE, int KP, int NTERMS>
__global__ void __launch_bounds__(Geo<KP>::NTHR, 1)
    k_fused_half(const __grid_constant__ FusedMaps maps, const FusedArgs args)
{
    using G = Geo<KP>;
    constexpr int BR = G::BR;
    constexpr int NR = G::NR;
    constexpr uint32_t ACC_COLS = G::ACC;
    if (args.st && *(volatile const uint32_t *)&args.st->converged) return;

    extern __shared__ unsigned char smem_raw[];
    uint32_t const base_u32 = (smem_u32(smem_raw) + 1023u) & ~1023u;
    unsigned char *const base = smem_raw + (base_u32 - smem_u32(smem_raw));
    unsigned char *const sY = base;                                 // [YST][Yh | Yl]
    unsigned char *const sYT = sY + G::YST * G::YSTAGE;             // [YST][YTh | YTl]
    unsigned char *const sYB = sYT + G::YST * G::YTSTAGE;           // [YST][bf16 Y | bf16 Y^T]
    unsigned char *const sV = sYB + G::YST * G::YBSTAGE;            // [VST][VBYTES]
    uint64_t *const bars = reinterpret_cast<uint64_t *>(sV + G::VST * G::VBYTES);
    uint64_t *const vfull = bars;                   // [VST]  TMA -> epilogue
    uint64_t *const vempty = vfull + G::VST;        // [VST]  epilogue -> V producer
    uint64_t *const yfull = vempty + G::VST;        // [YST]  TMA (Yh, Yl, Y^T) -> MMA1 / MMA2
    uint64_t *const yempty = yfull + G::YST;        // [YST]  MMA2 commit -> Y producer
    uint64_t *const dfull = yempty + G::YST;        // [NDB]  MMA1 commit -> R warps
    uint64_t *const rfull = dfull + G::NDB;         // [NDB]  R warps -> MMA2
    uint64_t *const accrdy = rfull + G::NDB;        // [2]    MMA2 commit -> accumulator warps
    uint64_t *const accfree = accrdy + 2;           // [2]    accumulator warps -> MMA2
    uint64_t *const xready = accfree + 2;           // [1]    X split into TMEM -> MMA1
    uint64_t *const mdrain = xready + 1;            // [1]    issuer's final commit (drain)
    uint32_t *const tmem_slot = reinterpret_cast<uint32_t *>(mdrain + 1);
    volatile uint32_t *const abort_flag = tmem_slot + 1;

    uint32_t const warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    uint32_t const oblk = blockIdx.x / args.nsplit;
    uint32_t const split = blockIdx.x % args.nsplit;
    uint32_t const o0 = oblk * BO;
    uint32_t const T_all = (args.R + BR - 1) / BR;
    uint32_t const t_begin = split * args.tiles_per_split;
    uint32_t const t_end = min(T_all, t_begin + args.tiles_per_split);
    uint32_t const T = t_end > t_begin ? t_end - t_begin : 0;
#ifdef NMFB_FUSED_DEBUG
    // Per-tile event times of block 0 (ns since kernel start), 8 events x 64 tiles.
    unsigned long long const ts0 = globaltimer();
    unsigned long long *const dts = args.dbg ? reinterpret_cast<unsigned long long *>(args.dbg + 4 * BO * 64) : nullptr;
#define DBG_TS(ev, t)                                                                              \
    do {                                                                                           \
        if (dts && blockIdx.x == 0 && (t) < 64) dts[(ev) * 64 + (t)] = globaltimer() - ts0;        \
    } while (0)
#define DBG_PH(ph, t)                                                                                 \
    do {                                                                                              \
        if (dts && blockIdx.x == 0 && warp == 5 && lane == 0 && (t) < 64)                             \
            dts[1536 + (ph) * 64 + (t)] = clock64();                                                  \
    } while (0)
#else
#define DBG_TS(ev, t) do { } while (0)
#define DBG_PH(ph, t) do { } while (0)
#endif

    if (threadIdx.x == 0) {
        for (int s = 0; s < G::VST; s++) {
            mbar_init(&vfull[s], 1);
            mbar_init(&vempty[s], NR / 2);   // one team reads each V tile
        }
        for (int s = 0; s < G::YST; s++) {
            mbar_init(&yfull[s], 1);
            mbar_init(&yempty[s], 1);
        }
        for (uint32_t b = 0; b < G::NDB; b++) {
            mbar_init(&dfull[b], 1);
            mbar_init(&rfull[b], NR / 2);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&accrdy[b], 1);
            mbar_init(&accfree[b], 4);
        }
        mbar_init(xready, 4);
        mbar_init(mdrain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t const tmem = *tmem_slot;

    if (T == 0 && warp < 4 + NR) {
        // idle (the accumulator warps write a zero partial)
    } else if (warp == 0) {
        // ------------------------------------------------------------ V producer
        if (lane == 0) {
            uint64_t const pol = policy_evict_first();
            uint32_t issued = 0;
            for (uint32_t t = 0; t < T; t++) {
                uint32_t const s = t % G::VST;
                if (t >= (uint32_t)G::VST &&
                    !mbar_wait(&vempty[s], ((t / G::VST) - 1) & 1, abort_flag, args.err, 1u, args.wait_ns))
                    break;
                issued = t + 1;
                unsigned char *sv = sV + s * G::VBYTES;
                int const r0 = (int)((t_begin + t) * BR);
                DBG_TS(0, t);
                mbar_expect_tx(&vfull[s], G::VBYTES);
                if (HSIDE) {
                    tma_load_2d(sv, &maps.v, &vfull[s], (int)o0, r0, pol);     // V[r0:r0+BR][o0:o0+128]
                } else {
#pragma unroll
                    for (int b = 0; b < BR / 32; b++)                          // V[o0:o0+128][r0+32b : +32]
                        tma_load_2d(sv + b * (BO * 128), &maps.v, &vfull[s], r0 + 32 * b, (int)o0, pol);
                }
            }
            // drain: the last load into every stage has landed (each earlier one
            // had to, before its stage was released for reuse)
            for (uint32_t t = issued > (uint32_t)G::VST ? issued - G::VST : 0; t < issued; t++)
                mbar_drain(&vfull[t % G::VST], (t / G::VST) & 1);
        }
    } else if (warp == 2) {
        // ------------------------------------------------------------ Y producer
        if (lane == 0) {
            uint64_t const pol = policy_evict_last();
            uint32_t issued = 0;
            for (uint32_t t = 0; t < T; t++) {
                uint32_t const s = t % G::YST;
                if (t >= (uint32_t)G::YST &&
                    !mbar_wait(&yempty[s], ((t / G::YST) - 1) & 1, abort_flag, args.err, 2u, args.wait_ns))
                    break;
                issued = t + 1;
                unsigned char *syh = sY + s * G::YSTAGE;
                int const r0 = (int)((t_begin + t) * BR);
                DBG_TS(1, t);
                mbar_expect_tx(&yfull[s], G::YBYTES + G::YTSTAGE + (NTERMS == 3 ? G::YBSTAGE : 0));
                for (int b = 0; b < G::NB; b++) tma_load_2d(syh + b * G::YBLK, &maps.y, &yfull[s], b * G::CB, r0, pol);
                if (NTERMS == 3) {
                    unsigned char *syb = sYB + s * G::YBSTAGE;
                    tma_load_2d(syb, &maps.ylb, &yfull[s], 0, r0, pol);
                    tma_load_2d(syb + G::YBB, &maps.yb, &yfull[s], 0, r0, pol);
                    tma_load_2d(syb + 2 * G::YBB, &maps.ybt, &yfull[s], 0, (int)((t_begin + t) * KP), pol);
                }
                // Y^T: the BR / 32 row blocks of this tile, 2 KP rows of 128 B each
                tma_load_2d(sYT + s * G::YTSTAGE, &maps.yt, &yfull[s], 0, (r0 / 32) * 2 * KP, pol);
            }
            for (uint32_t t = issued > (uint32_t)G::YST ? issued - G::YST : 0; t < issued; t++)
                mbar_drain(&yfull[t % G::YST], (t / G::YST) & 1);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        // Two issue queues, polled without blocking (shortest nanosleep between polls):
        //   MMA2(n2): needs the R warps' R(n2) and, for n2 >= 2, the accumulator
        //             warps to have read Acc[n2 % 2] of tile n2-2;
        //   MMA1(n1): needs Y(n1) loaded and a free D buffer (MMA2(n1-NDB)
        //             issued, i.e. n1 < n2 + NDB); A = X from TMEM.
        // The Y stage of tile t is released when MMA2(t), the last reader, completes.
        if (lane == 0) {
            constexpr uint32_t IDESC1 = idesc_tf32(BO, BR, 0);
            constexpr uint32_t IDESC1B = idesc_bf16xf32(BO, BR);
            constexpr uint32_t IDESC2 = idesc_tf32(BO, KP, 0);
            constexpr uint32_t IDESC2W = idesc_tf32(BO, 2 * KP, 0);
            constexpr uint32_t IDESC2B = idesc_bf16xf32(BO, KP);
            // Shared-memory descriptors are built once; a k-step or stage offset is
            // added to the start-address field (16-byte units, no carry out of it:
            // every operand lies below 256 KB).
            uint64_t const dY0 = smem_desc(smem_u32(sY), 16, 8 * G::ROWB, G::LAYOUT);
            uint64_t const dYT0 = smem_desc(smem_u32(sYT), 16, 1024, 2u);
            uint64_t const dYB0 = smem_desc(smem_u32(sYB), 16, 8 * 2 * KP, G::BLAYOUT);
            uint64_t const dYBT0 = smem_desc(smem_u32(sYB + 2 * G::YBB), 16, 8 * 2 * BR, G::BTLAYOUT);
            bool ok = mbar_wait(xready, 0, abort_flag, args.err, 3u, args.wait_ns);
            tc_fence_after();
            uint32_t n1 = 0, n2 = 0;
            unsigned long long last = globaltimer();
            while (ok && n2 < T) {
                bool progressed = false;
                if (n2 < n1 && mbar_test(&rfull[n2 % G::NDB], (n2 / G::NDB) & 1) &&
                    (n2 < 2 || mbar_test(&accfree[n2 & 1], ((n2 >> 1) - 1) & 1))) {
                    tc_fence_after();
                    uint32_t const sp = n2 % G::YST, bp = n2 & 1, db = n2 % G::NDB;
                    uint64_t const dYT = dYT0 + ((sp * G::YTSTAGE) >> 4);
                    uint32_t const rh = tmem + G::DA0 + db * BR;
                    uint32_t const rl = tmem + G::RL0 + db * (BR / 2);
                    uint32_t const dacc = tmem + bp * ACC_COLS;
                    // MMA2 for this tile only, K = BR reduction rows:
                    //   Acc[bp][0:2KP] (+)= Rh [Y^T_hi; Y^T_lo]     (kind::tf32, N = 2 KP, k-steps of 8)
                    //   Acc[bp][0:KP]   += bf16(Rl) bf16(Y)^T      (kind::f16, N = KP, k-steps of 16;
                    //                      column group g of the R warps = k-step g, A at rl + 8 g)
                    // so Acc[0:KP] + Acc[KP:2KP] = Rh Yh + Rh Yl + Rl Y (summed by the
                    // accumulator warps in FP32 registers).
#pragma unroll
                    for (int ks = 0; ks < BR / 8; ks++) {
                        uint32_t const ob = ((ks / 4) * G::YTPAIR + (ks % 4) * 32) >> 4;
                        mma_ts(dacc, rh + ks * 8, dYT + ob, NTERMS == 3 ? IDESC2W : IDESC2, ks > 0 ? 1u : 0u);
                    }
                    if (NTERMS == 3) {
                        uint64_t const dYBT = dYBT0 + ((sp * G::YBSTAGE) >> 4);
#pragma unroll
                        for (int g = 0; g < BR / 16; g++) mma_ts_bf16(dacc, rl + g * 8, dYBT + g * 2, IDESC2B, 1u);
                    }
                    tc_commit(&accrdy[bp]);
                    tc_commit(&yempty[sp]);
                    DBG_TS(3, n2);
                    n2++;
                    progressed = true;
                }
                if (n1 < T && n1 < n2 + G::NDB && mbar_test(&yfull[n1 % G::YST], (n1 / G::YST) & 1)) {
                    tc_fence_after();
                    uint32_t const s = n1 % G::YST, db = n1 % G::NDB;
                    uint64_t const dYh = dY0 + ((s * G::YSTAGE) >> 4);
                    uint32_t const dcol = tmem + G::DA0 + db * BR;
                    uint32_t const xh = tmem + G::XC0;
                    // MMA1, K = KP:  D = Xh Yh^T (TF32, k-steps of 8 per column block), then
                    // D += [bf16(Xh) | bf16(Xl)] [bf16(Yl) ; bf16(Y)]^T (K = 2 KP, k-steps of 16:
                    // the first KP / 16 read bf16(Yl), the rest bf16(Y)).
#pragma unroll
                    for (int ks = 0; ks < KP / 8; ks++) {
                        constexpr int KPB = G::CB / 8;     // k-steps per swizzle column block
                        uint32_t const ob = ((ks / KPB) * G::YBLK + (ks % KPB) * 32) >> 4;
                        mma_ts(dcol, xh + ks * 8, dYh + ob, IDESC1, ks > 0 ? 1u : 0u);
                    }
                    if (NTERMS == 3) {
                        uint64_t const dYB = dYB0 + ((s * G::YBSTAGE) >> 4);
#pragma unroll
                        for (int j = 0; j < KP / 8; j++) {
                            uint32_t const ob = ((j / (KP / 16)) * G::YBB + (j % (KP / 16)) * 32) >> 4;
                            mma_ts_bf16(dcol, tmem + G::XB0 + j * 8, dYB + ob, IDESC1B, 1u);
                        }
                    }
                    tc_commit(&dfull[db]);
                    DBG_TS(2, n1);
                    n1++;
                    progressed = true;
                }
                if (progressed) {
                    last = globaltimer();
                } else if (*abort_flag) {
                    ok = false;
                } else if (globaltimer() - last > args.wait_ns) {
                    *abort_flag = 1;
                    atomicExch(args.err, 4u);
                    ok = false;
                } else {
                    __nanosleep(0);
                }
            }
            // drain: every MMA issued above has completed (and with it its reads of
            // shared memory and writes of tensor memory) before the CTA frees them
            mma_drain(mdrain);
        }
    } else if (warp >= 4 && warp < 4 + NR) {
        // ------------------------------------------------------------ R warps
        // Two teams of NR/2 warps take alternate tiles (team 0 even, team 1 odd), so
        // one team's load latency overlaps the other's arithmetic.  Within a team,
        // warp (quad, grp) handles TMEM lanes 32 quad .. +31 and CW = BR / GPT tile
        // columns, in chunks of 16 (one BF16 k-step of MMA2 each).
        constexpr int TW = NR / 2;                     // warps per team
        constexpr int GPT = TW / 4;                    // column groups per team
        constexpr int CW = BR / GPT;                   // tile columns per warp
        static_assert(CW % 16 == 0, "16-column chunks");
        uint32_t const quad = warp & 3;
        uint32_t const jg = (warp - 4) >> 2;
        uint32_t const team = jg / GPT, grp = jg % GPT;
        uint32_t const row = quad * 32 + lane;        // TMEM lane = output row within the block
        uint32_t const lane_addr = tmem + ((quad * 32) << 16);
        for (uint32_t t = team; t < T; t += 2) {
            uint32_t const s = t % G::VST, b = t % G::NDB;
            if (warp == 4 && lane == 0) DBG_TS(4, t);
            DBG_PH(0, t);
            if (!mbar_wait(&dfull[b], (t / G::NDB) & 1, abort_flag, args.err, 6u, args.wait_ns)) break;
            DBG_PH(1, t);
            if (!mbar_wait(&vfull[s], (t / G::VST) & 1, abort_flag, args.err, 7u, args.wait_ns)) break;
            tc_fence_after();
            DBG_PH(2, t);
            if (warp == 4 && lane == 0) DBG_TS(5, t);
            const unsigned char *sv = sV + s * G::VBYTES;
            bool const edge = (t_begin + t + 1) * BR > args.R;   // the partial last reduction tile
            int const valid = (int)(args.R - (t_begin + t) * BR);          // its columns before R
#pragma unroll 1
            for (int ch = 0; ch < CW / 16; ch++) {
                int const col0 = grp * CW + ch * 16;                          // first tile column of the chunk
                uint32_t const dcol = G::DA0 + b * BR + col0;                 // its columns of D
                uint32_t const rlcol = G::RL0 + b * (BR / 2) + (col0 / 16) * 8;  // and of bf16(Rl)
                uint32_t d[32];   // D, then the TF32 hi part of R
                uint32_t v[32];   // V, then the lo part of R
                tmem_ld16(lane_addr + dcol, d);
                if (HSIDE) {
                    // V tile [BR rows][128 cols], row-major; this thread's column = row.
                    const float *vs = reinterpret_cast<const float *>(sv) + col0 * BO + row;
#pragma unroll
                    for (int c = 0; c < 16; c++) v[c] = __float_as_uint(vs[c * BO]);
                } else {
                    // V boxes of [128 rows][32 floats], 128B swizzle.
                    int const qb = col0 / 32;
                    int const c0 = (col0 % 32) / 4;      // 16-byte chunk offset within the box
                    const unsigned char *vb = sv + qb * (BO * 128) + row * 128;
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        uint4 const x = *reinterpret_cast<const uint4 *>(vb + (((c + c0) ^ (row & 7)) << 4));
                        v[4 * c + 0] = x.x;
                        v[4 * c + 1] = x.y;
                        v[4 * c + 2] = x.z;
                        v[4 * c + 3] = x.w;
                    }
                }
                if (ch == CW / 16 - 1) {
#ifdef NMFB_FUSED_DEBUG
                    {   // debug timing only: consume the loaded V values before the next phase mark
                        uint32_t x = 0;
#pragma unroll
                        for (int c = 0; c < 16; c++) x ^= v[c];
                        asm volatile("" ::"r"(x));
                        if (x == 0x7fffffffu && dts) dts[0] = x;
                    }
#endif
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&vempty[s]);      // V stage consumed (values are in registers)
                    DBG_PH(3, t);
                }
                tmem_wait_ld_dep(d);
                if (ch == CW / 16 - 1) DBG_PH(4, t);
                if (edge) {
                    // Columns past R are zero-filled (V = 0, WH = 0): WH = 1 there makes R 0
                    // instead of 0 * inf, which MMA2 would carry into every row's sum.
#pragma unroll
                    for (int c = 0; c < 16; c++)
                        if (col0 + c >= valid) {
                            d[c] = 0x3f800000u;
                            v[c] = 0u;
                        }
                }
                uint32_t pl[8];   // bf16(R lo), packed in column pairs
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    // R = V / WH as V * (1/WH): the approximate reciprocal (<= 1 ulp) runs at
                    // full rate, the fast-division intrinsic at a third of it.  A zero WH of
                    // the data behaves as in the reference's division (V / 0 = inf, 0 / 0 = NaN).
                    float const vv = __uint_as_float(v[c]);
                    float const wh = __uint_as_float(d[c]);
                    float const r = vv * rcp_approx(wh);
                    float const h = tf32_rna(r);
#ifdef NMFB_FUSED_DEBUG
                    if (args.dbg && blockIdx.x == 0 && t == 0) {
                        args.dbg[row * 64 + col0 + c] = wh;
                        args.dbg[BO * 64 + row * 64 + col0 + c] = vv;
                        args.dbg[2 * BO * 64 + row * 64 + col0 + c] = h;
                    }
#endif
                    d[c] = __float_as_uint(h);
                    v[c] = __float_as_uint(r - h);
                }
                if (NTERMS == 3) {
#pragma unroll
                    for (int j = 0; j < 8; j++) pl[j] = bf16x2_rn(__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1]));
                }
                if (ch == CW / 16 - 1) DBG_PH(5, t);
                tmem_st16(lane_addr + dcol, d);
                if (NTERMS == 3) tmem_st8(lane_addr + rlcol, pl);
            }
            tmem_wait_st();
            DBG_PH(6, t);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&rfull[b]);
            DBG_PH(7, t);
            if (warp == 4 && lane == 0) DBG_TS(6, t);
#ifdef NMFB_FUSED_DEBUG
            if (lane == 0 && dts && blockIdx.x == 0 && t < 64 && warp < 12) dts[512 + (warp - 4) * 64 + t] = globaltimer() - ts0;
#endif
        }
    } else if (warp >= 4 + NR) {
        // ------------------------------------------------------------ accumulator warps
        // Warp 4+NR+q owns TMEM lanes 32q..32q+31: sums the per-tile Acc into FP32
        // registers, and (all four together) splits X once.
        uint32_t const quad = warp & 3;
        uint32_t const row = quad * 32 + lane;
        uint32_t const lane_addr = tmem + ((quad * 32) << 16);
        float sum[KP];
#pragma unroll
        for (int c = 0; c < KP; c++) sum[c] = 0.0f;
        bool ok = true;
        if (T > 0) {   // this thread's row of X as TF32 hi and bf16(hi) | bf16(lo), into TMEM lanes = rows
            uint32_t const o = o0 + row;
            const float *xr = args.X + (size_t)o * KP;
#pragma unroll
            for (int c0 = 0; c0 < KP; c0 += 16) {
                uint32_t h[32], hb[8], lb[8];
#pragma unroll
                for (int c = 0; c < 16; c += 4) {
                    float4 const x = (o < args.O) ? *reinterpret_cast<const float4 *>(xr + c0 + c)
                                                  : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    float const xs[4] = {x.x, x.y, x.z, x.w};
                    float hv[4], lo[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        hv[i] = tf32_rna(xs[i]);
                        h[c + i] = __float_as_uint(hv[i]);
                        lo[i] = xs[i] - hv[i];
                    }
                    hb[c / 2] = bf16x2_rn(hv[0], hv[1]);
                    hb[c / 2 + 1] = bf16x2_rn(hv[2], hv[3]);
                    lb[c / 2] = bf16x2_rn(lo[0], lo[1]);
                    lb[c / 2 + 1] = bf16x2_rn(lo[2], lo[3]);
                }
                tmem_st16(lane_addr + G::XC0 + c0, h);
                if (NTERMS == 3) {
                    tmem_st8(lane_addr + G::XB0 + c0 / 2, hb);
                    tmem_st8(lane_addr + G::XB0 + KP / 2 + c0 / 2, lb);
                }
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(xready);
        }
        for (uint32_t t = 0; ok && t < T; t++) {
            uint32_t const bp = t & 1;
            if (!mbar_wait(&accrdy[bp], (t >> 1) & 1, abort_flag, args.err, 8u, args.wait_ns)) { ok = false; break; }
            tc_fence_after();
            // Acc columns [0, KP) and, for the 3-term arm, [KP, 2 KP) both add to sum.
#pragma unroll
            for (int part = 0; part < (NTERMS == 3 ? 2 : 1); part++) {
#pragma unroll
                for (int c0 = 0; c0 < KP; c0 += 32) {
                    uint32_t a[32];
                    if (KP - c0 >= 32) tmem_ld32(lane_addr + bp * ACC_COLS + part * KP + c0, a);
                    else tmem_ld16(lane_addr + bp * ACC_COLS + part * KP + c0, a);
                    tmem_wait_ld_dep(a);
#pragma unroll
                    for (int c = 0; c < 32; c++)
                        if (c0 + c < KP) sum[c0 + c] += __uint_as_float(a[c]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&accfree[bp]);
            if (warp == 4 + NR && lane == 0) DBG_TS(7, t);
#ifdef NMFB_FUSED_DEBUG
            if (lane == 0 && dts && blockIdx.x == 0 && t < 64) dts[1024 + (warp - 4 - NR) * 64 + t] = globaltimer() - ts0;
#endif
        }
#ifdef NMFB_FUSED_DEBUG
        if (ok && args.dbg && blockIdx.x == 0)
            for (int c = 0; c < KP; c++) args.dbg[3 * BO * 64 + row * KP + c] = sum[c];
#endif
        // this split's partial (zero for an idle split); k_finish sums the splits
        if (ok) {
            uint32_t const o = o0 + row;
            if (o < args.O) {
                float *dst = args.part + ((size_t)split * args.O + o) * KP;
#pragma unroll
                for (int c = 0; c < KP; c += 4)
                    *reinterpret_cast<float4 *>(dst + c) = make_float4(sum[c], sum[c + 1], sum[c + 2], sum[c + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

int encode_2d(nmfb_ctx *ctx, CUtensorMap *map, const void *base, uint64_t inner, uint64_t outer, uint64_t row_bytes,
              uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle sw,
              CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32)
{
    auto fn = encode_fn();
    if (!fn) return nmfb_fail(ctx, NMFB_ENODEV, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(map, dt, 2, (void *)base, dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nmfb_fail(ctx, NMFB_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return NMFB_OK;
}

// Layout of one factor's split copies (k_split_factor's outputs), in one buffer:
// hi (rows x kp FP32) | transposed hi/lo per 32 rows | bf16(lo) (rows x kp) |
// bf16(y) (rows x kp) | bf16(y) transposed per br rows.
struct SplitLayout {
    size_t t, bl, b, bt, floats;   // offsets in floats (bl, b, bt: start of the BF16 parts)
    uint32_t br, nblk32, nblkbr;
    SplitLayout(uint32_t rows, uint32_t kp)
    {
        br = (kp >= 64) ? 32 : 64;
        nblk32 = (rows + 31) / 32;
        nblkbr = (rows + br - 1) / br;
        size_t const f = (size_t)rows * kp;
        t = f;
        bl = t + (size_t)nblk32 * 64 * kp;
        b = bl + f / 2;                                   // rows * kp BF16 = f / 2 floats (kp is even)
        bt = b + f / 2;
        floats = bt + ((size_t)nblkbr * kp * br + 1) / 2;
    }
};

struct FusedPlan {
    FusedMaps mapsH, mapsW;  // update_H (HSIDE) and update_W
    uint32_t *dErr;
    float *dSplitW, *dSplitH;  // split copies of W and of H (k_split_factor, SplitLayout)
    double *dCs;               // [row blocks + chunks][kp] column-sum partials of k_finish
    uint32_t *dTick;           // [chunks + 1] retirement counters of k_finish
    uint32_t nticks, csoff;
#ifdef NMFB_FUSED_DEBUG
    float *dDbg;
#endif
};

template <bool HSIDE, int KP, int NTERMS>
int launch_fused(nmfb_ctx *ctx, const FusedMaps &maps, int adjust)
{
    using G = Geo<KP>;
    constexpr int BR = G::BR;
    auto kern = k_fused_half<HSIDE, KP, NTERMS>;
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    uint32_t const O = HSIDE ? ctx->m : ctx->n;
    uint32_t const R = HSIDE ? ctx->n : ctx->m;
    uint32_t const oblocks = (O + BO - 1) / BO;
    uint32_t const T = (R + BR - 1) / BR;
    // Splits of the reduction: one CTA per SM at a time, so the launch takes
    // ceil(CTAs / SMs) waves of (tiles per split + pipeline fill) tile times;
    // pick the split count that minimises that (fill ~ 6 tiles: TMEM
    // allocation, X load and split, pipeline ramp, partial write; measured
    // best among 1, 3 and 6).
    uint32_t tps = T, best = 0xffffffffu;
    for (uint32_t want = 1; want <= NMFB_MAX_SPLIT && want <= T; want++) {
        uint32_t const t_ps = (T + want - 1) / want;
        uint32_t const ns = (T + t_ps - 1) / t_ps;
        if ((size_t)ns * O * KP > ctx->part_items) break;
        uint32_t const waves = (oblocks * ns + (uint32_t)ctx->sm_count - 1) / (uint32_t)ctx->sm_count;
        uint32_t const cost = waves * (t_ps + 6);
        if (cost < best) {
            best = cost;
            tps = t_ps;
        }
    }
    uint32_t const nsplit = (T + tps - 1) / tps;
    if ((size_t)nsplit * O * KP > ctx->part_items)
        return nmfb_fail(ctx, NMFB_EINVAL, "fused: partial buffer too small (%u splits)", nsplit);
    FusedArgs args;
    args.O = O;
    args.R = R;
    args.tiles_per_split = tps;
    args.nsplit = nsplit;
    args.part = ctx->dPart;
    args.err = plan->dErr;
    args.st = ctx->dState;
    args.X = HSIDE ? ctx->dH : ctx->dW;
    args.wait_ns = ctx->wait_ns ? ctx->wait_ns : WAIT_LIMIT_NS;
#ifdef NMFB_FUSED_DEBUG
    args.dbg = plan->dDbg;
#endif
    int const main = HSIDE ? 0 : 1;
    int rc = nmfb_prof_begin(ctx, main);
    if (rc) return rc;
    kern<<<oblocks * nsplit, G::NTHR, G::SMEM, ctx->stream>>>(maps, args);
    NMFB_LAUNCH_CHECK(ctx);
    if ((rc = nmfb_prof_end(ctx, main))) return rc;

    FinishArgs fa;
    float *xsp = HSIDE ? plan->dSplitH : plan->dSplitW;
    SplitLayout const L(O, KP);
    fa.O = O;
    fa.nsplit = nsplit;
    fa.k = ctx->k;
    fa.adjust = adjust;
    fa.part = ctx->dPart;
    fa.X = HSIDE ? ctx->dH : ctx->dW;
    fa.accY = HSIDE ? ctx->dAccW : ctx->dAccH;
    fa.xhi = xsp;
    fa.xT = xsp + L.t;
    fa.xBl = reinterpret_cast<__nv_bfloat16 *>(xsp + L.bl);
    fa.xB = reinterpret_cast<__nv_bfloat16 *>(xsp + L.b);
    fa.xBT = reinterpret_cast<__nv_bfloat16 *>(xsp + L.bt);
    fa.xnblk32 = L.nblk32;
    fa.xnblkbr = L.nblkbr;
    fa.cs = plan->dCs;
    fa.csoff = plan->csoff;
    fa.accX = HSIDE ? ctx->dAccH : ctx->dAccW;
    fa.tick = plan->dTick;
    fa.st = ctx->dState;
    uint32_t const fblocks = fin_blocks(O, fin_rpt(nsplit));
    if (fblocks > plan->csoff || (fblocks + FIN_ECH - 1) / FIN_ECH + 1 > plan->nticks)
        return nmfb_fail(ctx, NMFB_EINVAL, "fused: column-sum buffers too small");
    fin_launch<KP, BR, 0>(fa, ctx->stream);
    NMFB_LAUNCH_CHECK(ctx);
    return (int)nsplit;
}

template <bool HSIDE>
int dispatch(nmfb_ctx *ctx, const FusedMaps &maps, int adjust)
{
    bool const x3 = ctx->arm == NMFB_ARM_FUSED;
    switch (ctx->kp) {
    case 16: return x3 ? launch_fused<HSIDE, 16, 3>(ctx, maps, adjust) : launch_fused<HSIDE, 16, 1>(ctx, maps, adjust);
    case 32: return x3 ? launch_fused<HSIDE, 32, 3>(ctx, maps, adjust) : launch_fused<HSIDE, 32, 1>(ctx, maps, adjust);
    case 64: return x3 ? launch_fused<HSIDE, 64, 3>(ctx, maps, adjust) : launch_fused<HSIDE, 64, 1>(ctx, maps, adjust);
    default: return nmfb_fail(ctx, NMFB_EINVAL, "fused arm: unsupported padded rank %u", ctx->kp);
    }
}

// Split copies and column sums of a factor, for a half-iteration that reads
// it as Y when the previous half-iteration's epilogue did not produce them.
int prepare_factor(nmfb_ctx *ctx, bool w)
{
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    const float *F = w ? ctx->dW : ctx->dH;
    uint32_t const rows = w ? ctx->n : ctx->m;
    int rc = nmfb_colsum(ctx, F, rows, w ? ctx->dAccW : ctx->dAccH, w ? 0 : 1);
    if (rc) return rc;
    float *sp = w ? plan->dSplitW : plan->dSplitH;
    SplitLayout const L(rows, ctx->kp);
    k_split_factor<<<L.nblkbr, 256, 0, ctx->stream>>>(F, rows, ctx->kp, L.br, sp, sp + L.t,
                                                     reinterpret_cast<__nv_bfloat16 *>(sp + L.bl),
                                                     reinterpret_cast<__nv_bfloat16 *>(sp + L.b),
                                                     reinterpret_cast<__nv_bfloat16 *>(sp + L.bt), ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    ctx->fz_ok[w ? 0 : 1] = 1;
    return NMFB_OK;
}

// One half-iteration: a single launch when the other factor's split copies and
// column sums are current (the previous half-iteration's epilogue wrote them).
int fused_half(nmfb_ctx *ctx, bool is_H, int adjust)
{
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    if (!plan) return nmfb_fail(ctx, NMFB_ESTATE, "fused arm not prepared");
    int const whole = is_H ? 2 : 3;
    int rc = nmfb_prof_begin(ctx, whole);
    if (rc) return rc;
    bool const yw = is_H;   // Y = W for update_H
    if (!ctx->fz_ok[yw ? 0 : 1] && (rc = prepare_factor(ctx, yw))) return rc;
    int const nsplit = is_H ? dispatch<true>(ctx, plan->mapsH, adjust) : dispatch<false>(ctx, plan->mapsW, adjust);
    if (nsplit < 0) return nsplit;
    ctx->fz_ok[is_H ? 1 : 0] = 1;
    return nmfb_prof_end(ctx, whole);
}

}  // namespace

template <int KP>
int set_smem_attrs(nmfb_ctx *ctx)
{
    int const smem = Geo<KP>::SMEM;
    NMFB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_fused_half<true, KP, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    NMFB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_fused_half<false, KP, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    NMFB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_fused_half<true, KP, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    NMFB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_fused_half<false, KP, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return NMFB_OK;
}

int nmfb_fused_prepare(nmfb_ctx *ctx)
{
    if (ctx->tmaps) return NMFB_OK;
    uint32_t const kp = ctx->kp;
    if (kp != 16 && kp != 32 && kp != 64)
        return nmfb_fail(ctx, NMFB_EINVAL, "the fused arm supports ranks up to 64 (k=%u); use the plain arm", ctx->k);
    int rc = (kp == 16) ? set_smem_attrs<16>(ctx) : (kp == 32) ? set_smem_attrs<32>(ctx) : set_smem_attrs<64>(ctx);
    if (rc) return rc;
    FusedPlan *plan = (FusedPlan *)calloc(1, sizeof(FusedPlan));
    if (!plan) return nmfb_fail(ctx, NMFB_ENOMEM, "fused plan");
    ctx->tmaps = plan;
    cudaError_t e = nmfb_malloc(ctx, (void **)&plan->dErr, sizeof(uint32_t));
    if (e != cudaSuccess) return nmfb_fail(ctx, NMFB_ENOMEM, "fused error word: %s", cudaGetErrorString(e));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(plan->dErr, 0, sizeof(uint32_t), ctx->own_stream));
#ifdef NMFB_FUSED_DEBUG
    NMFB_CUDA_TRY(ctx, nmfb_malloc(ctx, (void **)&plan->dDbg, (4 * BO * 64 + 8192) * sizeof(float)));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(plan->dDbg, 0, (4 * BO * 64 + 8192) * sizeof(float), ctx->own_stream));
#endif
    uint32_t const cb = (kp == 16) ? 16 : 32;
    CUtensorMapSwizzle const fsw = (kp == 16) ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    auto const sw_for = [](uint32_t bytes) {
        return bytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B : bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    };
    CUtensorMapDataType const BF16 = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    uint64_t const vrow = ctx->ldv * sizeof(float), frow = (uint64_t)kp * sizeof(float);
    SplitLayout const LW(ctx->n, kp), LH(ctx->m, kp);
    uint32_t const br = LW.br;
    e = nmfb_malloc(ctx, (void **)&plan->dSplitW, LW.floats * sizeof(float));
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&plan->dSplitH, LH.floats * sizeof(float));
    uint32_t const maxblk = fin_blocks(ctx->n > ctx->m ? ctx->n : ctx->m, 1);   // k_finish's most row blocks
    plan->csoff = maxblk;
    plan->nticks = (maxblk + FIN_ECH - 1) / FIN_ECH + 1;
    if (e == cudaSuccess)
        e = nmfb_malloc(ctx, (void **)&plan->dCs, (size_t)(maxblk + (maxblk + FIN_ECH - 1) / FIN_ECH) * kp * sizeof(double));
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&plan->dTick, plan->nticks * sizeof(uint32_t));
    if (e != cudaSuccess) return nmfb_fail(ctx, NMFB_ENOMEM, "fused split buffers: %s", cudaGetErrorString(e));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(plan->dTick, 0, plan->nticks * sizeof(uint32_t), ctx->own_stream));
    // Maps over one factor's split copies: Y (the other factor, `rows` rows).
    auto const y_maps = [&](FusedMaps &mp, const float *sp, const SplitLayout &L, uint32_t rows) -> int {
        int r;
        if ((r = encode_2d(ctx, &mp.y, sp, kp, rows, frow, cb, br, fsw))) return r;
        if ((r = encode_2d(ctx, &mp.ylb, sp + L.bl, kp, rows, (uint64_t)kp * 2, kp, br, sw_for(2 * kp), BF16)))
            return r;
        if ((r = encode_2d(ctx, &mp.yt, sp + L.t, 32, (uint64_t)L.nblk32 * 2 * kp, 128, 32, 2 * kp * (br / 32),
                           CU_TENSOR_MAP_SWIZZLE_128B)))
            return r;
        if ((r = encode_2d(ctx, &mp.yb, sp + L.b, kp, rows, (uint64_t)kp * 2, kp, br, sw_for(2 * kp), BF16))) return r;
        return encode_2d(ctx, &mp.ybt, sp + L.bt, br, (uint64_t)L.nblkbr * kp, (uint64_t)br * 2, br, kp,
                         sw_for(2 * br), BF16);
    };
    // update_H: X = H (rows m), Y = W (rows n); V tile [br rows of V][128 cols].
    FusedMaps &mh = plan->mapsH;
    if ((rc = encode_2d(ctx, &mh.v, ctx->dV, ctx->m, ctx->n, vrow, BO, br, CU_TENSOR_MAP_SWIZZLE_NONE))) return rc;
    if ((rc = y_maps(mh, plan->dSplitW, LW, ctx->n))) return rc;
    // update_W: X = W (rows n), Y = H (rows m); V tile [128 rows][32 cols] x (br/32), 128B swizzle.
    FusedMaps &mw = plan->mapsW;
    if ((rc = encode_2d(ctx, &mw.v, ctx->dV, ctx->m, ctx->n, vrow, 32, BO, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = y_maps(mw, plan->dSplitH, LH, ctx->m))) return rc;
    return NMFB_OK;
}

int nmfb_fused_release(nmfb_ctx *ctx)
{
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    if (!plan) return NMFB_OK;
    if (plan->dErr) nmfb_free(ctx, plan->dErr);
    if (plan->dSplitW) nmfb_free(ctx, plan->dSplitW);
    if (plan->dSplitH) nmfb_free(ctx, plan->dSplitH);
    if (plan->dCs) nmfb_free(ctx, plan->dCs);
    if (plan->dTick) nmfb_free(ctx, plan->dTick);
    free(plan);
    ctx->tmaps = nullptr;
    return NMFB_OK;
}

int nmfb_fused_update_H(nmfb_ctx *ctx, int adjust) { return fused_half(ctx, true, adjust); }

// Makes W's split copies and column sums current (before a test block is
// replayed as a graph, which holds no preparation launch).
int nmfb_fused_ready_W(nmfb_ctx *ctx)
{
    if (!ctx->tmaps || ctx->fz_ok[0]) return NMFB_OK;
    return prepare_factor(ctx, true);
}
int nmfb_fused_update_W(nmfb_ctx *ctx, int adjust) { return fused_half(ctx, false, adjust); }

uint32_t *nmfb_fused_err_word(nmfb_ctx *ctx)
{
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    return plan ? plan->dErr : nullptr;
}

// Reads the fused kernels' error word (the site of the first bounded wait that
// ran out, 0 if none) and clears it, so each expiry is reported once and the
// context stays usable.
int nmfb_fused_error(nmfb_ctx *ctx, uint32_t *code)
{
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    *code = 0;
    if (!plan) return NMFB_OK;
    NMFB_CUDA_TRY(ctx, cudaMemcpyAsync(code, plan->dErr, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (*code) {
        // an aborted launch may have left retirement counters and factor copies behind
        NMFB_CUDA_TRY(ctx, cudaMemsetAsync(plan->dErr, 0, sizeof(uint32_t), ctx->stream));
        NMFB_CUDA_TRY(ctx, cudaMemsetAsync(plan->dTick, 0, plan->nticks * sizeof(uint32_t), ctx->stream));
        ctx->fz_ok[0] = ctx->fz_ok[1] = 0;
        NMFB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return NMFB_OK;
}

#ifdef NMFB_FUSED_DEBUG
extern "C" int nmfb_debug_dump(nmfb_ctx *ctx, float *host)
{
    FusedPlan *plan = (FusedPlan *)ctx->tmaps;
    NMFB_CUDA_TRY(ctx, cudaMemcpy(host, plan->dDbg, (4 * BO * 64 + 8192) * sizeof(float), cudaMemcpyDeviceToHost));
    return NMFB_OK;
}
#endif
