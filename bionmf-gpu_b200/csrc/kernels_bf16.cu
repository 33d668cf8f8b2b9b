// kernels_bf16.cu -- the BF16 fused half-iteration arms (NMFB_ARM_BF16,
// NMFB_ARM_SPLIT_BF16 and NMFB_ARM_BF16X3).
//
// Same method and data flow as the FP32 arm (kernels_fused.cu): for 128 rows
// of the factor X being updated and a range of the reduction dimension, each
// 64-row tile of the other factor Y and the matching V tile give
//   D   = X Y^T                      (MMA1, TMEM, FP32 accumulate)
//   R   = V / D                      (R warps, FP32 registers)
//   Acc = R Y                        (MMA2, TMEM, FP32 accumulate)
// and Acc is summed per tile into FP32 registers; k_finish (finish.cuh) then
// applies X = X .* (sum of splits) ./ colsum(Y) and writes X's BF16 copies and
// column sums for the next half-iteration.  What changes is the operand type of
// the two contractions (tcgen05.mma kind::f16, BF16 A and B, K = 16 per
// instruction, FP32 accumulation):
//   NMFB_ARM_BF16       : X, Y, R rounded to BF16 (one product each);
//   NMFB_ARM_SPLIT_BF16 : the WH denominator from a split-BF16 product,
//                         x = xh + xl (xh = BF16(x), xl = BF16(x - xh)),
//                         D = Xh Yh^T + Xh Yl^T + Xl Yh^T (16 significant bits:
//                         small WH entries amplify denominator error in the
//                         quotient); MMA2 stays one BF16 product;
//   NMFB_ARM_BF16X3     : both contractions split, MMA2 = Rh Yh + Rh Yl + Rl Yh
//                         (FP32-class results from BF16 tensor instructions,
//                         K = 16 per instruction against 8 for TF32).
// The quotient, the per-tile sums and the updates stay FP32.  BF16 keeps FP32's
// 8-bit exponent, so a per-column rescaling of the factors would change no
// rounding error and is not applied.
//
// All operands reach shared memory by TMA in the layout the MMA reads: BF16
// hi / lo copies of X and Y (rows x KP, K-major) and, per 64-row block, the
// transposed hi block followed by the transposed lo block (64 rows -> 2 KP rows
// of 64 values) that MMA2 reads K-major -- written by k_finish when the factor
// is updated, or by k_split_bf16 when it is not current (start of a run, after
// the test's EPS adjust of H).  The R warps work in two teams on alternate tiles.
// R goes to shared memory (128B-swizzled, K-major), so both MMAs take A and B
// from shared memory.
//
// Warp roles (768 threads): 0 = V producer, 1 = MMA issuer / TMEM owner,
// 2 = X and Y producer, 3 = idle, 4..19 = R warps, 20..23 = accumulator warps.
// Every wait is bounded (1 s); on expiry the kernel records an error word that
// the host turns into NMFB_ETIMEOUT.  No TMA multicast is used.
#include "nmfb_internal.cuh"
#include "fused_common.cuh"
#include "finish.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <float.h>

using nmfb::ConvState;
using namespace nmfb_tc;

namespace {

// kind::f16 instruction descriptor: BF16 A and B, both K-major, FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// Two floats to a BF16 pair (round to nearest even); `first` in the low half,
// i.e. at the lower address.
__device__ __forceinline__ uint32_t pack_bf16x2(float first, float second)
{
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(second), "f"(first));
    return r;
}

// MODE 0: BF16 x BF16 in both contractions; 1: split-BF16 WH denominator;
// 2: split-BF16 in both contractions.
template <int KP, int MODE>
struct GeoB {
    static constexpr int BR = 64;                           // reduction rows per tile
    static constexpr int ROWB = 2 * KP;                     // bytes per X / Y row
    static constexpr uint32_t LAYOUT = (KP == 16) ? 6u : (KP == 32) ? 4u : 2u;   // SW32 / SW64 / SW128
    static constexpr int XBYTES = BO * KP * 2;
    static constexpr int YBYTES = BR * KP * 2;              // = KP rows of 128 B: one Y^T part
    static constexpr int YTROWS = (MODE == 2 ? 2 : 1) * KP; // Y^T hi (and lo) rows per tile
    static constexpr int YSTAGE = 2 * YBYTES + YTROWS * 128;   // Yh | Yl | Y^T
    static constexpr int RBYTES = BO * BR * 2;              // one R part
    static constexpr int RSTAGE = (MODE == 2 ? 2 : 1) * RBYTES;  // Rh (| Rl)
    static constexpr int VBYTES = BO * BR * 4;
    static constexpr int YST = (KP == 64 && MODE == 2) ? 2 : 3;
    static constexpr int NRB = 2;                           // R stages
    static constexpr uint32_t NDB = 4;                      // D buffers in TMEM
    static constexpr int FIXED = 1024 + 512;
    static constexpr int VAVAIL = (SMEM_LIMIT - FIXED - 2 * XBYTES - YST * YSTAGE - NRB * RSTAGE) / VBYTES;
    static constexpr int VST = VAVAIL > 6 ? 6 : VAVAIL;
    static_assert(VST >= 2, "shared-memory ring too small");
    static constexpr int SMEM = FIXED + 2 * XBYTES + YST * YSTAGE + NRB * RSTAGE + VST * VBYTES;
    static constexpr int NR = 16;                           // R warps
    static constexpr int NTHR = (4 + NR + 4) * 32;
    static constexpr uint32_t ACCW = (MODE == 2 ? 2 : 1) * KP;   // TMEM columns of one accumulator
    static constexpr uint32_t DB0 = 2 * ACCW;               // Acc[0..1] at 0 and ACCW; D[b] at DB0 + b*BR
    static_assert(DB0 + NDB * BR <= TMEM_COLS, "TMEM columns exceeded");
    static_assert(YBYTES % 1024 == 0 && YSTAGE % 1024 == 0 && XBYTES % 1024 == 0, "1024-byte stage alignment");
};

struct MapsB {
    CUtensorMap v;        // V (FP32), as in the FP32 arm
    CUtensorMap xh, xl;   // X hi / lo (BF16, rows x KP), box [KP x 128]
    CUtensorMap yh, yl;   // Y hi / lo (BF16, rows x KP), box [KP x 64]
    CUtensorMap yt;       // Y^T blocks (BF16, [rows/64][hi, lo][KP][64]), box [64 x KP] or [64 x 2 KP]
};

struct ArgsB {
    uint32_t O, R;
    uint32_t tiles_per_split, nsplit;
    float *part;
    uint32_t *err;
    const ConvState *st;
    unsigned long long wait_ns;  // limit of every bounded wait (%globaltimer ns)
};

// BF16 hi / lo copies of a factor (rows x kp FP32, padding columns zero) and,
// when T is given, per 64-row block the transposed hi block (kp rows of 64)
// followed by the transposed lo block, rows past the end zero.  One CTA per
// 64-row block.
__global__ void __launch_bounds__(256) k_split_bf16(const float *__restrict__ Y, uint32_t rows, uint32_t kp,
                                                    __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                                    __nv_bfloat16 *__restrict__ T, const ConvState *st)
{
    if (st && *(volatile const uint32_t *)&st->converged) return;
    __shared__ __nv_bfloat16 th[64][66], tl[64][66];
    uint32_t const r0 = blockIdx.x * 64;
    for (uint32_t e = threadIdx.x; e < 64 * kp; e += blockDim.x) {
        uint32_t const r = e / kp, c = e % kp;
        bool const in = r0 + r < rows;
        float const y = in ? Y[(size_t)(r0 + r) * kp + c] : 0.0f;
        __nv_bfloat16 const h = __float2bfloat16_rn(y);
        __nv_bfloat16 const l = __float2bfloat16_rn(y - __bfloat162float(h));
        if (in) {
            hi[(size_t)(r0 + r) * kp + c] = h;
            lo[(size_t)(r0 + r) * kp + c] = l;
        }
        th[r][c] = h;
        tl[r][c] = l;
    }
    if (!T) return;
    __syncthreads();
    __nv_bfloat16 *dst = T + (size_t)blockIdx.x * 2 * kp * 64;
    for (uint32_t e = threadIdx.x; e < 2 * kp * 64; e += blockDim.x) {
        uint32_t const row = e / 64, rr = e % 64;
        dst[e] = row < kp ? th[rr][row] : tl[rr][row - kp];
    }
}

template <bool HSIDE, int KP, int MODE>
__global__ void __launch_bounds__(GeoB<KP, MODE>::NTHR, 1)
    k_fused_bf16(const __grid_constant__ MapsB maps, const ArgsB args)
{
    using G = GeoB<KP, MODE>;
    constexpr int BR = G::BR;
    constexpr int NR = G::NR;
    constexpr bool SPLIT = MODE >= 1;                // MMA1 split
    constexpr bool SPLIT2 = MODE == 2;               // MMA2 split
    constexpr int NTERMS = SPLIT ? 3 : 1;
    if (args.st && *(volatile const uint32_t *)&args.st->converged) return;

    extern __shared__ unsigned char smem_raw[];
    uint32_t const base_u32 = (smem_u32(smem_raw) + 1023u) & ~1023u;
    unsigned char *const base = smem_raw + (base_u32 - smem_u32(smem_raw));
    unsigned char *const sX = base;                                  // Xh | Xl
    unsigned char *const sY = sX + 2 * G::XBYTES;                    // [YST][Yh | Yl | Y^T]
    unsigned char *const sR = sY + G::YST * G::YSTAGE;               // [NRB][Rh | Rl]
    unsigned char *const sV = sR + G::NRB * G::RSTAGE;               // [VST][V]
    uint64_t *const bars = reinterpret_cast<uint64_t *>(sV + G::VST * G::VBYTES);
    uint64_t *const vfull = bars;                    // [VST]  TMA -> R warps
    uint64_t *const vempty = vfull + G::VST;         // [VST]  R warps -> V producer
    uint64_t *const yfull = vempty + G::VST;         // [YST]  TMA -> MMA1 / MMA2
    uint64_t *const yempty = yfull + G::YST;         // [YST]  MMA2 commit -> Y producer
    uint64_t *const dfull = yempty + G::YST;         // [NDB]  MMA1 commit -> R warps
    uint64_t *const rfull = dfull + G::NDB;          // [NRB]  R warps -> MMA2
    uint64_t *const rempty = rfull + G::NRB;         // [NRB]  MMA2 commit -> R warps
    uint64_t *const accrdy = rempty + G::NRB;        // [2]    MMA2 commit -> accumulator warps
    uint64_t *const accfree = accrdy + 2;            // [2]    accumulator warps -> MMA2
    uint64_t *const xfull = accfree + 2;             // [1]    TMA -> MMA1
    uint64_t *const mdrain = xfull + 1;              // [1]    issuer's final commit (drain)
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

    if (threadIdx.x == 0) {
        for (int s = 0; s < G::VST; s++) {
            mbar_init(&vfull[s], 1);
            mbar_init(&vempty[s], NR / 2);   // one team reads each V tile
        }
        for (int s = 0; s < G::YST; s++) {
            mbar_init(&yfull[s], 1);
            mbar_init(&yempty[s], 1);
        }
        for (uint32_t b = 0; b < G::NDB; b++) mbar_init(&dfull[b], 1);
        for (int b = 0; b < G::NRB; b++) {
            mbar_init(&rfull[b], NR / 2);
            mbar_init(&rempty[b], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&accrdy[b], 1);
            mbar_init(&accfree[b], 4);
        }
        mbar_init(xfull, 1);
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

    if (T == 0) {
        // idle
    } else if (warp == 0) {
        // ------------------------------------------------------------ V producer
        if (lane == 0) {
            uint64_t const pol = policy_evict_first();
            uint32_t issued = 0;
            for (uint32_t t = 0; t < T; t++) {
                uint32_t const s = t % G::VST;
                if (t >= (uint32_t)G::VST &&
                    !mbar_wait(&vempty[s], ((t / G::VST) - 1) & 1, abort_flag, args.err, 21u, args.wait_ns))
                    break;
                issued = t + 1;
                unsigned char *sv = sV + s * G::VBYTES;
                int const r0 = (int)((t_begin + t) * BR);
                mbar_expect_tx(&vfull[s], G::VBYTES);
                if (HSIDE) {
                    tma_load_2d(sv, &maps.v, &vfull[s], (int)o0, r0, pol);     // V[r0:r0+BR][o0:o0+128]
                } else {
#pragma unroll
                    for (int b = 0; b < BR / 32; b++)                          // V[o0:o0+128][r0+32b : +32]
                        tma_load_2d(sv + b * (BO * 128), &maps.v, &vfull[s], r0 + 32 * b, (int)o0, pol);
                }
            }
            // drain: the last load into every stage has landed
            for (uint32_t t = issued > (uint32_t)G::VST ? issued - G::VST : 0; t < issued; t++)
                mbar_drain(&vfull[t % G::VST], (t / G::VST) & 1);
        }
    } else if (warp == 2) {
        // ------------------------------------------------------------ X and Y producer
        if (lane == 0) {
            uint64_t const pol = policy_evict_last();
            mbar_expect_tx(xfull, (SPLIT ? 2 : 1) * G::XBYTES);
            tma_load_2d(sX, &maps.xh, xfull, 0, (int)o0, pol);
            if (SPLIT) tma_load_2d(sX + G::XBYTES, &maps.xl, xfull, 0, (int)o0, pol);
            uint32_t issued = 0;
            for (uint32_t t = 0; t < T; t++) {
                uint32_t const s = t % G::YST;
                if (t >= (uint32_t)G::YST &&
                    !mbar_wait(&yempty[s], ((t / G::YST) - 1) & 1, abort_flag, args.err, 22u, args.wait_ns))
                    break;
                issued = t + 1;
                unsigned char *sy = sY + s * G::YSTAGE;
                int const r0 = (int)((t_begin + t) * BR);
                mbar_expect_tx(&yfull[s], (SPLIT ? 2 : 1) * G::YBYTES + G::YTROWS * 128);
                tma_load_2d(sy, &maps.yh, &yfull[s], 0, r0, pol);
                if (SPLIT) tma_load_2d(sy + G::YBYTES, &maps.yl, &yfull[s], 0, r0, pol);
                tma_load_2d(sy + 2 * G::YBYTES, &maps.yt, &yfull[s], 0, (int)((t_begin + t) * 2 * KP), pol);
            }
            // drain: X and the last load into every Y stage have landed
            mbar_drain(xfull, 0);
            for (uint32_t t = issued > (uint32_t)G::YST ? issued - G::YST : 0; t < issued; t++)
                mbar_drain(&yfull[t % G::YST], (t / G::YST) & 1);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        //   MMA2(n2): needs R(n2) in shared memory and, for n2 >= 2, Acc[n2 % 2]
        //             read by the accumulator warps (tile n2-2);
        //   MMA1(n1): needs Y(n1) and a free D buffer (n1 < n2 + NDB).
        // MMA2(t) is the last reader of Y stage t % YST and R stage t % NRB.
        if (lane == 0) {
            constexpr uint32_t IDESC1 = idesc_bf16(BO, BR);
            constexpr uint32_t IDESC2 = idesc_bf16(BO, KP);
            constexpr uint32_t IDESC2W = idesc_bf16(BO, 2 * KP);
            uint64_t const dXh = smem_desc(smem_u32(sX), 16, 8 * G::ROWB, G::LAYOUT);
            uint64_t const dXl = dXh + (G::XBYTES >> 4);
            uint64_t const dY0 = smem_desc(smem_u32(sY), 16, 8 * G::ROWB, G::LAYOUT);
            uint64_t const dYT0 = smem_desc(smem_u32(sY + 2 * G::YBYTES), 16, 1024, 2u);
            uint64_t const dR0 = smem_desc(smem_u32(sR), 16, 1024, 2u);
            bool ok = mbar_wait(xfull, 0, abort_flag, args.err, 23u, args.wait_ns);
            tc_fence_after();
            uint32_t n1 = 0, n2 = 0;
            unsigned long long last = globaltimer();
            while (ok && n2 < T) {
                bool progressed = false;
                if (n2 < n1 && mbar_test(&rfull[n2 % G::NRB], (n2 / G::NRB) & 1) &&
                    (n2 < 2 || mbar_test(&accfree[n2 & 1], ((n2 >> 1) - 1) & 1))) {
                    tc_fence_after();
                    uint32_t const ys = n2 % G::YST, rs = n2 % G::NRB, bp = n2 & 1;
                    uint64_t const dYT = dYT0 + ((ys * G::YSTAGE) >> 4);
                    uint64_t const dR = dR0 + ((rs * G::RSTAGE) >> 4);
                    uint32_t const dacc = tmem + bp * G::ACCW;
#pragma unroll
                    for (int ks = 0; ks < BR / 16; ks++) {
                        if (SPLIT2) {
                            // Acc[0:2KP] (+)= Rh [Y^T_hi; Y^T_lo];  Acc[0:KP] += Rl Y^T_hi
                            mma_bf16(dacc, dR + ks * 2, dYT + ks * 2, IDESC2W, ks > 0 ? 1u : 0u);
                            mma_bf16(dacc, dR + (G::RBYTES >> 4) + ks * 2, dYT + ks * 2, IDESC2, 1u);
                        } else {
                            mma_bf16(dacc, dR + ks * 2, dYT + ks * 2, IDESC2, ks > 0 ? 1u : 0u);
                        }
                    }
                    tc_commit(&accrdy[bp]);
                    tc_commit(&yempty[ys]);
                    tc_commit(&rempty[rs]);
                    n2++;
                    progressed = true;
                }
                if (n1 < T && n1 < n2 + G::NDB && mbar_test(&yfull[n1 % G::YST], (n1 / G::YST) & 1)) {
                    tc_fence_after();
                    uint32_t const s = n1 % G::YST, db = n1 % G::NDB;
                    uint64_t const dYh = dY0 + ((s * G::YSTAGE) >> 4);
                    uint64_t const dYl = dYh + (G::YBYTES >> 4);
                    uint32_t const dcol = tmem + G::DB0 + db * BR;
                    // D = Xl Yh^T + Xh Yl^T + Xh Yh^T (split arms; small terms first), K = KP in steps of 16.
#pragma unroll
                    for (int tt = 0; tt < NTERMS; tt++) {
                        int const term = NTERMS - 1 - tt;   // 2: Xl*Yh, 1: Xh*Yl, 0: Xh*Yh
                        uint64_t const xa = (term == 2) ? dXl : dXh;
                        uint64_t const yb = (term == 1) ? dYl : dYh;
#pragma unroll
                        for (int ks = 0; ks < KP / 16; ks++)
                            mma_bf16(dcol, xa + ks * 2, yb + ks * 2, IDESC1, (tt > 0 || ks > 0) ? 1u : 0u);
                    }
                    tc_commit(&dfull[db]);
                    n1++;
                    progressed = true;
                }
                if (progressed) {
                    last = globaltimer();
                } else if (*abort_flag) {
                    ok = false;
                } else if (globaltimer() - last > args.wait_ns) {
                    *abort_flag = 1;
                    atomicExch(args.err, 24u);
                    ok = false;
                } else {
                    __nanosleep(64);
                }
            }
            // drain: every MMA issued above has completed before the CTA frees
            // the shared and tensor memory it reads and writes
            mma_drain(mdrain);
        }
    } else if (warp >= 4 && warp < 4 + NR) {
        // ------------------------------------------------------------ R warps
        // Two teams of NR/2 warps take alternate tiles (team 0 even, team 1 odd), so
        // one team's load latency overlaps the other's arithmetic; a warp handles
        // TMEM lanes 32 quad .. +31 and CW tile columns in chunks of 16.
        constexpr int GPT = NR / 8;                     // column groups per team
        constexpr int CW = BR / GPT;                    // tile columns per warp
        static_assert(CW % 16 == 0, "16-column chunks");
        uint32_t const quad = warp & 3;
        uint32_t const jg = (warp - 4) >> 2;
        uint32_t const team = jg / GPT, grp = jg % GPT;
        uint32_t const row = quad * 32 + lane;          // TMEM lane = output row within the block
        uint32_t const lane_addr = tmem + ((quad * 32) << 16);
        for (uint32_t t = team; t < T; t += 2) {
            uint32_t const s = t % G::VST, b = t % G::NDB, rs = t % G::NRB;
            if (!mbar_wait(&dfull[b], (t / G::NDB) & 1, abort_flag, args.err, 25u, args.wait_ns)) break;
            if (!mbar_wait(&vfull[s], (t / G::VST) & 1, abort_flag, args.err, 26u, args.wait_ns)) break;
            if (t >= (uint32_t)G::NRB &&
                !mbar_wait(&rempty[rs], ((t / G::NRB) - 1) & 1, abort_flag, args.err, 27u, args.wait_ns))
                break;
            tc_fence_after();
            const unsigned char *sv = sV + s * G::VBYTES;
            bool const edge = (t_begin + t + 1) * BR > args.R;   // the partial last reduction tile
            int const valid = (int)(args.R - (t_begin + t) * BR);          // its columns before R
#pragma unroll 1
            for (int ch = 0; ch < CW / 16; ch++) {
                int const col0 = grp * CW + ch * 16;
                uint32_t d[32];
                float v[16];
                tmem_ld16(lane_addr + G::DB0 + b * BR + col0, d);
                if (HSIDE) {
                    // V tile [BR rows][128 cols], row-major; this thread's column = row.
                    const float *vs = reinterpret_cast<const float *>(sv) + col0 * BO + row;
#pragma unroll
                    for (int c = 0; c < 16; c++) v[c] = vs[c * BO];
                } else {
                    // V boxes of [128 rows][32 floats], 128B swizzle.
                    int const qb = col0 / 32;
                    int const c0 = (col0 % 32) / 4;
                    const unsigned char *vb = sv + qb * (BO * 128) + row * 128;
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        float4 const x = *reinterpret_cast<const float4 *>(vb + (((c + c0) ^ (row & 7)) << 4));
                        v[4 * c + 0] = x.x;
                        v[4 * c + 1] = x.y;
                        v[4 * c + 2] = x.z;
                        v[4 * c + 3] = x.w;
                    }
                }
                if (ch == CW / 16 - 1) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&vempty[s]);
                }
                tmem_wait_ld_dep(d);
                if (edge) {
                    // Columns past R are zero-filled (V = 0, WH = 0): WH = 1 there makes R 0
                    // instead of 0 * inf, which the second contraction would carry into every row.
#pragma unroll
                    for (int c = 0; c < 16; c++)
                        if (col0 + c >= valid) {
                            d[c] = 0x3f800000u;
                            v[c] = 0.0f;
                        }
                }
                uint32_t pk[8], pl[8];
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    // R = V * (1/WH); a zero WH of the data behaves as in the reference's division.
                    float const r0 = v[c] * rcp_approx(__uint_as_float(d[c]));
                    float const r1 = v[c + 1] * rcp_approx(__uint_as_float(d[c + 1]));
                    pk[c / 2] = pack_bf16x2(r0, r1);
                    if (SPLIT2) {
                        float const h0 = __uint_as_float(pk[c / 2] << 16), h1 = __uint_as_float(pk[c / 2] & 0xffff0000u);
                        pl[c / 2] = pack_bf16x2(r0 - h0, r1 - h1);
                    }
                }
                // R row `row`, columns col0 .. +16: 16-byte chunks of a 128-byte K-major row, 128B swizzle.
                unsigned char *rrow = sR + rs * G::RSTAGE + row * 128;
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    uint32_t const off = ((col0 / 8 + q) ^ (row & 7)) << 4;
                    *reinterpret_cast<uint4 *>(rrow + off) = make_uint4(pk[4 * q + 0], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
                    if (SPLIT2)
                        *reinterpret_cast<uint4 *>(rrow + G::RBYTES + off) =
                            make_uint4(pl[4 * q + 0], pl[4 * q + 1], pl[4 * q + 2], pl[4 * q + 3]);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&rfull[rs]);
        }
    } else if (warp >= 4 + NR) {
        // ------------------------------------------------------------ accumulator warps
        uint32_t const quad = warp & 3;
        uint32_t const row = quad * 32 + lane;
        uint32_t const lane_addr = tmem + ((quad * 32) << 16);
        float sum[KP];
#pragma unroll
        for (int c = 0; c < KP; c++) sum[c] = 0.0f;
        bool ok = true;
        for (uint32_t t = 0; ok && t < T; t++) {
            uint32_t const bp = t & 1;
            if (!mbar_wait(&accrdy[bp], (t >> 1) & 1, abort_flag, args.err, 28u, args.wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int part = 0; part < (SPLIT2 ? 2 : 1); part++) {
#pragma unroll
                for (int c0 = 0; c0 < KP; c0 += 16) {
                    uint32_t a[32];
                    tmem_ld16(lane_addr + bp * G::ACCW + part * KP + c0, a);
                    tmem_wait_ld_dep(a);
#pragma unroll
                    for (int c = 0; c < 16; c++) sum[c0 + c] += __uint_as_float(a[c]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&accfree[bp]);
        }
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
    if (T == 0 && warp >= 4 + NR) {
        uint32_t const o = o0 + (warp & 3) * 32 + lane;
        if (o < args.O) {
            float *dst = args.part + ((size_t)split * args.O + o) * KP;
            for (int c = 0; c < KP; c++) dst[c] = 0.0f;
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
PFN_cuTensorMapEncodeTiled_v12000 encode_fn_b()
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

int encode_map(nmfb_ctx *ctx, CUtensorMap *map, CUtensorMapDataType dt, const void *base, uint64_t inner,
               uint64_t outer, uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle sw)
{
    auto fn = encode_fn_b();
    if (!fn) return nmfb_fail(ctx, NMFB_ENODEV, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(map, dt, 2, (void *)base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nmfb_fail(ctx, NMFB_ECUDA, "cuTensorMapEncodeTiled (bf16 arm) failed (%d)", (int)r);
    return NMFB_OK;
}

struct PlanB {
    MapsB mapsH, mapsW;
    __nv_bfloat16 *wsplit, *hsplit;   // hi | lo | transposed hi/lo blocks, for W and for H
    uint32_t *dErr;                   // shared with the FP32 arm's error word
    int arm;                          // arm the Y^T maps were encoded for
    double *dCs;                      // k_finish's column-sum partials (row blocks, then chunks)
    uint32_t *dTick;                  // k_finish's retirement counters
    uint32_t nticks, csoff;
};

template <int KP, int MODE>
int set_attrs_mode(nmfb_ctx *ctx)
{
    int const smem = GeoB<KP, MODE>::SMEM;
    NMFB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_fused_bf16<true, KP, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    NMFB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_fused_bf16<false, KP, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return NMFB_OK;
}

template <int KP>
int set_attrs_b(nmfb_ctx *ctx)
{
    int rc = set_attrs_mode<KP, 0>(ctx);
    if (!rc) rc = set_attrs_mode<KP, 1>(ctx);
    if (!rc) rc = set_attrs_mode<KP, 2>(ctx);
    return rc;
}

template <bool HSIDE, int KP, int MODE>
int launch_b(nmfb_ctx *ctx, const MapsB &maps, uint32_t *err)
{
    using G = GeoB<KP, MODE>;
    constexpr int BR = G::BR;
    uint32_t const O = HSIDE ? ctx->m : ctx->n;
    uint32_t const R = HSIDE ? ctx->n : ctx->m;
    uint32_t const oblocks = (O + BO - 1) / BO;
    uint32_t const T = (R + BR - 1) / BR;
    // Same wave model as the FP32 arm: minimise waves x (tiles per split + fill).
    uint32_t tps = T, best = 0xffffffffu;
    for (uint32_t want = 1; want <= NMFB_MAX_SPLIT && want <= T; want++) {
        uint32_t const t_ps = (T + want - 1) / want;
        uint32_t const ns = (T + t_ps - 1) / t_ps;
        if ((size_t)ns * O * KP > ctx->part_items) break;
        uint32_t const waves = (oblocks * ns + (uint32_t)ctx->sm_count - 1) / (uint32_t)ctx->sm_count;
        uint32_t const cost = waves * (t_ps + 3);
        if (cost < best) {
            best = cost;
            tps = t_ps;
        }
    }
    uint32_t const nsplit = (T + tps - 1) / tps;
    if ((size_t)nsplit * O * KP > ctx->part_items)
        return nmfb_fail(ctx, NMFB_EINVAL, "bf16 arm: partial buffer too small (%u splits)", nsplit);
    ArgsB args;
    args.O = O;
    args.R = R;
    args.tiles_per_split = tps;
    args.nsplit = nsplit;
    args.part = ctx->dPart;
    args.err = err;
    args.st = ctx->dState;
    args.wait_ns = ctx->wait_ns ? ctx->wait_ns : WAIT_LIMIT_NS;
    int const main = HSIDE ? 0 : 1;
    int rc = nmfb_prof_begin(ctx, main);
    if (rc) return rc;
    k_fused_bf16<HSIDE, KP, MODE><<<oblocks * nsplit, G::NTHR, G::SMEM, ctx->stream>>>(maps, args);
    NMFB_LAUNCH_CHECK(ctx);
    if ((rc = nmfb_prof_end(ctx, main))) return rc;
    return (int)nsplit;
}

template <bool HSIDE, int KP>
int dispatch_kp(nmfb_ctx *ctx, const MapsB &maps, uint32_t *err)
{
    switch (ctx->arm) {
    case NMFB_ARM_BF16: return launch_b<HSIDE, KP, 0>(ctx, maps, err);
    case NMFB_ARM_SPLIT_BF16: return launch_b<HSIDE, KP, 1>(ctx, maps, err);
    default: return launch_b<HSIDE, KP, 2>(ctx, maps, err);
    }
}

template <bool HSIDE>
int dispatch_b(nmfb_ctx *ctx, const MapsB &maps, uint32_t *err)
{
    switch (ctx->kp) {
    case 16: return dispatch_kp<HSIDE, 16>(ctx, maps, err);
    case 32: return dispatch_kp<HSIDE, 32>(ctx, maps, err);
    case 64: return dispatch_kp<HSIDE, 64>(ctx, maps, err);
    default: return nmfb_fail(ctx, NMFB_EINVAL, "bf16 arms: unsupported padded rank %u", ctx->kp);
    }
}

int split_factor(nmfb_ctx *ctx, const float *F, uint32_t rows, __nv_bfloat16 *dst, bool with_t)
{
    size_t const part = (size_t)rows * ctx->kp;
    k_split_bf16<<<(rows + 63) / 64, 256, 0, ctx->stream>>>(F, rows, ctx->kp, dst, dst + part,
                                                            with_t ? dst + 2 * part : nullptr, ctx->dState);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

int encode_maps_b(nmfb_ctx *ctx, PlanB *plan)
{
    uint32_t const kp = ctx->kp;
    size_t const wsz = (size_t)ctx->n * kp, hsz = (size_t)ctx->m * kp;
    uint64_t const wblk = (ctx->n + 63) / 64, hblk = (ctx->m + 63) / 64;
    uint32_t const ytrows = (ctx->arm == NMFB_ARM_BF16X3 ? 2 : 1) * kp;
    CUtensorMapSwizzle const fsw = (kp == 16) ? CU_TENSOR_MAP_SWIZZLE_32B
                                 : (kp == 32) ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    CUtensorMapDataType const BF = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    uint64_t const vrow = ctx->ldv * sizeof(float), frow = (uint64_t)kp * 2;
    int rc;
    // update_H: X = H (rows m), Y = W (rows n)
    MapsB &mh = plan->mapsH;
    if ((rc = encode_map(ctx, &mh.v, F32, ctx->dV, ctx->m, ctx->n, vrow, BO, 64, CU_TENSOR_MAP_SWIZZLE_NONE))) return rc;
    if ((rc = encode_map(ctx, &mh.xh, BF, plan->hsplit, kp, ctx->m, frow, kp, BO, fsw))) return rc;
    if ((rc = encode_map(ctx, &mh.xl, BF, plan->hsplit + hsz, kp, ctx->m, frow, kp, BO, fsw))) return rc;
    if ((rc = encode_map(ctx, &mh.yh, BF, plan->wsplit, kp, ctx->n, frow, kp, 64, fsw))) return rc;
    if ((rc = encode_map(ctx, &mh.yl, BF, plan->wsplit + wsz, kp, ctx->n, frow, kp, 64, fsw))) return rc;
    if ((rc = encode_map(ctx, &mh.yt, BF, plan->wsplit + 2 * wsz, 64, wblk * 2 * kp, 128, 64, ytrows,
                         CU_TENSOR_MAP_SWIZZLE_128B)))
        return rc;
    // update_W: X = W (rows n), Y = H (rows m)
    MapsB &mw = plan->mapsW;
    if ((rc = encode_map(ctx, &mw.v, F32, ctx->dV, ctx->m, ctx->n, vrow, 32, BO, CU_TENSOR_MAP_SWIZZLE_128B))) return rc;
    if ((rc = encode_map(ctx, &mw.xh, BF, plan->wsplit, kp, ctx->n, frow, kp, BO, fsw))) return rc;
    if ((rc = encode_map(ctx, &mw.xl, BF, plan->wsplit + wsz, kp, ctx->n, frow, kp, BO, fsw))) return rc;
    if ((rc = encode_map(ctx, &mw.yh, BF, plan->hsplit, kp, ctx->m, frow, kp, 64, fsw))) return rc;
    if ((rc = encode_map(ctx, &mw.yl, BF, plan->hsplit + hsz, kp, ctx->m, frow, kp, 64, fsw))) return rc;
    if ((rc = encode_map(ctx, &mw.yt, BF, plan->hsplit + 2 * hsz, 64, hblk * 2 * kp, 128, 64, ytrows,
                         CU_TENSOR_MAP_SWIZZLE_128B)))
        return rc;
    plan->arm = ctx->arm;
    return NMFB_OK;
}

// A factor's BF16 copies (hi, lo, transposed blocks) and column sums, when the
// previous half-iteration's k_finish did not produce them.
int prepare_b(nmfb_ctx *ctx, bool w)
{
    PlanB *plan = (PlanB *)ctx->bplan;
    const float *F = w ? ctx->dW : ctx->dH;
    uint32_t const rows = w ? ctx->n : ctx->m;
    int rc = nmfb_colsum(ctx, F, rows, w ? ctx->dAccW : ctx->dAccH, w ? 0 : 1);
    if (!rc) rc = split_factor(ctx, F, rows, w ? plan->wsplit : plan->hsplit, true);
    if (!rc) ctx->fz_ok[w ? 0 : 1] = 1;
    return rc;
}

template <int KP>
int launch_finish_b(nmfb_ctx *ctx, bool is_H, uint32_t nsplit, int adjust)
{
    PlanB *plan = (PlanB *)ctx->bplan;
    uint32_t const O = is_H ? ctx->m : ctx->n;
    uint32_t const fblocks = fin_blocks(O, fin_rpt(nsplit));
    if (fblocks > plan->csoff || (fblocks + FIN_ECH - 1) / FIN_ECH + 1 > plan->nticks)
        return nmfb_fail(ctx, NMFB_EINVAL, "bf16 arms: column-sum buffers too small");
    __nv_bfloat16 *xs = is_H ? plan->hsplit : plan->wsplit;
    size_t const sz = (size_t)O * KP;
    FinishArgs fa = {};
    fa.O = O;
    fa.nsplit = nsplit;
    fa.k = ctx->k;
    fa.adjust = adjust;
    fa.part = ctx->dPart;
    fa.X = is_H ? ctx->dH : ctx->dW;
    fa.accY = is_H ? ctx->dAccW : ctx->dAccH;
    fa.bhi = xs;
    fa.blo = xs + sz;
    fa.bT = xs + 2 * sz;
    fa.bnblk64 = (O + 63) / 64;
    fa.cs = plan->dCs;
    fa.csoff = plan->csoff;
    fa.accX = is_H ? ctx->dAccH : ctx->dAccW;
    fa.tick = plan->dTick;
    fa.st = ctx->dState;
    fin_launch<KP, 64, 1>(fa, ctx->stream);
    NMFB_LAUNCH_CHECK(ctx);
    return NMFB_OK;
}

// One half-iteration: the fused BF16 kernel and k_finish (which writes X's BF16
// copies and column sums for the next half-iteration); the copies of X and Y
// are prepared first only when they are not current.
int bf16_half(nmfb_ctx *ctx, bool is_H, int adjust)
{
    PlanB *plan = (PlanB *)ctx->bplan;
    if (!plan) return nmfb_fail(ctx, NMFB_ESTATE, "bf16 arm not prepared");
    int rc;
    if (plan->arm != ctx->arm && (rc = encode_maps_b(ctx, plan))) return rc;
    int const whole = is_H ? 2 : 3;
    if ((rc = nmfb_prof_begin(ctx, whole))) return rc;
    if (!ctx->fz_ok[is_H ? 0 : 1] && (rc = prepare_b(ctx, is_H))) return rc;    // Y
    if (!ctx->fz_ok[is_H ? 1 : 0] && (rc = prepare_b(ctx, !is_H))) return rc;   // X
    int const nsplit = is_H ? dispatch_b<true>(ctx, plan->mapsH, plan->dErr) : dispatch_b<false>(ctx, plan->mapsW, plan->dErr);
    if (nsplit < 0) return nsplit;
    switch (ctx->kp) {
    case 16: rc = launch_finish_b<16>(ctx, is_H, (uint32_t)nsplit, adjust); break;
    case 32: rc = launch_finish_b<32>(ctx, is_H, (uint32_t)nsplit, adjust); break;
    default: rc = launch_finish_b<64>(ctx, is_H, (uint32_t)nsplit, adjust); break;
    }
    if (rc) return rc;
    ctx->fz_ok[is_H ? 1 : 0] = 1;
    return nmfb_prof_end(ctx, whole);
}

}  // namespace

int nmfb_bf16_prepare(nmfb_ctx *ctx)
{
    if (ctx->bplan) return NMFB_OK;
    uint32_t const kp = ctx->kp;
    if (kp != 16 && kp != 32 && kp != 64)
        return nmfb_fail(ctx, NMFB_EINVAL, "the bf16 arms support ranks up to 64 (k=%u)", ctx->k);
    int rc = (kp == 16) ? set_attrs_b<16>(ctx) : (kp == 32) ? set_attrs_b<32>(ctx) : set_attrs_b<64>(ctx);
    if (rc) return rc;
    PlanB *plan = (PlanB *)calloc(1, sizeof(PlanB));
    if (!plan) return nmfb_fail(ctx, NMFB_ENOMEM, "bf16 plan");
    ctx->bplan = plan;
    plan->arm = -1;
    plan->dErr = nmfb_fused_err_word(ctx);
    if (!plan->dErr) return nmfb_fail(ctx, NMFB_ESTATE, "bf16 arm needs the fused error word");
    // per factor: hi (rows x kp) | lo (rows x kp) | transposed hi and lo blocks (ceil(rows/64) x 2 kp x 64)
    size_t const wsz = (size_t)ctx->n * kp, hsz = (size_t)ctx->m * kp;
    size_t const wt = (size_t)((ctx->n + 63) / 64) * 128 * kp, ht = (size_t)((ctx->m + 63) / 64) * 128 * kp;
    cudaError_t e = nmfb_malloc(ctx, (void **)&plan->wsplit, (2 * wsz + wt) * sizeof(__nv_bfloat16));
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&plan->hsplit, (2 * hsz + ht) * sizeof(__nv_bfloat16));
    uint32_t const maxblk = fin_blocks(ctx->n > ctx->m ? ctx->n : ctx->m, 1);   // k_finish's most row blocks
    plan->csoff = maxblk;
    plan->nticks = (maxblk + FIN_ECH - 1) / FIN_ECH + 1;
    if (e == cudaSuccess)
        e = nmfb_malloc(ctx, (void **)&plan->dCs, (size_t)(maxblk + (maxblk + FIN_ECH - 1) / FIN_ECH) * kp * sizeof(double));
    if (e == cudaSuccess) e = nmfb_malloc(ctx, (void **)&plan->dTick, plan->nticks * sizeof(uint32_t));
    if (e != cudaSuccess) return nmfb_fail(ctx, NMFB_ENOMEM, "bf16 split buffers: %s", cudaGetErrorString(e));
    NMFB_CUDA_TRY(ctx, cudaMemsetAsync(plan->dTick, 0, plan->nticks * sizeof(uint32_t), ctx->own_stream));
    return NMFB_OK;
}

int nmfb_bf16_release(nmfb_ctx *ctx)
{
    PlanB *plan = (PlanB *)ctx->bplan;
    if (!plan) return NMFB_OK;
    if (plan->wsplit) nmfb_free(ctx, plan->wsplit);
    if (plan->hsplit) nmfb_free(ctx, plan->hsplit);
    if (plan->dCs) nmfb_free(ctx, plan->dCs);
    if (plan->dTick) nmfb_free(ctx, plan->dTick);
    free(plan);
    ctx->bplan = nullptr;
    return NMFB_OK;
}

int nmfb_bf16_update_H(nmfb_ctx *ctx, int adjust) { return bf16_half(ctx, true, adjust); }
int nmfb_bf16_update_W(nmfb_ctx *ctx, int adjust) { return bf16_half(ctx, false, adjust); }

// Makes W's BF16 copies and column sums current (before a test block is
// replayed as a graph).
int nmfb_bf16_ready_W(nmfb_ctx *ctx)
{
    if (!ctx->bplan || ctx->fz_ok[0]) return NMFB_OK;
    return prepare_b(ctx, true);
}
