// rowpass_mma.cuh -- the fused Golub-Kahan pass over a staged fp16 plane
// with both products on the tensor cores (mma.sync m16n8k16, fp16 inputs,
// FP32 accumulation).
//
// Per row i of A (as rowpass.cuh):
//     ut_i = cp (A p)_i + cu u_i            written to u_out
//     q   += ut_i A[i, :]                   per-CTA partial of A^T ut
//     ss  += ut_i^2                         per-CTA partial, FP64
//
// The CUDA-core pass converts every element and spends per-row
// instructions on shuffles and the FP64 ut; at 2 bytes an element that
// kept it issue-bound near two thirds of HBM bandwidth.  Here a stage is
// 32 rows (two m16 tiles: the per-stage barrier round trips between the
// MMA warps and the ut warp are paid once per 32 rows, and every lane of
// the ut warp has a row) and both products are tensor-core tiles read
// straight from the staged rows with ldmatrix, so an element costs no
// instruction of its own:
//
//   product 1   D1[32 rows x 8] = A_stage[32 x 16k] . B1[16k x 8]
//               B1's columns 0 and 1 are p_hi and p_lo:
//               p * 2^sp = p_hi + p_lo * 2^-11 (fp16 each), 2^sp putting
//               max|p| near 2^14 -- 22 significant bits of p, exact
//               products, FP32 sums
//   ut          32 lanes of the ut warp: dot_i = (sum over warps of D1[i][0] +
//               D1[i][1] 2^-11) 2^-sp in FP64, ut_i as rowpass.cuh
//   product 2   D2[16 cols x 8] += A_stage^T[16 x 32 rows] . B2[32 x 8]
//               (ldmatrix.trans), B2's columns ut_hi and ut_lo split the
//               same way against a running CTA exponent E: a stage whose
//               max|ut| raises E first rescales every D2 by the power of
//               two it moved (exact), so q = (D2[.][0] + D2[.][1] 2^-11)
//               2^(E-14) at the end
//
// Warp w of the 12 MMA warps owns k-tiles (16 columns each) w*TPW ..
// w*TPW+TPW-1 for both products, so its D2 tiles are whole columns of the
// CTA's A^T ut partial and no cross-warp reduction of q is needed.  A 13th
// warp computes ut, and the stages are software-pipelined around it:
//
//   MMA warps, step t:  product 1 of stage t -> partials[t&1],
//                       arrive A[t&1]; wait B[(t-1)&1];
//                       product 2 of stage t-1, release stage t-1
//   ut warp, step t:    wait A[t&1]; ut of stage t -> B2[t&1]; arrive B[t&1]
//
// (named barriers with arrive / sync halves), so the ut of one stage runs
// beside the products of its neighbours.  The producer warp and the stage
// ring are as in rowpass.cuh;
// the ring is zeroed before the first copy.  The rows past the CTA's range
// in its last stage hold stale values and are masked in the product-2
// fragments (an infinity there would meet a zero ut).  The columns past n
// that the last 16-wide tile of product 1 reads are the next row's first
// values and meet zeros of p: only an infinite HALF-tier value there (an
// element beyond the fp16 range, which makes the HALF-tier operator itself
// non-finite) could turn the product into a NaN, so they are not masked
// (masking cost 5% of the pass).  Every mbarrier wait is bounded.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "fused.cuh"
#include "mbarrier.cuh"

namespace tomos_b200 {

constexpr int kMmaWarps = 12;  // MMA warps; warp 12 computes ut, warp 13 copies
constexpr int kMmaUtWarp = kMmaWarps;
constexpr int kMmaProducer = kMmaWarps + 1;
constexpr int kMmaThreads = (kMmaWarps + 2) * 32;
constexpr int kMmaRows = 32;   // rows per stage at most: two m16 tiles (k = 32 for product 2)
constexpr int kMmaMaxStages = 12;
constexpr size_t kMmaSmemBudget = 200 * 1024;  // the tensor-core pass's stage ring
constexpr int kMmaMaxTpw = 11; // k-tiles per warp: n <= 12 * 11 * 16 = 2112

struct MmaPassParams {
    FusedParams f;
    int* err;       // set nonzero on a pipeline timeout
    int nstage;
    int cb;         // bytes copied per row (16-byte multiple)
    int pitch;      // shared-memory bytes between rows (cb, or cb + 16)
};

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t (&r)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

// D += A B for one m16n8k16 tile (fp16 or, BF, bf16 inputs; FP32
// accumulators).
template <bool BF>
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
    if constexpr (BF) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
            "{%8, %9}, {%0, %1, %2, %3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    } else {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
            "{%8, %9}, {%0, %1, %2, %3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
}

// x = hi + mid + lo exactly with bf16 parts (8 significant bits each;
// bf16 has the FP32 exponent range, so no scaling).  Returns part k.
__device__ __forceinline__ uint16_t split_bf16_part(float x, int k) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(hi);
    const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
    const __nv_bfloat16 lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
    return __bfloat16_as_ushort(k == 0 ? hi : (k == 1 ? mid : lo));
}

__device__ __forceinline__ void named_bar_arrive(int id, int count) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ uint32_t pack_half2(__half lo, __half hi) {
    return (uint32_t)__half_as_ushort(lo) | ((uint32_t)__half_as_ushort(hi) << 16);
}

// x * 2^s = hi + lo * 2^-11 with hi, lo fp16 (x * 2^s within fp16 range).
__device__ __forceinline__ void split_half(float x, int s, __half& hi, __half& lo) {
    const float v = ldexpf(x, s);
    hi = __float2half_rn(v);
    lo = __float2half_rn((v - __half2float(hi)) * 2048.0f);
}

// Zeroes the fp16 halves of a fragment register whose index (column of
// product 1, row of product 2) is not below `lim`.
__device__ __forceinline__ uint32_t mask_pair(uint32_t v, int i0, int lim) {
    return v & ((i0 < lim ? 0x0000FFFFu : 0u) | (i0 + 1 < lim ? 0xFFFF0000u : 0u));
}

// BF: the A plane is bf16 (an FP32_BF16 wh plane read in place) and p, ut
// enter as three exact bf16 parts (columns 0-2 of B1 / B2) instead of the
// scaled fp16 pair; the running exponent is not needed.
// ROWS: rows per stage, 32 (two m16 tiles) where two such stages fit the
// ring, else 16.
template <int TPW, bool BF, int ROWS>
__global__ void __launch_bounds__(kMmaThreads, 1) fused_rows_mma_kernel(MmaPassParams T) {
    const FusedParams& P = T.f;
    if (P.skip && *P.skip) return;

    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kMmaMaxStages];
    __shared__ __align__(8) uint64_t empty[kMmaMaxStages];
    __shared__ float2 red[2][kMmaWarps][kMmaRows];    // partial dots (hi, lo) per warp
    __shared__ float red3[2][kMmaWarps][kMmaRows];    // BF: the third part's partial dots
    __shared__ __align__(4) uint16_t ub[2][3][kMmaRows];  // B2: the parts of ut of a stage
    __shared__ int e_move[2];                         // the running exponent's last move
    __shared__ int e_final;                           // the running exponent at the end
    __shared__ float pmax_w[kMmaWarps + 2];
    __shared__ double ssw;
    __shared__ int abort_flag;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nstage = T.nstage;
    const int cb = T.cb;
    const int pitch = T.pitch;
    const size_t stage_bytes = (size_t)ROWS * pitch;
    const int64_t n = P.n;
    const int ktiles = (int)((n + 15) / 16);
    constexpr int kBar = (kMmaWarps + 1) * 32;  // MMA warps + the ut warp

    const int64_t rows_per_cta = (P.m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    int64_t r1 = r0 + rows_per_cta;
    if (r1 > P.m) r1 = P.m;
    const int64_t nrows = r1 > r0 ? r1 - r0 : 0;
    const int ntiles = (int)((nrows + ROWS - 1) / ROWS);

    // Zero the ring and its 64-byte tail (read by the last row's last
    // tile) and find max|p|.
    {
        uint4* z = reinterpret_cast<uint4*>(smem);
        const size_t nz = (nstage * stage_bytes + 64) / 16;
        for (size_t i = threadIdx.x; i < nz; i += kMmaThreads) z[i] = make_uint4(0, 0, 0, 0);
        float pm = 0.0f;
        for (int64_t j = threadIdx.x; j < n; j += kMmaThreads) pm = fmaxf(pm, fabsf(__ldg(P.p + j)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pm = fmaxf(pm, __shfl_xor_sync(0xffffffffu, pm, o));
        if (lane == 0) pmax_w[warp] = pm;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kMmaWarps);
        }
        abort_flag = 0;
        ssw = 0.0;
        fence_barrier_init();
    }
    __syncthreads();
    float pmax = 0.0f;
#pragma unroll
    for (int w = 0; w < kMmaWarps + 2; ++w) pmax = fmaxf(pmax, pmax_w[w]);
    // 2^sp brings max|p| to [2^13, 2^14) (fp16 only)
    const int sp = (!BF && pmax > 0.0f) ? 13 - ilogbf(pmax) : 0;

    if (warp == kMmaProducer) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            const bool contiguous = pitch == cb && (int64_t)P.ld * 2 == cb;
            int issued = 0;
            int s = 0;
            uint32_t ph = 0;
            for (int t = 0; t < ntiles; ++t) {
                if (!mbar_wait(&empty[s], ph ^ 1u)) {
                    atomicExch(T.err, 1);
                    break;
                }
                if (*(volatile int*)&abort_flag) break;
                const int64_t i0 = r0 + (int64_t)t * ROWS;
                const int rows = (int)((r1 - i0) < ROWS ? (r1 - i0) : ROWS);
                uint8_t* st = smem + (size_t)s * stage_bytes;
                mbar_expect_tx(&full[s], (uint32_t)(rows * cb));
                if (contiguous) {
                    bulk_g2s(st, static_cast<const uint8_t*>(P.hi) + (size_t)i0 * P.ld * 2,
                             (uint32_t)(rows * cb), &full[s]);
                } else {
                    for (int r = 0; r < rows; ++r)
                        bulk_g2s(st + (size_t)r * pitch,
                                 static_cast<const uint8_t*>(P.hi) + (size_t)(i0 + r) * P.ld * 2,
                                 (uint32_t)cb, &full[s]);
                }
                issued = t + 1;
                if (++s == nstage) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            // Drain: every issued stage must land before the CTA may exit.
            for (int t = (issued > nstage ? issued - nstage : 0); t < issued; ++t) {
                if (!mbar_wait(&full[t % nstage], (uint32_t)(t / nstage) & 1u)) {
                    atomicExch(T.err, 2);
                    break;
                }
            }
        }
    } else if (warp == kMmaUtWarp) {
        // ------------------------------------------------------------- ut
        const double cp = P.coef[0];
        const double cu = P.coef[1];
        double ss = 0.0;
        int e_cur = -1000;  // running exponent: |ut| < 2^e_cur so far
        float unext = (lane < ROWS && r0 + lane < r1) ? __ldg(P.u_in + r0 + lane) : 0.0f;  // a row a lane
        for (int t = 0; t < ntiles; ++t) {
            const int b = t & 1;
            const int64_t i = r0 + (int64_t)t * ROWS + lane;
            const bool has = lane < ROWS && i < r1;
            const float ucur = unext;
            const int64_t inx = i + ROWS;
            unext = (lane < ROWS && inx < r1) ? __ldg(P.u_in + inx) : 0.0f;
            named_bar_sync(1 + b, kBar);  // partials of stage t are in
            float ut = 0.0f;
            if (has) {
                double hs = 0.0, ls = 0.0, ts = 0.0;
#pragma unroll
                for (int w = 0; w < kMmaWarps; ++w) {
                    const float2 v = red[b][w][lane];
                    hs += (double)v.x;
                    ls += (double)v.y;
                    if (BF) ts += (double)red3[b][w][lane];
                }
                const double dot = BF ? hs + ls + ts : ldexp(hs + ls * (1.0 / 2048.0), -sp);
                ut = (float)(cp * dot + cu * (double)ucur);
                P.u_out[i] = ut;
                ss += (double)ut * (double)ut;
            }
            int e_new = e_cur;
            if constexpr (BF) {
#pragma unroll
                for (int k = 0; k < 3; ++k) ub[b][k][lane] = split_bf16_part(ut, k);
                e_new = 14;  // no scaling: q = the sum of D2's columns
                e_cur = 14;
            } else {
                float m = fabsf(ut);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                e_new = m > 0.0f ? max(e_cur, ilogbf(m) + 1) : e_cur;
                {
                    __half hi = __float2half_rn(0.0f), lo = hi;
                    if (e_new > -1000) split_half(ut, 14 - e_new, hi, lo);
                    ub[b][0][lane] = __half_as_ushort(hi);
                    ub[b][1][lane] = __half_as_ushort(lo);
                }
            }
            if (lane == 0) e_move[b] = e_new - e_cur;
            e_cur = e_new;
            named_bar_arrive(3 + b, kBar);  // B2 of stage t is out
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        if (lane == 0) {
            ssw = ss;
            e_final = e_cur;
        }
        named_bar_arrive(5, kBar);
    } else {
        // ------------------------------------------------------------ MMA
        const int g = lane >> 2, tq = lane & 3;
        // B1 fragments of this warp's k-tiles: lanes 0-3 carry p_hi, lanes
        // 4-7 p_lo (BF: lanes 8-11 the third part), the rest zero.
        constexpr int NPART = BF ? 3 : 2;
        uint32_t b1[TPW][2];
#pragma unroll
        for (int tt = 0; tt < TPW; ++tt) {
            const int kt = warp * TPW + tt;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t v = 0;
                if (g < NPART && kt < ktiles) {
                    uint16_t e2[2];
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int64_t col = (int64_t)kt * 16 + 8 * h + 2 * tq + q;
                        const float x = col < n ? __ldg(P.p + col) : 0.0f;
                        if constexpr (BF) {
                            e2[q] = split_bf16_part(x, g);
                        } else {
                            __half hi, lo;
                            split_half(x, sp, hi, lo);
                            e2[q] = __half_as_ushort(g == 0 ? hi : lo);
                        }
                    }
                    v = (uint32_t)e2[0] | ((uint32_t)e2[1] << 16);
                }
                b1[tt][h] = v;
            }
        }
        float d2[TPW][4];
#pragma unroll
        for (int tt = 0; tt < TPW; ++tt) d2[tt][0] = d2[tt][1] = d2[tt][2] = d2[tt][3] = 0.0f;
        // ldmatrix row addresses (relative to a stage): product 1 blocks are
        // (rows 0-7 | 8-15) x (cols 0-7 | 8-15) in the order a0..a3, the
        // transposed product 2 blocks (rows 0-7 | 8-15 as k) likewise.
        const int mi = lane >> 3, mr = lane & 7;
        const uint32_t off1 = (uint32_t)((mr + 8 * (mi & 1)) * pitch + 16 * (mi >> 1));
        const uint32_t off2 = (uint32_t)((mr + 8 * (mi >> 1)) * pitch + 16 * (mi & 1));
        const uint32_t ring = smem_addr(smem);
        bool failed = false;
        int s = 0;
        uint32_t ph = 0;
        // product 2 of the stage before (its B2 from the ut warp), then
        // release that stage
        // valid rows of stage tp (16 but in the CTA's last stage)
        auto rows_of = [&](int tp) {
            const int64_t left = r1 - (r0 + (int64_t)tp * ROWS);
            return left < ROWS ? (int)left : ROWS;
        };
        auto product2 = [&](int tp, int sp_slot, int rv) {
            const int b = tp & 1;
            named_bar_sync(3 + b, kBar);
            const int de = e_move[b];
            if (de != 0) {
                const float f = de > 126 ? 0.0f : ldexpf(1.0f, -de);
#pragma unroll
                for (int tt = 0; tt < TPW; ++tt)
#pragma unroll
                    for (int q = 0; q < 4; ++q) d2[tt][q] *= f;
            }
            // B2 fragments of the two k16 steps (rows 0-15, 16-31)
            uint32_t bb0 = 0, bb1 = 0, bc0 = 0, bc1 = 0;
            if (g < NPART) {
                bb0 = *reinterpret_cast<const uint32_t*>(&ub[b][g][2 * tq]);
                bb1 = *reinterpret_cast<const uint32_t*>(&ub[b][g][2 * tq + 8]);
                bc0 = *reinterpret_cast<const uint32_t*>(&ub[b][g][16 + 2 * tq]);
                bc1 = *reinterpret_cast<const uint32_t*>(&ub[b][g][16 + 2 * tq + 8]);
            }
            const uint32_t st = ring + (uint32_t)(sp_slot * stage_bytes);
            const uint32_t st2 = st + (uint32_t)(16 * pitch);
            if (!failed && rv == ROWS) {
#pragma unroll
                for (int tt = 0; tt < TPW; ++tt) {
                    const int mt = warp * TPW + tt;
                    if (mt < ktiles) {
                        uint32_t a[4];
                        ldsm_x4_t(st + off2 + (uint32_t)(mt * 32), a);
                        mma16816<BF>(d2[tt], a, bb0, bb1);
                        if constexpr (ROWS == 32) {
                            uint32_t c[4];
                            ldsm_x4_t(st2 + off2 + (uint32_t)(mt * 32), c);
                            mma16816<BF>(d2[tt], c, bc0, bc1);
                        }
                    }
                }
            } else if (!failed) {
                const int rv2 = rv - 16;  // valid rows of the second k16 step
#pragma unroll
                for (int tt = 0; tt < TPW; ++tt) {
                    const int mt = warp * TPW + tt;
                    if (mt < ktiles) {
                        uint32_t a[4];
                        ldsm_x4_t(st + off2 + (uint32_t)(mt * 32), a);
                        // rows past the CTA's last row hold stale values (an
                        // infinity among them would meet a zero ut)
                        a[0] = mask_pair(a[0], 2 * tq, rv);
                        a[1] = mask_pair(a[1], 2 * tq, rv);
                        a[2] = mask_pair(a[2], 2 * tq + 8, rv);
                        a[3] = mask_pair(a[3], 2 * tq + 8, rv);
                        mma16816<BF>(d2[tt], a, bb0, bb1);
                        if (ROWS == 32 && rv2 > 0) {
                            ldsm_x4_t(st2 + off2 + (uint32_t)(mt * 32), a);
                            a[0] = mask_pair(a[0], 2 * tq, rv2);
                            a[1] = mask_pair(a[1], 2 * tq, rv2);
                            a[2] = mask_pair(a[2], 2 * tq + 8, rv2);
                            a[3] = mask_pair(a[3], 2 * tq + 8, rv2);
                            mma16816<BF>(d2[tt], a, bc0, bc1);
                        }
                    }
                }
            }
            // every read of the stage is done: it may be refilled
            __syncwarp();
            if (lane == 0 && !failed) mbar_arrive(&empty[sp_slot]);
        };
        int prev_slot = 0;
        for (int t = 0; t < ntiles; ++t) {
            if (!failed && !mbar_wait(&full[s], ph)) {
                atomicExch(T.err, 3);
                abort_flag = 1;
                failed = true;
            }
            const uint32_t st = ring + (uint32_t)(s * stage_bytes);
            // product 1: this warp's partial dots of the stage's 32 rows (two
            // m16 tiles; two accumulator sets each halve the dependent chain)
            float d1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, d1b[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            float d1c[4] = {0.0f, 0.0f, 0.0f, 0.0f}, d1d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (!failed) {
                const uint32_t st2 = st + (uint32_t)(16 * pitch);
#pragma unroll
                for (int tt = 0; tt < TPW; ++tt) {
                    const int kt = warp * TPW + tt;
                    if (kt < ktiles) {
                        uint32_t a[4];
                        ldsm_x4(st + off1 + (uint32_t)(kt * 32), a);
                        if (tt & 1)
                            mma16816<BF>(d1b, a, b1[tt][0], b1[tt][1]);
                        else
                            mma16816<BF>(d1, a, b1[tt][0], b1[tt][1]);
                        if constexpr (ROWS == 32) {
                            uint32_t c[4];
                            ldsm_x4(st2 + off1 + (uint32_t)(kt * 32), c);
                            if (tt & 1)
                                mma16816<BF>(d1d, c, b1[tt][0], b1[tt][1]);
                            else
                                mma16816<BF>(d1c, c, b1[tt][0], b1[tt][1]);
                        }
                    }
                }
            }
            if (tq == 0) {
                red[t & 1][warp][g] = make_float2(d1[0] + d1b[0], d1[1] + d1b[1]);
                red[t & 1][warp][g + 8] = make_float2(d1[2] + d1b[2], d1[3] + d1b[3]);
                if (ROWS == 32) {
                    red[t & 1][warp][g + 16] = make_float2(d1c[0] + d1d[0], d1c[1] + d1d[1]);
                    red[t & 1][warp][g + 24] = make_float2(d1c[2] + d1d[2], d1c[3] + d1d[3]);
                }
            }
            if (BF && tq == 1) {  // column 2: the third part
                red3[t & 1][warp][g] = d1[0] + d1b[0];
                red3[t & 1][warp][g + 8] = d1[2] + d1b[2];
                if (ROWS == 32) {
                    red3[t & 1][warp][g + 16] = d1c[0] + d1d[0];
                    red3[t & 1][warp][g + 24] = d1c[2] + d1d[2];
                }
            }
            named_bar_arrive(1 + (t & 1), kBar);
            if (t > 0) product2(t - 1, prev_slot, rows_of(t - 1));
            prev_slot = s;
            if (++s == nstage) {
                s = 0;
                ph ^= 1u;
            }
        }
        if (ntiles > 0) product2(ntiles - 1, prev_slot, rows_of(ntiles - 1));
        // q partial: column g (+8) of each tile from lanes with tq == 0,
        // scaled by the ut warp's final exponent
        named_bar_sync(5, kBar);
        const int e_fin = e_final;
        const float qs = e_fin > -1000 ? ldexpf(1.0f, e_fin - 14) : 0.0f;
        float* qout = P.qpart + (size_t)blockIdx.x * P.qstride;
#pragma unroll
        for (int tt = 0; tt < TPW; ++tt) {
            const int mt = warp * TPW + tt;
            // BF: column 2 (the third part) sits in the lane with tq == 1
            const float t0 = __shfl_down_sync(0xffffffffu, d2[tt][0], 1);
            const float t2 = __shfl_down_sync(0xffffffffu, d2[tt][2], 1);
            if (tq == 0 && mt < ktiles) {
                const int64_t c0 = (int64_t)mt * 16 + g;
                if constexpr (BF) {
                    if (c0 < n) qout[c0] = (d2[tt][0] + d2[tt][1]) + t0;
                    if (c0 + 8 < n) qout[c0 + 8] = (d2[tt][2] + d2[tt][3]) + t2;
                } else {
                    if (c0 < n) qout[c0] = (d2[tt][0] + d2[tt][1] * (1.0f / 2048.0f)) * qs;
                    if (c0 + 8 < n) qout[c0 + 8] = (d2[tt][2] + d2[tt][3] * (1.0f / 2048.0f)) * qs;
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) P.sspart[blockIdx.x] = ssw;
}

// Dynamic shared memory of one launch: the stage ring and its tail.
inline size_t fused_rows_mma_smem(int nstage, int rows, int pitch) {
    return (size_t)nstage * rows * pitch + 64;
}

}  // namespace tomos_b200
