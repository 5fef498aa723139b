// rowpass.cuh -- the fused Golub-Kahan pass over a row-major A, staged
// through shared memory by bulk asynchronous copies (cp.async.bulk).
//
// Per row i of A (same arithmetic as fused.cuh):
//     ut_i = cp (A p)_i + cu u_i            written to u_out
//     q   += ut_i A[i, :]                   per-CTA partial of A^T ut
//     ss  += ut_i^2                         per-CTA partial, FP64
// so the two products of an LSQR iteration cost one read of A.
//
// Roles (one CTA per SM, CW + 1 warps; CW = 12, or 8 for ACC64 over one
// plane):
//   producer (warp CW, lane 0)           consumers (warps 0..CW-1)
//   wait empty[s]                        wait full[s]
//   expect_tx(full[s], bytes)            copy its row part to registers,
//   cp.async.bulk per plane (one per       decode, arrive empty[s]
//   stage when rows are contiguous,
//   else one per row)
//                                        dot with p (packed FP32x2 FMAs),
//                                        shuffle reduce, ut,
//                                        q += ut * row (packed FMAs)
// A stage holds RS = CW / G rows.  G consumer warps share a row when n is
// wider than one warp's columns (1024, 512 for the two-plane ACC64
// passes; G divides CW); their partial dots meet in shared memory behind
// a named barrier per row.  Lane l of part g owns the 16-byte chunks
// g*32*NCH + k*32 + l (k < NCH) of its row, so p and the q accumulators
// live in registers and every shared-memory read is a conflict-free
// 16-byte access.
//
// FP32_16 wh words with the control bit set (values outside the fp16
// range) are rare; one OR over a chunk's words tests for them, and only a
// chunk that has one rewrites them to their fp32_16_half_only bits before
// the fp16 conversion.
//
// ACC64 (the exact tiers, restart residuals, backward errors) forms every
// product exactly and sums it in FP64, as the reference's accurate tier
// does: p is held in FP64 registers, so an element costs one conversion
// and one DFMA, and the dot runs as four independent FP64 chains.  Those
// registers are why a one-plane ACC64 CTA has 8 consumer warps (each warp
// still covers 1024 columns); the two-plane exact decodes keep 12 warps
// at 512 columns a warp.  HALF-tier and FP32 passes accumulate in FP32.
//
// Every mbarrier wait is bounded.  A consumer whose wait expires records
// the failure in *err and stops waiting (it still runs the remaining
// named barriers, so its row partners never block); the producer stops
// issuing and drains what it issued (bounded again).  The results of such
// a launch are garbage and the host reports the error.
#pragma once

#include <cuda_fp16.h>

#include "common.cuh"
#include "fused.cuh"
#include "mbarrier.cuh"

namespace tomos_b200 {

template <Elem E>
struct RowPlanes {
    static constexpr int value = (E == Elem::A16 || E == Elem::AB16 || E == Elem::AB16R) ? 2 : 1;
};

// What one launch of fused_rows_kernel computes.
enum RowMode : int {
    kRowBoth = 0,  // the LSQR pass: ut = cp A p + cu u, partials of A^T ut and ||ut||^2
    kRowDot = 1,   // ut = cp A p + cu u only (a product whose lines are dots)
    kRowAxpy = 2,  // partials of A^T (cu u) only (a product that sums lines)
    kRowBothRuns = 3,  // kRowBoth with ACC64: the row dots as FP32 products
                       // over runs of at most 8 (a lane's float2 chains),
                       // summed in FP64, instead of one FP64 product an
                       // element; the backward error of a dot is then at
                       // most gamma_8 = 4.8e-7 (gamma_4 for two-plane rows)
};

// Passes that hold an FP64 register per column of a lane: the LSQR pass
// with FP64 products (p in FP64) and the FP64-accumulating A^T product.
template <bool ACC64, int MODE>
struct RowF64Regs {
    static constexpr bool value = ACC64 && (MODE == kRowBoth || MODE == kRowAxpy);
};

// Consumer warps of a pass.  13 warps (with the producer) leave 128
// registers a thread, 17 warps 96; the passes with FP64 registers per
// column over one plane keep a whole row part per lane, and run 8
// consumers (9 warps: up to 168 registers) so that a warp still covers
// 1024 columns; over two planes they keep 16 warps (a warp covering 512
// columns) to hide the exact decode's latency.  The plain 16-bit planes,
// and FP32_16's wh plane in the standalone products, take 16 warps; the
// LSQR pass over a wh plane keeps 12 (at 96 registers it would spill).
template <Elem E, bool ACC64, int MODE>
struct RowWarps {
    static constexpr bool wide16 = E == Elem::F16 || E == Elem::B16 || (E == Elem::H16 && MODE != kRowBoth);
    static constexpr int value = !RowF64Regs<ACC64, MODE>::value ? (wide16 ? 16 : 12)
                                                                 : (RowPlanes<E>::value == 1 ? 8 : 16);
};
constexpr int kRowWarps = 16;  // the widest configuration (shared arrays)

// 16-byte chunks a lane takes per row part at most (a warp covers 32 x
// that x VEC columns).
template <Elem E, bool ACC64, int MODE>
struct RowNchMax {
    static constexpr int base = (E == Elem::F32) ? 8 : 4;
    static constexpr int value = (RowF64Regs<ACC64, MODE>::value && RowPlanes<E>::value == 2) ? base / 2 : base;
};
constexpr int kRowMaxStages = 12;
constexpr size_t kRowSmemBudget = 216 * 1024;
// Bytes a bulk copy of one plane of a stage aims at: each copy carries a
// fixed cost beside its bytes (measured about a microsecond a stage for
// 24-48 KB copies), so stages of one tile of short 16-bit rows would bound
// the pass below the memory rate.
constexpr size_t kRowCopyTarget = 48 * 1024;

struct RowPassParams {
    FusedParams f;
    int* err;        // set nonzero on a pipeline timeout
    int nstage;
    int copy_bytes;  // bytes copied per row and plane (16-byte multiple)
    int tiles_per_stage;  // row tiles (CW / G rows each) a stage holds
    double* qpart64; // kRowAxpy with ACC64: FP64 partials (gridDim.x x qstride)
};

// kRowAxpy with ACC64 sums FP32 products over this many rows of a warp,
// then adds them into FP64 accumulators.
constexpr int kRowPromote = 8;

__device__ __forceinline__ uint4 lds128(const uint8_t* p) {
    return *reinterpret_cast<const uint4*>(p);
}

// Decodes this lane's NCH chunks of one row part from shared memory into
// float pairs (the operands of the packed FMAs).  Chunks past the end of
// the row (live bit clear) are not read and decode to zeros.
template <Elem E, int NCH>
__device__ __forceinline__ void decode_row(const uint8_t* hrow, const uint8_t* lrow,
                                           const int* coff, uint32_t live,
                                           float2 (&a)[NCH * ChunkElems<E>::value / 2]) {
    constexpr int VEC = ChunkElems<E>::value;
    constexpr int HV = VEC / 2;
    if constexpr (E == Elem::A16) {
        // Control-0 words (all but ~0.35 % of the bench matrix) decode as
        // the fp16 conversion of wh plus mant_lo minus the round flag at
        // bit 14, both added to the converted bits (decode_pair_fp32_16):
        // five operations an element.  Words with a control bit are redone
        // by the exact decode, one word at a time and only where a lane of
        // the warp holds one.
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            const bool lv = (live >> k) & 1u;
            uint4 h = make_uint4(0, 0, 0, 0), r = make_uint4(0, 0, 0, 0);
            if (lv) {
                h = lds128(hrow + coff[k]);
                r = lds128(lrow + coff[k]);
            }
            float f[8];
            {
                const float2 p0 = decode_pair_fp32_16(h.x, r.x), p1 = decode_pair_fp32_16(h.y, r.y);
                const float2 p2 = decode_pair_fp32_16(h.z, r.z), p3 = decode_pair_fp32_16(h.w, r.w);
                f[0] = p0.x; f[1] = p0.y; f[2] = p1.x; f[3] = p1.y;
                f[4] = p2.x; f[5] = p2.y; f[6] = p3.x; f[7] = p3.y;
            }
            // one bit per element with a control bit (bits 0..3: low
            // halves of words x..w, bits 16..19: high halves); a loop, so
            // the rare fix is a branch and not predicated code every warp
            // runs
            uint32_t flags = (h.x & 0x00010001u) | ((h.y & 0x00010001u) << 1) |
                             ((h.z & 0x00010001u) << 2) | ((h.w & 0x00010001u) << 3);
            while (flags) {
                const int bit = __ffs(flags) - 1;
                flags &= flags - 1;
                const int wi = bit & 3, hi = bit >> 4;   // word, half
                const uint32_t ww = wi == 0 ? h.x : wi == 1 ? h.y : wi == 2 ? h.z : h.w;
                const uint32_t rw = wi == 0 ? r.x : wi == 1 ? r.y : wi == 2 ? r.z : r.w;
                const float v = decode_fp32_16_exact_nb((ww >> (hi * 16)) & 0xFFFFu, (rw >> (hi * 16)) & 0xFFFFu);
                const int q = 2 * wi + hi;
#pragma unroll
                for (int e = 0; e < 8; ++e) f[e] = e == q ? v : f[e];
            }
#pragma unroll
            for (int e = 0; e < HV; ++e) a[k * HV + e] = make_float2(f[2 * e], f[2 * e + 1]);
        }
    } else if constexpr (E == Elem::H16) {
        // wh words without a control bit are fp16 values: a chunk that
        // holds a control bit (rare) has those words rewritten to their
        // fp32_16_half_only bits first, then every word converts as fp16.
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            uint4 h = (live >> k) & 1u ? lds128(hrow + coff[k]) : make_uint4(0, 0, 0, 0);
            if ((h.x | h.y | h.z | h.w) & 0x00010001u) fix_half_chunk(h);
            a[k * 4 + 0] = h2f2(h.x);
            a[k * 4 + 1] = h2f2(h.y);
            a[k * 4 + 2] = h2f2(h.z);
            a[k * 4 + 3] = h2f2(h.w);
        }
    } else {
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            if ((live >> k) & 1u) {
                const uint4 h = lds128(hrow + coff[k]);
                if constexpr (E == Elem::F16) {
                    a[k * 4 + 0] = h2f2(h.x);
                    a[k * 4 + 1] = h2f2(h.y);
                    a[k * 4 + 2] = h2f2(h.z);
                    a[k * 4 + 3] = h2f2(h.w);
                } else if constexpr (E == Elem::F32) {
                    a[k * 2 + 0] = make_float2(__uint_as_float(h.x), __uint_as_float(h.y));
                    a[k * 2 + 1] = make_float2(__uint_as_float(h.z), __uint_as_float(h.w));
                } else {
                    uint4 r = h;
                    if (RowPlanes<E>::value == 2) r = lds128(lrow + coff[k]);
                    float f[VEC];
                    ChunkDecoder<E>::decode(h, r, f);
#pragma unroll
                    for (int e = 0; e < HV; ++e) a[k * HV + e] = make_float2(f[2 * e], f[2 * e + 1]);
                }
            } else {
#pragma unroll
                for (int e = 0; e < HV; ++e) a[k * HV + e] = make_float2(0.0f, 0.0f);
            }
        }
    }
}

template <Elem E, int NCH, int G, bool ACC64, int MODE>
__global__ void __launch_bounds__((RowWarps<E, ACC64, MODE>::value + 1) * 32, 1) fused_rows_kernel(RowPassParams T) {
    constexpr int CW = RowWarps<E, ACC64, MODE>::value;  // consumer warps
    constexpr bool DOT = MODE != kRowAxpy;         // forms the row dots
    constexpr bool AXPY = MODE != kRowDot;         // accumulates A^T ut
    constexpr bool BOTH = MODE == kRowBoth || MODE == kRowBothRuns;  // an LSQR pass
    // FP64 p and per-element FP64 products: the exact LSQR passes of the
    // RELRES rule (a consistent system's residual keeps its digits).  The
    // standalone FP64 tiers (kRowDot, kRowAxpy with ACC64) and kRowBothRuns
    // form FP32 products over short runs and sum those in FP64.
    constexpr bool P64 = ACC64 && MODE == kRowBoth;
    constexpr int NTHREADS = (CW + 1) * 32;
    static_assert(CW % G == 0, "G divides the consumer warps");
    const FusedParams& P = T.f;
    if (P.skip && *P.skip) return;
    constexpr int VEC = ChunkElems<E>::value;
    constexpr int PER = NCH * VEC;      // columns per lane
    constexpr int WCOLS = 32 * PER;     // columns per consumer warp
    constexpr int RS = CW / G;          // rows per tile (one per row group of warps)
    constexpr int PLANES = RowPlanes<E>::value;
    constexpr int ESZ = (E == Elem::F32) ? 4 : 2;
    static_assert(PER % 4 == 0, "pairs of pairs");

    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kRowMaxStages];
    __shared__ __align__(8) uint64_t empty[kRowMaxStages];
    __shared__ double ssw[kRowWarps];
    __shared__ double xdot[2][kRowWarps];
    __shared__ int abort_flag;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nstage = T.nstage;
    const int cb = T.copy_bytes;
    // A stage holds tps row tiles: each bulk copy then moves tps times a
    // tile's bytes (a copy carries a fixed cost beside its bytes).
    const int tps = T.tiles_per_stage;
    const size_t plane_bytes = (size_t)RS * tps * cb;
    const size_t stage_bytes = plane_bytes * PLANES;

    const int64_t rows_per_cta = (P.m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    int64_t r1 = r0 + rows_per_cta;
    if (r1 > P.m) r1 = P.m;
    const int64_t nrows = r1 > r0 ? r1 - r0 : 0;
    const int ntiles = (int)((nrows + RS - 1) / RS);               // row tiles
    const int nstages_total = (int)((nrows + RS * tps - 1) / (RS * tps));  // stage loads

    if (threadIdx.x == 0) {
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CW);
        }
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();

    float2 acc[PER / 2];
#pragma unroll
    for (int j = 0; j < PER / 2; ++j) acc[j] = make_float2(0.0f, 0.0f);
    // kRowAxpy with ACC64: FP64 sums of the FP32 run sums held in acc
    constexpr int NACC64 = (AXPY && ACC64 && !BOTH) ? PER : 1;
    double acc64[NACC64];
#pragma unroll
    for (int j = 0; j < NACC64; ++j) acc64[j] = 0.0;
    double ss = 0.0;
    const int rg = warp / G;    // row of the stage
    const int part = warp % G;  // column part of the row

    if (warp == CW) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            const bool contiguous = (int64_t)P.ld * ESZ == cb;
            int issued = 0;
            int s = 0;
            uint32_t ph = 0;
            for (int t = 0; t < nstages_total; ++t) {
                if (!mbar_wait(&empty[s], ph ^ 1u)) {
                    atomicExch(T.err, 1);
                    break;
                }
                if (*(volatile int*)&abort_flag) break;
                const int64_t i0 = r0 + (int64_t)t * RS * tps;
                const int rows = (int)((r1 - i0) < RS * tps ? (r1 - i0) : RS * tps);
                uint8_t* st = smem + (size_t)s * stage_bytes;
                mbar_expect_tx(&full[s], (uint32_t)(rows * cb * PLANES));
                if (contiguous) {
                    // rows of A are back to back: one copy per plane and stage
                    const size_t goff = (size_t)i0 * (size_t)P.ld * ESZ;
                    bulk_g2s(st, static_cast<const uint8_t*>(P.hi) + goff, (uint32_t)(rows * cb),
                             &full[s]);
                    if (PLANES == 2)
                        bulk_g2s(st + plane_bytes, static_cast<const uint8_t*>(P.lo) + goff,
                                 (uint32_t)(rows * cb), &full[s]);
                } else {
                    for (int r = 0; r < rows; ++r) {
                        const size_t goff = (size_t)(i0 + r) * (size_t)P.ld * ESZ;
                        bulk_g2s(st + (size_t)r * cb, static_cast<const uint8_t*>(P.hi) + goff,
                                 (uint32_t)cb, &full[s]);
                        if (PLANES == 2)
                            bulk_g2s(st + plane_bytes + (size_t)r * cb,
                                     static_cast<const uint8_t*>(P.lo) + goff, (uint32_t)cb, &full[s]);
                    }
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
    } else {
        // --------------------------------------------------------- consumers
        const double cp = P.coef ? P.coef[0] : P.cp;
        const double cu = P.coef ? P.coef[1] : P.cu;
        // a product with cu == 0 never reads u (it may hold NaN)
        const bool use_u = BOTH || cu != 0.0;
        const int64_t n = P.n;
        const int64_t nchunks = (n + VEC - 1) / VEC;
        int coff[NCH];
        uint32_t live = 0;
        // p for this lane's columns: FP32 pairs, or FP64 for P64
        using PT = typename std::conditional<P64, double, float2>::type;
        PT pv[P64 ? PER : PER / 2];
        // The lane holding the row's last, partly filled chunk zeroes the
        // elements from zero_from on (the copy's tail past column n-1).
        int zero_from = PER;
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            const int64_t c = (int64_t)part * 32 * NCH + (int64_t)k * 32 + lane;
            coff[k] = (int)(c * 16);
            if (c < nchunks) live |= 1u << k;
            if (c == nchunks - 1 && n % VEC != 0) zero_from = k * VEC + (int)(n - c * VEC);
#pragma unroll
            for (int e = 0; e < VEC; e += 2) {
                const int64_t col = c * VEC + e;
                const float x0 = (DOT && col < n) ? __ldg(P.p + col) : 0.0f;
                const float x1 = (DOT && col + 1 < n) ? __ldg(P.p + col + 1) : 0.0f;
                if constexpr (P64) {
                    pv[k * VEC + e] = (double)x0;
                    pv[k * VEC + e + 1] = (double)x1;
                } else {
                    pv[(k * VEC + e) / 2] = make_float2(x0, x1);
                }
            }
        }

        bool failed = false;
        // u of this warp's row, fetched two tiles ahead
        float ua = 0.f, ub = 0.f;
        if (use_u) {
            const int64_t a0 = r0 + rg, b0 = r0 + RS + rg;
            if (a0 < r1) ua = __ldg(P.u_in + a0);
            if (b0 < r1) ub = __ldg(P.u_in + b0);
        }
        int s = 0;
        uint32_t ph = 0;
        int sub = 0;  // row tile within the stage
        for (int t = 0; t < ntiles; ++t) {
            const int64_t i = r0 + (int64_t)t * RS + rg;
            const bool has = i < r1;
            const float ucur = ua;
            ua = ub;
            ub = (use_u && i + 2 * RS < r1) ? __ldg(P.u_in + i + 2 * RS) : 0.0f;
            if (sub == 0 && !failed && !mbar_wait(&full[s], ph)) {
                atomicExch(T.err, 3);
                abort_flag = 1;
                failed = true;
            }
            const uint8_t* hrow = smem + (size_t)s * stage_bytes + (size_t)(sub * RS + rg) * cb;
            float2 a[PER / 2];
            if (has && !failed) {
                decode_row<E, NCH>(hrow, hrow + plane_bytes, coff, live, a);
                if (zero_from < PER) {
#pragma unroll
                    for (int e = 0; e < PER; e += 2) {
                        if (e >= zero_from) a[e / 2].x = 0.0f;
                        if (e + 1 >= zero_from) a[e / 2].y = 0.0f;
                    }
                }
            } else {
#pragma unroll
                for (int e = 0; e < PER / 2; ++e) a[e] = make_float2(0.0f, 0.0f);
            }
            // The stage may be refilled once every consumer warp holds its
            // row of the stage's last tile (or of the CTA's last tile).
            if (++sub == tps || t + 1 == ntiles) {
                __syncwarp();
                if (lane == 0 && !failed) mbar_arrive(&empty[s]);
                sub = 0;
                if (++s == nstage) {
                    s = 0;
                    ph ^= 1u;
                }
            }

            double dsum = 0.0;
            if constexpr (!DOT) {
                // no dot: ut = cu u
            } else if constexpr (P64) {
                double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
#pragma unroll
                for (int j = 0; j < PER / 2; j += 2) {
                    d0 = fma((double)a[j].x, pv[2 * j], d0);
                    d1 = fma((double)a[j].y, pv[2 * j + 1], d1);
                    d2 = fma((double)a[j + 1].x, pv[2 * j + 2], d2);
                    d3 = fma((double)a[j + 1].y, pv[2 * j + 3], d3);
                }
                double dd = (d0 + d1) + (d2 + d3);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) dd += __shfl_xor_sync(0xffffffffu, dd, o);
                dsum = dd;
            } else {
                float2 d0 = make_float2(0.f, 0.f), d1 = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < PER / 2; j += 2) {
                    d0 = __ffma2_rn(a[j], pv[j], d0);
                    d1 = __ffma2_rn(a[j + 1], pv[j + 1], d1);
                }
                if constexpr (ACC64) {
                    // FP32 products summed over the lane's run, then FP64
                    double dd = ((double)d0.x + (double)d1.x) + ((double)d0.y + (double)d1.y);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) dd += __shfl_xor_sync(0xffffffffu, dd, o);
                    dsum = dd;
                } else {
                    float d = (d0.x + d1.x) + (d0.y + d1.y);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
                    dsum = (double)d;
                }
            }
            if constexpr (DOT && G > 1) {
                // partial dots of the row's G parts, summed in part order
                if (lane == 0) xdot[t & 1][warp] = dsum;
                named_bar_sync(1 + rg, G * 32);
                double tot = 0.0;
#pragma unroll
                for (int g = 0; g < G; ++g) tot += xdot[t & 1][rg * G + g];
                dsum = tot;
            }
            float ut;
            if constexpr (DOT)
                ut = has ? (float)(cp * dsum + (use_u ? cu * (double)ucur : 0.0)) : 0.0f;
            else
                ut = has ? (float)(cu * (double)ucur) : 0.0f;
            if constexpr (DOT) {
                if (lane == 0 && part == 0 && has) {
                    P.u_out[i] = ut;
                    if constexpr (BOTH) ss += (double)ut * (double)ut;
                }
            }
            if constexpr (AXPY) {
                const float2 ut2 = make_float2(ut, ut);
#pragma unroll
                for (int j = 0; j < PER / 2; ++j) acc[j] = __ffma2_rn(a[j], ut2, acc[j]);

                if constexpr (ACC64 && !BOTH) {
                    if ((t + 1) % kRowPromote == 0) {
#pragma unroll
                        for (int j = 0; j < PER / 2; ++j) {
                            acc64[2 * j] += (double)acc[j].x;
                            acc64[2 * j + 1] += (double)acc[j].y;
                            acc[j] = make_float2(0.0f, 0.0f);
                        }
                    }
                }
            }
        }
        if constexpr (AXPY && ACC64 && !BOTH) {
#pragma unroll
            for (int j = 0; j < PER / 2; ++j) {
                acc64[2 * j] += (double)acc[j].x;
                acc64[2 * j + 1] += (double)acc[j].y;
            }
        }
    }

    if constexpr (MODE == kRowDot) return;  // u_out is all a dot product writes
    // Epilogue: the producer waited for every copy it issued, so the stage
    // memory can hold the cross-warp reduction.
    __syncthreads();
    if constexpr (NACC64 > 1) {
        double* red64 = reinterpret_cast<double*>(smem);
        if (warp < CW) {
#pragma unroll
            for (int k = 0; k < NCH; ++k)
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                    red64[(size_t)warp * WCOLS + (k * 32 + lane) * VEC + e] = acc64[k * VEC + e];
        }
        __syncthreads();
        double* qout64 = T.qpart64 + (size_t)blockIdx.x * P.qstride;
        for (int64_t j = threadIdx.x; j < P.n; j += NTHREADS) {
            const int g = (int)(j / WCOLS);
            const int loc = (int)(j % WCOLS);
            double sum = 0.0;
#pragma unroll
            for (int r = 0; r < RS; ++r) sum += red64[(size_t)(r * G + g) * WCOLS + loc];
            qout64[j] = sum;
        }
        return;
    }
    float* red = reinterpret_cast<float*>(smem);
    if (warp < CW) {
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            float4* dst = reinterpret_cast<float4*>(&red[(size_t)warp * WCOLS + (k * 32 + lane) * VEC]);
#pragma unroll
            for (int e = 0; e < VEC; e += 4) {
                const int j = (k * VEC + e) / 2;
                dst[e / 4] = make_float4(acc[j].x, acc[j].y, acc[j + 1].x, acc[j + 1].y);
            }
        }
        if (lane == 0) ssw[warp] = ss;
    }
    __syncthreads();
    float* qout = P.qpart + (size_t)blockIdx.x * P.qstride;
    for (int64_t j = threadIdx.x; j < P.n; j += NTHREADS) {
        const int g = (int)(j / WCOLS);
        const int loc = (int)(j % WCOLS);
        float sum = 0.0f;
#pragma unroll
        for (int r = 0; r < RS; ++r) sum += red[(size_t)(r * G + g) * WCOLS + loc];
        qout[j] = sum;
    }
    if (BOTH && threadIdx.x == 0) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < CW; ++w) sum += ssw[w];
        P.sspart[blockIdx.x] = sum;
    }
}

// Dynamic shared memory of one launch: the stage ring, at least the
// cross-warp reduction buffer.
template <Elem E, int NCH, bool ACC64, int MODE>
inline size_t fused_rows_smem(int nstage, int rows_per_stage, int copy_bytes) {
    constexpr int VEC = ChunkElems<E>::value;
    const size_t ring = (size_t)nstage * rows_per_stage * copy_bytes * RowPlanes<E>::value;
    const size_t esz = (ACC64 && MODE == kRowAxpy) ? sizeof(double) : sizeof(float);
    const size_t red = (size_t)RowWarps<E, ACC64, MODE>::value * NCH * 32 * VEC * esz;
    return ring > red ? ring : red;
}

}  // namespace tomos_b200
