// rowpass_launch.cuh -- host-side launch of the row pass
// (fused_rows_kernel, rowpass.cuh): the stage ring sized to the shared
// memory budget, and the (element type, chunks per lane, warps per row,
// FP64 flag, mode) instantiations behind a run-time choice.  lsqr.cu
// launches the LSQR mode, rowpass_gemv.cu the standalone-product modes, each
// instantiating only what it uses.
#pragma once

#include "common.cuh"
#include "fused.cuh"
#include "rowpass.cuh"

namespace tomos_b200 {

template <Elem E, int NCH, int G, bool ACC64, int MODE>
inline tomos_status launch_fused_t(const FusedParams& P, int* err, int grid, cudaStream_t st,
                                   double* qpart64 = nullptr) {
    constexpr int ESZ = (E == Elem::F32) ? 4 : 2;
    constexpr int CW = RowWarps<E, ACC64, MODE>::value;
    constexpr int RS = CW / G;
    RowPassParams T;
    T.f = P;
    T.err = err;
    T.qpart64 = qpart64;
    T.copy_bytes = (int)((((int64_t)P.n * ESZ) + 15) / 16 * 16);
    const size_t tile = (size_t)RS * T.copy_bytes * RowPlanes<E>::value;
    const size_t budget = kRowSmemBudget;
    // tiles per stage: enough that a copy moves about kRowCopyTarget bytes
    // a plane, while the ring still holds two stages
    int tps = (int)((kRowCopyTarget + (size_t)RS * T.copy_bytes - 1) / ((size_t)RS * T.copy_bytes));
    while (tps > 1 && 2 * tile * tps > budget) --tps;
    if (tps < 1) tps = 1;
    T.tiles_per_stage = tps;
    const size_t stage = tile * tps;
    int ns = (int)(budget / stage);
    if (ns > kRowMaxStages) ns = kRowMaxStages;
    if (ns < 2) return fail(TOMOS_ERR_UNSUPPORTED, "fused pass: rows too long for the stage ring");
    T.nstage = ns;
    const size_t smem = fused_rows_smem<E, NCH, ACC64, MODE>(ns, RS * tps, T.copy_bytes);
    auto kern = fused_rows_kernel<E, NCH, G, ACC64, MODE>;
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, (CW + 1) * 32, smem, st>>>(T);
    TOMOS_LAUNCH_CHECK("fused_rows_kernel");
    return TOMOS_OK;
}

inline bool elem_two_planes(Elem e) {
    return e == Elem::A16 || e == Elem::AB16 || e == Elem::AB16R;
}

// Host mirrors of RowF64Regs, RowNchMax and RowWarps for a pass of
// element type e, FP64 flag acc64 and mode (RowMode).
inline bool fused_f64regs(bool acc64, int mode) { return acc64 && (mode == kRowBoth || mode == kRowAxpy); }

inline int fused_nch_max(Elem e, bool acc64, int mode) {
    const int base = (e == Elem::F32) ? 8 : 4;
    return (fused_f64regs(acc64, mode) && elem_two_planes(e)) ? base / 2 : base;
}

inline int fused_warps(Elem e, bool acc64, int mode) {
    if (fused_f64regs(acc64, mode)) return elem_two_planes(e) ? 16 : 8;
    const bool wide16 = e == Elem::F16 || e == Elem::B16 || (e == Elem::H16 && mode != kRowBoth);
    return wide16 ? 16 : 12;
}

// Warps per row a pass may split a row over (divisors of its consumer
// warps).
inline const int* fused_g_list(Elem e, bool acc64, int mode, int* count) {
    static const int g12[] = {2, 3, 4, 6, 12};
    static const int g8[] = {2, 4, 8};
    static const int g16[] = {2, 4, 8, 16};
    const int w = fused_warps(e, acc64, mode);
    *count = w == 8 ? 3 : (w == 16 ? 4 : 5);
    return w == 8 ? g8 : (w == 16 ? g16 : g12);
}

// How the row pass covers lines of `inner` elements at leading dimension
// ld: chunks per lane (nch) and warps per line (g), or false when the
// lines are not 16-byte aligned (both planes for two-plane types), too
// long for the consumer warps, or too long for a stage ring of two.
inline bool plan_row_lines(Elem e, bool acc64, int mode, int64_t inner, int64_t ld, const void* hi,
                           const void* lo, int* nch_out, int* g_out) {
    const int vec = (e == Elem::F32) ? 4 : 8;
    const int wbytes = (e == Elem::F32) ? 4 : 2;
    if (inner <= 0 || (ld * wbytes) % 16 != 0 || reinterpret_cast<uintptr_t>(hi) % 16 != 0) return false;
    if (elem_two_planes(e) && reinterpret_cast<uintptr_t>(lo) % 16 != 0) return false;
    int nch = 0, g = 1;
    const int nmax = fused_nch_max(e, acc64, mode);
    for (int c : {1, 2, 4, 8}) {
        if (c > nmax) break;
        if ((int64_t)32 * c * vec >= inner) {
            nch = c;
            break;
        }
    }
    if (nch == 0) {
        int ng = 0;
        const int* gl = fused_g_list(e, acc64, mode, &ng);
        for (int q = 0; q < ng; ++q) {
            if ((int64_t)gl[q] * 32 * nmax * vec >= inner) {
                nch = nmax;
                g = gl[q];
                break;
            }
        }
    }
    if (nch == 0) return false;
    const int64_t rows_per_stage = fused_warps(e, acc64, mode) / g;
    const int64_t stage = rows_per_stage * ((inner * wbytes + 15) / 16 * 16) * (elem_two_planes(e) ? 2 : 1);
    if (2 * stage > (int64_t)kRowSmemBudget) return false;
    *nch_out = nch;
    *g_out = g;
    return true;
}

// CTAs of a pass over `outer` lines: one per SM, at least 64 lines each.
inline int row_pass_grid(int64_t outer) {
    int64_t grid = sm_count();
    const int64_t gr = (outer + 63) / 64;
    if (grid > gr) grid = gr;
    return grid < 1 ? 1 : (int)grid;
}

// (nch, g) pairs with an instantiation: one warp per row with 1..NCHMAX
// chunks per lane, or G warps per row (fused_g_list) at NCHMAX.
template <Elem E, bool ACC64, int MODE>
inline tomos_status launch_fused_e(const FusedParams& P, int* err, int nch, int g, int grid,
                                   cudaStream_t st, double* qpart64 = nullptr) {
    constexpr int NMAX = RowNchMax<E, ACC64, MODE>::value;
    if (g == 1) {
        switch (nch) {
            case 1: return launch_fused_t<E, 1, 1, ACC64, MODE>(P, err, grid, st, qpart64);
            case 2: return launch_fused_t<E, 2, 1, ACC64, MODE>(P, err, grid, st, qpart64);
            case 4:
                if constexpr (NMAX >= 4) return launch_fused_t<E, 4, 1, ACC64, MODE>(P, err, grid, st, qpart64);
                break;
            case 8:
                if constexpr (NMAX == 8) return launch_fused_t<E, 8, 1, ACC64, MODE>(P, err, grid, st, qpart64);
                break;
            default: break;
        }
    } else if (nch == NMAX) {
        if constexpr (RowWarps<E, ACC64, MODE>::value == 8) {
            switch (g) {
                case 2: return launch_fused_t<E, NMAX, 2, ACC64, MODE>(P, err, grid, st, qpart64);
                case 4: return launch_fused_t<E, NMAX, 4, ACC64, MODE>(P, err, grid, st, qpart64);
                case 8: return launch_fused_t<E, NMAX, 8, ACC64, MODE>(P, err, grid, st, qpart64);
                default: break;
            }
        } else if constexpr (RowWarps<E, ACC64, MODE>::value == 16) {
            switch (g) {
                case 2: return launch_fused_t<E, NMAX, 2, ACC64, MODE>(P, err, grid, st, qpart64);
                case 4: return launch_fused_t<E, NMAX, 4, ACC64, MODE>(P, err, grid, st, qpart64);
                case 8: return launch_fused_t<E, NMAX, 8, ACC64, MODE>(P, err, grid, st, qpart64);
                case 16: return launch_fused_t<E, NMAX, 16, ACC64, MODE>(P, err, grid, st, qpart64);
                default: break;
            }
        } else {
            switch (g) {
                case 2: return launch_fused_t<E, NMAX, 2, ACC64, MODE>(P, err, grid, st, qpart64);
                case 3: return launch_fused_t<E, NMAX, 3, ACC64, MODE>(P, err, grid, st, qpart64);
                case 4: return launch_fused_t<E, NMAX, 4, ACC64, MODE>(P, err, grid, st, qpart64);
                case 6: return launch_fused_t<E, NMAX, 6, ACC64, MODE>(P, err, grid, st, qpart64);
                case 12: return launch_fused_t<E, NMAX, 12, ACC64, MODE>(P, err, grid, st, qpart64);
                default: break;
            }
        }
    }
    return fail(TOMOS_ERR_UNSUPPORTED, "fused pass: no instantiation");
}

}  // namespace tomos_b200
