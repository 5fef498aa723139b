// C-ABI entry layer over the reference's own CPU path (test infrastructure).
//
// Compiled together with the reference's sources by oracle/Makefile into
// oracle/_ref/libtomos_ref.so; the Python tests load it with ctypes to pin
// the oracle restatement (oracle.c) and the CUDA product against the
// reference itself.  Every function here only marshals plain buffers into
// the reference's public C++ objects (tomos::Dense, tomos::Workspace, ...)
// and calls the reference's own entry points; no algorithm lives here.
//
// Functions return 0 on success and -1 if the reference threw.

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <vector>

#include "blas.hpp"
#include "context.hpp"
#include "countsketch_kernels.hpp"
#include "fp32_16_kernels.hpp"
#include "fp32_16_pack.hpp"
#include "fp32_bf16_pack.hpp"
#include "matrix.hpp"
#include "sketch_qr.hpp"
#include "solver.hpp"
#include "workspace.hpp"

using namespace tomos;

namespace {

void fill_colmajor(Dense& D, const float* src, size_t rows, size_t cols) {
    auto v = as_strided_view<float>(D);
    for (size_t j = 0; j < cols; ++j)
        for (size_t i = 0; i < rows; ++i)
            v.values_[i + j * v.lead_dim_] = src[i + j * rows];
}

void read_colmajor(Dense& D, float* dst, size_t rows, size_t cols) {
    auto v = as_strided_view<float>(D);
    for (size_t j = 0; j < cols; ++j)
        for (size_t i = 0; i < rows; ++i)
            dst[i + j * rows] = v.values_[i + j * v.lead_dim_];
}

}  // namespace

extern "C" {

// fp32_16_pack.hpp: fp32_16_split (full-carry encoder) element-wise.
void ref_fp32_16_split(const float* src, size_t n, uint16_t* wh, uint16_t* wr) {
    for (size_t i = 0; i < n; ++i) fp32_16_split(src[i], wh[i], wr[i]);
}

// fp32_16_pack.hpp: fp32_16_combine element-wise.
void ref_fp32_16_combine(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst) {
    for (size_t i = 0; i < n; ++i) dst[i] = fp32_16_combine(wh[i], wr[i]);
}

// fp32_16_pack.hpp: fp32_16_half_only element-wise; returns the half bits.
void ref_fp32_16_half_only(const uint16_t* wh, size_t n, uint16_t* half_bits) {
    for (size_t i = 0; i < n; ++i) {
        __half h = fp32_16_half_only(wh[i]);
        std::memcpy(&half_bits[i], &h, sizeof(uint16_t));
    }
}

// fp32_bf16_pack.hpp: truncating and rounding splits / combines.
void ref_fp32_bf16_split(const float* src, size_t n, uint16_t* wh, uint16_t* wr) {
    for (size_t i = 0; i < n; ++i) fp32_bf16_split(src[i], wh[i], wr[i]);
}
void ref_fp32_bf16_split_rounded(const float* src, size_t n, uint16_t* wh, uint16_t* wr) {
    for (size_t i = 0; i < n; ++i) fp32_bf16_split_rounded(src[i], wh[i], wr[i]);
}
void ref_fp32_bf16_combine(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst) {
    for (size_t i = 0; i < n; ++i) dst[i] = fp32_bf16_combine(wh[i], wr[i]);
}
void ref_fp32_bf16_combine_rounded(const uint16_t* wh, const uint16_t* wr, size_t n,
                                   float* dst) {
    for (size_t i = 0; i < n; ++i) dst[i] = fp32_bf16_combine_rounded(wh[i], wr[i]);
}

// countsketch_kernels.cpp: hash CountSketch, Y (m x B, col-major) +=
// S * X (n x B, col-major).  Y is accumulated into (the caller zeroes it).
void ref_countsketch_apply_f32(size_t n, size_t B, const float* X, size_t ldx,
                               size_t m, float* Y, size_t ldy) {
    cpu::countsketch_apply_impl<float>({n, B}, X, ldx, {m, B}, Y, ldy);
}
void ref_countsketch_apply_f64(size_t n, size_t B, const double* X, size_t ldx,
                               size_t m, double* Y, size_t ldy) {
    cpu::countsketch_apply_impl<double>({n, B}, X, ldx, {m, B}, Y, ldy);
}

// fp32_16_kernels.cpp: the reference's CPU FP32_16 GEMV tiers on a
// col-major packed A.  tier: 0 = pure_half, 1 = fast, 2 = accurate.
int ref_mv_fp32_16(int tier, int trans, double alpha, size_t m, size_t n,
                   const uint16_t* wh, const uint16_t* wr, size_t ld,
                   const float* x, double beta, float* y) {
    try {
        TransposeType t = trans ? TRANSPOSE : NO_TRANSPOSE;
        if (tier == 0)
            cpu::mv_fp32_16_pure_half(t, alpha, {m, n}, wh, ld, x, 1, beta, y, 1);
        else if (tier == 1)
            cpu::mv_fp32_16_fast(t, alpha, {m, n}, wh, ld, x, 1, beta, y, 1);
        else
            cpu::mv_fp32_16_accurate(t, alpha, {m, n}, wh, wr, ld, x, 1, beta, y, 1);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// blas.cpp mv_apply on a CPU FP32 col-major Dense (cblas_sgemv).
int ref_mv_f32(int trans, double alpha, size_t m, size_t n, const float* A,
               const float* x, double beta, float* y) {
    try {
        Context ctx(Device::CPU);
        Dense dA = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {m, n});
        fill_colmajor(dA, A, m, n);
        size_t lx = trans ? m : n, ly = trans ? n : m;
        Dense dx = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {lx, 1});
        Dense dy = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {ly, 1});
        fill_colmajor(dx, x, lx, 1);
        fill_colmajor(dy, y, ly, 1);
        mv_apply(Device::CPU, trans ? TRANSPOSE : NO_TRANSPOSE, alpha, dA, dx, beta, dy);
        read_colmajor(dy, y, ly, 1);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// sketch_qr.cpp generate_sketch_qr_precond on a CPU col-major k x n matrix:
// on return the leading n x n block of SA holds R^{-1}.  fp64 selects the
// FP64 (dgeqrf/dtrtri) or FP32 (sgeqrf/strtri) path.
int ref_sketch_qr_f64(size_t k, size_t n, double* SA) {
    try {
        Context ctx(Device::CPU);
        Dense d = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP64, {k, n});
        auto v = as_strided_view<double>(d);
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < k; ++i) v.values_[i + j * v.lead_dim_] = SA[i + j * k];
        Sparse S = Sparse::create_csr(ctx, NumericType::FP64, IntType::INT32, {k, k}, k);
        generate_sketch_qr_precond(S, d);
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < k; ++i) SA[i + j * k] = v.values_[i + j * v.lead_dim_];
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// lsqr.cpp lsqr_solve on the CPU, FP32 everywhere (A col-major m x n, b, x),
// optionally right-preconditioned by an FP32 col-major n x n Rinv.
// history (length >= restarts*max_iters, may be NULL) receives the
// relative residual |phi_bar|/||b|| of every completed iteration.
int ref_lsqr_solve_f32(size_t m, size_t n, const float* A, const float* b,
                       float* x, const float* Rinv, double tol, int max_iters,
                       double max_relres, int restarts, int* iterations,
                       double* history) {
    try {
        Context ctx(Device::CPU);
        Dense dA = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {m, n});
        fill_colmajor(dA, A, m, n);
        Dense db = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {m, 1});
        fill_colmajor(db, b, m, 1);
        Dense dx = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {n, 1});
        Dense dR = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {n, n});
        Workspace ws = create_lsqr_workspace(ctx, {m, n}, NumericType::FP32);
        if (Rinv) {
            fill_colmajor(dR, Rinv, n, n);
            add_precond(dR, ws);
        }
        std::vector<double> hist;
        int its = 0;
        lsqr_solve(ctx, dA, db, dx, ws, tol, max_iters, max_relres, &its,
                   history ? &hist : nullptr, restarts);
        read_colmajor(dx, x, n, 1);
        if (iterations) *iterations = its;
        if (history)
            for (size_t i = 0; i < hist.size(); ++i) history[i] = hist[i];
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// ref_lsqr_solve_f32 with the setup (copies into the reference's Dense
// objects, workspace creation, add_precond) outside the timed region:
// *seconds receives the wall time of the lsqr_solve call alone.
int ref_lsqr_solve_f32_timed(size_t m, size_t n, const float* A, const float* b, float* x,
                             const float* Rinv, double tol, int max_iters, double max_relres,
                             int restarts, int* iterations, double* seconds) {
    try {
        Context ctx(Device::CPU);
        Dense dA = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {m, n});
        fill_colmajor(dA, A, m, n);
        Dense db = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {m, 1});
        fill_colmajor(db, b, m, 1);
        Dense dx = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {n, 1});
        Dense dR = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {n, n});
        Workspace ws = create_lsqr_workspace(ctx, {m, n}, NumericType::FP32);
        if (Rinv) {
            fill_colmajor(dR, Rinv, n, n);
            add_precond(dR, ws);
        }
        int its = 0;
        const auto t0 = std::chrono::steady_clock::now();
        lsqr_solve(ctx, dA, db, dx, ws, tol, max_iters, max_relres, &its, nullptr, restarts);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        read_colmajor(dx, x, n, 1);
        if (iterations) *iterations = its;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// ref_sketch_qr_f64 with the copies in and out of the reference's Dense
// outside the timed region: *seconds receives the wall time of
// generate_sketch_qr_precond alone.
int ref_sketch_qr_f64_timed(size_t k, size_t n, double* SA, double* seconds) {
    try {
        Context ctx(Device::CPU);
        Dense d = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP64, {k, n});
        auto v = as_strided_view<double>(d);
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < k; ++i) v.values_[i + j * v.lead_dim_] = SA[i + j * k];
        Sparse S = Sparse::create_csr(ctx, NumericType::FP64, IntType::INT32, {k, k}, k);
        const auto t0 = std::chrono::steady_clock::now();
        generate_sketch_qr_precond(S, d);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < k; ++i) SA[i + j * k] = v.values_[i + j * v.lead_dim_];
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// Same as ref_lsqr_solve_f32, but stopping after exactly max_iters inner
// iterations (tol = max_relres = 0) -- used to time the per-iteration cost
// of the reference CPU path on a bounded sample.
int ref_lsqr_iterate_f32(size_t m, size_t n, const float* A, const float* b,
                         float* x, const float* Rinv, int iters) {
    return ref_lsqr_solve_f32(m, n, A, b, x, Rinv, 0.0, iters, 0.0, 1, nullptr,
                              nullptr);
}

}  // extern "C"
