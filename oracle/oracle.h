/* oracle.h -- CPU restatement of the reference (TOMOS) algorithms on the
 * LSQR hot path.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check and
 * the CPU-baseline leg of bench.py load this as the checker.  The product
 * library never links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function below
 * against the reference's own CPU build (oracle/_ref, when present) and
 * against the committed golden vectors in tests/golden/.
 *
 * Matrices are column-major unless a `row_major` flag says otherwise; ld is
 * the leading dimension in elements. */
#ifndef TOMOS_ORACLE_H
#define TOMOS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FP32_16 pack format (src/core/matrix/fp32_16_pack.hpp). */
void or_fp32_16_split(const float* src, size_t n, uint16_t* wh, uint16_t* wr);
void or_fp32_16_combine(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst);
void or_fp32_16_half_only(const uint16_t* wh, size_t n, uint16_t* half_bits);
/* The value fp32_16_half_only decodes to, widened to float. */
void or_fp32_16_half_only_f32(const uint16_t* wh, size_t n, float* dst);

/* FP32_BF16 pack format (src/core/matrix/fp32_bf16_pack.hpp). */
void or_fp32_bf16_split(const float* src, size_t n, uint16_t* wh, uint16_t* wr);
void or_fp32_bf16_split_rounded(const float* src, size_t n, uint16_t* wh, uint16_t* wr);
void or_fp32_bf16_combine(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst);
void or_fp32_bf16_combine_rounded(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst);

/* CountSketch hash (src/kernels/cpu/sketch/countsketch_kernels.cpp:59-85). */
uint64_t or_splitmix64(uint64_t x);
void or_countsketch_hash(size_t nrows, size_t s, uint64_t bucket_seed,
                         uint64_t sign_seed, int32_t* bucket, int8_t* sign);
/* SA (s x n, col-major, zeroed by the caller) += S * A, FP64 accumulate.
 * A is m x n with leading dimension ld, column-major or row-major. */
void or_countsketch_apply_f32(size_t m, size_t n, const float* A, size_t ld,
                              int row_major, size_t s, uint64_t bucket_seed,
                              uint64_t sign_seed, double* SA);
void or_countsketch_apply_f64(size_t m, size_t n, const float* A, size_t ld,
                              int row_major, size_t s, uint64_t bucket_seed,
                              uint64_t sign_seed, double* SA);

/* Unblocked FP64 Householder QR (LAPACK dgeqr2 convention, as called by
 * src/core/precond/sketch_qr.cpp:38-64): on return A's upper triangle holds
 * R, below it the reflectors; tau has n entries.  Requires m >= n. */
int or_householder_qr_f64(size_t m, size_t n, double* A, size_t ld, double* tau);
/* Inverse of an n x n upper-triangular R (col-major) into Rinv. */
int or_trtri_upper_f64(size_t n, const double* R, size_t ldr, double* Rinv, size_t ldi);

/* Plain LSQR, restating src/core/solver/lsqr.cpp:418-747 (fused_lsqr_impl
 * with FP32 working vectors and FP32-stored Givens scalars, as the
 * reference's FP32 instantiation does).  A is m x n col-major FP32, Rinv an
 * optional n x n col-major right preconditioner.  history (may be NULL)
 * receives |phi_bar|/||b|| per completed iteration. */
int or_lsqr_f32(size_t m, size_t n, const float* A, size_t lda, const float* b,
                float* x, const float* Rinv, double tol, int max_iters,
                double max_relres, int restarts, int* iterations, double* history);

#ifdef __cplusplus
}
#endif
#endif
