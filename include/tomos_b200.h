/* tomos_b200.h -- C ABI of the B200 (sm_100a) LSQR hot path.
 *
 * Every entry point takes plain pointers and sizes, never throws, and
 * returns a tomos_status (0 on success).  tomos_last_error() gives the
 * message of the calling thread's last failure.  Device pointers are CUDA
 * device memory on the current device; `stream` is a cudaStream_t passed as
 * void* (NULL = the legacy default stream).  Calls are asynchronous on
 * `stream` unless documented otherwise; tomos_sync() blocks.
 *
 * Enum values mirror the reference (TOMOS) so a binding can pass the
 * reference's own enums through unchanged:
 *   NumericType  include/core/precision.hpp:43-50 (FP32_BF16 is new, slot 5)
 *   Layout       include/core/precision.hpp:51
 *   TransposeType src/core/matrix/transpose.hpp
 */
#ifndef TOMOS_B200_H
#define TOMOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int tomos_status;
enum {
    TOMOS_OK = 0,
    TOMOS_ERR_INVALID = -1,     /* std::invalid_argument in the reference  */
    TOMOS_ERR_UNSUPPORTED = -2, /* std::runtime_error "no kernel registered" */
    TOMOS_ERR_CUDA = -3,        /* CUDA runtime error                       */
    TOMOS_ERR_ALLOC = -4,       /* allocation failure                       */
    TOMOS_ERR_NUMERIC = -5      /* singular R / non-finite data             */
};

enum tomos_numeric {
    TOMOS_FP64 = 0, TOMOS_FP32 = 1, TOMOS_FP16 = 2, TOMOS_FP32_16 = 3,
    TOMOS_BF16 = 4, TOMOS_FP32_BF16 = 5
};
enum tomos_layout { TOMOS_ROW_MAJOR = 0, TOMOS_COL_MAJOR = 1 };
enum tomos_trans { TOMOS_NO_TRANSPOSE = 0, TOMOS_TRANSPOSE = 1 };

/* Compute tier of a product with A (reference dense_registries.cpp:350-362
 * and blas.hpp:160-172):
 *   NATIVE   -- A's own type (FP32 / FP64 storage).
 *   HALF     -- packed A read from its 16-bit wh plane only: FP32_16 decoded
 *               exactly as fp32_16_half_only (the reference's "fast" tier,
 *               fp32_16_kernels.cpp:102-123), FP32_BF16 as its bf16 word;
 *               FP32 accumulation.
 *   ACCURATE -- packed A reconstructed exactly from wh+wr (fp32_16_combine /
 *               fp32_bf16_combine[_rounded]); FP64 row accumulation.
 *   AUTO     -- the reference's default rule (blas.cpp:33-53): HALF for
 *               packed A, NATIVE otherwise. */
enum tomos_tier { TOMOS_TIER_AUTO = 0, TOMOS_TIER_NATIVE = 1, TOMOS_TIER_HALF = 2,
                  TOMOS_TIER_ACCURATE = 3,
                  /* tomos_mm only: A's 16-bit values (HALF tier, or native
                     FP16) times B rounded to the same 16-bit type -- the
                     operands of the reference's pure_half GEMM tier
                     (fp32_16_kernels.cpp:172-203), FP32 accumulation */
                  TOMOS_TIER_HALF_OPERANDS = 4 };

/* A strided dense matrix in device memory (non-owning; the reference's
 * StridedView, include/core/matrix.hpp:167-177).  For the packed types
 * `values` is the wh plane (uint16) and `values_lo` the wr plane; NULL
 * values_lo means the reference's planar layout (fp32_16_pack.hpp:861-874):
 * wr = wh + ld * (layout == COL_MAJOR ? cols : rows).  FP32_BF16 packs may
 * be truncating (rounded == 0, fp32_bf16_split) or rounding (rounded == 1,
 * fp32_bf16_split_rounded). */
typedef struct tomos_dense {
    int32_t numeric;
    int32_t layout;
    int64_t rows;
    int64_t cols;
    int64_t ld;
    void* values;
    void* values_lo;
    int32_t rounded;
    int32_t reserved;
} tomos_dense;

/* A CSR matrix in device memory (non-owning; CsrView, matrix.hpp:182-200).
 * index_type 0 = int32, 1 = int64 (IntType).  Packed values as above with
 * values_lo = values + nnz when NULL. */
typedef struct tomos_csr {
    int32_t numeric;
    int32_t index_type;
    int64_t rows;
    int64_t cols;
    int64_t nnz;
    void* values;
    void* values_lo;
    void* row_ptrs;
    void* col_idxs;
    int32_t rounded;
    int32_t reserved;
} tomos_csr;

const char* tomos_last_error(void);
const char* tomos_version(void);
tomos_status tomos_sync(void* stream);

/* ------------------------------------------------------------------ pack */

/* FP32 -> FP32_16 planes, bit-exact with fp32_16_split (the reference's
 * split_fp32_16 -> cuda::split_dense_fp32_16, fp32_16_cuda_kernels.cu:
 * 271-299; encoder fp32_16_pack.hpp:129-190).  src and dst share rows,
 * cols and layout; ld_src / ld_dst are their leading dimensions.
 * counts (device, may be NULL, 4 x uint64 accumulated into): elements
 * encoded [0] normal, [1] extended underflow, [2] extended overflow,
 * [3] saturated. */
tomos_status tomos_pack_fp32_16(const float* src, int32_t layout, int64_t rows,
                                int64_t cols, int64_t ld_src, uint16_t* wh,
                                uint16_t* wr, int64_t ld_dst,
                                unsigned long long* counts, void* stream);
/* FP32_16 planes -> FP32 (fp32_16_combine; combine_fp32_16,
 * fp32_16_registries.cpp:48-62). */
tomos_status tomos_unpack_fp32_16(const uint16_t* wh, const uint16_t* wr,
                                  int32_t layout, int64_t rows, int64_t cols,
                                  int64_t ld_src, float* dst, int64_t ld_dst,
                                  void* stream);
/* FP32 -> FP32_BF16 planes (fp32_bf16_split / fp32_bf16_split_rounded,
 * fp32_bf16_pack.hpp:68-73,117-145) and back (combine / combine_rounded). */
tomos_status tomos_pack_fp32_bf16(const float* src, int32_t layout, int64_t rows,
                                  int64_t cols, int64_t ld_src, uint16_t* wh,
                                  uint16_t* wr, int64_t ld_dst, int32_t rounded,
                                  void* stream);
/* FP32 -> native IEEE fp16 (round to nearest even, overflow to Inf): a
 * plain __half Dense, as the reference fills one (fill_dense_from_host<__half>
 * in lsqr_precision_runner.cu; the storage of --explicit-duplicates, whose
 * products the reference runs in mv_fp16_native, dense_registries.cpp:
 * 73-92, 329-333).  FP16 storage is read by every dense product, the
 * CountSketch and LSQR (iterations in FP32 arithmetic). */
tomos_status tomos_pack_fp16(const float* src, int32_t layout, int64_t rows, int64_t cols,
                             int64_t ld_src, uint16_t* dst, int64_t ld_dst, void* stream);
tomos_status tomos_unpack_fp32_bf16(const uint16_t* wh, const uint16_t* wr,
                                    int32_t layout, int64_t rows, int64_t cols,
                                    int64_t ld_src, float* dst, int64_t ld_dst,
                                    int32_t rounded, void* stream);

/* ------------------------------------------------------------------ GEMV */

/* y = alpha * op(A) x + beta * y (FP32 x, y), the reference's mv_apply
 * (src/core/blas/blas.cpp:23-31) resolved through dispatch::Dense::lookup_mv
 * (dense_registries.cpp:180-189) / Fp32_16 tiers (fp32_16_registries.cpp).
 * Deterministic: the transposed product of a row-major A (and the plain
 * product of a column-major A) reduces per-block partials in a fixed
 * order.  beta == 0 never reads y.  scratch: device buffer of at least
 * tomos_gemv_scratch_bytes() bytes (may be NULL when that is 0). */
size_t tomos_gemv_scratch_bytes(const tomos_dense* A, int32_t trans);
tomos_status tomos_gemv(int32_t trans, double alpha, const tomos_dense* A,
                        int32_t tier, const float* x, double beta, float* y,
                        void* scratch, size_t scratch_bytes, void* stream);

/* tomos_gemv without caller scratch and without allocating anything.  No
 * reference counterpart: the reference's mv_apply takes its workspace from
 * the caller or allocates it.  This entry is for callers that cannot
 * allocate device memory at call time -- a loop that runs under a device
 * memory budget fixed in advance, or code that must not risk the device-wide
 * synchronisation that cudaMalloc/cudaFree can cause.  Its scratch is one
 * 16 MiB buffer per device, built into the library; a product whose
 * tomos_gemv_scratch_bytes() exceeds 16 MiB (16777216) is rejected with
 * TOMOS_ERR_INVALID.  The first call made with a device current looks up that
 * device's buffer address, so make it before any stream capture.  All calls
 * on a device share the buffer: two calls that can overlap on the GPU (other
 * streams, or other host threads) race and may return wrong results; order
 * them on one stream or with events.  Results equal tomos_gemv's. */
tomos_status tomos_gemv_no_alloc(int32_t trans, double alpha, const tomos_dense* A,
                                 int32_t tier, const float* x, double beta, float* y,
                                 void* stream);

/* ------------------------------------------------------------------ GEMM */

/* C = alpha * op(A) op(B) + beta * C, the reference's mm_apply for a dense
 * A (src/core/blas/blas.cpp:98-106 through dispatch::Dense::lookup_mm,
 * dense_registries.cpp:396-405) and its FP32_16 tiers (blas.cpp:168-190,
 * fp32_16_registries.cpp:371-455).  A: FP32, FP16 or packed storage, any
 * layout; B and C: FP32, any layout (the reference's are column-major).
 * Runs on the tcgen05 tensor cores with FP32 accumulation:
 *   HALF_OPERANDS  16-bit A values x B rounded to 16 bits (pure_half
 *                  operands), one fp16/bf16 product;
 *   HALF / AUTO    16-bit A values x B kept to ~22 bits (the "fast" tier),
 *                  two TF32 products;
 *   ACCURATE / NATIVE (FP32 A)  A and B both kept to ~22 bits (the accurate
 *                  tier), three TF32 products.
 * An entry's error is a few units of 2^-22 times sum_l |op(A)_il op(B)_lj|
 * plus the FP32 summation over K, which one accumulator carries over the
 * whole of K (for K in the 10^5 range prefer tomos_mm_ex below, whose split
 * sums shorter runs).  beta == 0 never reads C.  Allocates nothing;
 * asynchronous on `stream`. */
tomos_status tomos_mm(int32_t trans_a, int32_t trans_b, double alpha, const tomos_dense* A,
                      int32_t tier, const tomos_dense* B, double beta, tomos_dense* C,
                      void* stream);

/* tomos_mm with caller scratch: a product with too few 128 x BN output tiles
 * to fill the GPU and a long K (e.g. A^T Q with A tall, the transposed
 * multi-right-hand-side product) splits K over CTAs, writes FP32 partial sums
 * to `scratch` and sums them in FP64 in a fixed order (deterministic).
 * tomos_mm_scratch_bytes gives the bytes (0: no split); with less scratch the
 * product runs unsplit, with the same result up to summation order. */
size_t tomos_mm_scratch_bytes(int32_t trans_a, int32_t trans_b, const tomos_dense* A,
                              int32_t tier, const tomos_dense* B);
tomos_status tomos_mm_ex(int32_t trans_a, int32_t trans_b, double alpha, const tomos_dense* A,
                         int32_t tier, const tomos_dense* B, double beta, tomos_dense* C,
                         void* scratch, size_t scratch_bytes, void* stream);

/* CSR y = alpha * op(A) x + beta * y (cuda::mv_csr, mv_cuda_kernels.cu:
 * 2029-2058; dispatch::Sparse::lookup_mv).  FP32, FP64 and packed values.
 * The transposed product is deterministic (no atomics). */
size_t tomos_csr_gemv_scratch_bytes(const tomos_csr* A, int32_t trans);
tomos_status tomos_csr_gemv(int32_t trans, double alpha, const tomos_csr* A,
                            int32_t tier, const float* x, double beta, float* y,
                            void* scratch, size_t scratch_bytes, void* stream);

/* ----------------------------------------------------------- CountSketch */

#define TOMOS_CS_BUCKET_SEED 0x12345678abcdef00ull
#define TOMOS_CS_SIGN_SEED 0xf00dd00d42babe55ull

/* Row i of A -> bucket splitmix64(i ^ bucket_seed) mod s, sign + if bit 0 of
 * splitmix64(i ^ sign_seed) is set (countsketch_kernels.cpp:59-85,
 * countsketch_cuda_kernels.cu:267-286).  Device outputs, m entries each. */
tomos_status tomos_countsketch_hash(int64_t m, int64_t s, uint64_t bucket_seed,
                                    uint64_t sign_seed, int32_t* bucket,
                                    int8_t* sign, void* stream);
/* SA (s x cols, column-major FP64, leading dimension ld_sa) = S * A, with
 * S the hash CountSketch above (replaces apply_count_sketch,
 * src/core/sketch/countsketch.cpp:20-26, whose dense-source CUDA path the
 * reference omits, sketch_registries.cpp:29-41).  Deterministic: each
 * bucket is summed by one owner in increasing row order in FP32 (bit for
 * bit the reference's countsketch_apply_impl<float>,
 * countsketch_kernels.cpp:70-83), stored as FP64.  Packed A is read at
 * `tier` (HALF reads only wh).
 * fro2 (device, may be NULL) receives sum(A_ij^2) of the values read and
 * colsq (device, may be NULL, cols entries) the sum of squares of every
 * column, both in the same pass. */
size_t tomos_countsketch_scratch_bytes(int64_t m, int64_t cols, int64_t s);
tomos_status tomos_countsketch_apply(const tomos_dense* A, int32_t tier, int64_t s,
                                     uint64_t bucket_seed, uint64_t sign_seed,
                                     double* SA, int64_t ld_sa, double* fro2,
                                     double* colsq, void* scratch,
                                     size_t scratch_bytes, void* stream);
/* tomos_countsketch_apply at the HALF tier of a row-major FP32_16 A (rows
 * 16-byte aligned) that also writes, in the same pass, the fp32_16_half_only
 * fp16 copy of A's wh plane (fp32_16_pack.hpp:553-571) to `plane` (device,
 * 16-byte aligned, m x ld_plane halves, ld_plane a multiple of 8 and >=
 * cols).  Passed to tomos_lsqr_solve_dense as opts.staged_plane, it spares
 * the solve the staging pass over A its HALF-tier iterations need.  No
 * reference counterpart (the reference's HALF tier decodes wh in every
 * GEMV). */
tomos_status tomos_countsketch_apply_stage(const tomos_dense* A, int64_t s,
                                           uint64_t bucket_seed, uint64_t sign_seed,
                                           double* SA, int64_t ld_sa, double* fro2,
                                           double* colsq, void* plane, int64_t ld_plane,
                                           void* scratch, size_t scratch_bytes,
                                           void* stream);
tomos_status tomos_countsketch_apply_csr(const tomos_csr* A, int32_t tier, int64_t s,
                                         uint64_t bucket_seed, uint64_t sign_seed,
                                         double* SA, int64_t ld_sa, double* fro2,
                                         double* colsq, void* scratch,
                                         size_t scratch_bytes, void* stream);

/* The column scale of the BACKWARD stopping rule from column sums of
 * squares (tomos_countsketch_apply's colsq, device, n doubles): d_j =
 * sqrt(colsq_j), 1 for an empty column, and ||A D^{-1}||_F = sqrt(number of
 * non-empty columns) in *anorm (device, one double).  On the device, no
 * host round trip.  No reference counterpart (the reference stops on
 * |phi_bar| / ||b|| only, lsqr.cpp:418-425). */
tomos_status tomos_column_scale(const double* colsq, int64_t n, double* d, double* anorm,
                                void* stream);

/* Row-sharded CountSketch: as tomos_countsketch_apply, for a row shard of
 * the whole problem whose row i is row row0 + i of the whole A (the hash
 * takes that index, so the shards' SA summed over ranks -- e.g. with
 * tomos_comm_allreduce_f64 -- is the whole problem's SA bit for bit up to
 * the summation order of the ranks).  plane (may be NULL): the staged fp16
 * copy of a row-major FP32_16 shard's wh plane, as
 * tomos_countsketch_apply_stage.  No reference counterpart (the reference
 * runs on one GPU). */
tomos_status tomos_countsketch_apply_shard(const tomos_dense* A, int32_t tier, int64_t s,
                                           uint64_t bucket_seed, uint64_t sign_seed, int64_t row0,
                                           double* SA, int64_t ld_sa, double* fro2, double* colsq,
                                           void* plane, int64_t ld_plane, void* scratch,
                                           size_t scratch_bytes, void* stream);

/* ------------------------------------------------------------- sketch QR */

/* FP64 Householder QR of the k x n (k >= n) column-major SA, then the
 * explicit inverse of R: on return the leading n x n block of SA holds
 * R^{-1} (upper triangular, zeros below), exactly the contract of
 * generate_sketch_qr_precond (src/core/precond/sketch_qr.hpp:19,
 * sketch_qr.cpp:38-64: geqrf + trtri).  R (device, may be NULL, n x n
 * column-major, ld n) receives R itself. */
size_t tomos_sketch_qr_scratch_bytes(int64_t k, int64_t n);
tomos_status tomos_sketch_qr_precond_f64(int64_t k, int64_t n, double* SA, int64_t ld,
                                         double* R, void* scratch,
                                         size_t scratch_bytes, void* stream);

/* Flags of tomos_sketch_qr_precond_ex_f64.  TOMOS_QR_ANY_SIGNS: the rows of
 * R may carry other signs than LAPACK's (R = S R_lapack, S diagonal +-1, so
 * R^{-1} = R_lapack^{-1} S differs by the signs of its columns).  A right-
 * preconditioned LSQR is invariant under such S (the iterates x_k of A R^{-1}
 * S and A R^{-1} agree in exact arithmetic), and the path that returns
 * positive pivots skips the sign reconstruction (a second n x n
 * factorisation). */
#define TOMOS_QR_ANY_SIGNS 1
tomos_status tomos_sketch_qr_precond_ex_f64(int64_t k, int64_t n, double* SA, int64_t ld,
                                            double* R, int32_t flags, void* scratch,
                                            size_t scratch_bytes, void* stream);

/* ------------------------------------------------------------------ LSQR */

/* Stopping rules.  RELRES is the reference's (lsqr.cpp:418-425, :723-729):
 * stop when |phi_bar| / ||b|| < tol or < max_relres.  BACKWARD stops when
 * the normwise backward error
 *   eta = min( ||r|| / (||A||_F ||x|| + ||b||),  ||A^T r|| / (||A||_F ||r||) )
 * of the current x, recomputed from an ACCURATE-tier residual at every
 * restart boundary, is <= tol.  With a column scale D (opts.col_scale) the
 * same quantity is taken for the column-scaled problem (A D^{-1}, b, D x):
 *   eta_D = min( ||r|| / (||A D^{-1}||_F ||D x|| + ||b||),
 *                ||D^{-1} A^T r|| / (||A D^{-1}||_F ||r||) ),
 * which is invariant to the scaling of A's columns; with D the column
 * norms it is the backward error of the equilibrated problem.  With
 * BACKWARD at tol >= 1e-6 the accurate-tier passes form their row dots
 * as FP32 products over runs of at most 8, summed in FP64 (a backward
 * error of at most 4.8e-7 an element); below 1e-6, and under RELRES, as
 * one FP64 product an element. */
enum tomos_stop { TOMOS_STOP_RELRES = 0, TOMOS_STOP_BACKWARD = 1 };

typedef struct tomos_lsqr_opts {
    double tol;              /* lsqr_solve's tol                          */
    int32_t max_iters;       /* iterations per restart                     */
    int32_t restarts;        /* outer cycles (lsqr_solve's restarts)       */
    double max_relres;       /* lsqr_solve's max_relres                    */
    int32_t stop_rule;       /* enum tomos_stop                            */
    int32_t iter_tier;       /* per-iteration products (Workspace::
                                mv_compute_type_); AUTO = reference rule   */
    int32_t implicit_duplicate; /* Workspace::use_implicit_duplicate_: the
                                restart residual reads packed A ACCURATE    */
    int32_t warm_start;      /* 0: x zeroed first (lsqr_registries.cpp:156) */
    double inner_rtol;       /* BACKWARD rule: an inner cycle ends once its
                                residual estimate fell by this factor (0 =
                                run max_iters)                              */
    double anorm_fro;        /* ||A||_F (||A D^{-1}||_F with a column
                                scale) if already known, e.g. from
                                tomos_countsketch_apply; 0 = the BACKWARD
                                rule computes it (one pass)                  */
    const double* col_scale; /* device, n entries, may be NULL: the column
                                scale D of the BACKWARD rule                 */
    double* history;         /* host, may be NULL: |phi_bar|/||b|| per
                                completed iteration (residual_history)     */
    int32_t history_cap;
    int32_t profile;         /* nonzero: time every pass over A with CUDA
                                events on the solver stream (the reference's
                                TOMOS_LSQR_TIMING buckets, lsqr.cpp:85-166);
                                iterations then run as plain launches
                                instead of graph replays                    */
    const void* staged_plane; /* device, may be NULL: the fixed fp16 copy of
                                a row-major FP32_16 A's wh plane that
                                tomos_countsketch_apply_stage wrote (m x
                                staged_ld halves); HALF-tier iterations read
                                it instead of staging their own copy. The
                                caller keeps it equal to A's wh plane.      */
    int64_t staged_ld;
    const double* anorm_fro_dev; /* device, may be NULL: ||A||_F (or
                                ||A D^{-1}||_F) as one device double, e.g.
                                from tomos_column_scale; read on the device,
                                so the solve needs no host round trip before
                                its first pass.  Takes precedence over
                                anorm_fro.                                   */
    const tomos_dense* refine; /* may be NULL: lsqr_solve's
                                mtx_refine_precision (--explicit-duplicates):
                                a copy of A at higher precision (FP32, or
                                packed read exactly) that the initial and
                                restart passes read instead of A; it takes
                                precedence over implicit_duplicate
                                (lsqr.cpp:459-473)                          */
    struct tomos_comm* comm; /* may be NULL: the ranks of a row-sharded solve
                                (A, b this rank's rows; x replicated)        */
    double inner_eta_factor; /* BACKWARD rule: an inner cycle also ends once
                                its estimate |phi_bar| / (||A|| ||x|| + ||b||)
                                is below tol times this (0 = 1).  Below 1 with
                                refinement (inner iterations on a 16-bit
                                plane), it leaves room for the plane's
                                perturbation, so that the cycle's exact
                                residual meets tol and no further cycle
                                (and exact pass) is needed.                  */
    const struct tomos_csr* refine_csr; /* may be NULL: the CSR solve's
                                mtx_refine_precision (lsqr_sparse_impl,
                                lsqr_registries.cpp:164-183): a copy of a
                                CSR A at higher precision (FP32 values, or
                                packed read exactly) that the initial and
                                restart passes read instead of A.  A dense
                                solve rejects it, and a CSR solve rejects
                                `refine`.                                    */
} tomos_lsqr_opts;

typedef struct tomos_lsqr_report {
    int32_t iterations;      /* completed inner iterations, all restarts   */
    int32_t restarts_used;
    int32_t converged;
    int32_t history_len;
    double relres;           /* |phi_bar| / ||b|| at exit                  */
    double rnorm;            /* last accurate ||b - A x||                   */
    double arnorm;           /* last accurate ||A^T (b - A x)||             */
    double anorm_fro;        /* ||A||_F                                     */
    double xnorm;
    double bnorm;
    double backward_error;   /* eta of the returned x (accurate residual)   */
    double elapsed_ms;       /* device time of the solve                    */
    int32_t accurate_passes; /* restart-boundary passes over A              */
    int32_t half_passes;     /* per-iteration passes over A                 */
    double iter_pass_ms;     /* profile: total device time of the
                                per-iteration passes over A                 */
    double init_pass_ms;     /* profile: same for the accurate-tier restart
                                passes (the first pass from x = 0 runs at
                                the iteration tier and is not counted)      */
    int32_t iter_pass_count;
    int32_t init_pass_count;
    int32_t kernel_launches; /* kernels the solve enqueued (graph replays
                                counted per kernel)                          */
    int32_t reserved;
} tomos_lsqr_report;

typedef struct tomos_workspace tomos_workspace;

/* ------------------------------------------------------- multi-GPU solves */

/* A communicator over the ranks of a row-sharded solve (one process per
 * GPU; NCCL over NVLink / NVSwitch).  Rank 0 makes an id
 * (tomos_comm_unique_id), every rank receives it by its own means (a
 * torch.distributed broadcast, MPI, a file) and calls tomos_comm_create with
 * its device current.  Passed as tomos_lsqr_opts.comm, the solve treats A
 * and b as rank's row shard of one problem and x as the whole solution
 * (replicated): after every pass over A the n + 1 partial sums (A^T u and
 * ||u||^2) are summed across ranks, once.  No reference counterpart (the
 * reference runs on one GPU; lsqr.cpp:561-621 are the products split). */
#define TOMOS_COMM_ID_BYTES 128
typedef struct tomos_comm tomos_comm;
tomos_status tomos_comm_unique_id(void* id /* TOMOS_COMM_ID_BYTES */);
tomos_status tomos_comm_create(int32_t nranks, int32_t rank, const void* id, tomos_comm** out);
tomos_status tomos_comm_destroy(tomos_comm* comm);
/* buf (device, count doubles) <- its sum over the ranks, on stream. */
tomos_status tomos_comm_allreduce_f64(tomos_comm* comm, double* buf, int64_t count, void* stream);

/* create_lsqr_workspace (src/core/solver/lsqr.cpp:389-406,
 * include/core/solver.hpp:15-25): owns the device arena for the m- and
 * n-vectors, the per-block partials of the transposed products and the
 * solver state.  value_type must be FP32; precond_type FP32 or FP64. */
tomos_status tomos_workspace_create(int64_t m, int64_t n, int32_t value_type,
                                    int32_t precond_type, tomos_workspace** ws);
tomos_status tomos_workspace_destroy(tomos_workspace* ws);
/* add_precond (include/core/workspace.hpp:112-120): attaches a non-owning
 * n x n right preconditioner R^{-1} (FP32 or FP64 Dense, any layout); its
 * numeric type must equal the workspace's precond_type.  NULL detaches. */
tomos_status tomos_workspace_add_precond(tomos_workspace* ws, const tomos_dense* Rinv);

/* lsqr_solve (include/core/solver.hpp:68-78; lsqr.cpp:785-801): solves
 * min ||A x - b|| with A m x n on the device, b (m) and x (n) FP32 device
 * vectors.  Synchronous on `stream` (the report is filled on return).
 * HALF-tier iterations over a row-major FP32_16 A stream an fp16 copy of
 * its wh plane that the solve writes into the workspace first (2 bytes per
 * element, allocated by the first such solve and kept); if that allocation
 * fails the iterations read A directly. */
tomos_status tomos_lsqr_solve_dense(const tomos_dense* A, const float* b, float* x,
                                    tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                    tomos_lsqr_report* report, void* stream);
tomos_status tomos_lsqr_solve_csr(const tomos_csr* A, const float* b, float* x,
                                  tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                  tomos_lsqr_report* report, void* stream);

/* Normwise backward error of x (FP64, ACCURATE tier): fills report's
 * rnorm, arnorm, anorm_fro, xnorm, bnorm and backward_error.  col_scale
 * (device, may be NULL) selects eta_D (see the stopping rules).  Needs a
 * workspace of A's shape for its partials. */
tomos_status tomos_backward_error_dense(const tomos_dense* A, const float* b,
                                        const float* x, const double* col_scale,
                                        tomos_workspace* ws, tomos_lsqr_report* report,
                                        void* stream);

/* --------------------------------------------------------------- adjoint */

/* Adjoint of x* = argmin ||A x - b|| (no reference counterpart: the
 * reference has no differentiation).  For a loss L with g = dL/dx*:
 *   lambda = (A^T A)^{-1} g,  dL/db = A lambda,
 *   dL/dA = r lambda^T - (A lambda) x*^T  with r = b - A x*.
 * tomos_lsqr_adjoint_dense: lambda (n, FP32 device) by preconditioned
 * conjugate gradients on R^{-T} A^T A R^{-1} (the normal-equations form of
 * LSQR) with the workspace's R^{-1} (tomos_workspace_add_precond; none means
 * plain CG), one pass over A per iteration.  opts: tol (stop when
 * ||g - A^T A lambda|| <= tol ||g||), max_iters, iter_tier (AUTO = the exact
 * values of a packed A).  report: iterations, converged, relres (the final
 * relative residual), elapsed_ms, kernel_launches.  Synchronous on stream. */
tomos_status tomos_lsqr_adjoint_dense(const tomos_dense* A, const float* g, float* lambda,
                                      tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                      tomos_lsqr_report* report, void* stream);
/* K adjoints at once: Lambda_k = (A^T A)^{-1} G_k for the K columns of G
 * (n x K column-major FP32, leading dimension ldg) into Lambda (n x K, ld
 * ldl).  The same preconditioned CG as tomos_lsqr_adjoint_dense, one
 * recurrence per column, sharing the products with A: every iteration
 * forms Q = A P and W = A^T Q for all K directions with two tensor-core
 * products (tomos_mm_ex), so A is read twice an iteration for all K
 * columns instead of once per column.  Products at ~2^-22 relative
 * (three TF32 terms for FP32 or exactly read packed A).  reports (K
 * entries, may be NULL): each column's iterations, converged, relres;
 * half_passes counts the shared products.  The workspace grows a buffer
 * for the K columns on first use.  Synchronous on stream. */
tomos_status tomos_lsqr_adjoint_batch_dense(const tomos_dense* A, int32_t K, const float* G,
                                            int64_t ldg, float* Lambda, int64_t ldl,
                                            tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                            tomos_lsqr_report* reports, void* stream);
/* The gradients for K right-hand sides in one pass over a row-major A:
 * B (m x K), X = x*_k (n x K), Lam = lambda_k (n x K), column-major with
 * leading dimensions ldb, ldx, ldl.  gradB (m x K, ld ldgb) = A Lam;
 * gradA (m x n row-major, ld ldga; may be NULL) = sum_k r_k lambda_k^T -
 * (A lambda_k) x_k^T.  Packed A is read at its exact values.  n * min(K, 8)
 * must fit 25600 (X and Lam staged in shared memory). */
tomos_status tomos_lsqr_adjoint_grad_dense(const tomos_dense* A, int64_t K, const float* B,
                                           int64_t ldb, const float* X, int64_t ldx,
                                           const float* Lam, int64_t ldl, float* gradB,
                                           int64_t ldgb, float* gradA, int64_t ldga,
                                           void* stream);

/* ------------------------------------------------------------ MatrixMarket */

/* Host-side MatrixMarket files: the reference reads its test systems with
 * the NIST mmio routines (src/io/mmio.c) through read_mtx_host
 * (benchmarks/solvers/cuda/lsqr_precision_runner.cu:101-125), an `array`
 * file's values into an m x n column-major FP64 buffer.  These read the
 * same files the same way (strtod per value) and also take `coordinate`
 * files, the integer and pattern fields and symmetric / skew-symmetric
 * storage (mirrored); complex and hermitian files are rejected.  Array
 * files, general coordinate files read as triplets, and writes run on all
 * host threads (TOMOS_MTX_THREADS in the environment sets their number);
 * the results are the sequential ones, bit for bit. */
enum tomos_mtx_format { TOMOS_MTX_ARRAY = 0, TOMOS_MTX_COORDINATE = 1 };
enum tomos_mtx_field { TOMOS_MTX_REAL = 0, TOMOS_MTX_INTEGER = 1, TOMOS_MTX_PATTERN = 2 };
enum tomos_mtx_symmetry { TOMOS_MTX_GENERAL = 0, TOMOS_MTX_SYMMETRIC = 1, TOMOS_MTX_SKEW = 2 };
typedef struct tomos_mtx_info {
    int64_t rows;
    int64_t cols;
    int64_t entries;   /* stored entries (coordinate: the nnz line; array:
                          rows*cols or the stored triangle)              */
    int32_t format;    /* enum tomos_mtx_format                         */
    int32_t field;     /* enum tomos_mtx_field                          */
    int32_t symmetry;  /* enum tomos_mtx_symmetry                       */
    int32_t reserved;
} tomos_mtx_info;
/* mm_read_banner + mm_read_mtx_array_size / mm_read_mtx_crd_size. */
tomos_status tomos_mtx_read_info(const char* path, tomos_mtx_info* info);
/* The whole matrix into host memory `out` (FP64, layout COL_MAJOR as
 * read_mtx_host, or ROW_MAJOR; leading dimension ld); coordinate entries
 * that repeat a position add. */
tomos_status tomos_mtx_read_dense(const char* path, int32_t layout, double* out, int64_t ld);
/* The entries as 0-based triplets in file order, each mirrored entry of a
 * symmetric file right after its stored one.  *count receives the number
 * of triplets; more than cap is an error (call with cap = 0 to size). */
tomos_status tomos_mtx_read_coo(const char* path, int64_t cap, int64_t* rows, int64_t* cols,
                                double* vals, int64_t* count);
/* An `array real general` file, column by column, 17 significant digits
 * (the format generate_tall_thin_mtx.m writes). */
tomos_status tomos_mtx_write_dense(const char* path, int32_t layout, int64_t rows, int64_t cols,
                                   const double* a, int64_t ld);

#ifdef __cplusplus
}
#endif
#endif /* TOMOS_B200_H */
