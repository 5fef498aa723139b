/* oracle.c -- CPU restatement of the reference (TOMOS) algorithms on the
 * LSQR hot path.  TEST INFRASTRUCTURE ONLY (see oracle.h): the checker the
 * tests, the smoke check and bench.py's CPU-baseline leg use; the product
 * never links it.  Each function cites the reference file:line it
 * restates.  Parity is pinned against the reference's own CPU build
 * (oracle/_ref) and the golden vectors in tests/golden/. */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static uint32_t f2u(float v) { uint32_t u; memcpy(&u, &v, 4); return u; }
static float u2f(uint32_t u) { float v; memcpy(&v, &u, 4); return v; }

/* ---------------------------------------------------------------------
 * FP32_16: wh = sign(1) | exponent field(5) | mant_hi(9) | control(1)
 *          wr = mant_lo(14) | reserved(1) | round_flag(1)
 * fp32 exponents 113..142 are stored directly (rebias 112, control 0);
 * up to 14 further steps either side are stored as direction + (steps-1)
 * with control 1; anything beyond saturates (steps field 14) to signed
 * Inf / signed 0.  mant_hi is the RNE-rounded top 9 mantissa bits and
 * round_flag records the round-up so the split is invertible.
 * ------------------------------------------------------------------- */

/* fp32_16_pack.hpp:129-190 (fp32_16_split, "full carry" encoder). */
static void split16(float value, uint16_t* wh, uint16_t* wr) {
    uint32_t bits = f2u(value);
    uint32_t sign = (bits >> 16) & 0x8000u;
    uint32_t e = (bits >> 23) & 0xFFu;
    uint32_t mant = bits & 0x7FFFFFu;
    if (e >= 99u && e <= 156u) {
        uint32_t hi = mant >> 14, lo = mant & 0x3FFFu;
        uint32_t up = ((lo >> 13) & 1u) && ((lo & 0x1FFFu) || (hi & 1u));
        uint32_t hr = hi + up;
        uint32_t carry = hr > 0x1FFu;
        uint32_t ee = e + carry;
        uint32_t hw = carry ? 0u : hr;
        if (ee >= 113u && ee <= 142u) {
            *wh = (uint16_t)(sign | ((ee - 112u) << 10) | (hw << 1));
            *wr = (uint16_t)((lo << 2) | up);
            return;
        }
        uint32_t dir = ee > 142u;
        uint32_t steps = dir ? ee - 142u : 113u - ee;
        if (steps >= 1u && steps <= 14u) {
            *wh = (uint16_t)(sign | (dir << 14) | ((steps - 1u) << 10) | (hw << 1) | 1u);
            *wr = (uint16_t)((lo << 2) | up);
            return;
        }
        *wh = (uint16_t)(sign | (dir << 14) | (14u << 10) | 1u);
        *wr = 0;
        return;
    }
    uint32_t dir = e > 142u;
    *wh = (uint16_t)(sign | (dir << 14) | (14u << 10) | 1u);
    *wr = 0;
}

/* fp32_16_pack.hpp:301-359 (fp32_16_combine). */
static float combine16(uint16_t wh, uint16_t wr) {
    uint32_t h = wh, r = wr;
    uint32_t sign = (h & 0x8000u) << 16;
    uint32_t mh = (h >> 1) & 0x1FFu, ml = (r >> 2) & 0x3FFFu, rf = r & 1u;
    uint32_t carry = rf && mh == 0u;
    uint32_t pre = carry ? 0x1FFu : mh - rf;
    uint32_t e;
    if (!(h & 1u)) {
        e = ((h >> 10) & 0x1Fu) + 112u - carry;
    } else {
        uint32_t s = (h >> 10) & 0xFu, dir = (h >> 14) & 1u;
        if (s == 14u) return u2f(dir ? (sign | 0x7F800000u) : sign);
        e = (dir ? 143u + s : 112u - s) - carry;
    }
    return u2f(sign | (e << 23) | (pre << 14) | ml);
}

/* fp32_16_pack.hpp:553-571 (fp32_16_half_only): wh as an fp16 value;
 * underflow steps become fp16 subnormals by right-shifting the 10-bit
 * significand, overflow becomes signed Inf. */
static uint16_t half_only(uint16_t wh) {
    uint32_t h = wh;
    if (!(h & 1u)) return wh;
    uint32_t sign = h & 0x8000u;
    if ((h >> 14) & 1u) return (uint16_t)(sign | 0x7C00u);
    uint32_t s = (h >> 10) & 0xFu;
    uint32_t sig = 0x200u | ((h >> 1) & 0x1FFu);
    return (uint16_t)(sign | ((sig >> s) & 0x3FFu));
}

/* IEEE binary16 bits -> float (normal, subnormal, Inf; NaN not produced). */
static float half_bits_to_f32(uint16_t hb) {
    uint32_t sign = (hb & 0x8000u) ? 1u : 0u;
    uint32_t e = (hb >> 10) & 0x1Fu, m = hb & 0x3FFu;
    float v;
    if (e == 0u) v = ldexpf((float)m, -24);
    else if (e == 31u) v = m ? NAN : INFINITY;
    else v = ldexpf((float)(0x400u | m), (int)e - 25);
    return sign ? -v : v;
}

void or_fp32_16_split(const float* src, size_t n, uint16_t* wh, uint16_t* wr) {
    for (size_t i = 0; i < n; ++i) split16(src[i], &wh[i], &wr[i]);
}
void or_fp32_16_combine(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst) {
    for (size_t i = 0; i < n; ++i) dst[i] = combine16(wh[i], wr[i]);
}
void or_fp32_16_half_only(const uint16_t* wh, size_t n, uint16_t* half_bits) {
    for (size_t i = 0; i < n; ++i) half_bits[i] = half_only(wh[i]);
}
void or_fp32_16_half_only_f32(const uint16_t* wh, size_t n, float* dst) {
    for (size_t i = 0; i < n; ++i) dst[i] = half_bits_to_f32(half_only(wh[i]));
}

/* ---------------------------------------------------------------------
 * FP32_BF16: wh = top 16 bits (a bf16), wr = low 16 bits.
 * ------------------------------------------------------------------- */

/* fp32_bf16_pack.hpp:68-81 (fp32_bf16_split / fp32_bf16_combine). */
void or_fp32_bf16_split(const float* src, size_t n, uint16_t* wh, uint16_t* wr) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t b = f2u(src[i]);
        wh[i] = (uint16_t)(b >> 16);
        wr[i] = (uint16_t)(b & 0xFFFFu);
    }
}
void or_fp32_bf16_combine(const uint16_t* wh, const uint16_t* wr, size_t n, float* dst) {
    for (size_t i = 0; i < n; ++i) dst[i] = u2f(((uint32_t)wh[i] << 16) | wr[i]);
}

/* fp32_bf16_pack.hpp:117-145 (fp32_bf16_split_rounded): wh rounded to
 * nearest-even, the round-up recorded in wr's bit 0 (which costs the
 * original mantissa's last bit). */
void or_fp32_bf16_split_rounded(const float* src, size_t n, uint16_t* wh, uint16_t* wr) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t b = f2u(src[i]);
        uint32_t t = b >> 16, lo = b & 0xFFFFu;
        uint32_t up = ((lo >> 15) & 1u) && ((lo & 0x7FFFu) || (t & 1u));
        wh[i] = (uint16_t)(t + up);
        wr[i] = (uint16_t)((lo & 0xFFFEu) | up);
    }
}

/* fp32_bf16_pack.hpp:180-186 (fp32_bf16_combine_rounded). */
void or_fp32_bf16_combine_rounded(const uint16_t* wh, const uint16_t* wr, size_t n,
                                  float* dst) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t rf = wr[i] & 1u;
        uint32_t t = ((uint32_t)wh[i] - rf) & 0xFFFFu;
        dst[i] = u2f((t << 16) | (wr[i] & 0xFFFEu));
    }
}

/* ---------------------------------------------------------------------
 * CountSketch (countsketch_kernels.cpp:59-85): row i of A goes to bucket
 * splitmix64(i ^ bucket_seed) mod s with sign +1 if bit 0 of
 * splitmix64(i ^ sign_seed) is set, else -1.
 * ------------------------------------------------------------------- */
uint64_t or_splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

void or_countsketch_hash(size_t nrows, size_t s, uint64_t bucket_seed,
                         uint64_t sign_seed, int32_t* bucket, int8_t* sign) {
    for (size_t i = 0; i < nrows; ++i) {
        bucket[i] = (int32_t)(or_splitmix64((uint64_t)i ^ bucket_seed) % (uint64_t)s);
        sign[i] = (or_splitmix64((uint64_t)i ^ sign_seed) & 1ull) ? 1 : -1;
    }
}

void or_countsketch_apply_f64(size_t m, size_t n, const float* A, size_t ld,
                              int row_major, size_t s, uint64_t bucket_seed,
                              uint64_t sign_seed, double* SA) {
    for (size_t i = 0; i < m; ++i) {
        size_t bkt = (size_t)(or_splitmix64((uint64_t)i ^ bucket_seed) % (uint64_t)s);
        double sg = (or_splitmix64((uint64_t)i ^ sign_seed) & 1ull) ? 1.0 : -1.0;
        for (size_t j = 0; j < n; ++j) {
            float a = row_major ? A[i * ld + j] : A[i + j * ld];
            SA[bkt + j * s] += sg * (double)a;
        }
    }
}

/* The reference's own float path (countsketch_kernels.cpp:70-83,
 * countsketch_apply_impl<float>): Y[bucket] += sign * x in FP32, rows in
 * increasing order.  SA is returned widened to FP64. */
void or_countsketch_apply_f32(size_t m, size_t n, const float* A, size_t ld,
                              int row_major, size_t s, uint64_t bucket_seed,
                              uint64_t sign_seed, double* SA) {
    float* acc = (float*)calloc(s * n, sizeof(float));
    for (size_t i = 0; i < m; ++i) {
        size_t bkt = (size_t)(or_splitmix64((uint64_t)i ^ bucket_seed) % (uint64_t)s);
        float sg = (or_splitmix64((uint64_t)i ^ sign_seed) & 1ull) ? 1.0f : -1.0f;
        for (size_t j = 0; j < n; ++j) {
            float a = row_major ? A[i * ld + j] : A[i + j * ld];
            acc[bkt + j * s] += sg * a;
        }
    }
    for (size_t e = 0; e < s * n; ++e) SA[e] = (double)acc[e];
    free(acc);
}

/* ---------------------------------------------------------------------
 * Householder QR, LAPACK dgeqr2/dlarfg convention (the reference calls
 * LAPACKE_dgeqrf at src/core/precond/sketch_qr.cpp:20-22,48): reflector
 * H_j = I - tau_j v_j v_j^T with v_j(0) = 1, R_jj = -sign(a_jj)*||a_j||.
 * ------------------------------------------------------------------- */
int or_householder_qr_f64(size_t m, size_t n, double* A, size_t ld, double* tau) {
    if (m < n) return -1;
    for (size_t j = 0; j < n; ++j) {
        double* col = A + j * ld;
        double alpha = col[j], xn = 0.0;
        for (size_t i = j + 1; i < m; ++i) xn = hypot(xn, col[i]);
        if (xn == 0.0) {
            tau[j] = 0.0;
            continue;
        }
        double beta = -copysign(hypot(alpha, xn), alpha);
        tau[j] = (beta - alpha) / beta;
        double sc = 1.0 / (alpha - beta);
        for (size_t i = j + 1; i < m; ++i) col[i] *= sc;
        col[j] = beta;
        for (size_t k = j + 1; k < n; ++k) {
            double* ck = A + k * ld;
            double w = ck[j];
            for (size_t i = j + 1; i < m; ++i) w += col[i] * ck[i];
            w *= tau[j];
            ck[j] -= w;
            for (size_t i = j + 1; i < m; ++i) ck[i] -= w * col[i];
        }
    }
    return 0;
}

/* Upper-triangular inverse (the reference's LAPACKE_dtrtri('U','N') step,
 * sketch_qr.cpp:27-29,59), by column-wise back substitution. */
int or_trtri_upper_f64(size_t n, const double* R, size_t ldr, double* Rinv, size_t ldi) {
    for (size_t j = 0; j < n; ++j)
        for (size_t i = 0; i < n; ++i) Rinv[i + j * ldi] = 0.0;
    for (size_t j = 0; j < n; ++j) {
        if (R[j + j * ldr] == 0.0) return -1;
        Rinv[j + j * ldi] = 1.0 / R[j + j * ldr];
        for (size_t ii = j; ii-- > 0;) {
            double acc = 0.0;
            for (size_t k = ii + 1; k <= j; ++k) acc += R[ii + k * ldr] * Rinv[k + j * ldi];
            Rinv[ii + j * ldi] = -acc / R[ii + ii * ldr];
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------
 * Plain LSQR (src/core/solver/lsqr.cpp).  FP32 vectors; BLAS-1 as the
 * reference's cblas_s* calls (float scale factors); GEMV accumulated in
 * double and rounded once; Givens scalars recomputed in double from the
 * float-stored LsqrScalars (lsqr_solver.hpp:42-45).
 * ------------------------------------------------------------------- */

/* y = alpha * op(A) x + beta * y, A m x n col-major FP32. */
static void sgemv(int trans, size_t m, size_t n, const float* A, size_t lda,
                  double alpha, const float* x, double beta, float* y) {
    size_t rows = trans ? n : m, cols = trans ? m : n;
    for (size_t i = 0; i < rows; ++i) {
        double acc = 0.0;
        for (size_t j = 0; j < cols; ++j) {
            float a = trans ? A[j + i * lda] : A[i + j * lda];
            acc += (double)a * (double)x[j];
        }
        y[i] = beta != 0.0 ? (float)(alpha * acc + beta * (double)y[i]) : (float)(alpha * acc);
    }
}
static double snrm2(size_t n, const float* x) {
    double acc = 0.0;
    for (size_t i = 0; i < n; ++i) acc += (double)x[i] * (double)x[i];
    return (double)(float)sqrt(acc);
}
static void sscal(size_t n, double a, float* x) {
    float fa = (float)a;
    for (size_t i = 0; i < n; ++i) x[i] *= fa;
}
static void saxpy(size_t n, double a, const float* x, float* y) {
    float fa = (float)a;
    for (size_t i = 0; i < n; ++i) y[i] += fa * x[i];
}

int or_lsqr_f32(size_t m, size_t n, const float* A, size_t lda, const float* b,
                float* x, const float* Rinv, double tol, int max_iters,
                double max_relres, int restarts, int* iterations, double* history) {
    float* u = (float*)calloc(m, sizeof(float));
    float* v = (float*)calloc(n, sizeof(float));
    float* w = (float*)calloc(n, sizeof(float));
    float* t1 = (float*)calloc(n, sizeof(float));
    float* pv = (float*)calloc(n, sizeof(float));
    if (!u || !v || !w || !t1 || !pv) return -1;
    int nhist = 0, done = 0;
    /* lsqr_registries.cpp:156 zeroes x before solving. */
    for (size_t j = 0; j < n; ++j) x[j] = 0.0f;
    double rhsnorm = snrm2(m, b);
    float s_alpha = 0.f, s_beta = 0.f, s_rho_bar = 0.f, s_phi_bar = 0.f;
    int completed = 0;
#define STOP_CHECK()                                                        \
    (completed == 0 ? 0                                                     \
     : rhsnorm == 0.0 ? 1                                                   \
     : (history ? (history[nhist++] = fabs((double)s_phi_bar) / rhsnorm) : 0, \
        fabs((double)s_phi_bar) / rhsnorm < tol ||                          \
            fabs((double)s_phi_bar) / rhsnorm < max_relres))
    for (int rs = 0; rs < restarts && !done; ++rs) {
        if (STOP_CHECK()) break;
        /* initialize(), lsqr.cpp:432-513: u = b - A x, restarted from x. */
        memcpy(u, b, m * sizeof(float));
        sgemv(0, m, n, A, lda, -1.0, x, 1.0, u);
        double beta = snrm2(m, u);
        sscal(m, 1.0 / beta, u);
        if (Rinv) {
            sgemv(1, m, n, A, lda, 1.0, u, 0.0, t1);
            sgemv(1, n, n, Rinv, n, 1.0, t1, 0.0, v);
        } else {
            sgemv(1, m, n, A, lda, 1.0, u, 0.0, v);
        }
        double alpha = snrm2(n, v);
        sscal(n, 1.0 / alpha, v);
        memcpy(w, v, n * sizeof(float));
        s_alpha = (float)alpha; s_beta = (float)beta;
        s_rho_bar = (float)alpha; s_phi_bar = (float)beta;
        /* fused_lsqr_impl's restart-boundary true-residual check, :723-729. */
        if (rhsnorm == 0.0) break;
        double true_relres = (double)s_beta / rhsnorm;
        if (true_relres < tol || true_relres < max_relres) break;
        for (int it = 0; it < max_iters; ++it) {
            /* step_1_orth_basis, lsqr.cpp:521-626. */
            alpha = (double)s_alpha;
            if (Rinv) {
                sgemv(0, n, n, Rinv, n, 1.0, v, 0.0, pv);
                sgemv(0, m, n, A, lda, 1.0, pv, -alpha, u);
                beta = snrm2(m, u);
                sscal(m, 1.0 / beta, u);
                sgemv(1, m, n, A, lda, 1.0, u, 0.0, t1);
                sgemv(1, n, n, Rinv, n, 1.0, t1, 0.0, pv);
                saxpy(n, -beta, v, pv);
                alpha = snrm2(n, pv);
                sscal(n, 1.0 / alpha, pv);
                memcpy(v, pv, n * sizeof(float));
            } else {
                memcpy(t1, v, n * sizeof(float));
                sgemv(0, m, n, A, lda, 1.0, t1, -alpha, u);
                beta = snrm2(m, u);
                sscal(m, 1.0 / beta, u);
                sgemv(1, m, n, A, lda, 1.0, u, 0.0, t1);
                saxpy(n, -beta, v, t1);
                alpha = snrm2(n, t1);
                sscal(n, 1.0 / alpha, t1);
                memcpy(v, t1, n * sizeof(float));
            }
            s_alpha = (float)alpha; s_beta = (float)beta;
            /* step_2_update_sol, lsqr.cpp:633-679. */
            double rho_bar = s_rho_bar, phi_bar = s_phi_bar;
            double a = s_alpha, bb = s_beta;
            double rho = hypot(rho_bar, bb);
            double c = rho_bar / rho, s = bb / rho;
            double theta = s * a;
            rho_bar = -c * a;
            double phi = c * phi_bar;
            phi_bar = s * phi_bar;
            if (Rinv) {
                sgemv(0, n, n, Rinv, n, 1.0, w, 0.0, pv);
                saxpy(n, phi / rho, pv, x);
            } else {
                saxpy(n, phi / rho, w, x);
            }
            sscal(n, -theta / rho, w);
            saxpy(n, 1.0, v, w);
            s_rho_bar = (float)rho_bar; s_phi_bar = (float)phi_bar;
            completed += 1;
            if (STOP_CHECK()) { done = 1; break; }
        }
    }
#undef STOP_CHECK
    if (iterations) *iterations = completed;
    free(u); free(v); free(w); free(t1); free(pv);
    return nhist;
}
