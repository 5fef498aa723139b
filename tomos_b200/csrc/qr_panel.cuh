// qr_panel.cuh -- Householder panel factorisation of the sketch QR by
// Cholesky QR and Householder reconstruction, in FP64.
//
// A panel P (k_rem x nb, nb <= 32) of the blocked Householder QR is
// factored in three row-parallel passes instead of nb column steps:
//
//   1. G1 = P^T P (partials written by the previous trailing update),
//      D = diag(G1)^1/2, D^-1 G1 D^-1 = Rh^T Rh, R1 = Rh D;
//      Q1 = P R1^-1 and G2 = Q1^T Q1                       (qr_hr_q1_kernel)
//   2. G2 = R2^T R2 (Cholesky QR, second pass: Q = Q1 R2^-1 is orthonormal
//      to working precision for cond(P D^-1) up to ~1e7), R = R2 R1;
//      Householder reconstruction: the LU factorisation without pivoting
//      Q_top - S = L U with s_i = -sign of the pivot (so |U_ii| in [1, 2])
//      gives the reflectors of LAPACK's dgeqr2 on P exactly:
//         V = [L; Q_bot U^-1],  T = -U S L^-T,  tau = diag(T),  R_h = S R
//      (Q_house = Q S; s_i = -sign(alpha_i) is dlarfg's beta sign, and
//      tau = 1 + |q_ii| lies in [1, 2] as dlarfg's does)    (qr_hr_v_kernel)
//
// Every CTA of a pass repeats the 32 x 32 work (the whole CTA, shared
// memory) on the same inputs in the same order, so they agree bit for bit
// and no grid-wide exchange is needed.  When either Cholesky meets a pivot below
// its floor (a panel too ill-conditioned for Cholesky QR, or a zero
// column), the panel is factored by plain Householder column steps in one
// CTA instead (qr_hr_v_kernel's fallback), from the untouched panel: pass
// 1 writes Q1 to scratch, never into A.
//
// Matrices are 32 x 32 in shared memory as m[row][col] with a padding
// column; a panel narrower than 32 is padded with the identity, which
// every step below keeps block-diagonal, so the padding never mixes into
// the leading nb x nb results.
#pragma once

#include "common.cuh"

namespace tomos_b200 {

constexpr int kHB = 32;
typedef double HMat[kHB][kHB + 1];

// The 32 x 32 steps below run on the whole CTA (256 threads).  Cholesky and
// the signed LU are right-looking: per column a pivot, a scaled row or
// column, and the trailing update spread over all threads.  Triangular
// inverses double the solved block size 1 -> 2 -> ... -> 32, each level two
// small block products (X_IJ = -X_II R_IJ X_JJ).

// G (symmetric, upper half read) = R^T R with R upper; G is left as it
// was.  Returns false if a pivot is not above `floor` (or not finite).
// Warp 0 runs the 32 right-looking steps on registers: lane l holds column
// l of G, row j of R reaches the other lanes by shuffles (the other warps
// wait at the end).
// (Not inlined: inside the one-launch QR the kernel's register pressure
// would otherwise put the lane's 32 values in local memory.)
__device__ __noinline__ bool cta_chol(const HMat& G, HMat& R, double floor, int* okf) {
    const int t = threadIdx.x;
    __syncthreads();
    if (t < 32) {
        const int l = t;
        double g[kHB];
#pragma unroll
        for (int i = 0; i < kHB; ++i) g[i] = G[i][l];
        int ok = 1;
#pragma unroll
        for (int j = 0; j < kHB; ++j) {
            const double d = __shfl_sync(0xffffffffu, g[j], j);
            const bool good = d > floor && isfinite(d);
            if (!good) ok = 0;
            // one reciprocal square root on the step's critical path:
            // R(j, j) = d / sqrt(d), R(j, l) = G(j, l) / sqrt(d)
            const double dd = good ? d : 1.0;
            const double ri = rsqrt(dd);
            const double rjl = l > j ? g[j] * ri : (l == j ? dd * ri : 0.0);
            R[j][l] = rjl;
            // G(i, l) -= R(j, i) R(j, l) for j < i <= l (entries below the
            // diagonal of G are never read)
#pragma unroll
            for (int i = j + 1; i < kHB; ++i) g[i] -= __shfl_sync(0xffffffffu, rjl, i) * rjl;
        }
        if (l == 0) *okf = ok;
    }
    __syncthreads();
    return *okf != 0;
}

// X = R^{-1} for upper triangular R (X must not alias R; Tmp is scratch).
// A level of block size b has kHB / (2b) pairs (I, J) of b x b blocks,
// I = [2bp, 2bp + b), J = [2bp + b, 2bp + 2b): X_IJ = -X_II (R_IJ X_JJ).
__device__ __forceinline__ void cta_inv_upper(const HMat& R, HMat& X, HMat& Tmp) {
    const int t = threadIdx.x;
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int i = e >> 5, j = e & 31;
        X[i][j] = i == j ? 1.0 / R[i][i] : 0.0;
    }
    for (int b = 1; b < kHB; b *= 2) {
        const int entries = kHB * b / 2;
        __syncthreads();
        for (int e = t; e < entries; e += blockDim.x) {
            const int p = e / (b * b), r = e % (b * b);
            const int i0 = 2 * b * p, i = i0 + r / b, j = i0 + b + r % b;
            double s = 0.0;
            for (int k = i0 + b; k <= j; ++k) s += R[i][k] * X[k][j];
            Tmp[i][j] = s;
        }
        __syncthreads();
        for (int e = t; e < entries; e += blockDim.x) {
            const int p = e / (b * b), r = e % (b * b);
            const int i0 = 2 * b * p, i = i0 + r / b, j = i0 + b + r % b;
            double s = 0.0;
            for (int k = i; k < i0 + b; ++k) s += X[i][k] * Tmp[k][j];
            X[i][j] = -s;
        }
    }
    __syncthreads();
}

// Y = L^{-1} for the unit lower triangular L held strictly below the
// diagonal of Q (Tmp is scratch).  Same levels with the blocks transposed:
// Y_JI = -Y_JJ (L_JI Y_II).
__device__ __forceinline__ void cta_inv_unit_lower(const HMat& Q, HMat& Y, HMat& Tmp) {
    const int t = threadIdx.x;
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int i = e >> 5, j = e & 31;
        Y[i][j] = i == j ? 1.0 : 0.0;
    }
    for (int b = 1; b < kHB; b *= 2) {
        const int entries = kHB * b / 2;
        __syncthreads();
        for (int e = t; e < entries; e += blockDim.x) {
            const int p = e / (b * b), r = e % (b * b);
            const int j0 = 2 * b * p, i = j0 + b + r / b, j = j0 + r % b;  // i in J, j in I
            double s = 0.0;
            for (int k = j; k < j0 + b; ++k) s += Q[i][k] * Y[k][j];
            Tmp[i][j] = s;
        }
        __syncthreads();
        for (int e = t; e < entries; e += blockDim.x) {
            const int p = e / (b * b), r = e % (b * b);
            const int j0 = 2 * b * p, i = j0 + b + r / b, j = j0 + r % b;
            double s = 0.0;
            for (int k = j0 + b; k <= i; ++k) s += Y[i][k] * Tmp[k][j];
            Y[i][j] = -s;
        }
    }
    __syncthreads();
}

// In place: Q - S = L U without pivoting, s_i = -sign(pivot) (sign(+0) =
// +1, as dlarfg's copysign); L strictly below the diagonal, U on and
// above it.  Step `keep` (if >= 0) is a reflector with nothing below its
// diagonal, which dlarfg leaves as the identity (tau = 0, R_jj = alpha):
// there s = +sign(pivot).  Warp 0 runs the 32 steps on registers: lane l
// holds row l, row i of U reaches the other lanes by shuffles.
__device__ __noinline__ void cta_lu_signed(HMat& Q, double* sgn, int keep) {
    __syncthreads();
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        double q[kHB];
#pragma unroll
        for (int c = 0; c < kHB; ++c) q[c] = Q[l][c];
#pragma unroll
        for (int i = 0; i < kHB; ++i) {
            const double qii = __shfl_sync(0xffffffffu, q[i], i);
            double si = qii >= 0.0 ? -1.0 : 1.0;
            if (i == keep) si = -si;
            const double u = qii - si;
            if (l == 0) sgn[i] = si;
            if (l == i) q[i] = u;
            const bool below = l > i;
            // 1/u with |u| in [1, 2] (|u| = |q_ii| + 1): the hardware's
            // approximate float reciprocal and two Newton steps in FP64 (no
            // division, whose out-of-line path is costly in this kernel)
            float uf;
            asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(uf) : "f"((float)u));
            double ui = (double)uf;
            ui = fma(ui, fma(-u, ui, 1.0), ui);
            ui = fma(ui, fma(-u, ui, 1.0), ui);
            if (u == 0.0) ui = 0.0;
            const double lm = below ? q[i] * ui : 0.0;
            if (below) q[i] = lm;
#pragma unroll
            for (int c = i + 1; c < kHB; ++c) {
                const double uic = __shfl_sync(0xffffffffu, q[c], i);
                if (below) q[c] -= lm * uic;
            }
        }
#pragma unroll
        for (int c = 0; c < kHB; ++c) Q[l][c] = q[c];
    }
    __syncthreads();
}

// C = A B over the whole CTA (256 threads, 4 entries each).
__device__ __forceinline__ void cta_mul(const HMat& A, const HMat& B, HMat& C) {
    const int t = threadIdx.x;
    const int i = t & 31, j0 = (t >> 5) * 4;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < kHB; ++k) {
        const double a = A[i][k];
#pragma unroll
        for (int q = 0; q < 4; ++q) s[q] += a * B[k][j0 + q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) C[i][j0 + q] = s[q];
}

struct HrArgs {
    double* A;          // the k x n matrix being factored (column-major)
    int64_t ld, k, j0;  // panel starts at (j0, j0)
    int nb;             // panel width
    int64_t rpc;        // panel rows per CTA (multiple of 32)
    const double* Gp;   // G1 partials (ngp x 32 x 32)
    int ngp;
    double* Qs;         // Q1 scratch, column-major k_rem x 32 (ld kq)
    int64_t kq;
    double* G2p;        // G2 partials (one per CTA of the panel passes)
    double* R1;         // 32 x 32 (row-major [i * 32 + j])
    int* fail;          // nonzero: fall back to Householder column steps
    double* T;          // nb x nb, T(a, b) at T[b * nb + a]
    double* tau;        // n
};

// Panel rows of CTA `cta` of the panel passes, [r0, r1) relative to j0.
__device__ __forceinline__ void hr_rows(const HrArgs& H, int cta, int64_t& r0, int64_t& r1) {
    const int64_t krem = H.k - H.j0;
    r0 = (int64_t)cta * H.rpc;
    r1 = r0 + H.rpc;
    if (r1 > krem) r1 = krem;
    if (r0 > krem) r0 = krem;
}

// Sums `np` 32 x 32 partials in order into G and pads it with the
// identity outside the leading nb x nb block.  blockDim.x == 256: four
// entries a thread, 64 loads in flight.
__device__ __forceinline__ void hr_reduce_gram(const double* part, int np, int nb, HMat& G) {
    const int t = threadIdx.x;
    bool in[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int e = t + 256 * c;
        in[c] = (e >> 5) < nb && (e & 31) < nb;
    }
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int p0 = 0; p0 < np; p0 += 16) {
        double v[16][4];
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                v[u][c] = (p0 + u < np && in[c]) ? __ldcg(part + (size_t)(p0 + u) * kHB * kHB + t + 256 * c) : 0.0;
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 4; ++c) s[c] += v[u][c];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int e = t + 256 * c, i = e >> 5, j = e & 31;
        G[i][j] = in[c] ? s[c] : (i == j ? 1.0 : 0.0);
    }
    __syncthreads();
}

// Pass 1: R1 from the G1 partials, Q1 = P R1^-1 into Qs, G2 partials.
// CTA `cta` of the pass (0 writes R1 and the fallback flag).
__device__ void hr_q1(const HrArgs& H, int cta, double* hsm) {
    HMat& G = *reinterpret_cast<HMat*>(hsm);
    HMat& R = *reinterpret_cast<HMat*>(hsm + 1 * kHB * (kHB + 1));
    HMat& X = *reinterpret_cast<HMat*>(hsm + 2 * kHB * (kHB + 1));
    HMat& Pt = *reinterpret_cast<HMat*>(hsm + 3 * kHB * (kHB + 1));
    double* dsc = hsm + 4 * kHB * (kHB + 1);  // 32 column scales
    __shared__ int okflag;
    const int t = threadIdx.x;
    const int nb = H.nb;

    hr_reduce_gram(H.Gp, H.ngp, nb, G);
    // D = diag(G1)^1/2 (dsc) and D^-1 (dinv, by rsqrt: no division)
    double* dinv = dsc + kHB;
    if (t < kHB) {
        const double g = G[t][t];
        const bool ok = t < nb && g > 0.0 && isfinite(g);
        const double ri = ok ? rsqrt(g) : 1.0;
        dinv[t] = ri;
        dsc[t] = ok ? g * ri : 1.0;
        if (t < nb && !ok) G[t][t] = 0.0;  // forces the fallback
    }
    __syncthreads();
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int i = e >> 5, j = e & 31;
        if (i < nb && j < nb) G[i][j] = G[i][j] * dinv[i] * dinv[j];
    }
    __syncthreads();
    cta_chol(G, R, 1e-12, &okflag);
    cta_inv_upper(R, X, Pt);
    // R1 = Rh D (columns scaled), R1^-1 = D^-1 Rh^-1 (rows scaled)
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int i = e >> 5, j = e & 31;
        R[i][j] *= dsc[j];
        X[i][j] *= dinv[i];
    }
    __syncthreads();
    if (cta == 0) {
        for (int e = t; e < kHB * kHB; e += blockDim.x) H.R1[e] = R[e >> 5][e & 31];
        if (t == 0) *H.fail = okflag ? 0 : 1;
    }
    double* g2 = H.G2p + (size_t)cta * kHB * kHB;
    if (!okflag) return;

    int64_t r0, r1;
    hr_rows(H, cta, r0, r1);
    const int i = t & 31, c0 = (t >> 5) * 4;  // Q1 tile: row i, columns c0..c0+3
    double acc[4] = {0.0, 0.0, 0.0, 0.0};     // G2 partial: (a = i, b = c0..c0+3)
    // The next 32-row panel tile is loaded while the current one is used
    // (blockDim.x == 256: four entries a thread).
    double pre[4];
    auto fetch = [&](int64_t rt) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = t + u * 256, r = e & 31, c = e >> 5;
            const int64_t row = rt + r;
            pre[u] = (row < r1 && c < nb) ? __ldcg(H.A + (size_t)(H.j0 + c) * H.ld + H.j0 + row) : 0.0;
        }
    };
    if (r0 < r1) fetch(r0);
    for (int64_t rt = r0; rt < r1; rt += kHB) {
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = t + u * 256;
            Pt[e & 31][e >> 5] = pre[u];
        }
        if (rt + kHB < r1) fetch(rt + kHB);
        __syncthreads();
        double q[4] = {0.0, 0.0, 0.0, 0.0};
        for (int kk = 0; kk < kHB; ++kk) {
            const double p = Pt[i][kk];
#pragma unroll
            for (int u = 0; u < 4; ++u) q[u] += p * X[kk][c0 + u];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) Pt[i][c0 + u] = q[u];
        __syncthreads();
        for (int e = t; e < kHB * kHB; e += blockDim.x) {
            const int r = e & 31, c = e >> 5;
            const int64_t row = rt + r;
            if (row < r1) H.Qs[(size_t)c * H.kq + row] = Pt[r][c];
        }
        for (int r = 0; r < kHB; ++r) {
            const double a = Pt[r][i];
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[u] += a * Pt[r][c0 + u];
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) g2[i * kHB + c0 + u] = acc[u];
}

// One CTA: Householder column steps (dgeqr2) on the untouched panel, then
// T (dlarft), for panels Cholesky QR cannot take.
__device__ void hr_fallback_panel(const HrArgs& H, HMat& Gram, HMat& Tm, double* red, double* bc) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nwarp = blockDim.x >> 5;
    const int nb = H.nb;
    const int64_t krem = H.k - H.j0;
    auto col = [&](int c) { return H.A + (size_t)(H.j0 + c) * H.ld + H.j0; };
    __shared__ double taul[kHB];
    __shared__ double wsum[kHB];
    for (int j = 0; j < nb; ++j) {
        double* a = col(j);
        double ss = 0.0;
        for (int64_t r = j + 1 + t; r < krem; r += blockDim.x) {
            const double v = __ldcg(a + r);
            ss += v * v;
        }
        ss = warp_sum(ss);
        if (lane == 0) red[warp] = ss;
        __syncthreads();
        if (t == 0) {
            double xn2 = 0.0;
            for (int w = 0; w < nwarp; ++w) xn2 += red[w];
            const double alpha = __ldcg(a + j);
            double tau = 0.0, beta = alpha, scal = 0.0;
            if (xn2 > 0.0) {
                beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                tau = (beta - alpha) / beta;
                scal = 1.0 / (alpha - beta);
            }
            bc[0] = tau;
            bc[1] = beta;
            bc[2] = scal;
        }
        __syncthreads();
        const double tau = bc[0], beta = bc[1], scal = bc[2];
        for (int64_t r = j + 1 + t; r < krem; r += blockDim.x) a[r] = __ldcg(a + r) * scal;
        __syncthreads();
        if (t == 0) {
            a[j] = beta;
            taul[j] = tau;
            H.tau[H.j0 + j] = tau;
        }
        // w_c = v^T a_c for the later columns, then a_c -= tau w_c v
        for (int c = j + 1 + warp; c < nb; c += nwarp) {
            const double* ac = col(c);
            double w = lane == 0 ? __ldcg(ac + j) : 0.0;
            for (int64_t r = j + 1 + lane; r < krem; r += 32) w += __ldcg(a + r) * __ldcg(ac + r);
            w = warp_sum(w);
            if (lane == 0) wsum[c] = w;
        }
        __syncthreads();
        for (int c = j + 1 + warp; c < nb; c += nwarp) {
            double* ac = col(c);
            const double tw = tau * wsum[c];
            if (lane == 0) ac[j] = __ldcg(ac + j) - tw;
            for (int64_t r = j + 1 + lane; r < krem; r += 32) ac[r] = __ldcg(ac + r) - tw * __ldcg(a + r);
        }
        __syncthreads();
    }
    // Gram of V (unit diagonal, zeros above), then T column by column.
    for (int e = warp; e < nb * nb; e += nwarp) {
        const int x = e % nb, y = e / nb;
        double g = 0.0;
        if (x < y) {
            const double* vx = col(x);
            const double* vy = col(y);
            for (int64_t r = y + lane; r < krem; r += 32) {
                const double ex = r == x ? 1.0 : __ldcg(vx + r);
                const double ey = r == y ? 1.0 : __ldcg(vy + r);
                g += ex * ey;
            }
            g = warp_sum(g);
        }
        if (lane == 0) Gram[x][y] = g;
    }
    __syncthreads();
    if (warp == 0) {
        // T(0:j, j) = -tau_j T(0:j, 0:j) Gram(0:j, j), T_jj = tau_j (dlarft)
        for (int i = 0; i < kHB; ++i) Tm[i][lane] = 0.0;
        __syncwarp();
        for (int j = 0; j < nb; ++j) {
            double tij = 0.0;
            if (lane < j) {
                double s2 = 0.0;
                for (int l = lane; l < j; ++l) s2 += Tm[lane][l] * Gram[l][j];
                tij = -taul[j] * s2;
            }
            __syncwarp();
            if (lane < j) Tm[lane][j] = tij;
            if (lane == j) Tm[j][j] = taul[j];
            __syncwarp();
        }
    }
    __syncthreads();
    for (int e = t; e < nb * nb; e += blockDim.x) {
        const int i = e % nb, j = e / nb;
        H.T[(size_t)j * nb + i] = Tm[i][j];
    }
}

// Pass 2: R2, the reconstruction (every CTA of the pass), the top block,
// T and tau (CTA `top`) and V below the top block (each CTA its rows);
// `ncta` CTAs ran pass 1 (its G2 partials).  A `top` CTA past them has no
// rows and does only the top block, beside the others' rows.
__device__ void hr_v(const HrArgs& H, int cta, int ncta, int top, double* hsm) {
    constexpr int MS = kHB * (kHB + 1);
    HMat& G = *reinterpret_cast<HMat*>(hsm);
    HMat& R2 = *reinterpret_cast<HMat*>(hsm + 1 * MS);
    HMat& X2 = *reinterpret_cast<HMat*>(hsm + 2 * MS);
    HMat& Qt = *reinterpret_cast<HMat*>(hsm + 3 * MS);
    HMat& Ui = *reinterpret_cast<HMat*>(hsm + 4 * MS);
    HMat& M = *reinterpret_cast<HMat*>(hsm + 5 * MS);
    double* sgn = hsm + 6 * MS;
    double* red = sgn + kHB;
    double* bc = red + kHB;
    __shared__ int okflag;
    const int t = threadIdx.x;
    const int nb = H.nb;

    bool ok = __ldcg(H.fail) == 0;
    if (ok) {
        hr_reduce_gram(H.G2p, ncta, nb, G);
        ok = cta_chol(G, R2, 0.25, &okflag);
        cta_inv_upper(R2, X2, Qt);
    }
    if (!ok) {
        if (cta == 0) hr_fallback_panel(H, G, R2, red, bc);
        return;
    }
    // Q_top = Q1_top R2^-1 (identity padding), then Q_top - S = L U.
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int r = e & 31, c = e >> 5;
        G[r][c] = (r < nb && c < nb) ? __ldcg(H.Qs + (size_t)c * H.kq + r) : (r == c ? 1.0 : 0.0);
    }
    __syncthreads();
    cta_mul(G, X2, Qt);
    __syncthreads();
    // The last column of a square matrix has no rows below its diagonal.
    const int keep = (H.k - H.j0 == nb) ? nb - 1 : -1;
    cta_lu_signed(Qt, sgn, keep);
    const bool rows = cta < ncta;
    if (rows) {
        // U^-1: U is the upper part of Qt (diagonal included)
        for (int e = t; e < kHB * kHB; e += blockDim.x) {
            const int i = e >> 5, j = e & 31;
            G[i][j] = i <= j ? Qt[i][j] : 0.0;
        }
        __syncthreads();
        cta_inv_upper(G, Ui, M);
        cta_mul(X2, Ui, M);  // V2 = Q1_bot R2^-1 U^-1
        __syncthreads();
    }

    if (cta == top) {
        // Y = L^-1 into G; T = -U S Y^T; R = R2 R1 -> R_h = S R.
        cta_inv_unit_lower(Qt, G, X2);
        for (int e = t; e < kHB * kHB; e += blockDim.x) X2[e >> 5][e & 31] = __ldcg(H.R1 + e);
        for (int e = t; e < nb * nb; e += blockDim.x) {
            const int i = e % nb, j = e / nb;
            // T(i, j) = -sum_k U(i, k) s_k Y(j, k), U(i, k) = Qt[i][k] for k >= i
            double s = 0.0;
            if (i <= j && j != keep)
                for (int k = i; k <= j; ++k) s += Qt[i][k] * sgn[k] * G[j][k];
            H.T[(size_t)j * nb + i] = -s + 0.0;
            if (i == j) H.tau[H.j0 + i] = -s + 0.0;
        }
        // R = R2 R1 into Ui (R1 in X2), then the top block:
        // R_h = S R on and above the diagonal, L strictly below.
        __syncthreads();
        for (int e = t; e < kHB * kHB; e += blockDim.x) {
            const int i = e >> 5, j = e & 31;
            double s = 0.0;
            for (int k = i; k <= j; ++k) s += R2[i][k] * X2[k][j];
            Ui[i][j] = i <= j ? s : 0.0;
        }
        __syncthreads();
        for (int e = t; e < nb * nb; e += blockDim.x) {
            const int i = e % nb, j = e / nb;
            const double v = i <= j ? sgn[i] * Ui[i][j] : Qt[i][j];
            H.A[(size_t)(H.j0 + j) * H.ld + H.j0 + i] = v;
        }
    }
    if (!rows) return;
    // V2 rows: local rows >= nb of this CTA's block.
    int64_t r0, r1;
    hr_rows(H, cta, r0, r1);
    if (r0 < nb) r0 = nb;
    HMat& Pt = G;
    const int i = t & 31, c0 = (t >> 5) * 4;
    double pre[4];  // the next Q1 tile (blockDim.x == 256: four entries a thread)
    auto fetch = [&](int64_t rt) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = t + u * 256, r = e & 31, c = e >> 5;
            const int64_t row = rt + r;
            pre[u] = (row < r1 && c < nb) ? __ldcg(H.Qs + (size_t)c * H.kq + row) : 0.0;
        }
    };
    if (r0 < r1) fetch(r0);
    for (int64_t rt = r0; rt < r1; rt += kHB) {
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = t + u * 256;
            Pt[e & 31][e >> 5] = pre[u];
        }
        if (rt + kHB < r1) fetch(rt + kHB);
        __syncthreads();
        double q[4] = {0.0, 0.0, 0.0, 0.0};
        for (int kk = 0; kk < kHB; ++kk) {
            const double p = Pt[i][kk];
#pragma unroll
            for (int u = 0; u < 4; ++u) q[u] += p * M[kk][c0 + u];
        }
        const int64_t row = rt + i;
        if (row < r1) {
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (c0 + u < nb) H.A[(size_t)(H.j0 + c0 + u) * H.ld + H.j0 + row] = q[u];
        }
    }
}

__global__ void __launch_bounds__(256) qr_hr_q1_kernel(HrArgs H) {
    extern __shared__ __align__(16) double hsm[];
    hr_q1(H, blockIdx.x, hsm);
}

__global__ void __launch_bounds__(256) qr_hr_v_kernel(HrArgs H) {
    extern __shared__ __align__(16) double hsm[];
    hr_v(H, blockIdx.x, gridDim.x, 0, hsm);
}

inline size_t hr_q1_smem() { return (4 * kHB * (kHB + 1) + 2 * kHB) * sizeof(double); }
inline size_t hr_v_smem() { return (6 * kHB * (kHB + 1) + 3 * kHB + 8) * sizeof(double); }

}  // namespace tomos_b200
