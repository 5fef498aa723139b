// qr_gemm.cuh -- FP64 products of the blocked QR on the tensor cores
// (mma.sync m16n8k8 f64), and the pieces that turn a block of panels into
// one compact-WY transform.
//
// A block of kQrBlock columns is factored panel by panel (32 columns, the
// trailing update restricted to the block); its reflectors V (k_rem x 256)
// and the panels' 32 x 32 factors T_p then make the block's
// H_1 ... H_256 = I - V T V^T, with T upper triangular and
//   T = [[T_<j, -T_<j (V_<j^T V_j) T_j], [0, T_j]]    (j = 1 .. 7),
// and the columns right of the block get C <- (I - V T^T V^T) C as three
// products: Z = V T, W = Z^T C, C -= V W.  Each reads C once per block
// instead of twice per panel.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "mbarrier.cuh"  // smem_addr

namespace tomos_b200 {

constexpr int kQrBlock = 256;     // columns per block of the blocked QR
constexpr int kGbm = 128;         // GEMM CTA tile rows
constexpr int kGbn = 64;          // GEMM CTA tile columns
constexpr int kGbk = 16;          // k per stage
constexpr int kGpad = 4;          // row padding (doubles) of the stage tiles
constexpr int kGstages = 3;
constexpr int kGmaxSplits = 16;
constexpr int kGa = kGbm * (kGbk + kGpad) > kGbk * (kGbm + kGpad) ? kGbm * (kGbk + kGpad)
                                                                 : kGbk * (kGbm + kGpad);
constexpr int kGb = kGbn * (kGbk + kGpad);
constexpr int kGstage = kGa + kGb;
constexpr size_t kGemmSmem = sizeof(double) * kGstage * kGstages;

__device__ __forceinline__ void g_cp_async8(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void g_cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void g_cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// D += A B for one m16n8k8 FP64 tile: with g = lane / 4, q = lane % 4,
// a = A[g][q], A[g + 8][q], A[g][q + 4], A[g + 8][q + 4]; b = B[q][g],
// B[q + 4][g]; d = D[g][2q], D[g][2q + 1], D[g + 8][2q], D[g + 8][2q + 1].
__device__ __forceinline__ void g_dmma1688(double* d, const double* a, const double* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// D (M x N, column-major, ld ldd) = alpha * op(A) B + beta * D, B
// column-major K x N.  KMAJOR: op(A) = A^T with A column-major K x M;
// otherwise A is column-major M x K.  CTA tile 128 x 64, k-steps of 16
// through kGstages shared-memory stages filled by 8-byte asynchronous
// copies (zero-filled past the edges); 8 warps, each 32 x 32 = two by
// four m16n8k8 tiles.  Split-K: CTA z sums k in [z kc, (z + 1) kc); with
// gridDim.z > 1 it writes its partial to P + z M N (ld M) for
// qr_gemm_reduce_kernel.  sub: D -= op(A) B instead (alpha and beta
// unused): the accumulators start from the D tile, loaded while the first
// stages are in flight, and A enters negated.
struct GemmArgs {
    const double* A;
    int64_t lda;
    const double* B;
    int64_t ldb;
    double* D;
    int64_t ldd;
    double* P;
    int64_t M, N, K, kc;
    double alpha, beta;
    int sub;
    int upper;  // skip the tiles wholly below the diagonal (a symmetric product's other half)
};

template <bool KMAJOR>
__global__ void __launch_bounds__(256, 2) qr_gemm_kernel(GemmArgs g) {
    extern __shared__ __align__(16) double gsm[];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int gq = lane >> 2, qq = lane & 3;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
    const int64_t m0 = (int64_t)blockIdx.x * kGbm, n0 = (int64_t)blockIdx.y * kGbn;
    if (g.upper && m0 > n0 + kGbn - 1) return;
    const int64_t kb = (int64_t)blockIdx.z * g.kc;
    const int64_t ke = kb + g.kc < g.K ? kb + g.kc : g.K;
    const int nk = ke > kb ? (int)((ke - kb + kGbk - 1) / kGbk) : 0;
    auto issue = [&](int s, int64_t k0) {
        double* As = gsm + s * kGstage;
        double* Bs = As + kGa;
#pragma unroll
        for (int i = 0; i < kGbm * kGbk / 256; ++i) {
            const int e = t + i * 256;
            int m, kk;
            if (KMAJOR) {
                m = e >> 4;
                kk = e & 15;
            } else {
                m = e & (kGbm - 1);
                kk = e >> 7;
            }
            const int64_t gm = m0 + m, gk = k0 + kk;
            const bool ok = gm < g.M && gk < ke;
            const double* src = KMAJOR ? g.A + gk + gm * g.lda : g.A + gm + gk * g.lda;
            double* dst = KMAJOR ? As + m * (kGbk + kGpad) + kk : As + kk * (kGbm + kGpad) + m;
            g_cp_async8(dst, ok ? src : g.A, ok);
        }
#pragma unroll
        for (int i = 0; i < kGbn * kGbk / 256; ++i) {
            const int e = t + i * 256, nn = e >> 4, kk = e & 15;
            const int64_t gn = n0 + nn, gk = k0 + kk;
            const bool ok = gn < g.N && gk < ke;
            g_cp_async8(Bs + nn * (kGbk + kGpad) + kk, ok ? g.B + gk + gn * g.ldb : g.B, ok);
        }
        g_cp_async_commit();
    };
    double acc[2][4][4];
#pragma unroll
    for (int s = 0; s < kGstages - 1; ++s) {
        if (s < nk) issue(s, kb + (int64_t)s * kGbk);
        else g_cp_async_commit();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t row = m0 + wm + a * 16 + gq + 8 * (u >> 1);
                const int64_t col = n0 + wn + b * 8 + 2 * qq + (u & 1);
                acc[a][b][u] = (g.sub && row < g.M && col < g.N) ? g.D[row + col * g.ldd] : 0.0;
            }
    const double asg = g.sub ? -1.0 : 1.0;
    for (int i = 0; i < nk; ++i) {
        const int ni = i + kGstages - 1;
        if (ni < nk) issue(ni % kGstages, kb + (int64_t)ni * kGbk);
        else g_cp_async_commit();
        g_cp_async_wait<kGstages - 1>();
        __syncthreads();
        const double* As = gsm + (i % kGstages) * kGstage;
        const double* Bs = As + kGa;
#pragma unroll
        for (int ks = 0; ks < kGbk / 8; ++ks) {
            double a[2][4], b[4][2];
#pragma unroll
            for (int im = 0; im < 2; ++im)
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int row = wm + im * 16 + gq + 8 * (u & 1), kk = ks * 8 + qq + 4 * (u >> 1);
                    a[im][u] = asg * (KMAJOR ? As[row * (kGbk + kGpad) + kk] : As[kk * (kGbm + kGpad) + row]);
                }
#pragma unroll
            for (int in = 0; in < 4; ++in)
#pragma unroll
                for (int u = 0; u < 2; ++u)
                    b[in][u] = Bs[(wn + in * 8 + gq) * (kGbk + kGpad) + ks * 8 + qq + 4 * u];
#pragma unroll
            for (int im = 0; im < 2; ++im)
#pragma unroll
                for (int in = 0; in < 4; ++in) g_dmma1688(acc[im][in], a[im], b[in]);
        }
        __syncthreads();  // the stage is refilled kGstages - 1 steps on
    }
    g_cp_async_wait<0>();
    const bool split = gridDim.z > 1;
#pragma unroll
    for (int im = 0; im < 2; ++im)
#pragma unroll
        for (int in = 0; in < 4; ++in)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t row = m0 + wm + im * 16 + gq + 8 * (u >> 1);
                const int64_t col = n0 + wn + in * 8 + 2 * qq + (u & 1);
                if (row >= g.M || col >= g.N) continue;
                if (split) {
                    g.P[(size_t)blockIdx.z * g.M * g.N + row + col * g.M] = acc[im][in][u];
                } else if (g.sub) {
                    g.D[row + col * g.ldd] = acc[im][in][u];
                } else {
                    double v = g.alpha * acc[im][in][u];
                    if (g.beta != 0.0) v += g.beta * g.D[row + col * g.ldd];
                    g.D[row + col * g.ldd] = v;
                }
            }
}

// D = alpha * sum_z P[z] + beta * D, the splits summed in order.
__global__ void qr_gemm_reduce_kernel(const double* __restrict__ P, int splits, int64_t M, int64_t N,
                                      double alpha, double beta, double* __restrict__ D, int64_t ldd) {
    const int64_t total = M * N;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < splits; ++z) s += P[(size_t)z * total + e];
        const int64_t row = e % M, col = e / M;
        double v = alpha * s;
        if (beta != 0.0) v += beta * D[row + col * ldd];
        D[row + col * ldd] = v;
    }
}

// Vb (krem x w, ld ldv) = the block's reflectors: V(i, a) = A[j0 + a][j0 + i]
// below the diagonal, 1 on it, 0 above.
__global__ void qr_copy_v_kernel(const double* __restrict__ A, int64_t ld, int64_t j0, int64_t krem, int w,
                                 double* __restrict__ Vb, int64_t ldv) {
    const int64_t total = krem * w;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % krem, a = e / krem;
        Vb[i + a * ldv] = i > a ? A[(size_t)(j0 + a) * ld + j0 + i] : (i == a ? 1.0 : 0.0);
    }
}

// The block's T (w x w, column-major ld w) before its off-diagonal blocks:
// the panels' factors Tp[p] (32 x 32, T(a, b) at [b * 32 + a]) on the
// diagonal, zeros elsewhere.  T is the inverse of the block upper
// triangular L with diagonal blocks T_p^{-1} and off-diagonal blocks those
// of V^T V (the merge T_<j,j = -T_<j (V_<j^T V_j) T_j); the recursive
// inversion levels of the triangular inverse fill the rest.
__global__ void qr_block_t_init_kernel(const double* __restrict__ Tp, int w, double* __restrict__ T) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < w * w; e += gridDim.x * blockDim.x) {
        const int r = e % w, c = e / w;
        T[e] = r / 32 == c / 32 ? Tp[(size_t)(c / 32) * 1024 + (c % 32) * 32 + (r % 32)] : 0.0;
    }
}

}  // namespace tomos_b200
