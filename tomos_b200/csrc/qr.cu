// qr.cu -- FP64 Householder QR of the sketch SA and the explicit R^{-1}
// (tomos_sketch_qr_precond_f64).
//
// Contract of the reference's generate_sketch_qr_precond
// (src/core/precond/sketch_qr.cpp:38-64: LAPACK geqrf, zero below the
// diagonal, trtri): on return the leading n x n block of the k x n
// column-major input holds R^{-1}.  Reflectors follow LAPACK's
// dgeqr2/dlarfg convention, H_j = I - tau_j v_j v_j^T with v_j(0) = 1 and
// R_jj = -sign(a_jj) ||a_j||, so R matches the reference's R to rounding.
//
// Blocked right-looking algorithm, panel width nb (32 when it fits):
//   panel    one 8-CTA thread-block cluster factors the (k-j0) x nb panel
//            held in the CTAs' shared memory (row blocks); the two
//            reductions of each column step (the norm below the diagonal
//            and the reflector's inner products with the later panel
//            columns) are exchanged through distributed shared memory
//            with cluster barriers.  The cluster also forms the compact-WY
//            factor T (H_1...H_nb = I - V T V^T).
//   update   C <- (I - V T^T V^T) C on the trailing columns in three
//            kernels: W = V^T C partials per row chunk, W <- T^T (sum),
//            C -= V W.
// R^{-1} is then formed column by column (a warp per column, back
// substitution on a transposed copy of R).
#include <cooperative_groups.h>

#include <string>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace tomos_b200 {

constexpr int kQrCluster = 8;
constexpr int kQrThreads = 256;
constexpr int kQrChunk = 64;      // rows per trailing-update block
constexpr int kQrTile = 32;       // columns per trailing-update block
constexpr int kQrMaxNb = 32;
constexpr size_t kQrPanelSmem = 196 * 1024;

struct QrScratch {
    double* tau;    // n
    double* T;      // kQrMaxNb^2
    double* Wp;     // chunks x nb x n   (W partials)
    double* W2;     // nb x n
    double* Rt;     // n x n  (R transposed: row i of R contiguous)
    int* flag;      // singular-R flag
    size_t bytes;
};

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

static QrScratch qr_layout(void* base, int64_t k, int64_t n) {
    QrScratch q;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t b) {
        char* r = p ? p + off : nullptr;
        off += a256(b);
        return r;
    };
    const int64_t chunks = (k + kQrChunk - 1) / kQrChunk;
    q.tau = reinterpret_cast<double*>(take(sizeof(double) * (n > 0 ? n : 1)));
    q.T = reinterpret_cast<double*>(take(sizeof(double) * kQrMaxNb * kQrMaxNb));
    q.Wp = reinterpret_cast<double*>(take(sizeof(double) * (chunks > 0 ? chunks : 1) * kQrMaxNb *
                                          (n > 0 ? n : 1)));
    q.W2 = reinterpret_cast<double*>(take(sizeof(double) * kQrMaxNb * (n > 0 ? n : 1)));
    q.Rt = reinterpret_cast<double*>(take(sizeof(double) * (n > 0 ? n * n : 1)));
    q.flag = reinterpret_cast<int*>(take(sizeof(int) * 4));
    q.bytes = off;
    return q;
}

// Panel width: the largest power of two <= 32 whose per-CTA share of the
// panel (rows_per_cta x nb doubles) fits the shared-memory budget.
static int qr_panel_nb(int64_t rows) {
    const int64_t rpc = (rows + kQrCluster - 1) / kQrCluster;
    int nb = kQrMaxNb;
    while (nb > 1 && (size_t)rpc * nb * sizeof(double) > kQrPanelSmem) nb >>= 1;
    if ((size_t)rpc * nb * sizeof(double) > kQrPanelSmem) return 0;
    return nb;
}

struct PanelArgs {
    double* A;
    int64_t ld, m, j0;
    int nb;
    int64_t rpc;     // rows per CTA
    double* tau;     // global, indexed by column
    double* T;       // nb x nb, column-major
};

// Shared memory of one panel CTA: the panel slice (column-major, rpc rows
// per column), then the exchange slots.
struct PanelXch {
    double norm[2][2];               // [parity][0 = sum sq below pivot, 1 = pivot value]
    double w[2][kQrMaxNb];           // [parity][column] partial V^T C
    double gram[kQrMaxNb * kQrMaxNb];
};

__global__ void __cluster_dims__(kQrCluster, 1, 1) __launch_bounds__(kQrThreads)
    qr_panel_kernel(PanelArgs P) {
    extern __shared__ __align__(16) double smem[];
    __shared__ PanelXch X;
    __shared__ double red[kQrThreads / 32];
    __shared__ double bcast[4];
    __shared__ double taul[kQrMaxNb];
    __shared__ double gsum[kQrMaxNb * kQrMaxNb];
    __shared__ double tmat[kQrMaxNb * kQrMaxNb];
    __shared__ double gath[2 * kQrCluster];
    __shared__ double wgath[kQrCluster][kQrMaxNb];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = P.nb;
    const int64_t rpc = P.rpc;
    const int64_t row0 = P.j0 + rank * rpc;  // first global row of this CTA
    int64_t nrows = P.m - row0;
    if (nrows > rpc) nrows = rpc;
    if (nrows < 0) nrows = 0;
    double* pan = smem;  // pan[c * rpc + r]

    for (int64_t idx = tid; idx < (int64_t)nb * rpc; idx += kQrThreads) {
        const int c = (int)(idx / rpc);
        const int64_t r = idx % rpc;
        pan[idx] = r < nrows ? P.A[(size_t)(P.j0 + c) * P.ld + row0 + r] : 0.0;
    }
    cluster.sync();

    for (int j = 0; j < nb; ++j) {
        const int par = j & 1;
        const int64_t piv = P.j0 + j;           // global pivot row
        const int64_t lp = piv - row0;          // local index of the pivot row
        const bool owner = lp >= 0 && lp < nrows;
        // 1. partial ||a_j below pivot||^2 and the pivot value.
        double ss = 0.0;
        for (int64_t r = tid; r < nrows; r += kQrThreads)
            if (row0 + r > piv) {
                const double a = pan[(size_t)j * rpc + r];
                ss += a * a;
            }
        ss = warp_sum(ss);
        if (lane == 0) red[warp] = ss;
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            for (int k = 0; k < kQrThreads / 32; ++k) t += red[k];
            X.norm[par][0] = t;
            X.norm[par][1] = owner ? pan[(size_t)j * rpc + lp] : 0.0;
        }
        cluster.sync();
        // 2. every CTA forms the same reflector from the 8 partials
        //    (one distributed-shared-memory read per partial, in parallel).
        if (tid < 2 * kQrCluster) {
            const PanelXch* rx = cluster.map_shared_rank(&X, tid >> 1);
            gath[tid] = rx->norm[par][tid & 1];
        }
        __syncthreads();
        if (tid == 0) {
            double xn2 = 0.0, alpha = 0.0;
            for (int c = 0; c < kQrCluster; ++c) {
                xn2 += gath[2 * c];
                alpha += gath[2 * c + 1];
            }
            double tau = 0.0, beta = alpha, scal = 0.0;
            if (xn2 > 0.0) {
                beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
                tau = (beta - alpha) / beta;
                scal = 1.0 / (alpha - beta);
            }
            bcast[0] = tau;
            bcast[1] = beta;
            bcast[2] = scal;
        }
        __syncthreads();
        const double tau = bcast[0], beta = bcast[1], scal = bcast[2];
        for (int64_t r = tid; r < nrows; r += kQrThreads)
            if (row0 + r > piv) pan[(size_t)j * rpc + r] *= scal;
        if (owner && tid == 0) pan[(size_t)j * rpc + lp] = beta;
        if (tid == 0) taul[j] = tau;
        if (rank == 0 && tid == 0) P.tau[piv] = tau;
        __syncthreads();
        // 3. partial w_c = v^T a_c for the later panel columns.
        for (int c = j + 1 + warp; c < nb; c += kQrThreads / 32) {
            double w = 0.0;
            for (int64_t r = lane; r < nrows; r += 32) {
                const int64_t g = row0 + r;
                if (g > piv)
                    w += pan[(size_t)j * rpc + r] * pan[(size_t)c * rpc + r];
                else if (g == piv)
                    w += pan[(size_t)c * rpc + r];
            }
            w = warp_sum(w);
            if (lane == 0) X.w[par][c] = w;
        }
        cluster.sync();
        // 4. a_c -= tau * w_c * v, w_c summed over the cluster in a fixed order.
        for (int e = tid; e < kQrCluster * nb; e += kQrThreads) {
            const int q = e / nb, c = e % nb;
            if (c > j) wgath[q][c] = cluster.map_shared_rank(&X, q)->w[par][c];
        }
        __syncthreads();
        for (int c = j + 1 + warp; c < nb; c += kQrThreads / 32) {
            double w = 0.0;
            for (int q = 0; q < kQrCluster; ++q) w += wgath[q][c];
            const double tw = tau * w;
            for (int64_t r = lane; r < nrows; r += 32) {
                const int64_t g = row0 + r;
                if (g > piv)
                    pan[(size_t)c * rpc + r] -= tw * pan[(size_t)j * rpc + r];
                else if (g == piv)
                    pan[(size_t)c * rpc + r] -= tw;
            }
        }
        __syncthreads();
    }

    // Gram matrix G = V^T V of the panel's reflectors (unit diagonal,
    // zeros above), partial per CTA: a warp per (a < b) pair, lanes over rows.
    for (int e = warp; e < nb * nb; e += kQrThreads / 32) {
        const int a = e % nb, b = e / nb;
        double g = 0.0;
        if (a < b) {
            for (int64_t r = lane; r < nrows; r += 32) {
                const int64_t row = row0 + r;
                const double va = row > P.j0 + a ? pan[(size_t)a * rpc + r] : (row == P.j0 + a ? 1.0 : 0.0);
                const double vb = row > P.j0 + b ? pan[(size_t)b * rpc + r] : (row == P.j0 + b ? 1.0 : 0.0);
                g += va * vb;
            }
            g = warp_sum(g);
        }
        if (lane == 0) X.gram[e] = g;
    }
    cluster.sync();
    if (rank == 0) {
        // Sum the Gram partials locally, then T (upper triangular,
        // column-major): T_jj = tau_j, T(0:j, j) = -tau_j T(0:j, 0:j) G(0:j, j)
        // (LAPACK dlarft, forward / columnwise).
        for (int e = tid; e < nb * nb; e += kQrThreads) {
            double gq[kQrCluster];
#pragma unroll
            for (int q = 0; q < kQrCluster; ++q) gq[q] = cluster.map_shared_rank(&X, q)->gram[e];
            double g = 0.0;
#pragma unroll
            for (int q = 0; q < kQrCluster; ++q) g += gq[q];
            gsum[e] = g;
        }
        __syncthreads();
        if (warp == 0) {
            for (int j = 0; j < nb; ++j) {
                // lane i computes T(i, j) for i < j from column-j inputs.
                double tij = 0.0;
                if (lane < j) {
                    double s2 = 0.0;
                    for (int l = lane; l < j; ++l) s2 += tmat[l * kQrMaxNb + lane] * gsum[j * nb + l];
                    tij = -taul[j] * s2;
                }
                __syncwarp();
                if (lane < j) tmat[j * kQrMaxNb + lane] = tij;
                if (lane == j) tmat[j * kQrMaxNb + j] = taul[j];
                __syncwarp();
            }
            for (int e = lane; e < kQrMaxNb * kQrMaxNb; e += 32) {
                const int i = e % kQrMaxNb, j = e / kQrMaxNb;
                P.T[j * nb + i] = (i < nb && j < nb) ? tmat[e] : 0.0;
            }
        }
    }
    for (int64_t idx = tid; idx < (int64_t)nb * rpc; idx += kQrThreads) {
        const int c = (int)(idx / rpc);
        const int64_t r = idx % rpc;
        if (r < nrows) P.A[(size_t)(P.j0 + c) * P.ld + row0 + r] = pan[idx];
    }
    cluster.sync();  // keep every CTA's shared memory alive until all reads are done
}

// V(i, a) of the panel starting at column j0 (i, a relative to j0).
__device__ __forceinline__ double vref(const double* A, int64_t ld, int64_t j0, int64_t i, int a) {
    if (i > a) return A[(size_t)(j0 + a) * ld + j0 + i];
    return i == a ? 1.0 : 0.0;
}

// W partials: Wp[chunk][a][c] = sum over the chunk's rows of V(i,a) C(i,c).
__global__ void __launch_bounds__(kQrThreads) qr_w_partial_kernel(const double* A, int64_t ld,
                                                                  int64_t m, int64_t n, int64_t j0,
                                                                  int nb, double* Wp) {
    __shared__ double Vs[kQrChunk][kQrMaxNb + 1];
    __shared__ double Cs[kQrChunk][kQrTile + 1];
    const int64_t c0 = j0 + nb + (int64_t)blockIdx.x * kQrTile;  // global column
    const int64_t i0 = (int64_t)blockIdx.y * kQrChunk;           // row relative to j0
    const int64_t rows = m - j0;
    for (int e = threadIdx.x; e < kQrChunk * kQrMaxNb; e += kQrThreads) {
        const int r = e / kQrMaxNb, a = e % kQrMaxNb;
        const int64_t i = i0 + r;
        Vs[r][a] = (a < nb && i < rows) ? vref(A, ld, j0, i, a) : 0.0;
    }
    for (int e = threadIdx.x; e < kQrChunk * kQrTile; e += kQrThreads) {
        const int r = e % kQrChunk, c = e / kQrChunk;
        const int64_t i = i0 + r, col = c0 + c;
        Cs[r][c] = (i < rows && col < n) ? A[(size_t)col * ld + j0 + i] : 0.0;
    }
    __syncthreads();
    const int a = threadIdx.x / 8, cq = (threadIdx.x % 8) * 4;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int r = 0; r < kQrChunk; ++r) {
        const double v = Vs[r][a];
        s0 += v * Cs[r][cq];
        s1 += v * Cs[r][cq + 1];
        s2 += v * Cs[r][cq + 2];
        s3 += v * Cs[r][cq + 3];
    }
    if (a < nb) {
        const int64_t nc = n - j0 - nb;
        double* out = Wp + ((size_t)blockIdx.y * kQrMaxNb + a) * (size_t)nc;
        const int64_t cc = (int64_t)blockIdx.x * kQrTile + cq;
        if (cc < nc) out[cc] = s0;
        if (cc + 1 < nc) out[cc + 1] = s1;
        if (cc + 2 < nc) out[cc + 2] = s2;
        if (cc + 3 < nc) out[cc + 3] = s3;
    }
}

// W2(:, c) = T^T * sum_chunks Wp(:, :, c): a block per 32 trailing
// columns, threads over (row of W, column) pairs, coalesced along columns.
__global__ void __launch_bounds__(256) qr_w_reduce_kernel(const double* Wp, int64_t chunks,
                                                          int64_t nc, int nb, const double* T,
                                                          double* W2) {
    __shared__ double Ws[kQrMaxNb][kQrTile + 1];
    __shared__ double Ts[kQrMaxNb][kQrMaxNb + 1];
    const int64_t c0 = (int64_t)blockIdx.x * kQrTile;
    for (int e = threadIdx.x; e < kQrMaxNb * kQrMaxNb; e += blockDim.x) {
        const int a = e % kQrMaxNb, b = e / kQrMaxNb;
        Ts[a][b] = (a < nb && b < nb) ? T[b * nb + a] : 0.0;  // T(a, b)
    }
    for (int e = threadIdx.x; e < kQrMaxNb * kQrTile; e += blockDim.x) {
        const int a = e / kQrTile, cc = e % kQrTile;
        const int64_t col = c0 + cc;
        double sum = 0.0;
        if (a < nb && col < nc) {
            const double* p = Wp + (size_t)a * nc + col;
            const size_t stride = (size_t)kQrMaxNb * nc;
            int64_t q = 0;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            for (; q + 3 < chunks; q += 4) {
                s0 += p[(size_t)q * stride];
                s1 += p[(size_t)(q + 1) * stride];
                s2 += p[(size_t)(q + 2) * stride];
                s3 += p[(size_t)(q + 3) * stride];
            }
            for (; q < chunks; ++q) s0 += p[(size_t)q * stride];
            sum = (s0 + s1) + (s2 + s3);
        }
        Ws[a][cc] = sum;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kQrMaxNb * kQrTile; e += blockDim.x) {
        const int b = e / kQrTile, cc = e % kQrTile;
        const int64_t col = c0 + cc;
        if (b >= nb || col >= nc) continue;
        double sum = 0.0;
        for (int a = 0; a <= b; ++a) sum += Ts[a][b] * Ws[a][cc];
        W2[(size_t)b * nc + col] = sum;
    }
}

// C(i, c) -= sum_a V(i, a) W2(a, c).
__global__ void __launch_bounds__(kQrThreads) qr_update_kernel(double* A, int64_t ld, int64_t m,
                                                               int64_t n, int64_t j0, int nb,
                                                               const double* W2) {
    __shared__ double Vs[kQrChunk][kQrMaxNb + 1];
    __shared__ double Ws[kQrMaxNb][kQrTile + 1];
    const int64_t cc0 = (int64_t)blockIdx.x * kQrTile;  // column relative to j0+nb
    const int64_t i0 = (int64_t)blockIdx.y * kQrChunk;
    const int64_t rows = m - j0, nc = n - j0 - nb;
    for (int e = threadIdx.x; e < kQrChunk * kQrMaxNb; e += kQrThreads) {
        const int r = e / kQrMaxNb, a = e % kQrMaxNb;
        const int64_t i = i0 + r;
        Vs[r][a] = (a < nb && i < rows) ? vref(A, ld, j0, i, a) : 0.0;
    }
    for (int e = threadIdx.x; e < kQrMaxNb * kQrTile; e += kQrThreads) {
        const int a = e / kQrTile, c = e % kQrTile;
        Ws[a][c] = (a < nb && cc0 + c < nc) ? W2[(size_t)a * nc + cc0 + c] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kQrChunk * kQrTile; e += kQrThreads) {
        const int r = e % kQrChunk, c = e / kQrChunk;
        const int64_t i = i0 + r, cc = cc0 + c;
        if (i >= rows || cc >= nc) continue;
        double s = 0.0;
#pragma unroll 8
        for (int a = 0; a < kQrMaxNb; ++a) s += Vs[r][a] * Ws[a][c];
        A[(size_t)(j0 + nb + cc) * ld + j0 + i] -= s;
    }
}

// Rt = R^T (R upper triangle of A), R_out = R (optional), singular flag.
__global__ void qr_extract_kernel(const double* A, int64_t ld, int64_t n, double* Rt,
                                  double* R_out, int* flag) {
    const int64_t total = n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        const double v = i <= j ? A[(size_t)j * ld + i] : 0.0;
        Rt[(size_t)i * n + j] = v;
        if (R_out) R_out[(size_t)j * n + i] = v;
        if (i == j && !(v != 0.0 && isfinite(v))) atomicOr(flag, 1);
    }
}

__global__ void qr_zero_lower_kernel(double* A, int64_t ld, int64_t n) {
    const int64_t total = n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        if (i > j) A[(size_t)j * ld + i] = 0.0;
    }
}

// R^{-1} in 32 x 32 blocks, written into the leading n x n block of A
// (whose strictly lower part qr_extract_kernel has zeroed).
// Diagonal blocks: a warp per block, lane j back-substitutes column j.
__global__ void __launch_bounds__(32) qr_trtri_diag_kernel(const double* Rt, int64_t n, double* A,
                                                           int64_t ld) {
    __shared__ double Rb[32][33];
    __shared__ double Xb[32][33];
    const int lane = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.x * 32;
    const int bs = (int)(n - i0 < 32 ? n - i0 : 32);
    for (int r = 0; r < 32; ++r)
        Rb[r][lane] = (r < bs && lane < bs && lane >= r) ? Rt[(size_t)(i0 + r) * n + i0 + lane] : 0.0;
    __syncwarp();
    const int j = lane;
    if (j < bs) {
        Xb[j][j] = 1.0 / Rb[j][j];
        for (int i = j - 1; i >= 0; --i) {
            double sum = 0.0;
            for (int k = i + 1; k <= j; ++k) sum += Rb[i][k] * Xb[k][j];
            Xb[i][j] = -sum / Rb[i][i];
        }
        for (int i = 0; i < bs; ++i) A[(size_t)(i0 + j) * ld + i0 + i] = i <= j ? Xb[i][j] : 0.0;
    }
}

// Off-diagonal blocks of block column J (8 columns per CTA):
// X_IJ = -X_II * sum_{K=I+1..J} R_IK X_KJ for I = J-1 down to 0.
__global__ void __launch_bounds__(256) qr_trtri_off_kernel(const double* Rt, int64_t n, double* A,
                                                           int64_t ld) {
    __shared__ double tmp[32][9];
    const int J = blockIdx.x;
    const int64_t j0 = (int64_t)J * 32 + blockIdx.y * 8;
    const int i = threadIdx.x / 8, jj = threadIdx.x % 8;
    const int64_t col = j0 + jj;
    const bool cv = col < n && blockIdx.y * 8 + jj < 32;
    for (int I = J - 1; I >= 0; --I) {
        const int64_t i0 = (int64_t)I * 32;
        double sum = 0.0;
        if (cv) {
            const double* rrow = Rt + (size_t)(i0 + i) * n;
            const double* xcol = A + (size_t)col * ld;
            for (int64_t k = i0 + 32; k <= col; ++k) sum += rrow[k] * xcol[k];
        }
        tmp[i][jj] = sum;
        __syncthreads();
        if (cv) {
            double out = 0.0;
            for (int l = i; l < 32; ++l) out += A[(size_t)(i0 + l) * ld + i0 + i] * tmp[l][jj];
            A[(size_t)col * ld + i0 + i] = -out;
        }
        __syncthreads();
    }
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

size_t tomos_sketch_qr_scratch_bytes(int64_t k, int64_t n) {
    if (k < 0 || n < 0) return 0;
    return qr_layout(nullptr, k, n).bytes;
}

tomos_status tomos_sketch_qr_precond_f64(int64_t k, int64_t n, double* SA, int64_t ld, double* R,
                                         void* scratch, size_t scratch_bytes, void* stream) {
    if (k < n)
        return fail(TOMOS_ERR_INVALID,
                    "generate_sketch_qr_precond: sketched_mtx must have at least as many rows as "
                    "columns (k >= n).");
    if (n < 0 || ld < k || ld < 1) return fail(TOMOS_ERR_INVALID, "sketch_qr: bad shape");
    if (n == 0) return TOMOS_OK;
    if (!SA) return fail(TOMOS_ERR_INVALID, "sketch_qr: null matrix");
    QrScratch need = qr_layout(nullptr, k, n);
    if (!scratch || scratch_bytes < need.bytes)
        return fail(TOMOS_ERR_INVALID,
                    "sketch_qr: scratch too small (need " + std::to_string(need.bytes) + " bytes)");
    QrScratch q = qr_layout(scratch, k, n);
    cudaStream_t st = as_stream(stream);
    const int nb_max = qr_panel_nb(k);
    if (nb_max == 0) return fail(TOMOS_ERR_UNSUPPORTED, "sketch_qr: k too large for the panel");
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(qr_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kQrPanelSmem));
    TOMOS_CUDA_TRY(cudaMemsetAsync(q.flag, 0, sizeof(int), st));
    for (int64_t j0 = 0; j0 < n; j0 += nb_max) {
        const int nb = (int)(n - j0 < nb_max ? n - j0 : nb_max);
        PanelArgs P;
        P.A = SA;
        P.ld = ld;
        P.m = k;
        P.j0 = j0;
        P.nb = nb;
        P.rpc = (k - j0 + kQrCluster - 1) / kQrCluster;
        P.tau = q.tau;
        P.T = q.T;
        const size_t smem = (size_t)P.rpc * nb * sizeof(double);
        qr_panel_kernel<<<kQrCluster, kQrThreads, smem, st>>>(P);
        TOMOS_LAUNCH_CHECK("qr_panel_kernel");
        const int64_t nc = n - j0 - nb;
        if (nc <= 0) continue;
        const int64_t chunks = (k - j0 + kQrChunk - 1) / kQrChunk;
        dim3 g1((unsigned)((nc + kQrTile - 1) / kQrTile), (unsigned)chunks);
        qr_w_partial_kernel<<<g1, kQrThreads, 0, st>>>(SA, ld, k, n, j0, nb, q.Wp);
        TOMOS_LAUNCH_CHECK("qr_w_partial_kernel");
        qr_w_reduce_kernel<<<(unsigned)((nc + kQrTile - 1) / kQrTile), 256, 0, st>>>(
            q.Wp, chunks, nc, nb, q.T, q.W2);
        TOMOS_LAUNCH_CHECK("qr_w_reduce_kernel");
        qr_update_kernel<<<g1, kQrThreads, 0, st>>>(SA, ld, k, n, j0, nb, q.W2);
        TOMOS_LAUNCH_CHECK("qr_update_kernel");
    }
    qr_extract_kernel<<<(unsigned)((n * n + 255) / 256 < 4096 ? (n * n + 255) / 256 : 4096), 256, 0,
                        st>>>(SA, ld, n, q.Rt, R, q.flag);
    TOMOS_LAUNCH_CHECK("qr_extract_kernel");
    int flag = 0;
    TOMOS_CUDA_TRY(cudaMemcpyAsync(&flag, q.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
    if (flag)
        return fail(TOMOS_ERR_NUMERIC,
                    "generate_sketch_qr_precond: trtri failed -- R is singular.");
    const int64_t nbk = (n + 31) / 32;
    qr_zero_lower_kernel<<<(unsigned)((n * n + 255) / 256 < 4096 ? (n * n + 255) / 256 : 4096), 256, 0,
                           st>>>(SA, ld, n);
    TOMOS_LAUNCH_CHECK("qr_zero_lower_kernel");
    qr_trtri_diag_kernel<<<(unsigned)nbk, 32, 0, st>>>(q.Rt, n, SA, ld);
    TOMOS_LAUNCH_CHECK("qr_trtri_diag_kernel");
    if (nbk > 1) {
        qr_trtri_off_kernel<<<dim3((unsigned)nbk, 4), 256, 0, st>>>(q.Rt, n, SA, ld);
    }
    TOMOS_LAUNCH_CHECK("qr_trtri_off_kernel");
    return TOMOS_OK;
}

}  // extern "C"
