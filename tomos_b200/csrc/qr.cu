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
// Blocked right-looking algorithm with 32-column panels:
//   panel    Cholesky QR twice and Householder reconstruction
//            (qr_panel.cuh): three row-parallel passes give the panel's
//            reflectors V, the compact-WY factor T (H_1...H_nb = I - V T V^T),
//            tau and R, in the layout dgeqrf leaves them.
//   update   C <- (I - V T^T V^T) C on the trailing columns in two kernels:
//            W = V^T C partials per row chunk (qr_w_part_kernel), then per
//            tile the fixed-order sum of the partials, W' = T^T W and
//            C -= V W' (qr_apply_kernel).  The tiles holding the next
//            panel's columns also leave that panel's Gram partials.
// R^{-1} is then formed recursively: 32 x 32 diagonal blocks by back
// substitution, then levels of X_IJ = -X_II R_IJ X_JJ with doubling block
// size, each two batched FP64 products.
#include <cmath>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "mbarrier.cuh"  // smem_addr
#include "qr_gemm.cuh"
#include "qr_panel.cuh"

namespace tomos_b200 {

constexpr int kQrThreads = 256;
constexpr int kQrNb = 32;        // panel width
constexpr int kQrWc = 64;        // trailing columns per update tile
constexpr int kQrChunks = 8;     // row chunks of the W partials
constexpr int kQrMaxChunks = 32; // ... when few column tiles leave SMs idle (one-launch QR)
constexpr int kQrRowTile = 256;  // rows per apply tile (and per Gram partial)
constexpr int kQrMinRowTile = 64; // ... halved down to this when tiles would leave CTAs idle
constexpr int64_t kTrtriGemmMin = 1024; // R^{-1} levels from this block size on run as GEMMs
constexpr int kQrPanelCtas = 128; // CTAs of the panel passes (~64 rows each)

struct QrScratch {
    double* tau;    // n
    double* T;      // 32 x 32
    double* R1;     // 32 x 32
    double* Gp;     // Gram partials of the next panel (k / 256 tiles)
    double* G2p;    // Gram partials of Q1 (kQrPanelCtas)
    double* Qs;     // Q1 of the current panel, k x 32 column-major
    double* Wp;     // kQrMaxChunks x 32 x n  (W partials)
    double* Wr;     // 32 x n, their sum when there are more than kQrChunks
    double* Rt;     // n x n  (R transposed: row i of R contiguous)
    double* Tb;     // products of one level of the recursive inversion
    int* flag;      // [0] singular R, [1] panel fallback
    void* gsync;    // grid barrier of the one-launch QR
    // blocked QR (n from kQrBlockedMinN): per block of kQrBlock columns
    double* Tp;     // the panels' T factors, kQrBlock / 32 x 32 x 32
    double* Vb;     // reflectors, k x kQrBlock
    double* Z;      // V T, k x kQrBlock
    double* Y;      // V^T V, kQrBlock x kQrBlock
    double* Tb2;    // the block's T, kQrBlock x kQrBlock
    double* Wb;     // Z^T C, kQrBlock x n
    double* Pk;     // split-K partials, kGmaxSplits x kQrBlock x max(n, kQrBlock)
    size_t pk_doubles;
    size_t bytes;
};

// Columns from which the blocked QR is used (TOMOS_QR_BLOCKED=0 turns it
// off, =1 uses it whenever there is more than one block).
constexpr int64_t kQrBlockedMinN = 1536;

static bool qr_blocked(int64_t n) {
    static int mode = -1;
    if (mode < 0) {
        const char* e = std::getenv("TOMOS_QR_BLOCKED");
        mode = e ? std::atoi(e) : 2;
    }
    if (mode == 0) return false;
    if (mode == 1) return n > kQrBlock;
    return n >= kQrBlockedMinN;
}

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

__host__ __device__ inline int64_t qr_row_tiles(int64_t rows) { return (rows + kQrRowTile - 1) / kQrRowTile; }

static QrScratch qr_layout(void* base, int64_t k, int64_t n) {
    QrScratch q;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t b) {
        char* r = p ? p + off : nullptr;
        off += a256(b);
        return r;
    };
    const size_t nn = n > 0 ? (size_t)n : 1, kk = k > 0 ? (size_t)k : 1;
    const size_t tiles = (size_t)((k > 0 ? k : 1) + kQrMinRowTile - 1) / kQrMinRowTile;
    q.tau = reinterpret_cast<double*>(take(sizeof(double) * nn));
    q.T = reinterpret_cast<double*>(take(sizeof(double) * kHB * kHB));
    q.R1 = reinterpret_cast<double*>(take(sizeof(double) * kHB * kHB));
    q.Gp = reinterpret_cast<double*>(take(sizeof(double) * tiles * kHB * kHB));
    q.G2p = reinterpret_cast<double*>(take(sizeof(double) * kQrPanelCtas * kHB * kHB));
    q.Qs = reinterpret_cast<double*>(take(sizeof(double) * kk * kHB));
    q.Wp = reinterpret_cast<double*>(take(sizeof(double) * kQrMaxChunks * kHB * nn));
    q.Wr = reinterpret_cast<double*>(take(sizeof(double) * kHB * nn));
    q.Rt = reinterpret_cast<double*>(take(sizeof(double) * nn * nn));
    size_t tb = 1;  // the largest level of the recursive inversion
    for (int64_t b = 32; b < n; b *= 2) {
        const size_t pairs = (size_t)((n - b + 2 * b - 1) / (2 * b));
        if (pairs * b * b > tb) tb = pairs * b * b;
    }
    q.Tb = reinterpret_cast<double*>(take(sizeof(double) * tb));
    q.flag = reinterpret_cast<int*>(take(sizeof(int) * 4));
    q.gsync = take(64);
    q.Tp = q.Vb = q.Z = q.Y = q.Tb2 = q.Wb = q.Pk = nullptr;
    q.pk_doubles = 0;
    if (qr_blocked(n)) {
        const size_t bb = kQrBlock, nw = nn > bb ? nn : bb;
        q.Tp = reinterpret_cast<double*>(take(sizeof(double) * (bb / kHB) * kHB * kHB));
        q.Vb = reinterpret_cast<double*>(take(sizeof(double) * kk * bb));
        q.Z = reinterpret_cast<double*>(take(sizeof(double) * kk * bb));
        q.Y = reinterpret_cast<double*>(take(sizeof(double) * bb * bb));
        q.Tb2 = reinterpret_cast<double*>(take(sizeof(double) * bb * bb));
        q.Wb = reinterpret_cast<double*>(take(sizeof(double) * bb * nn));
        q.pk_doubles = kGmaxSplits * bb * nw;
        q.Pk = reinterpret_cast<double*>(take(sizeof(double) * q.pk_doubles));
    }
    q.bytes = off;
    return q;
}

// V(i, a) of the panel starting at column j0 (i, a relative to j0): unit
// diagonal, zeros above, the stored reflector below.
__device__ __forceinline__ double vref(const double* A, int64_t ld, int64_t j0, int64_t i, int a) {
    if (i > a) return __ldcg(A + (size_t)(j0 + a) * ld + j0 + i);
    return i == a ? 1.0 : 0.0;
}

// D = A B + C for one m8n8k4 FP64 tile on the tensor cores.  Lane l holds
// A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Row stride (doubles) of the shared 32 x 32 tiles the trailing update reads
// as m8n8k4 fragments (V, T, the Gram tile).  A fragment read touches word
// 36 r + c for lane (r, c) in {0..3} x {0..3} (+ a constant); 36 = 4 mod 16
// puts the 16 lanes of each half-warp on 16 distinct 8-byte banks, either way
// round (a stride of 33 left up to four lanes on one bank).
constexpr int kQrVs = kHB + 4;

// Gram partials of the first panel: tile `tile` sums rows [256 t, 256 t + 256).
// Shared tiles of the phase functions below, carved from `sm` (dynamic
// shared memory of the calling kernel, 16-byte aligned).
// (the trailing update's W, T^T W and T tiles plus its copy stages)
constexpr int kQrTileSmemDoubles =
    2 * kHB * (kQrWc + 2) + kHB * kQrVs + 3 * (kHB * kQrVs + kHB * (kQrWc + 2));

__device__ void qr_gram_tile(const double* A, int64_t ld, int64_t k, int nb, int tile, double* Gp,
                             double* sm) {
    double (*Pt)[kHB + 1] = reinterpret_cast<double (*)[kHB + 1]>(sm);
    const int t = threadIdx.x;
    const int a = t & 31, b0 = (t >> 5) * 4;
    const int64_t r0 = (int64_t)tile * kQrRowTile;
    int64_t r1 = r0 + kQrRowTile;
    if (r1 > k) r1 = k;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t rt = r0; rt < r1; rt += kHB) {
        __syncthreads();
        for (int e = t; e < kHB * kHB; e += kQrThreads) {
            const int r = e & 31, c = e >> 5;
            const int64_t row = rt + r;
            Pt[r][c] = (row < r1 && c < nb) ? __ldcg(A + (size_t)c * ld + row) : 0.0;
        }
        __syncthreads();
        for (int r = 0; r < kHB; ++r) {
            const double x = Pt[r][a];
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[u] += x * Pt[r][b0 + u];
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) Gp[(size_t)tile * kHB * kHB + a * kHB + b0 + u] = acc[u];
    __syncthreads();
}

__global__ void __launch_bounds__(kQrThreads) qr_gram_kernel(const double* A, int64_t ld, int64_t k,
                                                             int nb, double* Gp) {
    extern __shared__ __align__(16) double qsm[];
    qr_gram_tile(A, ld, k, nb, blockIdx.x, Gp, qsm);
}

// Shared tiles of the trailing update keep an even row stride.
constexpr int kQrWs = kQrWc + 2;
// Sub-tiles (32 rows of V and of C) in flight in the trailing update.
constexpr int kQrStages = 3;
constexpr int kQrStageDoubles = kHB * kQrVs + kHB * kQrWs;

__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The V and C sub-tiles of rows [rt, rt + 32) (relative to j0) into one
// stage: V(i, a) = A[j0 + a][j0 + i] as stored (the unit diagonal and the
// zeros above it are set by qr_fix_v once the copies landed), C(i, c) the
// trailing columns c0 + c.  Rows past r1, reflectors past nb and columns
// past nc read as zeros.  One asynchronous copy group per call.
__device__ __forceinline__ void qr_issue_vc(const double* A, int64_t ld, int64_t j0, int nb, int64_t nc,
                                            int64_t c0, int64_t rt, int64_t r1, double* stage) {
    double (*Vs)[kQrVs] = reinterpret_cast<double (*)[kQrVs]>(stage);
    double (*Cs)[kQrWs] = reinterpret_cast<double (*)[kQrWs]>(stage + kHB * kQrVs);
    const int t = threadIdx.x;
#pragma unroll
    for (int i = 0; i < kHB * kHB / kQrThreads; ++i) {
        const int e = t + i * kQrThreads, r = e & 31, aa = e >> 5;
        const int64_t row = rt + r;
        const bool ok = row < r1 && aa < nb;
        cp_async8(&Vs[r][aa], ok ? A + (size_t)(j0 + aa) * ld + j0 + row : A, ok);
    }
#pragma unroll
    for (int i = 0; i < kHB * kQrWc / kQrThreads; ++i) {
        const int e = t + i * kQrThreads, r = e & 31, c = e >> 5;
        const int64_t row = rt + r, col = c0 + c;
        const bool ok = row < r1 && col < nc;
        cp_async8(&Cs[r][c], ok ? A + (size_t)(j0 + nb + col) * ld + j0 + row : A, ok);
    }
    cp_async_commit();
}

// The panel's first 32 rows of V: unit diagonal, zeros above it.
__device__ __forceinline__ void qr_fix_v(double* stage, int64_t rt) {
    if (rt != 0) return;
    double (*Vs)[kQrVs] = reinterpret_cast<double (*)[kQrVs]>(stage);
    for (int e = threadIdx.x; e < kHB * kHB; e += kQrThreads) {
        const int r = e & 31, aa = e >> 5;
        if (r <= aa) Vs[r][aa] = r == aa ? 1.0 : 0.0;
    }
}

// W partials: Wp[chunk][a][c] = sum over the chunk's rows of V(i, a) C(i, c),
// C the trailing columns j0 + nb + c.  A CTA: one row chunk x 64 columns,
// 32-row sub-tiles streamed through kQrStages shared-memory stages by
// asynchronous copies; warp w: all 32 reflectors x columns 8w..8w+7 as two
// m16n8 FP64 tensor-core tiles, 8 rows of a sub-tile per step.
__device__ void qr_w_part_tile(const double* A, int64_t ld, int64_t k, int64_t n, int64_t j0, int nb,
                               int64_t chunk_rows, double* Wp, int ct, int rc, double* sm) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5, g = lane >> 2, q = lane & 3;
    const int cw = warp * 8;
    const int64_t nc = n - j0 - nb, krem = k - j0;
    const int64_t c0 = (int64_t)ct * kQrWc;
    const int64_t r0 = (int64_t)rc * chunk_rows;
    int64_t r1 = r0 + chunk_rows;
    if (r1 > krem) r1 = krem;
    const int nsub = r1 > r0 ? (int)((r1 - r0 + kHB - 1) / kHB) : 0;
    double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
    __syncthreads();  // a previous tile of this CTA may still read the stages
#pragma unroll
    for (int i = 0; i < kQrStages - 1; ++i) {
        if (i < nsub) qr_issue_vc(A, ld, j0, nb, nc, c0, r0 + (int64_t)i * kHB, r1, sm + i * kQrStageDoubles);
        else cp_async_commit();
    }
    for (int i = 0; i < nsub; ++i) {
        const int ni = i + kQrStages - 1;
        if (ni < nsub)
            qr_issue_vc(A, ld, j0, nb, nc, c0, r0 + (int64_t)ni * kHB, r1, sm + (ni % kQrStages) * kQrStageDoubles);
        else
            cp_async_commit();
        cp_async_wait<kQrStages - 1>();  // this thread's copies of sub-tile i
        __syncthreads();                 // everyone's
        double* stage = sm + (i % kQrStages) * kQrStageDoubles;
        const int64_t rt = r0 + (int64_t)i * kHB;
        if (rt == 0) {
            qr_fix_v(stage, rt);
            __syncthreads();
        }
        double (*Vt)[kQrVs] = reinterpret_cast<double (*)[kQrVs]>(stage);
        double (*Ct)[kQrWs] = reinterpret_cast<double (*)[kQrWs]>(stage + kHB * kQrVs);
#pragma unroll
        for (int ks = 0; ks < kHB / 8; ++ks) {
            const int k0 = 8 * ks + q;
            const double b[2] = {Ct[k0][cw + g], Ct[k0 + 4][cw + g]};  // B[k][c] = C(row, col)
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {
                const int m0 = 16 * mb + g;
                const double a[4] = {Vt[k0][m0], Vt[k0][m0 + 8], Vt[k0 + 4][m0], Vt[k0 + 4][m0 + 8]};  // A[a][k] = V(row, a)
                g_dmma1688(acc[mb], a, b);
            }
        }
        __syncthreads();  // the stage is refilled two sub-tiles on
    }
    cp_async_wait<0>();
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int aa = 16 * mb + 8 * h + g;
            if (aa >= nb) continue;
            double* out = Wp + ((size_t)rc * kHB + aa) * (size_t)nc;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int64_t col = c0 + cw + 2 * q + u;
                if (col < nc) out[col] = acc[mb][2 * h + u];
            }
        }
    __syncthreads();
}

__global__ void __launch_bounds__(kQrThreads) qr_w_part_kernel(const double* A, int64_t ld,
                                                               int64_t k, int64_t n, int64_t j0,
                                                               int nb, int64_t chunk_rows,
                                                               double* Wp) {
    extern __shared__ __align__(16) double qsm[];
    qr_w_part_tile(A, ld, k, n, j0, nb, chunk_rows, Wp, blockIdx.x, blockIdx.y, qsm);
}

// C -= V (T^T W) on one tile of 256 rows x 64 trailing columns, W the
// fixed-order sum of the chunk partials.  The 32-row sub-tiles of V and C
// stream through kQrStages shared-memory stages by asynchronous copies;
// warp w: the 32 rows of a sub-tile x columns 8w..8w+7 as two m16n8 FP64
// tensor-core tiles (C the accumulator, A = -V, B = T^T W).  Tiles holding
// the next panel's columns (column tile 0) then write that panel's Gram
// partial over their rows below the current panel (rows j0 + nb on),
// again on the tensor cores (warp w: one 16 x 8 tile of the 32 x 32 Gram).
__device__ void qr_apply_tile(double* A, int64_t ld, int64_t k, int64_t n, int64_t j0, int nb,
                              int nchunks, const double* Wp, const double* T, int nb_next,
                              double* Gp_next, int ct, int rtile, int row_tile, double* sm) {
    double (*W0)[kQrWs] = reinterpret_cast<double (*)[kQrWs]>(sm);
    double (*Wt)[kQrWs] = reinterpret_cast<double (*)[kQrWs]>(sm + kHB * kQrWs);
    double (*Tt)[kQrVs] = reinterpret_cast<double (*)[kQrVs]>(sm + 2 * kHB * kQrWs);
    double (*Gt)[kQrVs] = Tt;  // the Gram tile reuses T's storage
    double* stages = sm + 2 * kHB * kQrWs + kHB * kQrVs;
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5, g = lane >> 2, q = lane & 3;
    const int cw = warp * 8;
    const int64_t nc = n - j0 - nb, krem = k - j0;
    const int64_t c0 = (int64_t)ct * kQrWc;
    const int64_t r0 = (int64_t)rtile * row_tile;
    int64_t r1 = r0 + row_tile;
    if (r1 > krem) r1 = krem;
    const int nsub = r1 > r0 ? (int)((r1 - r0 + kHB - 1) / kHB) : 0;
    __syncthreads();  // a previous tile of this CTA may still read the buffers
    // the first sub-tiles' copies fly while W and T^T W are formed
#pragma unroll
    for (int i = 0; i < kQrStages - 1; ++i) {
        if (i < nsub) qr_issue_vc(A, ld, j0, nb, nc, c0, r0 + (int64_t)i * kHB, r1, stages + i * kQrStageDoubles);
        else cp_async_commit();
    }
    // W: thread t sums column t % 64 of reflectors t / 64 + 4 i (i < 8), the
    // chunk partials in order, one chunk's eight loads in flight at a time
    {
        constexpr int kPer = kHB * kQrWc / kQrThreads;
        const int c = t % kQrWc, a0 = t / kQrWc;
        const int64_t col = c0 + c;
        double w[kPer];
#pragma unroll
        for (int i = 0; i < kPer; ++i) w[i] = 0.0;
        for (int qq = 0; qq < nchunks; ++qq) {
            double v[kPer];
#pragma unroll
            for (int i = 0; i < kPer; ++i) {
                const int aa = a0 + i * (kQrThreads / kQrWc);
                v[i] = (aa < nb && col < nc) ? __ldcg(Wp + ((size_t)qq * kHB + aa) * (size_t)nc + col) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < kPer; ++i) w[i] += v[i];
        }
#pragma unroll
        for (int i = 0; i < kPer; ++i) W0[a0 + i * (kQrThreads / kQrWc)][c] = w[i];
    }
    for (int e = t; e < kHB * kHB; e += kQrThreads) {
        const int aa = e & 31, b = e >> 5;
        Tt[aa][b] = (aa < nb && b < nb) ? __ldcg(T + (size_t)b * nb + aa) : 0.0;  // T(aa, b)
    }
    __syncthreads();
    // T^T W on the tensor cores: warp w, all 32 rows x columns 8w..8w+7;
    // A[b][aa] = T(aa, b) for aa <= b (T is upper triangular), B = W
    {
        double tw[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int ks = 0; ks < kHB / 4; ++ks) {
            const int aa = 4 * ks + q;
            const double bw = W0[aa][cw + g];
#pragma unroll
            for (int blk = 0; blk < 4; ++blk) {
                const int b = 8 * blk + g;
                dmma884(tw[blk][0], tw[blk][1], aa <= b ? Tt[aa][b] : 0.0, bw);
            }
        }
#pragma unroll
        for (int blk = 0; blk < 4; ++blk) {
            Wt[8 * blk + g][cw + 2 * q] = tw[blk][0];
            Wt[8 * blk + g][cw + 2 * q + 1] = tw[blk][1];
        }
    }
    const bool gram = Gp_next != nullptr && ct == 0;
    // Gram tile of warp w: rows 16 (w / 4) .., columns 8 (w % 4) ..
    const int gmb = warp >> 2, gnb = warp & 3;
    double gacc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < nsub; ++i) {
        const int ni = i + kQrStages - 1;
        if (ni < nsub)
            qr_issue_vc(A, ld, j0, nb, nc, c0, r0 + (int64_t)ni * kHB, r1,
                        stages + (ni % kQrStages) * kQrStageDoubles);
        else
            cp_async_commit();
        cp_async_wait<kQrStages - 1>();
        __syncthreads();  // sub-tile i of every thread; Wt (first pass); Gt free
        double* stage = stages + (i % kQrStages) * kQrStageDoubles;
        const int64_t rt = r0 + (int64_t)i * kHB;
        if (rt == 0) {
            qr_fix_v(stage, rt);
            __syncthreads();
        }
        double (*Vt)[kQrVs] = reinterpret_cast<double (*)[kQrVs]>(stage);
        double (*Ct)[kQrWs] = reinterpret_cast<double (*)[kQrWs]>(stage + kHB * kQrVs);
        // cur[2 blk + u] = C(8 blk + g, cw + 2q + u): rows 16 mb + g and
        // 16 mb + g + 8 of m16n8 tile mb are cur[4 mb + {0, 1}], cur[4 mb + {2, 3}]
        double cur[8];
#pragma unroll
        for (int blk = 0; blk < 4; ++blk) {
            cur[2 * blk] = Ct[8 * blk + g][cw + 2 * q];
            cur[2 * blk + 1] = Ct[8 * blk + g][cw + 2 * q + 1];
        }
#pragma unroll
        for (int ks = 0; ks < kHB / 8; ++ks) {
            const int k0 = 8 * ks + q;
            const double b[2] = {Wt[k0][cw + g], Wt[k0 + 4][cw + g]};  // B[a][c] = (T^T W)(a, col)
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {
                const int m0 = 16 * mb + g;
                const double a[4] = {-Vt[m0][k0], -Vt[m0 + 8][k0], -Vt[m0][k0 + 4], -Vt[m0 + 8][k0 + 4]};  // A = -V
                g_dmma1688(&cur[4 * mb], a, b);
            }
        }
#pragma unroll
        for (int blk = 0; blk < 4; ++blk) {
            const int rr = 8 * blk + g;
            const int64_t row = rt + rr;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int cl = cw + 2 * q + u;
                const int64_t col = c0 + cl;
                const bool in = row < r1 && col < nc;
                if (in) A[(size_t)(j0 + nb + col) * ld + j0 + row] = cur[2 * blk + u];
                if (gram && cl < kHB) Gt[rr][cl] = (in && row >= nb && cl < nb_next) ? cur[2 * blk + u] : 0.0;
            }
        }
        if (gram) {
            __syncthreads();
#pragma unroll
            for (int ks = 0; ks < kHB / 8; ++ks) {
                const int k0 = 8 * ks + q, m0 = 16 * gmb + g;
                const double a[4] = {Gt[k0][m0], Gt[k0][m0 + 8], Gt[k0 + 4][m0], Gt[k0 + 4][m0 + 8]};  // A[a][r] = C(r, a)
                const double b[2] = {Gt[k0][8 * gnb + g], Gt[k0 + 4][8 * gnb + g]};
                g_dmma1688(gacc, a, b);
            }
        }
        __syncthreads();  // the stage is refilled two sub-tiles on; Gt rewritten
    }
    cp_async_wait<0>();
    if (gram) {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int u = 0; u < 2; ++u)
                Gp_next[(size_t)rtile * kHB * kHB + (16 * gmb + 8 * h + g) * kHB + 8 * gnb + 2 * q + u] =
                    gacc[2 * h + u];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kQrThreads) qr_apply_kernel(double* A, int64_t ld, int64_t k,
                                                              int64_t n, int64_t j0, int nb,
                                                              int nchunks, const double* Wp,
                                                              const double* T, int nb_next,
                                                              double* Gp_next) {
    extern __shared__ __align__(16) double qsm[];
    qr_apply_tile(A, ld, k, n, j0, nb, nchunks, Wp, T, nb_next, Gp_next, blockIdx.x, blockIdx.y,
                  kQrRowTile, qsm);
}

// ------------------------------------------------------ one launch per QR
//
// Every read of data another CTA may have written earlier in the same
// launch (A, Q1, the Gram and W partials, T, R1) goes through __ldcg (L2,
// not the SM's non-coherent L1), in the phase functions above and in
// qr_panel.cuh.
//
// The same phases as the per-phase kernels above, run by one cooperative
// launch (one CTA per SM, all resident) that separates them with a grid
// barrier instead of kernel boundaries:
//   panel passes (hr_q1, hr_v) on up to kQrPanelCtas CTAs, then the W
//   partials and the apply tiles spread over every CTA.
// The barrier is a counter and a generation word in global memory; waits
// are bounded (kGridSpinLimit polls with a short sleep), and a CTA whose
// wait expires sets an error word and leaves, so a broken barrier ends the
// kernel with an error the host reports instead of hanging the GPU.

constexpr long long kGridSpinLimit = 1ll << 22;

struct GridSync {
    unsigned int arrive;
    unsigned int gen;
    int err;
    int pad;
};

__device__ bool grid_sync(GridSync* gs, unsigned int& gen, int* sflag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int g = gen;
        if (atomicAdd(&gs->arrive, 1u) == gridDim.x - 1) {
            atomicExch(&gs->arrive, 0u);
            __threadfence();
            atomicExch(&gs->gen, g + 1u);
        } else {
            long long k = 0;
            while (*(volatile unsigned int*)&gs->gen == g) {
                if (++k > kGridSpinLimit) {
                    atomicExch(&gs->err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        *sflag = *(volatile int*)&gs->err;
    }
    __syncthreads();
    gen += 1u;
    return *sflag == 0;
}

// One launch factors columns [jb, je): panels of 32, the trailing update
// restricted to the range.  Panel p's T goes to Tp + p * t_stride.
struct QrPersistArgs {
    double* A;
    int64_t ld, k, n;
    int64_t jb, je;
    double* Tp;
    int64_t t_stride;
    QrScratch q;
    GridSync* gs;
};

__global__ void __launch_bounds__(kQrThreads, 1) qr_persist_kernel(QrPersistArgs a) {
    extern __shared__ __align__(16) double hsm[];
    __shared__ int sflag;
    unsigned int gen = 0;
    const int cta = blockIdx.x, ncta = gridDim.x;
    const int64_t k = a.k, n = a.je;
    const int nb0 = (int)(n - a.jb < kQrNb ? n - a.jb : kQrNb);
    const int tiles0 = (int)qr_row_tiles(k - a.jb);
    for (int tl = cta; tl < tiles0; tl += ncta)
        qr_gram_tile(a.A + (size_t)a.jb * a.ld + a.jb, a.ld, k - a.jb, nb0, tl, a.q.Gp, hsm);
    if (!grid_sync(a.gs, gen, &sflag)) return;
    int ngp = tiles0;
    for (int64_t j0 = a.jb; j0 < n; j0 += kQrNb) {
        const int nb = (int)(n - j0 < kQrNb ? n - j0 : kQrNb);
        double* Tpan = a.Tp + (size_t)((j0 - a.jb) / kQrNb) * a.t_stride;
        const int64_t krem = k - j0;
        int gp = (int)((krem + 63) / 64);
        if (gp > kQrPanelCtas) gp = kQrPanelCtas;
        if (gp > ncta) gp = ncta;
        if (gp < 1) gp = 1;
        HrArgs H;
        H.A = a.A;
        H.ld = a.ld;
        H.k = k;
        H.j0 = j0;
        H.nb = nb;
        H.rpc = ((krem + gp - 1) / gp + kHB - 1) / kHB * kHB;
        H.Gp = a.q.Gp;
        H.ngp = ngp;
        H.Qs = a.q.Qs;
        H.kq = k;
        H.G2p = a.q.G2p;
        H.R1 = a.q.R1;
        H.fail = a.q.flag + 1;
        H.T = Tpan;
        H.tau = a.q.tau;
        if (cta < gp) hr_q1(H, cta, hsm);
        if (!grid_sync(a.gs, gen, &sflag)) return;
        const int top = gp < ncta ? gp : 0;  // the top block beside the rows
        if (cta < gp || cta == top) hr_v(H, cta, gp, top, hsm);
        if (!grid_sync(a.gs, gen, &sflag)) return;
        const int64_t nc = n - j0 - nb;
        if (nc <= 0) break;
        const int ctiles = (int)((nc + kQrWc - 1) / kQrWc);
        // row chunks: enough W-partial tiles for every CTA, up to kQrMaxChunks
        int want = ncta / ctiles;
        if (want < kQrChunks) want = kQrChunks;
        if (want > kQrMaxChunks) want = kQrMaxChunks;
        const int64_t chunk_rows = ((krem + want - 1) / want + kHB - 1) / kHB * kHB;
        const int nchunks = (int)((krem + chunk_rows - 1) / chunk_rows);
        for (int tl = cta; tl < ctiles * nchunks; tl += ncta)
            qr_w_part_tile(a.A, a.ld, k, n, j0, nb, chunk_rows, a.q.Wp, tl % ctiles, tl / ctiles, hsm);
        if (!grid_sync(a.gs, gen, &sflag)) return;
        const double* Wuse = a.q.Wp;
        int nuse = nchunks;
        if (nchunks > kQrChunks) {  // sum the partials once, in order
            for (int64_t e = (int64_t)cta * kQrThreads + threadIdx.x; e < (int64_t)kHB * nc;
                 e += (int64_t)ncta * kQrThreads) {
                double sum = 0.0;
                for (int c = 0; c < nchunks; ++c) sum += __ldcg(a.q.Wp + (size_t)c * kHB * nc + e);
                a.q.Wr[e] = sum;
            }
            if (!grid_sync(a.gs, gen, &sflag)) return;
            Wuse = a.q.Wr;
            nuse = 1;
        }
        const int nb_next = (int)(nc < kQrNb ? nc : kQrNb);
        // apply tiles: rows halved from 256 (down to 64) while CTAs would idle
        int row_tile = kQrRowTile;
        while (row_tile > kQrMinRowTile && (int64_t)ctiles * ((krem + row_tile - 1) / row_tile) < ncta)
            row_tile /= 2;
        const int rtiles = (int)((krem + row_tile - 1) / row_tile);
        for (int tl = cta; tl < ctiles * rtiles; tl += ncta)
            qr_apply_tile(a.A, a.ld, k, n, j0, nb, nuse, Wuse, Tpan, nb_next, a.q.Gp,
                          tl % ctiles, tl / ctiles, row_tile, hsm);
        ngp = rtiles;
        if (!grid_sync(a.gs, gen, &sflag)) return;
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

// One level of the recursive inversion X = R^{-1}: for every pair p of
// diagonal blocks I = [2bp, 2bp + b), J = [2bp + b, 2bp + 2b) (J clipped
// at n), X_IJ = -X_II R_IJ X_JJ, in two batched products
//   mode 0:  T_p  = R_IJ X_JJ      (R from Rt, row-major)
//   mode 1:  X_IJ = -X_II T_p
// X_II and X_JJ come from the previous level.  32 x 32 output tiles (many
// CTAs even at the widest level), k-steps of 32 through shared memory,
// each warp two m8n8 FP64 tensor-core tiles.
__global__ void __launch_bounds__(256) trtri_level_kernel(const double* Rt, int64_t n, double* X,
                                                          int64_t ldx, double* Tb, int64_t b,
                                                          int mode) {
    __shared__ double As[32][32 + 1];  // [k][row]
    __shared__ double Bs[32][32 + 1];  // [k][col]
    const int64_t p = blockIdx.z;
    const int64_t I0 = 2 * b * p, J0 = I0 + b;
    const int64_t Jn = n - J0 < b ? n - J0 : b;
    if (Jn <= 0) return;
    const int64_t M = b, N = Jn, K = mode == 0 ? Jn : b;
    const int64_t row0 = (int64_t)blockIdx.y * 32, col0 = (int64_t)blockIdx.x * 32;
    if (row0 >= M || col0 >= N) return;
    double* T = Tb + (size_t)p * b * b;  // b x Jn, column-major, ld b
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5, g = lane >> 2, q = lane & 3;
    const int mb = warp >> 1, nb0 = 2 * (warp & 1);
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int64_t k0 = 0; k0 < K; k0 += 32) {
        __syncthreads();
        for (int e = t; e < 32 * 32; e += 256) {
            int i, kk;
            double v = 0.0;
            if (mode == 0) {  // R row-major: consecutive threads along k
                i = e >> 5;
                kk = e & 31;
                if (row0 + i < M && k0 + kk < K) v = Rt[(size_t)(I0 + row0 + i) * n + J0 + k0 + kk];
            } else {          // X column-major: consecutive threads along rows
                i = e & 31;
                kk = e >> 5;
                if (row0 + i < M && k0 + kk < K) v = X[(size_t)(I0 + k0 + kk) * ldx + I0 + row0 + i];
            }
            As[kk][i] = v;
        }
        for (int e = t; e < 32 * 32; e += 256) {
            const int kk = e & 31, j = e >> 5;
            double v = 0.0;
            if (k0 + kk < K && col0 + j < N)
                v = mode == 0 ? X[(size_t)(J0 + col0 + j) * ldx + J0 + k0 + kk]
                              : T[(size_t)(col0 + j) * b + k0 + kk];
            Bs[kk][j] = v;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
            const double a = As[4 * ks + q][8 * mb + g];
#pragma unroll
            for (int nn = 0; nn < 2; ++nn)
                dmma884(acc[nn][0], acc[nn][1], a, Bs[4 * ks + q][8 * (nb0 + nn) + g]);
        }
    }
#pragma unroll
    for (int nn = 0; nn < 2; ++nn)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int64_t i = row0 + 8 * mb + g, j = col0 + 8 * (nb0 + nn) + 2 * q + u;
            if (i >= M || j >= N) continue;
            if (mode == 0)
                T[(size_t)j * b + i] = acc[nn][u];
            else
                X[(size_t)(J0 + j) * ldx + I0 + i] = -acc[nn][u];
        }
}

// D[i, j] = D[j, i] for i > j (n x n column-major).
__global__ void qr_mirror_lower_kernel(double* D, int64_t ldd, int64_t n) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        if (i > j) D[(size_t)j * ldd + i] = D[(size_t)i * ldd + j];
    }
}

// op(A) B products of the blocked QR (qr_gemm.cuh).  With a partial
// buffer P of pcap doubles, K is split over CTAs (partials summed in
// order) by the count that wastes the least of the last wave of resident
// CTAs (two per SM), each split keeping at least 16 k-stages and all
// partials fitting P.  sub: D -= op(A) B.  upper (a symmetric product,
// op(A) = B^T, square D): only the tiles that reach the diagonal or above
// are formed, and the lower triangle is then copied from the upper
// (qr_mirror_lower_kernel), exactly symmetric.
template <bool KMAJOR>
static tomos_status qr_gemm(const double* A, int64_t lda, const double* B, int64_t ldb, double* D,
                            int64_t ldd, int64_t M, int64_t N, int64_t K, double alpha, double beta,
                            double* P, size_t pcap, cudaStream_t st, int sub = 0, bool upper = false) {
    if (M <= 0 || N <= 0) return TOMOS_OK;
    const int64_t tm = (M + kGbm - 1) / kGbm, tn = (N + kGbn - 1) / kGbn;
    int64_t active = tm * tn;
    if (upper) {
        active = 0;
        for (int64_t i = 0; i < tm; ++i)
            for (int64_t j = 0; j < tn; ++j)
                if (i * kGbm <= j * kGbn + kGbn - 1) ++active;
    }
    int64_t splits = 1;
    if (P) {
        const int64_t slots = 2 * (int64_t)sm_count(), tiles = active;
        int64_t kmax = K / (16 * kGbk);
        if (kmax > kGmaxSplits) kmax = kGmaxSplits;
        const int64_t fit = (int64_t)(pcap / (size_t)(M * N));
        if (kmax > fit) kmax = fit;
        double best = -1.0;
        for (int64_t s = 1; s <= kmax; ++s) {
            const int64_t ctas = tiles * s, waves = (ctas + slots - 1) / slots;
            const double eff = (double)ctas / (double)(waves * slots);
            if (eff > best + 0.02) {  // more splits only for a clear gain
                best = eff;
                splits = s;
            }
        }
    }
    int64_t kc = (K + splits - 1) / splits;
    kc = (kc + kGbk - 1) / kGbk * kGbk;
    if (kc < kGbk) kc = kGbk;
    splits = (K + kc - 1) / kc;
    if (splits < 1) splits = 1;
    GemmArgs g;
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.D = D;
    g.ldd = ldd;
    g.P = P;
    g.M = M;
    g.N = N;
    g.K = K;
    g.kc = kc;
    g.alpha = alpha;
    g.beta = beta;
    g.sub = sub;
    g.upper = upper ? 1 : 0;
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(qr_gemm_kernel<KMAJOR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kGemmSmem));
    qr_gemm_kernel<KMAJOR><<<dim3((unsigned)tm, (unsigned)tn, (unsigned)splits), 256, kGemmSmem, st>>>(g);
    TOMOS_LAUNCH_CHECK("qr_gemm_kernel");
    if (splits > 1) {
        int64_t rb = (M * N + 255) / 256;
        if (rb > 4096) rb = 4096;
        qr_gemm_reduce_kernel<<<(unsigned)rb, 256, 0, st>>>(P, (int)splits, M, N, alpha, beta, D, ldd);
        TOMOS_LAUNCH_CHECK("qr_gemm_reduce_kernel");
    }
    if (upper) {
        const int64_t nn = M * M;
        const unsigned mb = (unsigned)((nn + 255) / 256 < 4096 ? (nn + 255) / 256 : 4096);
        qr_mirror_lower_kernel<<<mb, 256, 0, st>>>(D, ldd, M);
        TOMOS_LAUNCH_CHECK("qr_mirror_lower_kernel");
    }
    return TOMOS_OK;
}

// Columns [je, n) <- (I - V T^T V^T) [je, n) for the block [jb, je) just
// factored: V^T V, the block's T (recursive inversion levels), Z = V T,
// W = Z^T C, C -= V W.
static tomos_status qr_block_update(double* SA, int64_t ld, int64_t k, int64_t n, int64_t jb, int64_t je,
                                    const QrScratch& q, cudaStream_t st) {
    const int64_t krem = k - jb, nc = n - je;
    const int w = (int)(je - jb);
    int64_t cb = (krem * w + 255) / 256;
    if (cb > 4096) cb = 4096;
    qr_copy_v_kernel<<<(unsigned)cb, 256, 0, st>>>(SA, ld, jb, krem, w, q.Vb, k);
    TOMOS_LAUNCH_CHECK("qr_copy_v_kernel");
    tomos_status s = qr_gemm<true>(q.Vb, k, q.Vb, k, q.Y, w, w, w, krem, 1.0, 0.0, q.Pk, q.pk_doubles, st);
    if (s) return s;
    qr_block_t_init_kernel<<<(unsigned)((w * w + 255) / 256), 256, 0, st>>>(q.Tp, w, q.Tb2);
    TOMOS_LAUNCH_CHECK("qr_block_t_init_kernel");
    for (int64_t b = 32; b < w; b *= 2) {  // V^T V is symmetric: its storage is also row-major
        const int64_t pairs = (w - b + 2 * b - 1) / (2 * b);
        const dim3 g((unsigned)((b + 31) / 32), (unsigned)((b + 31) / 32), (unsigned)pairs);
        trtri_level_kernel<<<g, 256, 0, st>>>(q.Y, w, q.Tb2, w, q.Tb, b, 0);
        TOMOS_LAUNCH_CHECK("trtri_level_kernel");
        trtri_level_kernel<<<g, 256, 0, st>>>(q.Y, w, q.Tb2, w, q.Tb, b, 1);
        TOMOS_LAUNCH_CHECK("trtri_level_kernel");
    }
    s = qr_gemm<false>(q.Vb, k, q.Tb2, w, q.Z, k, krem, w, w, 1.0, 0.0, nullptr, 0, st);
    if (s) return s;
    double* C = SA + (size_t)je * ld + jb;
    s = qr_gemm<true>(q.Z, k, C, ld, q.Wb, w, w, nc, krem, 1.0, 0.0, q.Pk, q.pk_doubles, st);
    if (s) return s;
    return qr_gemm<false>(q.Vb, k, q.Wb, w, C, ld, krem, nc, w, -1.0, 1.0, nullptr, 0, st, 1);
}

// X (n x n, column-major, leading dimension ldx) = R^{-1} for the upper
// triangular R given row-major in Rt: zeros below the diagonal, 32 x 32
// diagonal blocks by back substitution, then levels X_IJ = -X_II R_IJ X_JJ
// of doubling block size (batched tiles, or two GEMMs a pair from
// kTrtriGemmMin on).  Tb holds one level's products; P (pcap doubles) the
// GEMMs' split-K partials.
static tomos_status trtri_rt(const double* Rt, int64_t n, double* X, int64_t ldx, double* Tb, double* P,
                             size_t pcap, cudaStream_t st) {
    const int64_t nbk = (n + 31) / 32;
    qr_zero_lower_kernel<<<(unsigned)((n * n + 255) / 256 < 4096 ? (n * n + 255) / 256 : 4096), 256, 0,
                           st>>>(X, ldx, n);
    TOMOS_LAUNCH_CHECK("qr_zero_lower_kernel");
    qr_trtri_diag_kernel<<<(unsigned)nbk, 32, 0, st>>>(Rt, n, X, ldx);
    TOMOS_LAUNCH_CHECK("qr_trtri_diag_kernel");
    for (int64_t b = 32; b < n; b *= 2) {
        const int64_t pairs = (n - b + 2 * b - 1) / (2 * b);
        if (b >= kTrtriGemmMin) {
            // few, large pairs: each product a qr_gemm_kernel launch
            //   T_p = R_IJ X_JJ  (R_IJ from the row-major copy of R),
            //   X_IJ = -X_II T_p
            for (int64_t p = 0; p < pairs; ++p) {
                const int64_t I0 = 2 * b * p, J0 = I0 + b;
                const int64_t Jn = n - J0 < b ? n - J0 : b;
                if (Jn <= 0) continue;
                double* Tp = Tb + (size_t)p * b * b;
                tomos_status gs = qr_gemm<true>(Rt + (size_t)I0 * n + J0, n, X + (size_t)J0 * ldx + J0, ldx,
                                                Tp, b, b, Jn, Jn, 1.0, 0.0, P, pcap, st);
                if (gs) return gs;
                gs = qr_gemm<false>(X + (size_t)I0 * ldx + I0, ldx, Tp, b, X + (size_t)J0 * ldx + I0, ldx, b, Jn,
                                    b, -1.0, 0.0, P, pcap, st);
                if (gs) return gs;
            }
            continue;
        }
        const dim3 g((unsigned)((b + 31) / 32), (unsigned)((b + 31) / 32), (unsigned)pairs);
        trtri_level_kernel<<<g, 256, 0, st>>>(Rt, n, X, ldx, Tb, b, 0);
        TOMOS_LAUNCH_CHECK("trtri_level_kernel");
        trtri_level_kernel<<<g, 256, 0, st>>>(Rt, n, X, ldx, Tb, b, 1);
        TOMOS_LAUNCH_CHECK("trtri_level_kernel");
    }
    return TOMOS_OK;
}


// ------------------------------------------------------------ wide path
//
// For sketches of up to kQrWideMaxN columns, the factorisation is formed
// from the whole sketch at once instead of 32-column panels (whose chains
// leave most SMs waiting at grid barriers):
//   G = SA^T SA                          (FP64 tensor-core GEMM)
//   D^-1 G D^-1 = U^T U, d_j = G_jj^1/2 (blocked Cholesky; R = U D is SA's
//                                        R with a positive diagonal)
//   R^-1 = D^-1 U^-1                     (trtri_rt)
//   Q_top = SA[0:n, :] R^-1, and the LU factorisation without pivoting
//   Q_top - S = L U' with s_j = -sign of the pivot: the Householder
//   reconstruction of the panel path applied to all n columns, whose S is
//   the sign LAPACK's dgeqr2 gives row j of R (R_h = S R, R_h^-1 = R^-1 S).
// It is Cholesky QR once, so it is used only when kappa_F(U) =
// ||U||_F ||U^-1||_F = sqrt(n) ||U^-1||_F is at most kQrWideMaxKappa (R then
// agrees with the Householder R to about kappa * 1e-16) and every Cholesky
// pivot is above kQrWideFloor; otherwise the panel path factors SA, which
// the wide path leaves untouched until it has passed both checks.
//
// The two n x n factorisations run in one cooperative launch each
// (fact_kernel): right-looking in 32-column blocks, one grid barrier a
// block.  CTA 0 updates the next diagonal block first and factors it
// (cta_chol / cta_lu_signed, and its inverses) while the other CTAs apply
// the current block to the rest of the trailing matrix in 32 x 32 tiles.

constexpr int64_t kQrWideMaxN = 2048;
constexpr double kQrWideMaxKappa = 1e6;
constexpr double kQrWideFloor = 1e-10;

struct WideScratch {
    double* G;     // n x n column-major: SA^T SA, equilibrated, then Q_top
    double* Ur;    // n x n row-major: U
    double* X;     // n x n column-major: U^-1, then R^-1
    double* d;     // n: column norms of SA
    double* sgn;   // n: S
    double* Xd;    // 2 x 2 x 32 x 32: a diagonal block's inverse factors (by block parity)
    double* kap;   // ||U^-1||_F^2
    double* Tb;    // trtri level products
    double* P;     // GEMM split-K partials
    size_t pcap;
    int* flag;     // [0] a Cholesky pivot failed or d_j == 0
    GridSync* gs;
    size_t bytes;
};

static WideScratch wide_layout(void* base, int64_t n) {
    WideScratch w;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t b) {
        char* r = p ? p + off : nullptr;
        off += a256(b);
        return r;
    };
    const size_t nn = n > 0 ? (size_t)n : 1;
    w.G = reinterpret_cast<double*>(take(sizeof(double) * nn * nn));
    w.Ur = reinterpret_cast<double*>(take(sizeof(double) * nn * nn));
    w.X = reinterpret_cast<double*>(take(sizeof(double) * nn * nn));
    w.d = reinterpret_cast<double*>(take(sizeof(double) * nn));
    w.sgn = reinterpret_cast<double*>(take(sizeof(double) * nn));
    w.Xd = reinterpret_cast<double*>(take(sizeof(double) * 4 * kHB * kHB));
    w.kap = reinterpret_cast<double*>(take(sizeof(double) * 2));
    size_t tb = 1;
    for (int64_t b = 32; b < n; b *= 2) {
        const size_t pairs = (size_t)((n - b + 2 * b - 1) / (2 * b));
        if (pairs * b * b > tb) tb = pairs * b * b;
    }
    w.Tb = reinterpret_cast<double*>(take(sizeof(double) * tb));
    w.pcap = 4 * nn * nn;
    w.P = reinterpret_cast<double*>(take(sizeof(double) * w.pcap));
    w.flag = reinterpret_cast<int*>(take(sizeof(int) * 4));
    w.gs = reinterpret_cast<GridSync*>(take(sizeof(GridSync)));
    w.bytes = off;
    return w;
}

// d_j = G_jj^1/2 (flag[0] set when a column of SA is zero or not finite).
__global__ void wide_colnorm_kernel(const double* G, int64_t n, double* d, int* flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double gi = G[i * n + i];
        const bool ok = gi > 0.0 && isfinite(gi);
        if (!ok) atomicOr(flag, 1);
        d[i] = ok ? sqrt(gi) : 1.0;
    }
}

// The upper half of D^-1 G D^-1 in place (d from wide_colnorm_kernel, so no
// thread reads a diagonal entry another one rescales).
__global__ void wide_equilibrate_kernel(double* G, int64_t n, const double* d) {
    const int64_t total = n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        if (i <= j) G[e] /= d[i] * d[j];
    }
}

// ||X||_F^2 of the n x n column-major X: block b sums its contiguous
// chunk into part[b], then one thread sums the parts in block order.
__global__ void wide_fro2_part_kernel(const double* X, int64_t total, double* part) {
    __shared__ double sm[32];
    const int64_t chunk = (total + gridDim.x - 1) / gridDim.x;
    const int64_t e0 = (int64_t)blockIdx.x * chunk;
    const int64_t e1 = e0 + chunk < total ? e0 + chunk : total;
    double s = 0.0;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) s += X[e] * X[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sm[w];
        part[blockIdx.x] = t;
    }
}

__global__ void wide_fro2_sum_kernel(const double* part, int np, double* out) {
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < np; ++b) t += part[b];
        *out = t;
    }
}

// X <- D^-1 X (rows scaled: U^-1 -> R^-1).
__global__ void wide_row_scale_kernel(double* X, int64_t n, const double* d) {
    const int64_t total = n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
        X[e] /= d[e % n];
}

// The outputs: R_h^-1 = R^-1 S in the leading n x n block of SA (zeros
// below the diagonal) and, when asked, R_h = S U D (column-major, ld n).
__global__ void wide_output_kernel(const double* X, const double* Ur, const double* d, const double* sgn,
                                   int64_t n, double* SA, int64_t ld, double* R) {
    const int64_t total = n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        const double sj = sgn ? sgn[j] : 1.0, si = sgn ? sgn[i] : 1.0;  // NULL: no signs
        SA[(size_t)j * ld + i] = i <= j ? X[e] * sj : 0.0;
        if (R) R[e] = i <= j ? si * Ur[(size_t)i * n + j] * d[j] : 0.0;
    }
}

struct FactArgs {
    double* M;      // n x n column-major (ld n), updated in place
    int64_t n;
    int mode;       // 0: Cholesky of the upper half (U to Ur); 1: signed LU (signs to sgn)
    double* Ur;
    double* Xd;
    double* sgn;
    int64_t keep;   // LU: the column dlarfg leaves as the identity, or -1
    double floor;
    int* fail;
    GridSync* gs;
};

constexpr int kFactSmemMats = 6;

// X = R^{-1} for an upper triangular 32 x 32 R in shared memory: lane c of
// warp 0 solves R x = e_c by back substitution on registers (rows of R are
// broadcast reads), two partial sums a row; the other warps wait at the end.
__device__ __forceinline__ void warp_inv_upper(const HMat& R, HMat& X, double* dinv) {
    const int t = threadIdx.x;
    if (t < kHB) dinv[t] = 1.0 / R[t][t];
    __syncthreads();
    if (t < kHB) {
        const int c = t;
        double x[kHB];
#pragma unroll
        for (int i = kHB - 1; i >= 0; --i) {
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = i + 1; k < kHB; k += 2) {
                s0 = fma(R[i][k], x[k], s0);
                if (k + 1 < kHB) s1 = fma(R[i][k + 1], x[k + 1], s1);
            }
            const double v = ((i == c ? 1.0 : 0.0) - (s0 + s1)) * dinv[i];
            x[i] = i > c ? 0.0 : v;
        }
#pragma unroll
        for (int i = 0; i < kHB; ++i) X[i][c] = x[i];
    }
    __syncthreads();
}

// Y = L^{-1} for the unit lower triangular L held strictly below the
// diagonal of Q: lane c of warp 0 solves L y = e_c by forward substitution.
__device__ __forceinline__ void warp_inv_unit_lower(const HMat& Q, HMat& Y) {
    const int t = threadIdx.x;
    if (t < kHB) {
        const int c = t;
        double y[kHB];
#pragma unroll
        for (int i = 0; i < kHB; ++i) {
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int k = 0; k < i; k += 2) {
                s0 = fma(Q[i][k], y[k], s0);
                if (k + 1 < i) s1 = fma(Q[i][k + 1], y[k + 1], s1);
            }
            const double v = (i == c ? 1.0 : 0.0) - (s0 + s1);
            y[i] = i < c ? 0.0 : v;
        }
#pragma unroll
        for (int i = 0; i < kHB; ++i) Y[i][c] = y[i];
    }
    __syncthreads();
}

// Factor the diagonal block of block column p (M's block already holds
// every earlier update): Cholesky U_pp (to Ur) and X = U_pp^-1, or the
// signed LU L\U of the block with X = U^-1, Y = L^-1; X (and Y) to
// Xd[p & 1] as row-major 32 x 32.
__device__ void fact_diag(const FactArgs& a, int64_t p, double* sm) {
    HMat& B = *reinterpret_cast<HMat*>(sm);
    HMat& R = *reinterpret_cast<HMat*>(sm + 1 * kHB * (kHB + 1));
    HMat& X = *reinterpret_cast<HMat*>(sm + 2 * kHB * (kHB + 1));
    HMat& Y = *reinterpret_cast<HMat*>(sm + 3 * kHB * (kHB + 1));
    __shared__ int okf;
    __shared__ double sg[kHB];
    const int t = threadIdx.x;
    const int64_t n = a.n, jb = p * kHB;
    const int nb = (int)(n - jb < kHB ? n - jb : kHB);
    __syncthreads();
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int r = e & 31, c = e >> 5;
        B[r][c] = (r < nb && c < nb) ? __ldcg(a.M + (size_t)(jb + c) * n + jb + r) : (r == c ? 1.0 : 0.0);
    }
    double* xd = a.Xd + (size_t)(p & 1) * 2 * kHB * kHB;
    __shared__ double dinv[kHB];
    if (a.mode == 0) {
        const bool ok = cta_chol(B, R, a.floor, &okf);
        if (!ok && t == 0) atomicExch(a.fail, 1);
        warp_inv_upper(R, X, dinv);
        for (int e = t; e < kHB * kHB; e += blockDim.x) {
            const int r = e >> 5, c = e & 31;
            if (r < nb && c < nb) a.Ur[(size_t)(jb + r) * n + jb + c] = r <= c ? R[r][c] : 0.0;
            xd[e] = X[r][c];
        }
    } else {
        const int64_t kk = a.keep - jb;
        cta_lu_signed(B, sg, (kk >= 0 && kk < nb) ? (int)kk : -1);
        for (int e = t; e < kHB * kHB; e += blockDim.x) {
            const int r = e >> 5, c = e & 31;
            R[r][c] = r <= c ? B[r][c] : 0.0;
        }
        if (t < nb) a.sgn[jb + t] = sg[t];
        __syncthreads();
        warp_inv_upper(R, X, dinv);
        warp_inv_unit_lower(B, Y);
        for (int e = t; e < kHB * kHB; e += blockDim.x) {
            const int r = e >> 5, c = e & 31;
            xd[e] = X[r][c];
            xd[kHB * kHB + e] = Y[r][c];
        }
    }
    __syncthreads();
}

// C = A^T B (TA) or A B over the CTA, 32 x 32 shared tiles.
template <bool TA>
__device__ __forceinline__ void fact_mm(const HMat& A, const HMat& B, HMat& C) {
    const int t = threadIdx.x;
    const int i = t & 31, j0 = (t >> 5) * 4;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < kHB; ++k) {
        const double x = TA ? A[k][i] : A[i][k];
#pragma unroll
        for (int q = 0; q < 4; ++q) s[q] += x * B[k][j0 + q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) C[i][j0 + q] = s[q];
}

// Trailing tile `tau` of block column p: Cholesky tiles (I <= J) in rows,
// LU tiles (I, J) row by row; tile 0 is the next diagonal block.
__device__ void fact_tile(const FactArgs& a, int64_t p, int64_t tau, double* sm) {
    HMat& A1 = *reinterpret_cast<HMat*>(sm);
    HMat& P1 = *reinterpret_cast<HMat*>(sm + 1 * kHB * (kHB + 1));
    HMat& A2 = *reinterpret_cast<HMat*>(sm + 2 * kHB * (kHB + 1));
    HMat& P2 = *reinterpret_cast<HMat*>(sm + 3 * kHB * (kHB + 1));
    HMat& F1 = *reinterpret_cast<HMat*>(sm + 4 * kHB * (kHB + 1));
    HMat& F2 = *reinterpret_cast<HMat*>(sm + 5 * kHB * (kHB + 1));
    const int t = threadIdx.x;
    const int64_t n = a.n, jb = p * kHB, t0 = jb + kHB;
    const int64_t nt = (n - t0 + kHB - 1) / kHB;
    int64_t I, J;
    if (a.mode == 0) {
        I = 0;
        int64_t rest = tau;
        while (rest >= nt - I) {
            rest -= nt - I;
            ++I;
        }
        J = I + rest;
    } else {
        I = tau / nt;
        J = tau % nt;
    }
    const int64_t I0 = t0 + I * kHB, J0 = t0 + J * kHB;
    const int wI = (int)(n - I0 < kHB ? n - I0 : kHB), wJ = (int)(n - J0 < kHB ? n - J0 : kHB);
    const double* xd = a.Xd + (size_t)(p & 1) * 2 * kHB * kHB;
    __syncthreads();
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int r = e & 31, c = e >> 5;
        F1[r][c] = __ldcg(xd + r * kHB + c);
        if (a.mode == 0) {
            // row panel of G: A1 = G[jb.., I cols], A2 = G[jb.., J cols]
            A1[r][c] = c < wI ? __ldcg(a.M + (size_t)(I0 + c) * n + jb + r) : 0.0;
            A2[r][c] = c < wJ ? __ldcg(a.M + (size_t)(J0 + c) * n + jb + r) : 0.0;
        } else {
            F2[r][c] = __ldcg(xd + kHB * kHB + r * kHB + c);
            // A1 = M[I rows, panel cols], A2 = M[panel rows, J cols]
            A1[r][c] = r < wI ? __ldcg(a.M + (size_t)(jb + c) * n + I0 + r) : 0.0;
            A2[r][c] = c < wJ ? __ldcg(a.M + (size_t)(J0 + c) * n + jb + r) : 0.0;
        }
    }
    __syncthreads();
    if (a.mode == 0) {
        fact_mm<true>(F1, A1, P1);   // U_pI = X^T G_pI
        if (I != J) fact_mm<true>(F1, A2, P2);  // U_pJ
        __syncthreads();
        const HMat& PJ = I != J ? P2 : P1;
        fact_mm<true>(P1, PJ, A1);   // U_pI^T U_pJ
        if (I == J)
            for (int e = t; e < kHB * kHB; e += blockDim.x) {
                const int r = e >> 5, c = e & 31;
                if (c < wJ) a.Ur[(size_t)(jb + r) * n + J0 + c] = P1[r][c];
            }
    } else {
        fact_mm<false>(A1, F1, P1);  // L_Ip = M_Ip U_pp^-1
        fact_mm<false>(F2, A2, P2);  // U_pJ = L_pp^-1 M_pJ
        __syncthreads();
        fact_mm<false>(P1, P2, A1);  // L_Ip U_pJ
    }
    __syncthreads();
    for (int e = t; e < kHB * kHB; e += blockDim.x) {
        const int r = e & 31, c = e >> 5;
        if (r < wI && c < wJ) a.M[(size_t)(J0 + c) * n + I0 + r] -= A1[r][c];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kQrThreads, 1) fact_kernel(FactArgs a) {
    extern __shared__ __align__(16) double fsm[];
    __shared__ int sflag;
    unsigned int gen = 0;
    const int64_t n = a.n;
    const int64_t np = (n + kHB - 1) / kHB;
    const int64_t G = gridDim.x;
    if (blockIdx.x == 0) fact_diag(a, 0, fsm);
    if (!grid_sync(a.gs, gen, &sflag)) return;
    for (int64_t p = 0; p + 1 < np; ++p) {
        const int64_t t0 = (p + 1) * kHB;
        const int64_t nt = (n - t0 + kHB - 1) / kHB;
        const int64_t ntiles = a.mode == 0 ? nt * (nt + 1) / 2 : nt * nt;
        if (blockIdx.x == 0) {
            fact_tile(a, p, 0, fsm);
            fact_diag(a, p + 1, fsm);
            if (G == 1)
                for (int64_t tau = 1; tau < ntiles; ++tau) fact_tile(a, p, tau, fsm);
        } else {
            for (int64_t tau = blockIdx.x; tau < ntiles; tau += G - 1) fact_tile(a, p, tau, fsm);
        }
        if (!grid_sync(a.gs, gen, &sflag)) return;
    }
}

// One cooperative launch of fact_kernel (one CTA per SM).
static tomos_status launch_fact(const FactArgs& fa, GridSync* gs, cudaStream_t st) {
    const size_t smem = sizeof(double) * kFactSmemMats * kHB * (kHB + 1);
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(fact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TOMOS_CUDA_TRY(cudaMemsetAsync(gs, 0, sizeof(GridSync), st));
    FactArgs a = fa;
    void* args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)fact_kernel, dim3((unsigned)sm_count()),
                                                dim3(kQrThreads), args, smem, st);
    if (e != cudaSuccess) return cuda_fail(e, "sketch_qr: cooperative launch (wide path)");
    return TOMOS_OK;
}

// The wide path (see above).  *done false: SA untouched, the panel path
// must factor it (not used for this size, a failed pivot, or kappa above
// kQrWideMaxKappa).
// any_signs: R is returned with a positive diagonal (the Cholesky factor
// scaled back) instead of LAPACK's row signs S, which skips Q_top and its
// signed LU (R^-1 then differs from the LAPACK one by the signs of its
// columns: R_h^-1 = R^-1 S).
static tomos_status qr_wide(int64_t k, int64_t n, double* SA, int64_t ld, double* R, const WideScratch& w,
                            cudaStream_t st, bool* done, bool any_signs) {
    *done = false;
    TOMOS_CUDA_TRY(cudaMemsetAsync(w.flag, 0, sizeof(int) * 4, st));
    // the Gram S^T S: its upper triangle, mirrored
    tomos_status s = qr_gemm<true>(SA, ld, SA, ld, w.G, n, n, n, k, 1.0, 0.0, w.P, w.pcap, st, 0, true);
    if (s) return s;
    const unsigned eb = (unsigned)((n * n + 255) / 256 < 4096 ? (n * n + 255) / 256 : 4096);
    wide_colnorm_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(w.G, n, w.d, w.flag);
    TOMOS_LAUNCH_CHECK("wide_colnorm_kernel");
    wide_equilibrate_kernel<<<eb, 256, 0, st>>>(w.G, n, w.d);
    TOMOS_LAUNCH_CHECK("wide_equilibrate_kernel");
    FactArgs fa;
    fa.M = w.G;
    fa.n = n;
    fa.mode = 0;
    fa.Ur = w.Ur;
    fa.Xd = w.Xd;
    fa.sgn = w.sgn;
    fa.keep = -1;
    fa.floor = kQrWideFloor;
    fa.fail = w.flag;
    fa.gs = w.gs;
    s = launch_fact(fa, w.gs, st);
    if (s) return s;
    s = trtri_rt(w.Ur, n, w.X, n, w.Tb, w.P, w.pcap, st);
    if (s) return s;
    {
        // the split-K partial buffer is free between the products
        const int np = w.pcap >= 256 ? 256 : (int)w.pcap;
        wide_fro2_part_kernel<<<np, 256, 0, st>>>(w.X, n * n, w.P);
        TOMOS_LAUNCH_CHECK("wide_fro2_part_kernel");
        wide_fro2_sum_kernel<<<1, 32, 0, st>>>(w.P, np, w.kap);
        TOMOS_LAUNCH_CHECK("wide_fro2_sum_kernel");
    }
    int flag = 0;
    double kap2 = 0.0;
    GridSync gsh{};
    TOMOS_CUDA_TRY(cudaMemcpyAsync(&flag, w.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaMemcpyAsync(&kap2, w.kap, sizeof(double), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaMemcpyAsync(&gsh, w.gs, sizeof(gsh), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
    if (gsh.err) return fail(TOMOS_ERR_CUDA, "sketch_qr: a bounded grid barrier wait expired");
    const double kappa = std::sqrt((double)n * kap2);
    if (flag || !(kappa <= kQrWideMaxKappa)) return TOMOS_OK;  // the panel path takes over
    wide_row_scale_kernel<<<eb, 256, 0, st>>>(w.X, n, w.d);
    TOMOS_LAUNCH_CHECK("wide_row_scale_kernel");
    if (any_signs) {
        wide_output_kernel<<<eb, 256, 0, st>>>(w.X, w.Ur, w.d, nullptr, n, SA, ld, R);
        TOMOS_LAUNCH_CHECK("wide_output_kernel");
        *done = true;
        return TOMOS_OK;
    }
    // Q_top = SA[0:n, :] R^-1 into G (no longer needed), then its signed LU
    s = qr_gemm<false>(SA, ld, w.X, n, w.G, n, n, n, n, 1.0, 0.0, w.P, w.pcap, st);
    if (s) return s;
    fa.mode = 1;
    fa.keep = k == n ? n - 1 : -1;
    s = launch_fact(fa, w.gs, st);
    if (s) return s;
    wide_output_kernel<<<eb, 256, 0, st>>>(w.X, w.Ur, w.d, w.sgn, n, SA, ld, R);
    TOMOS_LAUNCH_CHECK("wide_output_kernel");
    TOMOS_CUDA_TRY(cudaMemcpyAsync(&gsh, w.gs, sizeof(gsh), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
    if (gsh.err) return fail(TOMOS_ERR_CUDA, "sketch_qr: a bounded grid barrier wait expired");
    *done = true;
    return TOMOS_OK;
}

// Whether the wide path is tried: n from 64 to kQrWideMaxN columns.
// TOMOS_QR_WIDE=0 turns it off, =1 tries it at every size up to the max,
// =3 requires it there (a sketch it refuses is then an error; for tests).
static int qr_wide_mode() {
    static int mode = -1;
    if (mode < 0) {
        const char* e = std::getenv("TOMOS_QR_WIDE");
        mode = e ? std::atoi(e) : 2;
    }
    return mode;
}

static bool qr_wide_used(int64_t n) {
    const int mode = qr_wide_mode();
    if (mode == 0 || n > kQrWideMaxN) return false;
    return mode == 1 || mode == 3 ? n >= 1 : n >= 64;
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

size_t tomos_sketch_qr_scratch_bytes(int64_t k, int64_t n) {
    if (k < 0 || n < 0) return 0;
    const size_t panel = qr_layout(nullptr, k, n).bytes;
    return qr_wide_used(n) ? panel + wide_layout(nullptr, n).bytes : panel;
}

tomos_status tomos_sketch_qr_precond_ex_f64(int64_t k, int64_t n, double* SA, int64_t ld, double* R,
                                            int32_t flags, void* scratch, size_t scratch_bytes, void* stream) {
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
    if (qr_wide_used(n) && scratch_bytes >= need.bytes + wide_layout(nullptr, n).bytes) {
        bool done = false;
        tomos_status ws = qr_wide(k, n, SA, ld, R, wide_layout(static_cast<char*>(scratch) + need.bytes, n),
                                  st, &done, (flags & TOMOS_QR_ANY_SIGNS) != 0);
        if (ws) return ws;
        if (done) return TOMOS_OK;
        if (qr_wide_mode() == 3)
            return fail(TOMOS_ERR_NUMERIC, "sketch_qr: the wide path refused this sketch (TOMOS_QR_WIDE=3)");
    }
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(qr_hr_v_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)hr_v_smem()));
    TOMOS_CUDA_TRY(cudaMemsetAsync(q.flag, 0, sizeof(int) * 4, st));
    bool done = false;
    {
        // One cooperative launch when every CTA of a full wave can be resident.
        int dev = 0, coop = 0, per_sm = 0;
        TOMOS_CUDA_TRY(cudaGetDevice(&dev));
        TOMOS_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        const size_t psmem = hr_v_smem() > kQrTileSmemDoubles * sizeof(double)
                                 ? hr_v_smem()
                                 : kQrTileSmemDoubles * sizeof(double);
        TOMOS_CUDA_TRY(cudaFuncSetAttribute(qr_persist_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem));
        TOMOS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qr_persist_kernel,
                                                                     kQrThreads, psmem));
        if (coop && per_sm >= 1) {
            QrPersistArgs pa;
            pa.A = SA;
            pa.ld = ld;
            pa.k = k;
            pa.n = n;
            pa.q = q;
            pa.gs = static_cast<GridSync*>(q.gsync);
            const bool blocked = q.Vb != nullptr;
            const int64_t bw = blocked ? kQrBlock : n;
            for (int64_t jb = 0; jb < n; jb += bw) {
                const int64_t je = jb + bw < n ? jb + bw : n;
                pa.jb = jb;
                pa.je = je;
                pa.Tp = blocked ? q.Tp : q.T;
                pa.t_stride = blocked ? kHB * kHB : 0;
                // counter and generation start at 0; the error word is
                // cleared once, so an expired wait in any launch is reported
                TOMOS_CUDA_TRY(cudaMemsetAsync(q.gsync, 0, jb == 0 ? sizeof(GridSync) : 2 * sizeof(unsigned int), st));
                void* args[] = {&pa};
                cudaError_t e = cudaLaunchCooperativeKernel((const void*)qr_persist_kernel,
                                                            dim3((unsigned)sm_count()), dim3(kQrThreads),
                                                            args, psmem, st);
                if (e != cudaSuccess) {
                    cudaGetLastError();
                    if (jb == 0) break;  // fall back to the per-phase kernels
                    return cuda_fail(e, "sketch_qr: cooperative launch");
                }
                if (je == n) done = true;
                if (je < n) {
                    tomos_status bs = qr_block_update(SA, ld, k, n, jb, je, q, st);
                    if (bs) return bs;
                }
            }
        }
    }
    const size_t tile_smem = kQrTileSmemDoubles * sizeof(double);
    if (!done) {
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(qr_w_part_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tile_smem));
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(qr_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tile_smem));
    const int nb0 = (int)(n < kQrNb ? n : kQrNb);
    qr_gram_kernel<<<(unsigned)qr_row_tiles(k), kQrThreads, kHB * (kHB + 1) * sizeof(double), st>>>(
        SA, ld, k, nb0, q.Gp);
    TOMOS_LAUNCH_CHECK("qr_gram_kernel");
    int ngp = (int)qr_row_tiles(k);
    for (int64_t j0 = 0; j0 < n; j0 += kQrNb) {
        const int nb = (int)(n - j0 < kQrNb ? n - j0 : kQrNb);
        const int64_t krem = k - j0;
        int gp = (int)((krem + 63) / 64);
        if (gp > kQrPanelCtas) gp = kQrPanelCtas;
        if (gp < 1) gp = 1;
        HrArgs H;
        H.A = SA;
        H.ld = ld;
        H.k = k;
        H.j0 = j0;
        H.nb = nb;
        H.rpc = ((krem + gp - 1) / gp + kHB - 1) / kHB * kHB;
        H.Gp = q.Gp;
        H.ngp = ngp;
        H.Qs = q.Qs;
        H.kq = k;
        H.G2p = q.G2p;
        H.R1 = q.R1;
        H.fail = q.flag + 1;
        H.T = q.T;
        H.tau = q.tau;
        qr_hr_q1_kernel<<<(unsigned)gp, kQrThreads, hr_q1_smem(), st>>>(H);
        TOMOS_LAUNCH_CHECK("qr_hr_q1_kernel");
        qr_hr_v_kernel<<<(unsigned)gp, kQrThreads, hr_v_smem(), st>>>(H);
        TOMOS_LAUNCH_CHECK("qr_hr_v_kernel");
        const int64_t nc = n - j0 - nb;
        if (nc <= 0) continue;
        const int64_t chunk_rows = ((krem + kQrChunks - 1) / kQrChunks + kHB - 1) / kHB * kHB;
        const int nchunks = (int)((krem + chunk_rows - 1) / chunk_rows);
        const unsigned ctiles = (unsigned)((nc + kQrWc - 1) / kQrWc);
        qr_w_part_kernel<<<dim3(ctiles, (unsigned)nchunks), kQrThreads, tile_smem, st>>>(
            SA, ld, k, n, j0, nb, chunk_rows, q.Wp);
        TOMOS_LAUNCH_CHECK("qr_w_part_kernel");
        const int nb_next = (int)(nc < kQrNb ? nc : kQrNb);
        const unsigned rtiles = (unsigned)qr_row_tiles(krem);
        qr_apply_kernel<<<dim3(ctiles, rtiles), kQrThreads, tile_smem, st>>>(
            SA, ld, k, n, j0, nb, nchunks, q.Wp, q.T, nb_next, q.Gp);
        TOMOS_LAUNCH_CHECK("qr_apply_kernel");
        ngp = (int)rtiles;
    }
    }  // per-phase kernels
    qr_extract_kernel<<<(unsigned)((n * n + 255) / 256 < 4096 ? (n * n + 255) / 256 : 4096), 256, 0,
                        st>>>(SA, ld, n, q.Rt, R, q.flag);
    TOMOS_LAUNCH_CHECK("qr_extract_kernel");
    int flag = 0;
    GridSync gsh{};
    TOMOS_CUDA_TRY(cudaMemcpyAsync(&flag, q.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (done)
        TOMOS_CUDA_TRY(cudaMemcpyAsync(&gsh, q.gsync, sizeof(gsh), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
    if (gsh.err)
        return fail(TOMOS_ERR_CUDA, "sketch_qr: a bounded grid barrier wait expired");
    if (flag)
        return fail(TOMOS_ERR_NUMERIC,
                    "generate_sketch_qr_precond: trtri failed -- R is singular.");
    return trtri_rt(q.Rt, n, SA, ld, q.Tb, q.Pk, q.pk_doubles, st);
}

tomos_status tomos_sketch_qr_precond_f64(int64_t k, int64_t n, double* SA, int64_t ld, double* R,
                                         void* scratch, size_t scratch_bytes, void* stream) {
    return tomos_sketch_qr_precond_ex_f64(k, n, SA, ld, R, 0, scratch, scratch_bytes, stream);
}

}  // extern "C"
