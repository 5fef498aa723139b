// adjoint_batch.cu -- K adjoint solves at once: Lambda_k = (A^T A)^{-1} G_k.
//
// The same preconditioned conjugate gradients as tomos_lsqr_adjoint_dense
// (adjoint.cu: CG on R^{-T} A^T A R^{-1} mu = R^{-T} g, lambda = R^{-1} mu),
// one recurrence per right-hand side, but the products with A are shared:
// every iteration forms, for all K directions P (n x K) at once,
//   Q = A P      one tcgen05 product over A (tomos_mm_ex), and
//   W = A^T Q    a second one, its long K (the m rows) split over CTAs,
// so A is read twice an iteration for all K instead of once per right-hand
// side.  The n-side kernels run every column k in blockIdx.y; a column
// whose recurrence has stopped returns at once.  Scalars and vectors are
// FP64; the direction goes to the products as FP32.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "lsqr.cuh"

namespace tomos_b200 {

namespace {

struct AdjCol {  // the state of one right-hand side
    double rz;   // r . z of the current direction
    double gg;   // ||g||^2
    double rr;   // ||r||^2 after the last update
    int iter, done, converged, breakdown;
};

struct BArgs {
    int64_t n;
    int K;
    int nbp;  // partial sums per column (the larger of the two grids)
    double *lam, *r, *z, *t, *w, *pd;  // n x K, column k at + k n
    float *p32, *w32;                  // the direction / A^T A p in FP32
    AdjCol* col;
    double *rr_part, *rz_part, *pw_part;  // [K][nbp]
    const float* G;
    int64_t ldg;
    const double* Rcm;  // R^{-1} column-major (NULL: no preconditioner)
    const double* Rrm;  // R^{-1} row-major
    double tol;
    int max_iters;
};

__device__ __forceinline__ double* colv(double* base, const BArgs& a, int k) { return base + (size_t)k * a.n; }

// r = g, lambda = 0; partial ||g||^2.
__global__ void __launch_bounds__(256) bk_init_kernel(BArgs a) {
    __shared__ double sm[32];
    const int k = blockIdx.y;
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    double v = 0.0;
    if (i < a.n) {
        v = (double)a.G[(size_t)k * a.ldg + i];
        colv(a.r, a, k)[i] = v;
        colv(a.lam, a, k)[i] = 0.0;
    }
    const double s = block_sum(v * v, sm);
    if (threadIdx.x == 0) a.rr_part[(size_t)k * a.nbp + blockIdx.x] = s;
}

// t = R^{-T} r (a warp per entry).
__global__ void __launch_bounds__(256) bk_pt_kernel(BArgs a) {
    const int k = blockIdx.y;
    if (a.col[k].done) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * 8 + w;
    if (j >= a.n) return;
    const double* c = a.Rcm + (size_t)j * a.n;
    const double* r = colv(a.r, a, k);
    double s = 0.0;
    for (int64_t i = lane; i < a.n; i += 32) s += c[i] * r[i];
    s = warp_sum(s);
    if (lane == 0) colv(a.t, a, k)[j] = s;
}

// z = R^{-1} t (or z = r); partial r . z.
__global__ void __launch_bounds__(256) bk_p_kernel(BArgs a) {
    const int k = blockIdx.y;
    if (a.col[k].done) return;
    __shared__ double smz[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * 8 + w;
    double rz = 0.0;
    if (i < a.n) {
        const double* r = colv(a.r, a, k);
        double z;
        if (a.Rrm) {
            const double* row = a.Rrm + (size_t)i * a.n;
            const double* t = colv(a.t, a, k);
            double s = 0.0;
            for (int64_t j = lane; j < a.n; j += 32) s += row[j] * t[j];
            z = warp_sum(s);
        } else {
            z = r[i];
        }
        if (lane == 0) colv(a.z, a, k)[i] = z;
        rz = z * r[i];
    }
    if (lane == 0) smz[w] = rz;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) s += smz[q];
        a.rz_part[(size_t)k * a.nbp + blockIdx.x] = s;
    }
}

__device__ double sum_parts(const double* p, int count, double* sm) { return block_sum_array(p, count, sm); }

// One block a column: rz and ||g||^2, p = z, the state.
__global__ void __launch_bounds__(256) bk_start_kernel(BArgs a, int nb8, int nbu) {
    __shared__ double sm[32];
    const int k = blockIdx.x;
    const double rz = sum_parts(a.rz_part + (size_t)k * a.nbp, nb8, sm);
    const double gg = sum_parts(a.rr_part + (size_t)k * a.nbp, nbu, sm);
    const double* z = colv(a.z, a, k);
    double* pd = colv(a.pd, a, k);
    float* p32 = a.p32 + (size_t)k * a.n;
    for (int64_t i = threadIdx.x; i < a.n; i += blockDim.x) {
        pd[i] = z[i];
        p32[i] = (float)z[i];
    }
    if (threadIdx.x == 0) {
        AdjCol& c = a.col[k];
        c.rz = rz;
        c.gg = gg;
        c.rr = gg;
        c.iter = 0;
        c.converged = gg == 0.0 ? 1 : 0;
        c.breakdown = 0;
        c.done = (gg == 0.0 || a.max_iters == 0) ? 1 : 0;
    }
}

// w = (A^T A p) from the product (FP32 -> FP64); partial p . w.
__global__ void __launch_bounds__(256) bk_w_kernel(BArgs a) {
    const int k = blockIdx.y;
    if (a.col[k].done) return;
    __shared__ double sm[32];
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    double pw = 0.0;
    if (i < a.n) {
        const double w = (double)a.w32[(size_t)k * a.n + i];
        colv(a.w, a, k)[i] = w;
        pw = w * colv(a.pd, a, k)[i];
    }
    const double s = block_sum(pw, sm);
    if (threadIdx.x == 0) a.pw_part[(size_t)k * a.nbp + blockIdx.x] = s;
}

// alpha = rz / p.w; lambda += alpha p; r -= alpha w; partial ||r||^2.
__global__ void __launch_bounds__(256) bk_update_kernel(BArgs a, int nbu) {
    const int k = blockIdx.y;
    if (a.col[k].done) return;
    __shared__ double sm[32];
    const double pw = sum_parts(a.pw_part + (size_t)k * a.nbp, nbu, sm);
    const double alpha = pw > 0.0 ? a.col[k].rz / pw : 0.0;
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    double v = 0.0;
    if (i < a.n) {
        colv(a.lam, a, k)[i] += alpha * colv(a.pd, a, k)[i];
        double* r = colv(a.r, a, k);
        v = r[i] - alpha * colv(a.w, a, k)[i];
        r[i] = v;
    }
    const double s = block_sum(v * v, sm);
    if (threadIdx.x == 0) {
        a.rr_part[(size_t)k * a.nbp + blockIdx.x] = s;
        if (blockIdx.x == 0 && !(pw > 0.0)) a.col[k].breakdown = 1;
    }
}

// One block a column: the stopping rule, beta = rz' / rz, p = z + beta p.
__global__ void __launch_bounds__(256) bk_finish_kernel(BArgs a, int nb8, int nbu) {
    const int k = blockIdx.x;
    if (a.col[k].done) return;
    __shared__ double sm[32];
    __shared__ double bc[2];
    const double rr = sum_parts(a.rr_part + (size_t)k * a.nbp, nbu, sm);
    const double rz = sum_parts(a.rz_part + (size_t)k * a.nbp, nb8, sm);
    if (threadIdx.x == 0) {
        AdjCol& c = a.col[k];
        c.iter += 1;
        c.rr = rr;
        bc[0] = 0.0;
        bc[1] = 0.0;
        if (sqrt(rr) <= a.tol * sqrt(c.gg)) {
            c.converged = 1;
            c.done = 1;
        } else if (c.breakdown || c.iter >= a.max_iters || !(rz > 0.0)) {
            c.done = 1;
        } else {
            bc[0] = rz / c.rz;
            bc[1] = 1.0;
            c.rz = rz;
        }
    }
    __syncthreads();
    if (bc[1] == 0.0) return;
    const double beta = bc[0];
    const double* z = colv(a.z, a, k);
    double* pd = colv(a.pd, a, k);
    float* p32 = a.p32 + (size_t)k * a.n;
    for (int64_t i = threadIdx.x; i < a.n; i += blockDim.x) {
        const double p = z[i] + beta * pd[i];
        pd[i] = p;
        p32[i] = (float)p;
    }
}

__global__ void bk_out_kernel(const double* lam, int64_t n, int K, float* out, int64_t ldl) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * K) return;
    const int64_t k = t / n, i = t % n;
    out[(size_t)k * ldl + i] = (float)lam[t];
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

tomos_status tomos_lsqr_adjoint_batch_dense(const tomos_dense* A, int32_t K, const float* G, int64_t ldg,
                                            float* Lambda, int64_t ldl, tomos_workspace* ws,
                                            const tomos_lsqr_opts* opts, tomos_lsqr_report* reports,
                                            void* stream) {
    if (!A || !opts) return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_batch: null pointer");
    if (opts->max_iters < 0) return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_batch: negative max_iters");
    const int64_t m = A->rows, n = A->cols;
    if (K < 0 || m < 0 || n < 0 || (K > 0 && (ldg < n || ldl < n)))
        return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_batch: bad sizes");
    tomos_status s = workspace_check(ws, m, n);
    if (s) return s;
    if (reports && K > 0) std::memset(reports, 0, sizeof(tomos_lsqr_report) * (size_t)K);
    if (K == 0 || n == 0) return TOMOS_OK;
    if (!G || !Lambda || (!A->values && m * n > 0)) return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_batch: null pointer");
    const bool packed = A->numeric == TOMOS_FP32_16 || A->numeric == TOMOS_FP32_BF16;
    const int32_t tier =
        opts->iter_tier == TOMOS_TIER_AUTO ? (packed ? TOMOS_TIER_ACCURATE : TOMOS_TIER_AUTO) : opts->iter_tier;

    // the products' operands: P (n x K), Q (m x K), W (n x K), FP32 column-major
    tomos_dense P{TOMOS_FP32, TOMOS_COL_MAJOR, n, K, n, nullptr, nullptr, 0, 0};
    tomos_dense Q{TOMOS_FP32, TOMOS_COL_MAJOR, m, K, m > 0 ? m : 1, nullptr, nullptr, 0, 0};
    tomos_dense W{TOMOS_FP32, TOMOS_COL_MAJOR, n, K, n, nullptr, nullptr, 0, 0};
    const size_t mm1 = tomos_mm_scratch_bytes(TOMOS_NO_TRANSPOSE, TOMOS_NO_TRANSPOSE, A, tier, &P);
    const size_t mm2 = tomos_mm_scratch_bytes(TOMOS_TRANSPOSE, TOMOS_NO_TRANSPOSE, A, tier, &Q);
    const size_t mmb = mm1 > mm2 ? mm1 : mm2;
    const int nbu = (int)((n + 255) / 256), nb8 = (int)((n + 7) / 8);
    const int nbp = nbu > nb8 ? nbu : nb8;
    const size_t nk = (size_t)n * (size_t)K;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += a256(bytes);
        return o;
    };
    const size_t o_vec = take(sizeof(double) * nk * 6);
    const size_t o_p32 = take(sizeof(float) * nk);
    const size_t o_w32 = take(sizeof(float) * nk);
    const size_t o_q32 = take(sizeof(float) * (size_t)(m > 0 ? m : 1) * K);
    const size_t o_col = take(sizeof(AdjCol) * K);
    const size_t o_part = take(sizeof(double) * (size_t)K * nbp * 3);
    const size_t o_mm = take(mmb > 0 ? mmb : 1);
    if (off > ws->adjb_bytes) {
        if (ws->adjb) cudaFree(ws->adjb);
        ws->adjb = nullptr;
        ws->adjb_bytes = 0;
        if (cudaMalloc(&ws->adjb, off) != cudaSuccess) {
            cudaGetLastError();
            return fail(TOMOS_ERR_ALLOC, "lsqr_adjoint_batch: workspace allocation failed");
        }
        ws->adjb_bytes = off;
    }
    char* base = static_cast<char*>(ws->adjb);
    BArgs a;
    a.n = n;
    a.K = K;
    a.nbp = nbp;
    double* v = reinterpret_cast<double*>(base + o_vec);
    a.lam = v;
    a.r = v + nk;
    a.z = v + 2 * nk;
    a.t = v + 3 * nk;
    a.w = v + 4 * nk;
    a.pd = v + 5 * nk;
    a.p32 = reinterpret_cast<float*>(base + o_p32);
    a.w32 = reinterpret_cast<float*>(base + o_w32);
    float* q32 = reinterpret_cast<float*>(base + o_q32);
    a.col = reinterpret_cast<AdjCol*>(base + o_col);
    a.rr_part = reinterpret_cast<double*>(base + o_part);
    a.rz_part = a.rr_part + (size_t)K * nbp;
    a.pw_part = a.rz_part + (size_t)K * nbp;
    void* mmscratch = base + o_mm;
    a.G = G;
    a.ldg = ldg;
    a.tol = opts->tol > 0.0 ? opts->tol : 0.0;
    a.max_iters = opts->max_iters;
    P.values = a.p32;
    Q.values = q32;
    W.values = a.w32;

    cudaStream_t us = as_stream(stream);
    cudaStream_t st = ws->stream;
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, us));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_fence, 0));
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    const int64_t launches0 = ws->launches;
    s = refresh_precond(ws, st);
    if (s) return s;
    a.Rcm = ws->has_precond ? ws->Rcm : nullptr;
    a.Rrm = ws->has_precond ? ws->Rrm : nullptr;

    const dim3 gu((unsigned)nbu, (unsigned)K), g8((unsigned)nb8, (unsigned)K);
    TOMOS_CUDA_TRY(cudaMemsetAsync(a.col, 0, sizeof(AdjCol) * K, st));  // not done: the first kernels run
    bk_init_kernel<<<gu, 256, 0, st>>>(a);
    TOMOS_LAUNCH_CHECK("bk_init_kernel");
    if (a.Rcm) {
        bk_pt_kernel<<<g8, 256, 0, st>>>(a);
        TOMOS_LAUNCH_CHECK("bk_pt_kernel");
    }
    bk_p_kernel<<<g8, 256, 0, st>>>(a);
    TOMOS_LAUNCH_CHECK("bk_p_kernel");
    bk_start_kernel<<<(unsigned)K, 256, 0, st>>>(a, nb8, nbu);
    TOMOS_LAUNCH_CHECK("bk_start_kernel");
    ws->launches += a.Rcm ? 4 : 3;

    // iterations in batches of four direct launches, the K states read back
    // between batches (a finished column costs the shared products nothing
    // extra; a batch past the last column's convergence costs up to three)
    std::vector<AdjCol> h((size_t)K);
    const int batch = 4;
    int iters = 0;
    for (;;) {
        TOMOS_CUDA_TRY(cudaMemcpyAsync(h.data(), a.col, sizeof(AdjCol) * K, cudaMemcpyDeviceToHost, st));
        TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
        bool all = true;
        for (const AdjCol& c : h) all = all && c.done;
        if (all || iters >= opts->max_iters) break;
        const int left = opts->max_iters - iters;
        const int kk = batch < left ? batch : left;
        for (int it = 0; it < kk; ++it) {
            s = tomos_mm_ex(TOMOS_NO_TRANSPOSE, TOMOS_NO_TRANSPOSE, 1.0, A, tier, &P, 0.0, &Q, mmscratch, mmb, st);
            if (s) return s;
            s = tomos_mm_ex(TOMOS_TRANSPOSE, TOMOS_NO_TRANSPOSE, 1.0, A, tier, &Q, 0.0, &W, mmscratch, mmb, st);
            if (s) return s;
            bk_w_kernel<<<gu, 256, 0, st>>>(a);
            TOMOS_LAUNCH_CHECK("bk_w_kernel");
            bk_update_kernel<<<gu, 256, 0, st>>>(a, nbu);
            TOMOS_LAUNCH_CHECK("bk_update_kernel");
            if (a.Rcm) {
                bk_pt_kernel<<<g8, 256, 0, st>>>(a);
                TOMOS_LAUNCH_CHECK("bk_pt_kernel");
            }
            bk_p_kernel<<<g8, 256, 0, st>>>(a);
            TOMOS_LAUNCH_CHECK("bk_p_kernel");
            bk_finish_kernel<<<(unsigned)K, 256, 0, st>>>(a, nb8, nbu);
            TOMOS_LAUNCH_CHECK("bk_finish_kernel");
            ws->launches += a.Rcm ? 7 : 6;
        }
        iters += kk;
    }
    bk_out_kernel<<<(unsigned)((nk + 255) / 256), 256, 0, st>>>(a.lam, n, K, Lambda, ldl);
    TOMOS_LAUNCH_CHECK("bk_out_kernel");
    ws->launches += 1;
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
    TOMOS_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop);
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, st));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(us, ws->ev_fence, 0));
    if (reports) {
        for (int k = 0; k < K; ++k) {
            tomos_lsqr_report& R = reports[k];
            R.iterations = h[(size_t)k].iter;
            R.converged = h[(size_t)k].converged;
            R.relres = h[(size_t)k].gg > 0.0 ? std::sqrt(h[(size_t)k].rr / h[(size_t)k].gg) : 0.0;
            R.elapsed_ms = ms;
            R.half_passes = 2 * iters;  // shared: two products over A an iteration
            R.kernel_launches = (int32_t)(ws->launches - launches0);
        }
    }
    return TOMOS_OK;
}

}  // extern "C"
