// adjoint.cu -- the adjoint of x* = argmin ||A x - b||.  No reference
// counterpart: the reference has no differentiation.
//
// For a loss L(x*) with g = dL/dx*:
//   lambda = (A^T A)^{-1} g                          tomos_lsqr_adjoint_dense
//   dL/db  = A lambda                                tomos_lsqr_adjoint_grad_dense
//   dL/dA  = r lambda^T - (A lambda) x*^T,   r = b - A x*
//
// lambda comes from preconditioned conjugate gradients on
// R^{-T} A^T A R^{-1} mu = R^{-T} g, lambda = R^{-1} mu -- the
// normal-equations iteration LSQR carries out implicitly -- with the sketch
// preconditioner attached to the workspace.  Each iteration is one fused
// pass over A (ut = A p, q = A^T ut: rowpass.cuh / the generic GEMV pair),
// so A is read once per iteration, as in lsqr_solve; scalars and the
// direction are FP64 on the device, and the host reads the state only
// between batches of iterations.
//
// The gradient pass reads each row a_i of A once: the dots a_i x_k and
// a_i lambda_k give r_ik = b_ik - a_i x_k and w_ik = a_i lambda_k
// (= dL/db_k), and row i of dL/dA, sum_k r_ik lambda_k - w_ik x_k, is
// written while those 2K numbers are still in registers.
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "gemv.cuh"
#include "lsqr.cuh"

namespace tomos_b200 {

struct AdjDev {
    double coef[2];  // [cp, cu] = [1, 0] of the pass: ut = A p
    double rz;       // r . z of the current direction
    double gg;       // ||g||^2
    double rr;       // ||r||^2 after the last update
    double tol;      // stop when ||r|| <= tol ||g||
    int iter, max_iters, done, converged, breakdown, pad_;
};

struct AdjBufs {
    AdjDev* dev;
    double *lam, *r, *z, *t, *w, *pd;  // n each
    double *pw_part, *rr_part, *rz_part;
    int nb1, nbu, nb3;
    size_t bytes;
};

static size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

static AdjBufs adj_layout(void* base, int64_t n) {
    AdjBufs b;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* r = p ? p + off : nullptr;
        off += a256(bytes);
        return r;
    };
    const size_t nn = n > 0 ? (size_t)n : 1;
    b.nb1 = (int)((nn + 31) / 32);
    b.nbu = (int)((nn + 255) / 256);
    b.nb3 = (int)((nn + 7) / 8);
    b.dev = reinterpret_cast<AdjDev*>(take(sizeof(AdjDev)));
    double** vecs[] = {&b.lam, &b.r, &b.z, &b.t, &b.w, &b.pd};
    for (double** v : vecs) *v = reinterpret_cast<double*>(take(sizeof(double) * nn));
    b.pw_part = reinterpret_cast<double*>(take(sizeof(double) * b.nb1));
    b.rr_part = reinterpret_cast<double*>(take(sizeof(double) * (b.nbu > b.nb3 ? b.nbu : b.nb3)));
    b.rz_part = reinterpret_cast<double*>(take(sizeof(double) * (b.nbu > b.nb3 ? b.nbu : b.nb3)));
    b.bytes = off;
    return b;
}

struct AdjArgs {
    int64_t n;
    AdjBufs B;
    const float* g;
    float* p;            // FP32 copy of the direction (the pass reads it)
    const float* qpart;  // A^T ut partials of the pass
    int64_t qstride;
    int gq;
    const double* Rcm;   // R^{-1} column-major (NULL: no preconditioner)
    const double* Rrm;   // R^{-1} row-major
};

__device__ __forceinline__ bool adj_done(const AdjArgs& a) { return a.B.dev->done != 0; }

// r = g, lambda = 0; partial ||g||^2.
__global__ void __launch_bounds__(256) adj_init_kernel(AdjArgs a) {
    __shared__ double sm[32];
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    double v = 0.0;
    if (i < a.n) {
        v = (double)a.g[i];
        a.B.r[i] = v;
        a.B.lam[i] = 0.0;
    }
    const double s = block_sum(v * v, sm);
    if (threadIdx.x == 0) a.B.rr_part[blockIdx.x] = s;
}

// t = R^{-T} r (a warp per entry).
__global__ void __launch_bounds__(256) adj_pt_kernel(AdjArgs a) {
    if (adj_done(a)) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * 8 + w;
    if (j >= a.n) return;
    const double* col = a.Rcm + (size_t)j * a.n;
    double s = 0.0;
    for (int64_t i = lane; i < a.n; i += 32) s += col[i] * a.B.r[i];
    s = warp_sum(s);
    if (lane == 0) a.B.t[j] = s;
}

// z = R^{-1} t (or z = r without a preconditioner); partial r . z.
__global__ void __launch_bounds__(256) adj_p_kernel(AdjArgs a) {
    if (adj_done(a)) return;
    __shared__ double smz[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * 8 + w;
    double rz = 0.0;
    if (i < a.n) {
        double z;
        if (a.Rrm) {
            const double* row = a.Rrm + (size_t)i * a.n;
            double s = 0.0;
            for (int64_t j = lane; j < a.n; j += 32) s += row[j] * a.B.t[j];
            z = warp_sum(s);
        } else {
            z = a.B.r[i];
        }
        if (lane == 0) a.B.z[i] = z;
        rz = z * a.B.r[i];
    }
    if (lane == 0) smz[w] = rz;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += smz[k];
        a.B.rz_part[blockIdx.x] = s;
    }
}

// One block: rz and ||g||^2 from their partials, p = z.
__global__ void __launch_bounds__(256) adj_start_kernel(AdjArgs a) {
    __shared__ double sm[32];
    const double rz = block_sum_array(a.B.rz_part, a.B.nb3, sm);
    const double gg = block_sum_array(a.B.rr_part, a.B.nbu, sm);
    for (int64_t i = threadIdx.x; i < a.n; i += blockDim.x) {
        const double z = a.B.z[i];
        a.B.pd[i] = z;
        a.p[i] = (float)z;
    }
    if (threadIdx.x == 0) {
        AdjDev* d = a.B.dev;
        d->coef[0] = 1.0;
        d->coef[1] = 0.0;
        d->rz = rz;
        d->gg = gg;
        d->rr = gg;
        d->iter = 0;
        d->converged = gg == 0.0 ? 1 : 0;
        d->breakdown = 0;
        d->done = (gg == 0.0 || d->max_iters == 0) ? 1 : 0;
    }
}

// w = A^T A p from the pass partials (fixed order); partial p . w.
__global__ void __launch_bounds__(256) adj_w_kernel(AdjArgs a) {
    if (adj_done(a)) return;
    __shared__ double smq[8][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * 32 + lane;
    double q = 0.0;
    if (j < a.n)
        for (int c = w; c < a.gq; c += 8) q += (double)a.qpart[(size_t)c * a.qstride + j];
    smq[w][lane] = q;
    __syncthreads();
    if (w == 0) {
        double qs = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) qs += smq[k][lane];
        double pw = 0.0;
        if (j < a.n) {
            a.B.w[j] = qs;
            pw = qs * a.B.pd[j];
        }
        pw = warp_sum(pw);
        if (lane == 0) a.B.pw_part[blockIdx.x] = pw;
    }
}

// alpha = rz / p.w; lambda += alpha p; r -= alpha w; partial ||r||^2.
__global__ void __launch_bounds__(256) adj_update_kernel(AdjArgs a) {
    if (adj_done(a)) return;
    __shared__ double sm[32];
    const double pw = block_sum_array(a.B.pw_part, a.B.nb1, sm);
    const double alpha = pw > 0.0 ? a.B.dev->rz / pw : 0.0;
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    double v = 0.0;
    if (i < a.n) {
        a.B.lam[i] += alpha * a.B.pd[i];
        v = a.B.r[i] - alpha * a.B.w[i];
        a.B.r[i] = v;
    }
    const double s = block_sum(v * v, sm);
    if (threadIdx.x == 0) {
        a.B.rr_part[blockIdx.x] = s;
        if (blockIdx.x == 0 && !(pw > 0.0)) a.B.dev->breakdown = 1;
    }
}

// One block: stopping rule, beta = rz' / rz, p = z + beta p.
__global__ void __launch_bounds__(256) adj_finish_kernel(AdjArgs a) {
    if (adj_done(a)) return;
    __shared__ double sm[32];
    __shared__ double bc[2];
    const double rr = block_sum_array(a.B.rr_part, a.B.nbu, sm);
    const double rz = block_sum_array(a.B.rz_part, a.B.nb3, sm);
    if (threadIdx.x == 0) {
        AdjDev* d = a.B.dev;
        d->iter += 1;
        d->rr = rr;
        bc[0] = 0.0;
        bc[1] = 0.0;
        if (sqrt(rr) <= d->tol * sqrt(d->gg)) {
            d->converged = 1;
            d->done = 1;
        } else if (d->breakdown || d->iter >= d->max_iters || !(rz > 0.0)) {
            d->done = 1;
        } else {
            bc[0] = rz / d->rz;
            bc[1] = 1.0;
            d->rz = rz;
        }
    }
    __syncthreads();
    if (bc[1] == 0.0) return;
    const double beta = bc[0];
    for (int64_t i = threadIdx.x; i < a.n; i += blockDim.x) {
        const double p = a.B.z[i] + beta * a.B.pd[i];
        a.B.pd[i] = p;
        a.p[i] = (float)p;
    }
}

__global__ void adj_out_kernel(const double* lam, int64_t n, float* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)lam[i];
}

// Gradient pass over a row-major A, K right-hand sides (K <= 8 per launch;
// X and Lambda staged in shared memory as [column][k]).  A warp per row.
template <Elem E, int K>
__global__ void __launch_bounds__(256) adj_grad_kernel(const void* hi, const void* lo, int64_t m,
                                                       int64_t n, int64_t ld, const float* B,
                                                       int64_t ldb, const float* X, int64_t ldx,
                                                       const float* Lm, int64_t ldl, float* gradB,
                                                       int64_t ldgb, float* gradA, int64_t ldga,
                                                       int accumulate) {
    extern __shared__ float gsm[];
    float* xs = gsm;
    float* ls = gsm + (size_t)n * K;
    for (int64_t e = threadIdx.x; e < n * K; e += blockDim.x) {
        const int64_t j = e / K, k = e % K;
        xs[e] = X[(size_t)k * ldx + j];
        ls[e] = Lm[(size_t)k * ldl + j];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t i = (int64_t)blockIdx.x * 8 + warp; i < m; i += (int64_t)gridDim.x * 8) {
        float dx[K], dl[K];
#pragma unroll
        for (int k = 0; k < K; ++k) dx[k] = dl[k] = 0.0f;
        const size_t row = (size_t)i * ld;
        for (int64_t j = lane; j < n; j += 32) {
            const float a = load_elem<E>(hi, lo, row + j);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                dx[k] = fmaf(a, xs[j * K + k], dx[k]);
                dl[k] = fmaf(a, ls[j * K + k], dl[k]);
            }
        }
        float rk[K], wk[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            float sx = dx[k], sl = dl[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sx += __shfl_xor_sync(0xffffffffu, sx, o);
                sl += __shfl_xor_sync(0xffffffffu, sl, o);
            }
            rk[k] = B[(size_t)k * ldb + i] - sx;
            wk[k] = sl;
        }
        if (lane < K) {
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (k == lane) gradB[(size_t)k * ldgb + i] = wk[k];
        }
        if (gradA) {
            float* gr = gradA + (size_t)i * ldga;
            for (int64_t j = lane; j < n; j += 32) {
                float s = 0.0f;
#pragma unroll
                for (int k = 0; k < K; ++k) s = fmaf(rk[k], ls[j * K + k], fmaf(-wk[k], xs[j * K + k], s));
                gr[j] = accumulate ? gr[j] + s : s;
            }
        }
    }
}

template <Elem E>
static tomos_status launch_grad_e(int kk, const tomos_dense* A, const float* B, int64_t ldb,
                                  const float* X, int64_t ldx, const float* L, int64_t ldl,
                                  float* gB, int64_t ldgb, float* gA, int64_t ldga, int acc,
                                  cudaStream_t st) {
    const void* lo = elem_is_exact(E) ? dense_lo_plane(A) : nullptr;
    const size_t smem = (size_t)A->cols * kk * 2 * sizeof(float);
    int64_t grid = (A->rows + 7) / 8;
    const int64_t cap = (int64_t)sm_count() * 8;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
#define TOMOS_GRAD(KK)                                                                              \
    do {                                                                                            \
        auto kern = adj_grad_kernel<E, KK>;                                                         \
        TOMOS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                            (int)smem));                                            \
        kern<<<(unsigned)grid, 256, smem, st>>>(A->values, lo, A->rows, A->cols, A->ld, B, ldb, X,  \
                                                ldx, L, ldl, gB, ldgb, gA, ldga, acc);              \
    } while (0)
    switch (kk) {
        case 1: TOMOS_GRAD(1); break;
        case 2: TOMOS_GRAD(2); break;
        case 3: TOMOS_GRAD(3); break;
        case 4: TOMOS_GRAD(4); break;
        case 5: TOMOS_GRAD(5); break;
        case 6: TOMOS_GRAD(6); break;
        case 7: TOMOS_GRAD(7); break;
        case 8: TOMOS_GRAD(8); break;
        default: return fail(TOMOS_ERR_INVALID, "adjoint_grad: bad group size");
    }
#undef TOMOS_GRAD
    TOMOS_LAUNCH_CHECK("adj_grad_kernel");
    return TOMOS_OK;
}

static tomos_status ensure_adj(tomos_workspace* ws) {
    if (ws->adj) return TOMOS_OK;
    const AdjBufs need = adj_layout(nullptr, ws->n);
    if (cudaMalloc(&ws->adj, need.bytes) != cudaSuccess) {
        ws->adj = nullptr;
        cudaGetLastError();
        return fail(TOMOS_ERR_ALLOC, "adjoint workspace allocation failed");
    }
    return TOMOS_OK;
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

tomos_status tomos_lsqr_adjoint_dense(const tomos_dense* A, const float* g, float* lambda,
                                      tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                      tomos_lsqr_report* report, void* stream) {
    std::string why;
    bool dot;
    int64_t outer, inner;
    if (!gemv_shape(A, TOMOS_NO_TRANSPOSE, &dot, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "lsqr_adjoint: " + why);
    if (!opts) return fail(TOMOS_ERR_INVALID, "lsqr_adjoint: null options");
    if (opts->max_iters < 0) return fail(TOMOS_ERR_INVALID, "lsqr_adjoint: negative max_iters");
    tomos_status s = workspace_check(ws, A->rows, A->cols);
    if (s) return s;
    const int64_t m = A->rows, n = A->cols;
    if (n == 0) {
        if (report) std::memset(report, 0, sizeof(*report));
        return TOMOS_OK;
    }
    if (!g || !lambda || (!A->values && m * n > 0))
        return fail(TOMOS_ERR_INVALID, "lsqr_adjoint: null pointer");
    // Packed A: the exact (wh + wr) values unless a tier is asked for.
    const bool packed = A->numeric == TOMOS_FP32_16 || A->numeric == TOMOS_FP32_BF16;
    const int32_t tier = opts->iter_tier == TOMOS_TIER_AUTO
                             ? (packed ? TOMOS_TIER_ACCURATE : TOMOS_TIER_NATIVE)
                             : opts->iter_tier;
    Elem e;
    if (!resolve_elem(A, tier, &e, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_adjoint: " + why);
    s = ensure_adj(ws);
    if (s) return s;
    const PassPlan pl = plan_dense_pass(ws, A, e, false);
    if (!pl.fused) {
        s = ensure_scratch(ws, dense_pass_scratch(A));
        if (s) return s;
    }
    cudaStream_t us = as_stream(stream);
    cudaStream_t st = ws->stream;
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, us));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_fence, 0));
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    const int64_t launches0 = ws->launches;

    AdjArgs a;
    a.n = n;
    a.B = adj_layout(ws->adj, n);
    a.g = g;
    a.p = ws->p;
    a.qpart = ws->qpart;
    a.qstride = pl.qstride;
    a.gq = pl.gq;
    s = refresh_precond(ws, st);
    if (s) return s;
    a.Rcm = ws->has_precond ? ws->Rcm : nullptr;
    a.Rrm = ws->has_precond ? ws->Rrm : nullptr;

    AdjDev init{};
    init.tol = opts->tol > 0.0 ? opts->tol : 0.0;
    init.max_iters = opts->max_iters;
    TOMOS_CUDA_TRY(cudaMemcpyAsync(a.B.dev, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    TOMOS_CUDA_TRY(cudaMemsetAsync(ws->u, 0, sizeof(float) * m, st));
    TOMOS_CUDA_TRY(cudaMemsetAsync(&ws->st->pipe_err, 0, sizeof(int), st));
    adj_init_kernel<<<a.B.nbu, 256, 0, st>>>(a);
    TOMOS_LAUNCH_CHECK("adj_init_kernel");
    if (a.Rcm) {
        adj_pt_kernel<<<a.B.nb3, 256, 0, st>>>(a);
        TOMOS_LAUNCH_CHECK("adj_pt_kernel");
    }
    adj_p_kernel<<<a.B.nb3, 256, 0, st>>>(a);
    TOMOS_LAUNCH_CHECK("adj_p_kernel");
    adj_start_kernel<<<1, 256, 0, st>>>(a);
    TOMOS_LAUNCH_CHECK("adj_start_kernel");
    ws->launches += a.Rcm ? 4 : 3;

    // CG iterations in batches of direct launches (the pass and four or
    // five n-side kernels each; a converged state makes them return at
    // once), the state read back between batches.
    AdjDev h{};
    int batch = 4;
    for (;;) {
        int pe = 0;
        TOMOS_CUDA_TRY(cudaMemcpyAsync(&h, a.B.dev, sizeof(h), cudaMemcpyDeviceToHost, st));
        TOMOS_CUDA_TRY(cudaMemcpyAsync(&pe, &ws->st->pipe_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
        if (pe)
            return fail(TOMOS_ERR_CUDA, "lsqr_adjoint: a bounded pipeline wait expired (code " +
                                            std::to_string(pe) + ")");
        if (h.done) break;
        const int left = opts->max_iters - h.iter;
        const int k = batch < left ? batch : left;
        for (int i = 0; i < k; ++i) {
            s = enqueue_dense_pass(ws, A, pl, ws->p, ws->u, &a.B.dev->coef[0], &a.B.dev->done, st);
            if (s) return s;
            adj_w_kernel<<<a.B.nb1, 256, 0, st>>>(a);
            TOMOS_LAUNCH_CHECK("adj_w_kernel");
            adj_update_kernel<<<a.B.nbu, 256, 0, st>>>(a);
            TOMOS_LAUNCH_CHECK("adj_update_kernel");
            if (a.Rcm) {
                adj_pt_kernel<<<a.B.nb3, 256, 0, st>>>(a);
                TOMOS_LAUNCH_CHECK("adj_pt_kernel");
            }
            adj_p_kernel<<<a.B.nb3, 256, 0, st>>>(a);
            TOMOS_LAUNCH_CHECK("adj_p_kernel");
            adj_finish_kernel<<<1, 256, 0, st>>>(a);
            TOMOS_LAUNCH_CHECK("adj_finish_kernel");
            ws->launches += a.Rcm ? 5 : 4;
        }
        if (batch < 32) batch *= 2;
    }
    adj_out_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.B.lam, n, lambda);
    TOMOS_LAUNCH_CHECK("adj_out_kernel");
    ws->launches += 1;
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
    TOMOS_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop);
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, st));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(us, ws->ev_fence, 0));
    if (report) {
        std::memset(report, 0, sizeof(*report));
        report->iterations = h.iter;
        report->converged = h.converged;
        report->relres = h.gg > 0.0 ? std::sqrt(h.rr / h.gg) : 0.0;
        report->elapsed_ms = ms;
        report->half_passes = h.iter;
        report->kernel_launches = (int32_t)(ws->launches - launches0);
    }
    return TOMOS_OK;
}

tomos_status tomos_lsqr_adjoint_grad_dense(const tomos_dense* A, int64_t K, const float* B,
                                           int64_t ldb, const float* X, int64_t ldx,
                                           const float* Lam, int64_t ldl, float* gradB,
                                           int64_t ldgb, float* gradA, int64_t ldga,
                                           void* stream) {
    std::string why;
    bool dot;
    int64_t outer, inner;
    if (!gemv_shape(A, TOMOS_NO_TRANSPOSE, &dot, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_grad: " + why);
    if (A->layout != TOMOS_ROW_MAJOR)
        return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_adjoint_grad: row-major A only");
    const int64_t m = A->rows, n = A->cols;
    if (K < 0 || ldb < m || ldx < n || ldl < n || ldgb < m || (gradA && ldga < n))
        return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_grad: bad sizes");
    if (K == 0 || m == 0 || n == 0) return TOMOS_OK;
    if (!B || !X || !Lam || !gradB || !A->values)
        return fail(TOMOS_ERR_INVALID, "lsqr_adjoint_grad: null pointer");
    const bool packed = A->numeric == TOMOS_FP32_16 || A->numeric == TOMOS_FP32_BF16;
    Elem e;
    if (!resolve_elem(A, packed ? TOMOS_TIER_ACCURATE : TOMOS_TIER_NATIVE, &e, &why))
        return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_adjoint_grad: " + why);
    // X and Lambda of one group of right-hand sides must fit shared memory.
    int kg = 8;
    while (kg > 1 && (size_t)n * kg * 2 * sizeof(float) > 200 * 1024) kg /= 2;
    if ((size_t)n * kg * 2 * sizeof(float) > 200 * 1024)
        return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_adjoint_grad: n too large for one pass");
    cudaStream_t st = as_stream(stream);
    for (int64_t k0 = 0; k0 < K; k0 += kg) {
        const int kk = (int)(K - k0 < kg ? K - k0 : kg);
        const float* Bk = B + (size_t)k0 * ldb;
        const float* Xk = X + (size_t)k0 * ldx;
        const float* Lk = Lam + (size_t)k0 * ldl;
        float* gBk = gradB + (size_t)k0 * ldgb;
        tomos_status s;
        switch (e) {
            case Elem::F32: s = launch_grad_e<Elem::F32>(kk, A, Bk, ldb, Xk, ldx, Lk, ldl, gBk, ldgb, gradA, ldga, k0 > 0, st); break;
            case Elem::A16: s = launch_grad_e<Elem::A16>(kk, A, Bk, ldb, Xk, ldx, Lk, ldl, gBk, ldgb, gradA, ldga, k0 > 0, st); break;
            case Elem::AB16: s = launch_grad_e<Elem::AB16>(kk, A, Bk, ldb, Xk, ldx, Lk, ldl, gBk, ldgb, gradA, ldga, k0 > 0, st); break;
            case Elem::AB16R: s = launch_grad_e<Elem::AB16R>(kk, A, Bk, ldb, Xk, ldx, Lk, ldl, gBk, ldgb, gradA, ldga, k0 > 0, st); break;
            default: return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_adjoint_grad: element type");
        }
        if (s) return s;
    }
    return TOMOS_OK;
}

}  // extern "C"
