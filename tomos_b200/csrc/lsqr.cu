// lsqr.cu -- preconditioned LSQR on the device: workspace, the n-side
// kernels of one Golub-Kahan step, and the host driver behind
// tomos_lsqr_solve_dense / _csr and tomos_backward_error_dense.
//
// Algorithm: Paige-Saunders LSQR with a right preconditioner M = R^{-1}
// (the reference's fused_lsqr_impl, src/core/solver/lsqr.cpp:432-747),
// restarted from the current x, with two changes of formulation that
// leave the iterates mathematically unchanged:
//   * u is kept unnormalised: the A pass produces ut = A p - (alpha/beta) ut
//     (p = M v), so A^T u = A^T ut / beta comes from the same pass over A
//     (rowpass.cuh) instead of a second one;
//   * w is kept in x-space (wt = M w), so x += (phi/rho) wt and
//     wt = p - (theta/rho) wt need no third product with M per iteration.
// Every scalar of the recurrence (alpha, beta, rho, rho_bar, phi, phi_bar,
// c, s, theta) and every norm is FP64 and stays on the device; one
// iteration is five kernels with no host round trip, captured once into a
// CUDA graph and replayed.  The host only looks at the state at restart
// boundaries and between batches of iterations.
//
// Per iteration:
//   A pass   ut = A p + cu * ut, partials of A^T ut and ||ut||^2
//   N1       beta = ||ut||, t = A^T ut / beta (fixed-order partial reduce)
//   N2       z = M^T t, vh = z - beta v               (preconditioned only)
//   N3       alpha = ||vh||, v = vh / alpha, p = M v, Givens, x and wt
//   N4       state update, history, stopping rule, next cu = -alpha/beta
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "fused.cuh"
#include "gemv.cuh"
#include "lsqr.cuh"
#include "rowpass.cuh"
#include "rowpass_launch.cuh"
#include "rowpass_mma.cuh"

namespace tomos_b200 {

// ------------------------------------------------------------ reductions

__global__ void sumsq_partial_kernel(const float* __restrict__ x, int64_t n, const int* skip,
                                     double* __restrict__ part) {
    if (skip && *skip) return;
    __shared__ double sm[32];
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * per;
    int64_t i1 = i0 + per;
    if (i1 > n) i1 = n;
    double s = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        double v = x[i];
        s += v * v;
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void sum_to_scalar_kernel(const double* __restrict__ part, int64_t np,
                                     double* __restrict__ out) {
    __shared__ double sm[32];
    double s = block_sum_array(part, np, sm);
    if (threadIdx.x == 0) *out = s;
}

// sum of squares of every element of a strided matrix (its ||.||_F^2),
// read at element tag E; per-block partials.
template <Elem E>
__global__ void fro2_partial_kernel(const void* hi, const void* lo, int64_t outer, int64_t inner,
                                    int64_t ld, const double* dscale, int col_is_inner,
                                    double* part) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int64_t o = blockIdx.x; o < outer; o += gridDim.x)
        for (int64_t i = threadIdx.x; i < inner; i += blockDim.x) {
            double v = load_elem<E>(hi, lo, (size_t)o * ld + i);
            if (dscale) v /= dscale[col_is_inner ? i : o];
            s += v * v;
        }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ||b|| from its partials, and ||A||_F (from a device value, from
// ||A||_F^2, or left as the host set it) into the solver state.
__global__ void __launch_bounds__(256) state_norms_kernel(const double* __restrict__ bpart, int64_t np,
                                                          const double* anorm_dev, const double* fro2,
                                                          LsqrDev* st) {
    __shared__ double sm[32];
    const double bn = sqrt(block_sum_array(bpart, np, sm));
    if (threadIdx.x != 0) return;
    st->rhsnorm = bn;
    st->bnorm = bn;
    if (anorm_dev) st->anorm_fro = *anorm_dev;
    else if (fro2) st->anorm_fro = sqrt(*fro2);
}

__global__ void fill_f32_kernel(float* p, int64_t n, float v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// sum of (d_i x_i)^2 (d may be NULL), one block.
__global__ void scaled_sumsq_kernel(const float* __restrict__ x, const double* __restrict__ d,
                                    int64_t n, double* __restrict__ out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = (double)x[i] * (d ? d[i] : 1.0);
        s += v * v;
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *out = s;
}

// FP64 column-major and row-major copies of a dense n x n preconditioner.
// Both copies of the preconditioner; *lower_nz (zeroed before) becomes 1
// if any element below the diagonal is nonzero, else the n-side products
// skip the zero triangle of the (sketch QR's upper triangular) R^{-1}.
__global__ void precond_copy_kernel(const void* R, int numeric, int layout, int64_t ld, int64_t n,
                                    double* Rcm, double* Rrm, double* lower_nz) {
    const int64_t total = n * n;
    bool nz = false;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k % n, j = k / n;  // element (i, j)
        const size_t src = layout == TOMOS_COL_MAJOR ? (size_t)j * ld + i : (size_t)i * ld + j;
        double v = numeric == TOMOS_FP64 ? static_cast<const double*>(R)[src]
                                         : (double)static_cast<const float*>(R)[src];
        Rcm[(size_t)j * n + i] = v;
        Rrm[(size_t)i * n + j] = v;
        nz = nz || (i > j && v != 0.0);
    }
    if (nz) *lower_nz = 1.0;  // every writer stores the same value
}

// d_j = sqrt(colsq_j) (1 for an empty column) and ||A D^{-1}||_F =
// sqrt(#non-empty columns), one block.
__global__ void __launch_bounds__(256) column_scale_kernel(const double* __restrict__ colsq, int64_t n,
                                                           double* __restrict__ d, double* __restrict__ anorm) {
    __shared__ double sm[32];
    double cnt = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const double c = colsq[j];
        const bool nz = c > 0.0;
        d[j] = nz ? sqrt(c) : 1.0;
        cnt += nz ? 1.0 : 0.0;
    }
    cnt = block_sum(cnt, sm);
    if (threadIdx.x == 0) *anorm = sqrt(cnt);
}

// ------------------------------------------------------------- n-side

struct NSide {
    int64_t n;
    const float* qpart;
    int64_t qstride;
    int gq;
    const double* sspart;
    int gs;
    double* t;
    double* vhat;
    float* v;
    float* wt;
    float* p;
    float* x;
    double* vpart;
    double* xpart;
    double* qnpart;
    const double* Rcm;
    const double* Rrm;
    int has_precond;
    int init;
    int nb1;   // N1 blocks
    int nb3;   // N2/N3 blocks
    double* scal;
    LsqrDev* st;
    const int* skip;
    const double* dscale;  // column scale D of the backward-error rule, or NULL
    const double* qsum;    // row-sharded solves: A^T ut summed over ranks (n), else NULL
    // The iteration graph's while loop: N4 sets its condition (1: run the
    // body again) on every path, so the loop ends once the solver stops.
    cudaGraphConditionalHandle cond;
    int use_cond;
};

// Givens step of LSQR (lsqr.cpp:633-679), FP64.
struct Givens {
    double rho, c, s, theta, rho_bar, phi, phi_bar;
};
__device__ __forceinline__ Givens givens(double rho_bar, double phi_bar, double alpha, double beta) {
    Givens g;
    g.rho = hypot(rho_bar, beta);
    const double inv = g.rho > 0.0 ? 1.0 / g.rho : 0.0;
    g.c = rho_bar * inv;
    g.s = beta * inv;
    g.theta = g.s * alpha;
    g.rho_bar = -g.c * alpha;
    g.phi = g.c * phi_bar;
    g.phi_bar = g.s * phi_bar;
    return g;
}

// sum over k = lane, lane + 32, .. < len of a[k] b[k] (the lane's share of a
// warp's dot product over L2-resident vectors): eight independent FP64
// chains, so a lane has sixteen loads in flight instead of two.
__device__ __forceinline__ double strided_dot(const double* __restrict__ a, const double* __restrict__ b,
                                              int lane, int64_t len) {
    double z[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int64_t k = lane;
    for (; k + 7 * 32 < len; k += 8 * 32) {
        double av[8], bv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            av[u] = __ldg(a + k + 32 * u);
            bv[u] = __ldg(b + k + 32 * u);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) z[u] = fma(av[u], bv[u], z[u]);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
        if (k + 32 * u < len) z[u] = fma(__ldg(a + k + 32 * u), __ldg(b + k + 32 * u), z[u]);
    return ((z[0] + z[1]) + (z[2] + z[3])) + ((z[4] + z[5]) + (z[6] + z[7]));
}

// N1: beta and t = A^T ut / beta (no preconditioner: vh = t - beta v).
__global__ void __launch_bounds__(256) nside_reduce_kernel(NSide S) {
    if (S.skip && *S.skip) return;
    __shared__ double sm[32];
    __shared__ double smq[8][33];
    const double beta = sqrt(block_sum_array(S.sspart, S.gs, sm));
    const double inv = beta > 0.0 ? 1.0 / beta : 0.0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * 32 + lane;
    double q = 0.0;
    if (S.qsum)
        q = (w == 0 && j < S.n) ? S.qsum[j] : 0.0;
    else if (j < S.n) {
        double q1 = 0.0;
        int c = w;
        for (; c + 8 < S.gq; c += 16) {
            q += (double)S.qpart[(size_t)c * S.qstride + j];
            q1 += (double)S.qpart[(size_t)(c + 8) * S.qstride + j];
        }
        if (c < S.gq) q += (double)S.qpart[(size_t)c * S.qstride + j];
        q += q1;
    }
    smq[w][lane] = q;
    __syncthreads();
    if (w == 0) {
        double qs = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) qs += smq[k][lane];
        double vh2 = 0.0, qn = 0.0;
        if (j < S.n) {
            const double tj = qs * inv;
            if (S.has_precond) {
                S.t[j] = tj;
            } else {
                const double vh = S.init ? tj : tj - beta * (double)S.v[j];
                S.vhat[j] = vh;
                vh2 = vh * vh;
            }
            const double qd = S.dscale ? qs / S.dscale[j] : qs;
            qn = qd * qd;
        }
        vh2 = warp_sum(vh2);
        qn = warp_sum(qn);
        if (lane == 0) {
            if (!S.has_precond) S.vpart[blockIdx.x] = vh2;
            S.qnpart[blockIdx.x] = qn;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) S.scal[0] = beta;
}

// N2: z = M^T t (M = R^{-1}), vh = z - beta v.
__global__ void __launch_bounds__(256) nside_precond_t_kernel(NSide S) {
    if (S.skip && *S.skip) return;
    __shared__ double smv[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * 8 + w;
    const double beta = S.scal[0];
    double vh2 = 0.0;
    if (j < S.n) {
        const double* __restrict__ col = S.Rcm + (size_t)j * S.n;
        const double* __restrict__ tv = S.t;
        // an upper triangular M: column j ends at row j
        const int64_t ie = S.scal[7] != 0.0 ? S.n : j + 1;
        const double z = warp_sum(strided_dot(col, tv, lane, ie));
        const double vh = S.init ? z : z - beta * (double)S.v[j];
        if (lane == 0) S.vhat[j] = vh;
        vh2 = vh * vh;
    }
    if (lane == 0) smv[w] = vh2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += smv[k];
        S.vpart[blockIdx.x] = s;
    }
}

// N3: alpha, v, p = M v, and the x / wt update of the Givens step.
__global__ void __launch_bounds__(256) nside_update_kernel(NSide S) {
    if (S.skip && *S.skip) return;
    __shared__ double sm[32];
    __shared__ double smx[8];
    const int nvp = S.has_precond ? S.nb3 : S.nb1;
    const double alpha = sqrt(block_sum_array(S.vpart, nvp, sm));
    const double inva = alpha > 0.0 ? 1.0 / alpha : 0.0;
    const double beta = S.scal[0];
    Givens g = givens(S.st->rho_bar, S.st->phi_bar, alpha, beta);
    const double step_x = g.rho > 0.0 ? g.phi / g.rho : 0.0;
    const double step_w = g.rho > 0.0 ? g.theta / g.rho : 0.0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * 8 + w;
    double xs = 0.0;
    if (i < S.n) {
        double pi;
        if (S.has_precond) {
            const double* __restrict__ row = S.Rrm + (size_t)i * S.n;
            const double* __restrict__ vh = S.vhat;
            // an upper triangular M: row i starts at column i
            const int64_t j0 = S.scal[7] != 0.0 ? 0 : i;
            pi = warp_sum(strided_dot(row + j0, vh + j0, lane, S.n - j0)) * inva;
        } else {
            pi = S.vhat[i] * inva;
        }
        if (lane == 0) {
            S.v[i] = (float)(S.vhat[i] * inva);
            double xi = (double)S.x[i];
            if (S.init) {
                S.wt[i] = (float)pi;
            } else {
                const double wi = (double)S.wt[i];
                xi += step_x * wi;
                S.x[i] = (float)xi;
                S.wt[i] = (float)(pi - step_w * wi);
            }
            S.p[i] = (float)pi;
            const double xf = (double)(float)xi * (S.dscale ? S.dscale[i] : 1.0);
            xs = xf * xf;
        }
    }
    if (lane == 0) smx[w] = xs;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += smx[k];
        S.xpart[blockIdx.x] = s;
        if (blockIdx.x == 0) S.scal[1] = alpha;
    }
}

// N4: one block -- state update and the stopping rule.  In the iteration
// graph's while loop it also sets the loop's condition: 0 once the solver
// stopped (a skipped body, the stopping rule, a breakdown or the restart's
// max_iters iterations), so the loop runs at most max_iters + 1 bodies.
__global__ void __launch_bounds__(256) nside_finish_kernel(NSide S) {
    if (S.skip && *S.skip) {
        if (S.use_cond && threadIdx.x == 0) cudaGraphSetConditional(S.cond, 0u);
        return;
    }
    __shared__ double sm[32];
    const double xn = sqrt(block_sum_array(S.xpart, S.nb3, sm));
    const double qn = S.init ? sqrt(block_sum_array(S.qnpart, S.nb1, sm)) : 0.0;
    if (threadIdx.x != 0) return;
    LsqrDev* st = S.st;
    const double beta = S.scal[0], alpha = S.scal[1];
    st->xnorm = xn;
    st->coef[0] = 1.0;
    st->coef[1] = beta > 0.0 ? -alpha / beta : 0.0;
    if (S.init) {
        st->alpha = alpha;
        st->beta = beta;
        st->rho_bar = alpha;
        st->phi_bar = beta;
        st->beta_init = beta;
        st->arnorm = qn;
        st->iter_restart = 0;
        st->relres = st->rhsnorm > 0.0 ? beta / st->rhsnorm : 0.0;
        st->done = 0;
        st->breakdown = (alpha == 0.0 || beta == 0.0) ? 1 : 0;
        if (S.use_cond) cudaGraphSetConditional(S.cond, 0u);  // no loop runs init passes
        return;
    }
    Givens g = givens(st->rho_bar, st->phi_bar, alpha, beta);
    st->alpha = alpha;
    st->beta = beta;
    st->rho_bar = g.rho_bar;
    st->phi_bar = g.phi_bar;
    st->iter += 1;
    st->iter_restart += 1;
    const double relres = st->rhsnorm > 0.0 ? fabs(g.phi_bar) / st->rhsnorm : 0.0;
    st->relres = relres;
    if (st->history && st->iter - 1 < st->history_cap) st->history[st->iter - 1] = relres;
    int stop = 0;
    if (st->rhsnorm == 0.0) stop = 1;
    if (st->stop_rule == TOMOS_STOP_RELRES) {
        if (relres < st->tol || relres < st->max_relres) {
            stop = 1;
            st->converged = 1;
        }
    } else {
        const double den = st->anorm_fro * xn + st->bnorm;
        const double eta1 = den > 0.0 ? fabs(g.phi_bar) / den : 0.0;
        if (eta1 <= st->inner_tol) stop = 1;
        if (st->inner_rtol > 0.0 && fabs(g.phi_bar) <= st->inner_rtol * st->beta_init) stop = 1;
    }
    if (alpha == 0.0 || beta == 0.0) {
        stop = 1;
        st->breakdown = 1;
    }
    if (st->iter_restart >= st->max_iters) stop = 1;
    if (stop) st->done = 1;
    if (S.use_cond) cudaGraphSetConditional(S.cond, stop ? 0u : 1u);
}

// ------------------------------------------------------------ workspace

static void ws_free(tomos_workspace* ws) {
    void* ptrs[] = {ws->u,      ws->v,      ws->wt,     ws->p,    ws->qvec,   ws->t,
                    ws->vhat,   ws->qpart,  ws->sspart, ws->vpart, ws->xpart, ws->qnpart,
                    ws->scal,   ws->coef_init, ws->bpart, ws->fro2, ws->st,   ws->Rcm,
                    ws->Rrm,    ws->hist,   ws->scratch, ws->h16, ws->adj, ws->csc, ws->shard, ws->adjb,
                    ws->xg,     ws->dscale};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (ws->st_host) cudaFreeHost(ws->st_host);
    if (ws->graph) cudaGraphExecDestroy(ws->graph);
    if (ws->ev_start) cudaEventDestroy(ws->ev_start);
    if (ws->ev_stop) cudaEventDestroy(ws->ev_stop);
    if (ws->ev_fence) cudaEventDestroy(ws->ev_fence);
    if (ws->ev_pa) cudaEventDestroy(ws->ev_pa);
    if (ws->ev_pb) cudaEventDestroy(ws->ev_pb);
    if (ws->stream) cudaStreamDestroy(ws->stream);
}

template <typename T>
static cudaError_t alloc(T** p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(p), (count ? count : 1) * sizeof(T));
}

tomos_status ensure_scratch(tomos_workspace* ws, size_t bytes) {
    if (bytes <= ws->scratch_bytes) return TOMOS_OK;
    if (ws->scratch) cudaFree(ws->scratch);
    ws->scratch = nullptr;
    ws->scratch_bytes = 0;
    cudaError_t e = cudaMalloc(&ws->scratch, bytes);
    if (e != cudaSuccess) return fail(TOMOS_ERR_ALLOC, "workspace scratch allocation failed");
    ws->scratch_bytes = bytes;
    return TOMOS_OK;
}

static tomos_status ensure_history(tomos_workspace* ws, int cap) {
    if (cap <= ws->hist_cap) return TOMOS_OK;
    if (ws->hist) cudaFree(ws->hist);
    ws->hist = nullptr;
    ws->hist_cap = 0;
    if (alloc(&ws->hist, (size_t)cap) != cudaSuccess)
        return fail(TOMOS_ERR_ALLOC, "history allocation failed");
    ws->hist_cap = cap;
    return TOMOS_OK;
}

// ------------------------------------------------------------ A passes

// The LSQR pass (kRowBoth) for every element type and FP64 flag; runs:
// the FP64-summing passes of the FP32 and exact two-plane types form their
// row dots as FP32 products over short runs (kRowBothRuns).
static tomos_status launch_fused(Elem e, bool acc64, bool runs, const FusedParams& P, int* err,
                                 int nch, int g, int grid, cudaStream_t st) {
#define TOMOS_BOTH(EE)                                                                    \
    (runs ? launch_fused_e<EE, true, kRowBothRuns>(P, err, nch, g, grid, st)              \
          : launch_fused_e<EE, true, kRowBoth>(P, err, nch, g, grid, st))
    switch (e) {
        case Elem::F32:
            return acc64 ? TOMOS_BOTH(Elem::F32) : launch_fused_e<Elem::F32, false, kRowBoth>(P, err, nch, g, grid, st);
        case Elem::H16:
            return acc64 ? launch_fused_e<Elem::H16, true, kRowBoth>(P, err, nch, g, grid, st)
                         : launch_fused_e<Elem::H16, false, kRowBoth>(P, err, nch, g, grid, st);
        case Elem::B16:
            return acc64 ? launch_fused_e<Elem::B16, true, kRowBoth>(P, err, nch, g, grid, st)
                         : launch_fused_e<Elem::B16, false, kRowBoth>(P, err, nch, g, grid, st);
        case Elem::F16:
            return acc64 ? launch_fused_e<Elem::F16, true, kRowBoth>(P, err, nch, g, grid, st)
                         : launch_fused_e<Elem::F16, false, kRowBoth>(P, err, nch, g, grid, st);
        case Elem::A16: return TOMOS_BOTH(Elem::A16);
        case Elem::AB16: return TOMOS_BOTH(Elem::AB16);
        case Elem::AB16R: return TOMOS_BOTH(Elem::AB16R);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "fused pass: element type");
    }
#undef TOMOS_BOTH
}

// The staged-fp16 pass on the tensor cores (rowpass_mma.cuh).
template <int TPW, bool BF>
static tomos_status launch_fused_mma_t(const FusedParams& P, int* err, int grid, cudaStream_t st) {
    MmaPassParams T;
    T.f = P;
    T.err = err;
    T.cb = (int)((((int64_t)P.n * 2) + 15) / 16 * 16);
    // an odd number of 16-byte units between rows keeps ldmatrix free of
    // bank conflicts
    T.pitch = ((T.cb / 16) % 2 == 1) ? T.cb : T.cb + 16;
    // 32-row stages where two of them fit the ring, else 16-row stages
    const int rows = (size_t)2 * 32 * T.pitch + 64 <= kMmaSmemBudget ? 32 : 16;
    const size_t stage = (size_t)rows * T.pitch;
    int ns = (int)((kMmaSmemBudget - 64) / stage);
    if (ns > kMmaMaxStages) ns = kMmaMaxStages;
    if (ns < 2) return fail(TOMOS_ERR_UNSUPPORTED, "fused pass: rows too long for the stage ring");
    T.nstage = ns;
    const size_t smem = fused_rows_mma_smem(ns, rows, T.pitch);
    auto kern = rows == 32 ? fused_rows_mma_kernel<TPW, BF, 32> : fused_rows_mma_kernel<TPW, BF, 16>;
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, kMmaThreads, smem, st>>>(T);
    TOMOS_LAUNCH_CHECK("fused_rows_mma_kernel");
    return TOMOS_OK;
}

template <bool BF>
static tomos_status launch_fused_mma_b(const FusedParams& P, int* err, int tpw, int grid, cudaStream_t st) {
    switch (tpw) {
        case 1: return launch_fused_mma_t<1, BF>(P, err, grid, st);
        case 2: return launch_fused_mma_t<2, BF>(P, err, grid, st);
        case 3: return launch_fused_mma_t<3, BF>(P, err, grid, st);
        case 4: return launch_fused_mma_t<4, BF>(P, err, grid, st);
        case 5: return launch_fused_mma_t<5, BF>(P, err, grid, st);
        case 6: return launch_fused_mma_t<6, BF>(P, err, grid, st);
        case 7: return launch_fused_mma_t<7, BF>(P, err, grid, st);
        case 8: return launch_fused_mma_t<8, BF>(P, err, grid, st);
        case 9: return launch_fused_mma_t<9, BF>(P, err, grid, st);
        case 10: return launch_fused_mma_t<10, BF>(P, err, grid, st);
        case 11: return launch_fused_mma_t<11, BF>(P, err, grid, st);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "fused pass: no tensor-core instantiation");
    }
}

// The tensor-core pass over a 16-bit plane: fp16 (the staged FP32_16
// plane, or native FP16 storage) or bf16 (an FP32_BF16 wh plane).
static tomos_status launch_fused_mma(Elem e, const FusedParams& P, int* err, int tpw, int grid,
                                     cudaStream_t st) {
    return e == Elem::B16 ? launch_fused_mma_b<true>(P, err, tpw, grid, st)
                          : launch_fused_mma_b<false>(P, err, tpw, grid, st);
}

// wh plane of a row-major FP32_16 A -> IEEE fp16 words with the
// fp32_16_half_only values (fp32_16_pack.hpp:553-571), rows of ldh words;
// a block per row, a thread per 16-byte chunk.  Control-bit words are
// rare and scattered: here a chunk holding one costs that one thread a few
// instructions, where inside the LSQR pass the whole warp would wait on
// it every iteration.
__global__ void __launch_bounds__(128) stage_half_kernel(const uint16_t* __restrict__ wh,
                                                         int64_t m, int64_t ld, int64_t nch,
                                                         uint16_t* __restrict__ h16, int64_t ldh) {
    for (int64_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint4* src = reinterpret_cast<const uint4*>(wh + (size_t)r * ld);
        uint4* dst = reinterpret_cast<uint4*>(h16 + (size_t)r * ldh);
        for (int64_t c = threadIdx.x; c < nch; c += blockDim.x) {
            uint4 w = __ldcs(src + c);
            fix_half_chunk(w);
            dst[c] = w;
        }
    }
}

// Chooses the fused pass when A is row-major with 16-byte aligned rows
// and n fits the consumer warps (12288 columns; 8192 or 6144 for ACC64); otherwise
// the generic two-kernel path.
PassPlan plan_dense_pass(tomos_workspace* ws, const tomos_dense* A, Elem e, bool acc64, bool runs) {
    PassPlan pl;
    pl.e = e;
    pl.acc64 = acc64 || elem_is_exact(e);
    // run-summed dots: the FP32 and two-plane FP64-summing passes
    pl.runs = runs && pl.acc64 && (e == Elem::F32 || elem_two_planes(e));
    int nch = 0, g = 1;
    const bool ok = A->layout == TOMOS_ROW_MAJOR && A->cols > 0 &&
                    plan_row_lines(e, pl.acc64, pl.runs ? kRowBothRuns : kRowBoth, A->cols, A->ld, A->values,
                                   elem_is_exact(e) ? dense_lo_plane(A) : nullptr, &nch, &g);
    if (ok) {
        pl.fused = true;
        pl.nch = nch;
        pl.g = g;
        // a 16-bit plane read at the HALF tier (the staged fp16 plane,
        // native FP16, an FP32_BF16 wh plane): both products on the tensor
        // cores when n fits 12 warps x kMmaMaxTpw k-tiles
        const int64_t ktiles = (A->cols + 15) / 16;
        if ((e == Elem::F16 || e == Elem::B16) && !pl.acc64 && ktiles <= (int64_t)kMmaWarps * kMmaMaxTpw)
            pl.tpw = (int)((ktiles + kMmaWarps - 1) / kMmaWarps);
        pl.grid = row_pass_grid(A->rows);
        pl.gq = pl.grid;
        pl.gs = pl.grid;
        pl.qstride = ws->qstride;
    } else {
        pl.fused = false;
        pl.gq = 1;
        pl.qstride = A->cols;
        pl.gs = ws->gs_max;
    }
    return pl;
}

size_t dense_pass_scratch(const tomos_dense* A) {
    size_t a = gemv_scratch_bytes_max(A, TOMOS_NO_TRANSPOSE);
    size_t b = gemv_scratch_bytes_max(A, TOMOS_TRANSPOSE);
    return a > b ? a : b;
}

// Enqueues one A pass.  p: right vector; u_in: vector combined with cu;
// coef: device [cp, cu]; skip: device stop flag (NULL for unconditional).
tomos_status enqueue_dense_pass(tomos_workspace* ws, const tomos_dense* A,
                                       const PassPlan& pl, const float* p, const float* u_in,
                                       const double* coef, const int* skip, cudaStream_t st) {
    const void* lo = elem_is_exact(pl.e) ? dense_lo_plane(A) : nullptr;
    if (pl.fused) {
        FusedParams P;
        P.hi = A->values;
        P.lo = lo;
        P.m = A->rows;
        P.n = A->cols;
        P.ld = A->ld;
        P.p = p;
        P.u_in = u_in;
        P.u_out = ws->u;
        P.coef = coef;
        P.qpart = ws->qpart;
        P.sspart = ws->sspart;
        P.qstride = pl.qstride;
        P.skip = skip;
        tomos_status ls = pl.tpw > 0 ? launch_fused_mma(pl.e, P, &ws->st->pipe_err, pl.tpw, pl.grid, st)
                                     : launch_fused(pl.e, pl.acc64, pl.runs, P, &ws->st->pipe_err, pl.nch, pl.g,
                                                    pl.grid, st);
        if (ls) return ls;
        ws->launches += 1;
        return TOMOS_OK;
    }
    // Generic path: u = cp*A p + cu*u_in (u_in copied into u first when
    // they differ), ||u||^2, then q = A^T u.
    if (u_in != ws->u) {
        TOMOS_CUDA_TRY(cudaMemcpyAsync(ws->u, u_in, sizeof(float) * A->rows,
                                       cudaMemcpyDeviceToDevice, st));
    }
    GemvLaunch L;
    std::string why;
    if (!gemv_shape(A, TOMOS_NO_TRANSPOSE, &L.dot, &L.outer, &L.inner, &why))
        return fail(TOMOS_ERR_INVALID, why);
    L.hi = A->values;
    L.lo = lo;
    L.ld = A->ld;
    L.x = p;
    L.y = ws->u;
    L.coef = coef;
    L.skip = skip;
    L.scratch = ws->scratch;
    L.scratch_bytes = ws->scratch_bytes;
    tomos_status s = gemv_launch(L, pl.e, pl.acc64, st);
    if (s) return s;
    ws->launches += (L.dot ? 1 : 2) + 1 + 2;
    sumsq_partial_kernel<<<pl.gs, 256, 0, st>>>(ws->u, A->rows, skip, ws->sspart);
    TOMOS_LAUNCH_CHECK("sumsq_partial_kernel");
    GemvLaunch T;
    if (!gemv_shape(A, TOMOS_TRANSPOSE, &T.dot, &T.outer, &T.inner, &why))
        return fail(TOMOS_ERR_INVALID, why);
    T.hi = A->values;
    T.lo = lo;
    T.ld = A->ld;
    T.x = ws->u;
    T.y = ws->qpart;
    T.alpha = 1.0;
    T.beta = 0.0;
    T.skip = skip;
    T.scratch = ws->scratch;
    T.scratch_bytes = ws->scratch_bytes;
    return gemv_launch(T, pl.e, pl.acc64, st);
}

// ------------------------------------------------------------ n-side glue

static NSide make_nside(tomos_workspace* ws, const PassPlan& pl, float* x, bool init,
                        const int* skip, const double* dscale = nullptr) {
    NSide S;
    S.dscale = dscale;
    S.n = ws->n;
    S.qpart = ws->qpart;
    S.qstride = pl.qstride;
    S.gq = pl.gq;
    S.sspart = ws->sspart;
    S.gs = pl.gs;
    S.t = ws->t;
    S.vhat = ws->vhat;
    S.v = ws->v;
    S.wt = ws->wt;
    S.p = ws->p;
    S.x = x;
    S.vpart = ws->vpart;
    S.xpart = ws->xpart;
    S.qnpart = ws->qnpart;
    S.Rcm = ws->Rcm;
    S.Rrm = ws->Rrm;
    S.has_precond = ws->has_precond ? 1 : 0;
    S.init = init ? 1 : 0;
    S.nb1 = ws->nb1;
    S.nb3 = ws->nb3;
    S.scal = ws->scal;
    S.st = ws->st;
    S.skip = skip;
    S.qsum = nullptr;
    S.cond = 0;
    S.use_cond = 0;
    if (ws->comm) {  // the pass's partials were folded and summed across ranks
        S.qsum = ws->shard;
        S.sspart = ws->shard + ws->n;
        S.gs = 1;
    }
    return S;
}

static tomos_status enqueue_nside(tomos_workspace* ws, const NSide& S, cudaStream_t st) {
    nside_reduce_kernel<<<ws->nb1, 256, 0, st>>>(S);
    TOMOS_LAUNCH_CHECK("nside_reduce_kernel");
    if (S.has_precond) {
        nside_precond_t_kernel<<<ws->nb3, 256, 0, st>>>(S);
        TOMOS_LAUNCH_CHECK("nside_precond_t_kernel");
    }
    nside_update_kernel<<<ws->nb3, 256, 0, st>>>(S);
    TOMOS_LAUNCH_CHECK("nside_update_kernel");
    nside_finish_kernel<<<1, 256, 0, st>>>(S);
    TOMOS_LAUNCH_CHECK("nside_finish_kernel");
    ws->launches += S.has_precond ? 4 : 3;
    return TOMOS_OK;
}

// HALF-tier iterations over a row-major FP32_16 A read a staged fp16 copy
// of its wh plane (one conversion per solve, in the workspace, or the
// caller's staged_plane) -- on the tensor cores when n fits that pass.
// The restart passes read A itself.
struct DensePass : PassOps {
    tomos_workspace* ws;
    const tomos_dense* A;
    Elem iter_e, init_e;
    bool stage = false;
    tomos_dense staged{};
    DensePass(tomos_workspace* w, const tomos_dense* a, Elem ie, Elem ze)
        : ws(w), A(a), iter_e(ie), init_e(ze) {
        stage = ie == Elem::H16 && plan_dense_pass(ws, A, ie, false).fused;
        staged = *A;  // values set by prepare()
        staged.values_lo = nullptr;
        staged.ld = (A->cols + 7) / 8 * 8;
    }
    // A copy the caller staged already (tomos_countsketch_apply_stage).
    const void* given = nullptr;
    int64_t given_ld = 0;
    tomos_status prepare(cudaStream_t st) override {
        if (!stage) return TOMOS_OK;
        if (given) {
            staged = *A;
            staged.values = const_cast<void*>(given);  // read only
            staged.values_lo = nullptr;
            staged.ld = given_ld;
            return TOMOS_OK;
        }
        const int64_t m = A->rows, n = A->cols, ldh = (n + 7) / 8 * 8;
        const size_t bytes = (size_t)m * ldh * sizeof(uint16_t);
        if (bytes > ws->h16_bytes) {
            if (ws->h16) cudaFree(ws->h16);
            ws->h16 = nullptr;
            ws->h16_bytes = 0;
            if (cudaMalloc(&ws->h16, bytes) != cudaSuccess) {
                cudaGetLastError();
                stage = false;  // not enough memory: iterate on A itself
                return TOMOS_OK;
            }
            ws->h16_bytes = bytes;
        }
        staged = *A;
        staged.values = ws->h16;
        staged.values_lo = nullptr;
        staged.ld = ldh;
        int64_t grid = (int64_t)sm_count() * 16;
        if (grid > m) grid = m;
        if (grid < 1) grid = 1;
        stage_half_kernel<<<(unsigned)grid, 128, 0, st>>>(static_cast<const uint16_t*>(A->values), m,
                                                          A->ld, ldh / 8, static_cast<uint16_t*>(ws->h16),
                                                          ldh);
        TOMOS_LAUNCH_CHECK("stage_half_kernel");
        ws->launches += 1;
        return TOMOS_OK;
    }
    PassPlan plan(bool init) override {
        if (!init && stage) return plan_dense_pass(ws, &staged, Elem::F16, false);
        return plan_dense_pass(ws, A, init ? init_e : iter_e, init, init && runs);
    }
    tomos_status enqueue(const PassPlan& pl, const float* p, const float* u_in, const double* coef,
                         const int* skip, cudaStream_t st) override {
        // F16 passes read the staged plane only when this solve staged one;
        // native FP16 storage is read in place
        return enqueue_dense_pass(ws, (stage && pl.e == Elem::F16) ? &staged : A, pl, p, u_in, coef, skip, st);
    }
    tomos_status fro2(double* out, const double* d, cudaStream_t st) override {
        bool dot;
        int64_t outer, inner;
        std::string why;
        gemv_shape(A, TOMOS_NO_TRANSPOSE, &dot, &outer, &inner, &why);
        const void* lo = elem_is_exact(init_e) ? dense_lo_plane(A) : nullptr;
        const int g = ws->gs_max;
        const int ci = A->layout == TOMOS_ROW_MAJOR ? 1 : 0;
#define TOMOS_FRO2(EE) fro2_partial_kernel<EE><<<g, 256, 0, st>>>(A->values, lo, outer, inner, A->ld, d, ci, ws->bpart)
        switch (init_e) {
            case Elem::F32: TOMOS_FRO2(Elem::F32); break;
            case Elem::H16: TOMOS_FRO2(Elem::H16); break;
            case Elem::F16: TOMOS_FRO2(Elem::F16); break;
            case Elem::A16: TOMOS_FRO2(Elem::A16); break;
            case Elem::B16: TOMOS_FRO2(Elem::B16); break;
            case Elem::AB16: TOMOS_FRO2(Elem::AB16); break;
            case Elem::AB16R: TOMOS_FRO2(Elem::AB16R); break;
            default: return fail(TOMOS_ERR_UNSUPPORTED, "fro2: element type");
        }
#undef TOMOS_FRO2
        TOMOS_LAUNCH_CHECK("fro2_partial_kernel");
        sum_to_scalar_kernel<<<1, 256, 0, st>>>(ws->bpart, g, out);
        TOMOS_LAUNCH_CHECK("sum_to_scalar_kernel");
        return TOMOS_OK;
    }
    uint64_t key() override {
        return reinterpret_cast<uint64_t>(A->values) ^ ((uint64_t)A->layout << 60) ^
               ((uint64_t)A->ld << 20) ^
               (stage ? reinterpret_cast<uint64_t>(staged.values) * 31 ^ ((uint64_t)staged.ld << 40) : 0);
    }
    int64_t rows() override { return A->rows; }
    int64_t cols() override { return A->cols; }
};

// ------------------------------------------------------------ driver

tomos_status refresh_precond(tomos_workspace* ws, cudaStream_t st) {
    if (!ws->has_precond) return TOMOS_OK;
    TOMOS_CUDA_TRY(cudaMemsetAsync(ws->scal + 7, 0, sizeof(double), st));
    precond_copy_kernel<<<ws->gs_max, 256, 0, st>>>(ws->precond.values, ws->precond.numeric,
                                                   ws->precond.layout, ws->precond.ld, ws->n,
                                                   ws->Rcm, ws->Rrm, ws->scal + 7);
    TOMOS_LAUNCH_CHECK("precond_copy_kernel");
    ws->launches += 1;
    return TOMOS_OK;
}

static tomos_status sync_state(tomos_workspace* ws) {
    TOMOS_CUDA_TRY(cudaMemcpyAsync(ws->st_host, ws->st, sizeof(LsqrDev), cudaMemcpyDeviceToHost,
                                   ws->stream));
    TOMOS_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    if (ws->st_host->pipe_err)
        return fail(TOMOS_ERR_CUDA, "A pass: a bounded pipeline wait expired (code " +
                                        std::to_string(ws->st_host->pipe_err) + ")");
    return TOMOS_OK;
}

static double eta_of(const LsqrDev& s) {
    const double den1 = s.anorm_fro * s.xnorm + s.bnorm;
    const double e1 = den1 > 0.0 ? s.beta / den1 : 0.0;
    const double den2 = s.anorm_fro * s.beta;
    const double e2 = den2 > 0.0 ? s.arnorm / den2 : 0.0;
    return e1 < e2 ? e1 : e2;
}

tomos_status solve_driver(tomos_workspace* ws, PassOps& ops, const float* b, float* x_user,
                          const tomos_lsqr_opts* o, tomos_lsqr_report* rep, void* user_stream) {
    cudaStream_t us = as_stream(user_stream);
    cudaStream_t st = ws->stream;
    const int64_t m = ops.rows(), n = ops.cols();
    ws->comm = o->comm;
    struct CommScope {  // the communicator belongs to this solve only
        tomos_workspace* w;
        ~CommScope() {
            // A graph that captured the communicator's all-reduce must not
            // outlive it (the caller may destroy the communicator next).
            if (w->comm && w->graph) {
                cudaGraphExecDestroy(w->graph);
                w->graph = nullptr;
                w->graph_key.clear();
            }
            w->comm = nullptr;
        }
    } comm_scope{ws};
    // One pass over A; a row-sharded solve then sums its partials across ranks.
    auto pass = [&](const PassPlan& pl, const float* p, const float* u_in, const double* coef,
                    const int* skip) -> tomos_status {
        tomos_status ps = ops.enqueue(pl, p, u_in, coef, skip, st);
        if (ps || !ws->comm) return ps;
        return enqueue_shard_reduce(ws, ws->comm, ws->qpart, pl.gq, pl.qstride, ws->sspart, pl.gs, skip, st);
    };
    tomos_lsqr_report R;
    std::memset(&R, 0, sizeof(R));

    // Order against the caller's stream.
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, us));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_fence, 0));
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_start, st));

    const int64_t launches0 = ws->launches;
    const int max_iters = o->max_iters > 0 ? o->max_iters : 0;
    const int restarts = o->restarts > 0 ? o->restarts : 1;
    const int64_t hist_total = (int64_t)max_iters * restarts;
    tomos_status s = ensure_history(ws, (int)(hist_total > 0 ? hist_total : 1));
    if (s) return s;

    // Precondition copies (FP64, both orientations).
    s = refresh_precond(ws, st);
    if (s) return s;
    // The solve runs on the workspace's copy of x, so the iteration graph
    // (whose kernels hold x's address) is reused whatever buffer the
    // caller passes; the result is copied out at the end.
    float* x = ws->xg;
    if (o->warm_start)
        TOMOS_CUDA_TRY(cudaMemcpyAsync(x, x_user, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    else
        TOMOS_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(float) * n, st));
    s = ops.prepare(st);
    if (s) return s;

    // ||b|| and, for the backward-error rule, ||A||_F go into the device
    // state by a kernel (no host round trip before the first pass).
    int extra_passes = 0;
    // The column scale the n-side kernels read (the iteration graph holds
    // its address): the workspace's copy, so a graph captured by an earlier
    // solve never reads a caller's buffer that has since been freed.
    const double* dsc = nullptr;
    if (o->stop_rule == TOMOS_STOP_BACKWARD && o->col_scale) {
        TOMOS_CUDA_TRY(cudaMemcpyAsync(ws->dscale, o->col_scale, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        dsc = ws->dscale;
    }
    const bool need_fro = o->stop_rule == TOMOS_STOP_BACKWARD && !o->anorm_fro_dev && !(o->anorm_fro > 0.0);

    LsqrDev init_state;
    std::memset(&init_state, 0, sizeof(init_state));
    init_state.anorm_fro = o->anorm_fro;
    init_state.tol = o->tol;
    init_state.max_relres = o->max_relres;
    init_state.inner_rtol = o->stop_rule == TOMOS_STOP_BACKWARD ? o->inner_rtol : 0.0;
    init_state.inner_tol = o->tol * (o->inner_eta_factor > 0.0 ? o->inner_eta_factor : 1.0);
    init_state.max_iters = max_iters;
    init_state.stop_rule = o->stop_rule;
    init_state.history = ws->hist;
    init_state.history_cap = ws->hist_cap;
    init_state.done = 1;
    TOMOS_CUDA_TRY(cudaMemcpyAsync(ws->st, &init_state, sizeof(LsqrDev), cudaMemcpyHostToDevice, st));
    const double coef_init[2] = {-1.0, 1.0};
    TOMOS_CUDA_TRY(cudaMemcpyAsync(ws->coef_init, coef_init, sizeof(coef_init),
                                   cudaMemcpyHostToDevice, st));
    sumsq_partial_kernel<<<ws->gs_max, 256, 0, st>>>(b, m, nullptr, ws->bpart);
    TOMOS_LAUNCH_CHECK("sumsq_partial_kernel");
    ws->launches += 2;
    const double* bsum = ws->bpart;
    int64_t nbsum = ws->gs_max;
    if (ws->comm) {  // ||b||^2 over every rank's rows
        sum_to_scalar_kernel<<<1, 256, 0, st>>>(ws->bpart, ws->gs_max, ws->scal + 2);
        TOMOS_LAUNCH_CHECK("sum_to_scalar_kernel");
        s = comm_allreduce(ws->comm, ws->scal + 2, 1, st);
        if (s) return s;
        bsum = ws->scal + 2;
        nbsum = 1;
    }
    if (need_fro) {
        s = ops.fro2(ws->scal + 3, dsc, st);
        if (s) return s;
        if (ws->comm) {
            s = comm_allreduce(ws->comm, ws->scal + 3, 1, st);
            if (s) return s;
        }
        extra_passes = 1;
        ws->launches += 2;
    }
    state_norms_kernel<<<1, 256, 0, st>>>(bsum, nbsum, o->anorm_fro_dev,
                                          need_fro ? ws->scal + 3 : nullptr, ws->st);
    TOMOS_LAUNCH_CHECK("state_norms_kernel");

    // Under the BACKWARD rule at a tolerance of 1e-6 or above, the accurate
    // passes' dots need only a backward error below it: FP32 products over
    // runs of at most 8, summed in FP64 (gamma_8 = 4.8e-7), the accuracy of
    // the FP32 tier's own passes, instead of one FP64 conversion and product
    // an element.  RELRES keeps the FP64 products: the residual of a
    // consistent system is far below the rounding of its products.
    ops.runs = o->stop_rule == TOMOS_STOP_BACKWARD && o->tol >= kRunsTolMin;
    PassPlan pl_init = ops.plan(true);
    PassPlan pl_iter = ops.plan(false);

    // Capture (or reuse) the graph of one iteration.
    std::vector<uint64_t> key = {ops.key(),
                                 (uint64_t)pl_iter.fused,
                                 (uint64_t)pl_iter.e,
                                 (uint64_t)pl_iter.nch,
                                 (uint64_t)pl_iter.g,
                                 (uint64_t)pl_iter.grid,
                                 (uint64_t)pl_iter.tpw,
                                 reinterpret_cast<uint64_t>(x),
                                 reinterpret_cast<uint64_t>(dsc),
                                 (uint64_t)ws->has_precond,
                                 (uint64_t)n,
                                 (uint64_t)m,
                                 reinterpret_cast<uint64_t>(o->comm)};
    if (!ws->graph || ws->graph_key != key) {
        if (ws->graph) cudaGraphExecDestroy(ws->graph);
        ws->graph = nullptr;
        ws->graph_loop = false;
        // A graph whose one node is a while loop over the iteration: its
        // condition starts at 1 at each launch and N4 sets it, so one
        // launch runs a restart's iterations to the stopping rule with no
        // host round trip.  Row-sharded solves (an NCCL call in the
        // iteration) and a runtime without conditional nodes replay the
        // plain iteration graph in batches instead.
        if (!o->comm) {
            const int64_t before = ws->launches;
            cudaGraph_t g = nullptr;
            cudaGraphConditionalHandle h = 0;
            cudaGraphNodeParams cp = {};
            cudaGraphNode_t node = nullptr;
            bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
                      cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
            if (ok) {
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = h;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                ok = cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess;
            }
            if (ok)
                ok = cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                const int* skip = &ws->st->done;
                NSide S = make_nside(ws, pl_iter, x, false, skip, dsc);
                S.cond = h;
                S.use_cond = 1;
                tomos_status cs = pass(pl_iter, ws->p, ws->u, ws->st->coef, skip);
                if (!cs) cs = enqueue_nside(ws, S, st);
                cudaGraph_t body = nullptr;
                const cudaError_t ce = cudaStreamEndCapture(st, &body);
                if (cs) {
                    cudaGraphDestroy(g);
                    return cs;
                }
                ok = ce == cudaSuccess;
            }
            if (ok) ok = cudaGraphInstantiate(&ws->graph, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
            if (ok) {
                ws->graph_loop = true;
                ws->graph_key = key;
                ws->graph_kernels = ws->launches - before;
            } else {
                cudaGetLastError();  // not sticky: fall back to the plain graph
                if (ws->graph) cudaGraphExecDestroy(ws->graph);
                ws->graph = nullptr;
                ws->launches = before;
            }
        }
    }
    if (!ws->graph || ws->graph_key != key) {
        if (ws->graph) cudaGraphExecDestroy(ws->graph);
        ws->graph = nullptr;
        ws->graph_loop = false;
        cudaGraph_t g = nullptr;
        const int64_t before = ws->launches;
        TOMOS_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int* skip = &ws->st->done;
        tomos_status cs = pass(pl_iter, ws->p, ws->u, ws->st->coef, skip);
        if (!cs) cs = enqueue_nside(ws, make_nside(ws, pl_iter, x, false, skip, dsc), st);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (cs) {
            if (g) cudaGraphDestroy(g);
            return cs;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&ws->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
        ws->graph_key = key;
        ws->graph_kernels = ws->launches - before;
    }

    std::vector<double> hist_host;
    int hist_read = 0;
    int accurate_passes = extra_passes, iter_passes = 0;
    bool converged = false;
    int restarts_used = 0;
    LsqrDev& H = *ws->st_host;

    for (int rs = 0; rs < restarts; ++rs) {
        // Restart-boundary stopping check on the running estimate
        // (check_stopping_criteria at the top of each restart, lsqr.cpp:705-708).
        if (rs > 0 && o->stop_rule == TOMOS_STOP_RELRES && H.iter > 0) {
            double rel = H.rhsnorm == 0.0 ? 0.0 : std::fabs(H.phi_bar) / H.rhsnorm;
            hist_host.push_back(rel);
            if (H.rhsnorm == 0.0 || rel < o->tol || rel < o->max_relres) {
                converged = true;
                break;
            }
        }
        // initialize(): ut = b - A x (restarted from the current x).  From
        // x = 0 the pass only forms A^T b, so it runs at the iteration tier
        // (the operator the inner iterations then use); later restarts
        // need the residual of the accurate A.
        restarts_used = rs + 1;
        const PassPlan& pz = (rs == 0 && !o->warm_start) ? pl_iter : pl_init;
        if (o->profile) TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_pa, st));
        s = pass(pz, x, b, ws->coef_init, nullptr);
        if (s) return s;
        if (o->profile) TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_pb, st));
        s = enqueue_nside(ws, make_nside(ws, pz, x, true, nullptr, dsc), st);
        if (s) return s;
        if (&pz == &pl_init && (elem_is_exact(pz.e) || pz.e != pl_iter.e || pz.acc64 != pl_iter.acc64))
            ++accurate_passes;
        else
            ++iter_passes;
        s = sync_state(ws);
        if (s) return s;
        if (o->profile) {
            // restart passes at the accurate tier only (the x = 0 pass is
            // an iteration-tier pass)
            float pm = 0.0f;
            TOMOS_CUDA_TRY(cudaEventElapsedTime(&pm, ws->ev_pa, ws->ev_pb));
            if (&pz == &pl_init) {
                R.init_pass_ms += pm;
                R.init_pass_count += 1;
            }
        }
        if (H.rhsnorm == 0.0) {
            converged = true;
            break;
        }
        if (o->stop_rule == TOMOS_STOP_RELRES) {
            const double true_relres = H.beta / H.rhsnorm;
            if (true_relres < o->tol || true_relres < o->max_relres) {
                converged = true;
                break;
            }
        } else {
            R.rnorm = H.beta;
            R.arnorm = H.arnorm;
            R.xnorm = H.xnorm;
            R.backward_error = eta_of(H);
            if (R.backward_error <= o->tol || H.beta == 0.0) {
                converged = true;
                break;
            }
        }
        if (H.breakdown || max_iters == 0) continue;
        // Inner iterations in batches of graph launches; the device stops
        // doing work once its stopping rule fires.  The profiling mode
        // launches each iteration directly and times its pass over A.
        int batch = 4;
        int done_iters = 0;
        while (o->profile && done_iters < max_iters) {
            const int* skip = &ws->st->done;
            TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_pa, st));
            s = pass(pl_iter, ws->p, ws->u, ws->st->coef, skip);
            if (s) return s;
            TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_pb, st));
            s = enqueue_nside(ws, make_nside(ws, pl_iter, x, false, skip, dsc), st);
            if (s) return s;
            s = sync_state(ws);
            if (s) return s;
            float pm = 0.0f;
            TOMOS_CUDA_TRY(cudaEventElapsedTime(&pm, ws->ev_pa, ws->ev_pb));
            R.iter_pass_ms += pm;
            R.iter_pass_count += 1;
            done_iters = H.iter_restart;
            if (H.done) break;
        }
        if (!o->profile && ws->graph_loop) {
            // one launch: the device loops to the stopping rule
            TOMOS_CUDA_TRY(cudaGraphLaunch(ws->graph, st));
            s = sync_state(ws);
            if (s) return s;
            ws->launches += (int64_t)H.iter_restart * ws->graph_kernels;
            done_iters = max_iters;
        }
        while (!o->profile && done_iters < max_iters) {
            int k = batch < max_iters - done_iters ? batch : max_iters - done_iters;
            for (int i = 0; i < k; ++i) TOMOS_CUDA_TRY(cudaGraphLaunch(ws->graph, st));
            ws->launches += (int64_t)k * ws->graph_kernels;
            s = sync_state(ws);
            if (s) return s;
            done_iters = H.iter_restart;
            if (H.done) break;
            if (batch < 32) batch *= 2;
        }
        iter_passes += H.iter_restart;
        if (H.iter > hist_read) {
            int cnt = (H.iter < ws->hist_cap ? H.iter : ws->hist_cap) - hist_read;
            if (cnt > 0) {
                std::vector<double> tmp(cnt);
                TOMOS_CUDA_TRY(cudaMemcpy(tmp.data(), ws->hist + hist_read, sizeof(double) * cnt,
                                          cudaMemcpyDeviceToHost));
                hist_host.insert(hist_host.end(), tmp.begin(), tmp.end());
                hist_read += cnt;
            }
        }
        if (o->stop_rule == TOMOS_STOP_RELRES && H.converged) {
            converged = true;
            break;
        }
    }
    // The backward-error rule reports the accurate eta of the returned x.
    if (o->stop_rule == TOMOS_STOP_BACKWARD && !converged) {
        s = pass(pl_init, x, b, ws->coef_init, nullptr);
        if (s) return s;
        s = enqueue_nside(ws, make_nside(ws, pl_init, x, true, nullptr, dsc), st);
        if (s) return s;
        ++accurate_passes;
        s = sync_state(ws);
        if (s) return s;
        R.rnorm = H.beta;
        R.arnorm = H.arnorm;
        R.xnorm = H.xnorm;
        R.backward_error = eta_of(H);
        converged = R.backward_error <= o->tol;
    }
    TOMOS_CUDA_TRY(cudaMemcpyAsync(x_user, x, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
    TOMOS_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop);
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, st));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(us, ws->ev_fence, 0));

    const double anorm = H.anorm_fro, bnorm = H.bnorm;
    R.iterations = H.iter;
    R.restarts_used = restarts_used;
    R.converged = converged ? 1 : 0;
    R.relres = H.relres;
    if (o->stop_rule == TOMOS_STOP_RELRES) R.relres = H.rhsnorm > 0 ? std::fabs(H.phi_bar) / H.rhsnorm : 0.0;
    R.anorm_fro = anorm;
    R.bnorm = bnorm;
    if (o->stop_rule != TOMOS_STOP_BACKWARD) R.xnorm = H.xnorm;
    R.elapsed_ms = ms;
    R.accurate_passes = accurate_passes;
    R.half_passes = iter_passes;
    R.kernel_launches = (int32_t)(ws->launches - launches0);
    if (o->history && o->history_cap > 0) {
        int cnt = (int)hist_host.size() < o->history_cap ? (int)hist_host.size() : o->history_cap;
        for (int i = 0; i < cnt; ++i) o->history[i] = hist_host[i];
        R.history_len = cnt;
    }
    if (rep) *rep = R;
    return TOMOS_OK;
}

tomos_status workspace_check(tomos_workspace* ws, int64_t m, int64_t n) {
    if (!ws) return fail(TOMOS_ERR_INVALID, "lsqr_solve: null workspace");
    if (ws->m != m || ws->n != n)
        return fail(TOMOS_ERR_INVALID, "lsqr_solve: workspace is sized for " +
                                           std::to_string(ws->m) + "x" + std::to_string(ws->n) +
                                           ", matrix is " + std::to_string(m) + "x" +
                                           std::to_string(n));
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != ws->device)
        return fail(TOMOS_ERR_INVALID, "lsqr_solve: workspace belongs to another device");
    return TOMOS_OK;
}

bool opts_ok(const tomos_lsqr_opts* o, std::string* why) {
    if (!o) {
        *why = "null options";
        return false;
    }
    if (o->stop_rule != TOMOS_STOP_RELRES && o->stop_rule != TOMOS_STOP_BACKWARD) {
        *why = "unknown stop rule";
        return false;
    }
    if (o->max_iters < 0) {
        *why = "negative max_iters";
        return false;
    }
    return true;
}

// Tier used for the restart-boundary residual.
static int32_t init_tier_for(int32_t numeric, const tomos_lsqr_opts* o, int32_t iter_tier) {
    const bool packed = numeric == TOMOS_FP32_16 || numeric == TOMOS_FP32_BF16;
    if (packed && (o->implicit_duplicate || o->stop_rule == TOMOS_STOP_BACKWARD))
        return TOMOS_TIER_ACCURATE;
    return iter_tier;
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

tomos_status tomos_workspace_create(int64_t m, int64_t n, int32_t value_type,
                                    int32_t precond_type, tomos_workspace** out) {
    if (!out) return fail(TOMOS_ERR_INVALID, "tomos_workspace_create: null output");
    *out = nullptr;
    if (m < 0 || n < 0) return fail(TOMOS_ERR_INVALID, "tomos_workspace_create: negative size");
    if (value_type != TOMOS_FP32)
        return fail(TOMOS_ERR_UNSUPPORTED,
                    "tomos_workspace_create: only FP32 working vectors are registered");
    if (precond_type != TOMOS_FP32 && precond_type != TOMOS_FP64)
        return fail(TOMOS_ERR_UNSUPPORTED,
                    "tomos_workspace_create: precond_type must be FP32 or FP64");
    tomos_workspace* ws = new tomos_workspace();
    ws->m = m;
    ws->n = n;
    ws->value_type = value_type;
    ws->precond_type = precond_type;
    cudaGetDevice(&ws->device);
    const int sms = sm_count();
    ws->gmax = sms * 4;
    ws->qstride = ((n + 31) / 32) * 32;
    if (ws->qstride < 32) ws->qstride = 32;
    ws->nb1 = (int)((n + 31) / 32);
    ws->nb3 = (int)((n + 7) / 8);
    if (ws->nb1 < 1) ws->nb1 = 1;
    if (ws->nb3 < 1) ws->nb3 = 1;
    ws->gs_max = sms * 2;
    bool ok = true;
    auto A = [&](cudaError_t e) { ok = ok && e == cudaSuccess; };
    A(alloc(&ws->u, (size_t)m));
    A(alloc(&ws->v, (size_t)n));
    A(alloc(&ws->wt, (size_t)n));
    A(alloc(&ws->p, (size_t)n));
    A(alloc(&ws->qvec, (size_t)n));
    A(alloc(&ws->t, (size_t)n));
    A(alloc(&ws->vhat, (size_t)n));
    size_t qp = (size_t)ws->gmax * ws->qstride;
    if (qp < (size_t)n) qp = n;
    A(alloc(&ws->qpart, qp));
    size_t sp = (size_t)(ws->gmax > ws->gs_max ? ws->gmax : ws->gs_max);
    A(alloc(&ws->sspart, sp));
    A(alloc(&ws->vpart, (size_t)(ws->nb1 > ws->nb3 ? ws->nb1 : ws->nb3)));
    A(alloc(&ws->xpart, (size_t)ws->nb3));
    A(alloc(&ws->qnpart, (size_t)ws->nb1));
    A(alloc(&ws->scal, 8));
    A(alloc(&ws->coef_init, 2));
    A(alloc(&ws->bpart, (size_t)ws->gs_max));
    A(alloc(&ws->fro2, 1));
    A(alloc(&ws->st, 1));
    A(alloc(&ws->shard, (size_t)n + 1));
    A(alloc(&ws->xg, (size_t)n));
    A(alloc(&ws->dscale, (size_t)n));
    A(cudaMallocHost(reinterpret_cast<void**>(&ws->st_host), sizeof(LsqrDev)));
    A(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
    A(cudaEventCreate(&ws->ev_start));
    A(cudaEventCreate(&ws->ev_stop));
    A(cudaEventCreate(&ws->ev_pa));
    A(cudaEventCreate(&ws->ev_pb));
    A(cudaEventCreateWithFlags(&ws->ev_fence, cudaEventDisableTiming));
    if (!ok) {
        ws_free(ws);
        delete ws;
        return fail(TOMOS_ERR_ALLOC, "tomos_workspace_create: device allocation failed");
    }
    std::memset(ws->st_host, 0, sizeof(LsqrDev));
    cudaMemset(ws->st, 0, sizeof(LsqrDev));
    *out = ws;
    return TOMOS_OK;
}

tomos_status tomos_column_scale(const double* colsq, int64_t n, double* d, double* anorm, void* stream) {
    if (n < 0) return fail(TOMOS_ERR_INVALID, "column_scale: negative n");
    if (!anorm || (n > 0 && (!colsq || !d))) return fail(TOMOS_ERR_INVALID, "column_scale: null pointer");
    column_scale_kernel<<<1, 256, 0, as_stream(stream)>>>(colsq, n, d, anorm);
    TOMOS_LAUNCH_CHECK("column_scale_kernel");
    return TOMOS_OK;
}

tomos_status tomos_workspace_destroy(tomos_workspace* ws) {
    if (!ws) return TOMOS_OK;
    cudaStreamSynchronize(ws->stream);
    ws_free(ws);
    delete ws;
    return TOMOS_OK;
}

tomos_status tomos_workspace_add_precond(tomos_workspace* ws, const tomos_dense* Rinv) {
    if (!ws) return fail(TOMOS_ERR_INVALID, "add_precond: null workspace");
    if (!Rinv) {
        ws->has_precond = false;
        return TOMOS_OK;
    }
    if (Rinv->numeric != ws->precond_type)
        return fail(TOMOS_ERR_INVALID,
                    "add_precond: precond's NumericType doesn't match the precond_type the "
                    "workspace was created with.");
    if (Rinv->rows != ws->n || Rinv->cols != ws->n)
        return fail(TOMOS_ERR_INVALID, "add_precond: preconditioner must be n x n");
    if (Rinv->layout != TOMOS_ROW_MAJOR && Rinv->layout != TOMOS_COL_MAJOR)
        return fail(TOMOS_ERR_INVALID, "add_precond: bad layout");
    if (Rinv->ld < ws->n) return fail(TOMOS_ERR_INVALID, "add_precond: bad leading dimension");
    if (!ws->Rcm) {
        bool ok = alloc(&ws->Rcm, (size_t)ws->n * ws->n) == cudaSuccess &&
                  alloc(&ws->Rrm, (size_t)ws->n * ws->n) == cudaSuccess;
        if (!ok) return fail(TOMOS_ERR_ALLOC, "add_precond: allocation failed");
    }
    ws->precond = *Rinv;
    ws->has_precond = true;
    return TOMOS_OK;
}

tomos_status tomos_lsqr_solve_dense(const tomos_dense* A, const float* b, float* x,
                                    tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                    tomos_lsqr_report* report, void* stream) {
    std::string why;
    bool dot;
    int64_t outer, inner;
    if (!gemv_shape(A, TOMOS_NO_TRANSPOSE, &dot, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "lsqr_solve: " + why);
    if (!opts_ok(opts, &why)) return fail(TOMOS_ERR_INVALID, "lsqr_solve: " + why);
    if (opts->refine_csr)
        return fail(TOMOS_ERR_INVALID, "lsqr_solve: a sparse mtx_refine_precision for a dense A");
    tomos_status s = workspace_check(ws, A->rows, A->cols);
    if (s) return s;
    if (!b || !x || (!A->values && A->rows * A->cols > 0))
        return fail(TOMOS_ERR_INVALID, "lsqr_solve: null pointer");
    if (opts->implicit_duplicate && A->numeric != TOMOS_FP32_16 && A->numeric != TOMOS_FP32_BF16)
        return fail(TOMOS_ERR_INVALID,
                    "lsqr_solve: Workspace::use_implicit_duplicate_ requires A to be stored "
                    "packed (FP32_16 or FP32_BF16).");
    Elem ie, ze;
    if (!resolve_elem(A, opts->iter_tier, &ie, &why))
        return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_solve: " + why);
    int32_t it = opts->iter_tier == TOMOS_TIER_AUTO
                     ? ((A->numeric == TOMOS_FP32) ? TOMOS_TIER_NATIVE : TOMOS_TIER_HALF)
                     : opts->iter_tier;
    if (!resolve_elem(A, init_tier_for(A->numeric, opts, it), &ze, &why))
        return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_solve: " + why);
    if (A->rows == 0 || A->cols == 0) {
        if (A->cols > 0 && !opts->warm_start) cudaMemsetAsync(x, 0, sizeof(float) * A->cols, as_stream(stream));
        if (report) std::memset(report, 0, sizeof(*report));
        if (report) report->converged = 1;
        return TOMOS_OK;
    }
    // An explicit duplicate takes precedence over the implicit one for the
    // restart residual, as in the reference (lsqr.cpp:459-473: the explicit
    // branch is tested first; lsqr_registries.cpp:102-112 sets both flags).
    if (opts->refine) {
        const tomos_dense* Rf = opts->refine;
        if (!gemv_shape(Rf, TOMOS_NO_TRANSPOSE, &dot, &outer, &inner, &why))
            return fail(TOMOS_ERR_INVALID, "lsqr_solve: mtx_refine_precision: " + why);
        if (Rf->rows != A->rows || Rf->cols != A->cols || (!Rf->values && Rf->rows * Rf->cols > 0))
            return fail(TOMOS_ERR_INVALID, "lsqr_solve: mtx_refine_precision must have A's size");
        Elem re;
        const int32_t rt = Rf->numeric == TOMOS_FP32 ? TOMOS_TIER_NATIVE : TOMOS_TIER_ACCURATE;
        if (!resolve_elem(Rf, rt, &re, &why))
            return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_solve: mtx_refine_precision: " + why);
        if (A->rows == 0 || A->cols == 0) {
            if (A->cols > 0 && !opts->warm_start) cudaMemsetAsync(x, 0, sizeof(float) * A->cols, as_stream(stream));
            if (report) std::memset(report, 0, sizeof(*report));
            if (report) report->converged = 1;
            return TOMOS_OK;
        }
        if (opts->staged_plane) return fail(TOMOS_ERR_INVALID, "lsqr_solve: staged_plane with mtx_refine_precision");
        DensePass pa(ws, A, ie, ie), pr(ws, Rf, re, re);
        RefinePass ops(pa, pr);
        PassPlan a = ops.plan(true), b2 = ops.plan(false);
        if (!a.fused || !b2.fused) {
            const size_t sa = dense_pass_scratch(A), sr = dense_pass_scratch(Rf);
            s = ensure_scratch(ws, sa > sr ? sa : sr);
            if (s) return s;
        }
        return solve_driver(ws, ops, b, x, opts, report, stream);
    }
    DensePass ops(ws, A, ie, ze);
    if (opts->staged_plane) {
        if (A->numeric != TOMOS_FP32_16 || A->layout != TOMOS_ROW_MAJOR)
            return fail(TOMOS_ERR_INVALID, "lsqr_solve: staged_plane needs a row-major FP32_16 A");
        if (reinterpret_cast<uintptr_t>(opts->staged_plane) % 16 != 0 || opts->staged_ld < A->cols ||
            opts->staged_ld % 8 != 0)
            return fail(TOMOS_ERR_INVALID,
                        "lsqr_solve: staged_plane must be 16-byte aligned with staged_ld a multiple "
                        "of 8 and >= cols");
        ops.given = opts->staged_plane;
        ops.given_ld = opts->staged_ld;
    }
    PassPlan a = ops.plan(true), b2 = ops.plan(false);
    if (!a.fused || !b2.fused) {
        s = ensure_scratch(ws, dense_pass_scratch(A));
        if (s) return s;
    }
    return solve_driver(ws, ops, b, x, opts, report, stream);
}

tomos_status tomos_backward_error_dense(const tomos_dense* A, const float* b, const float* x,
                                        const double* col_scale, tomos_workspace* ws,
                                        tomos_lsqr_report* report, void* stream) {
    std::string why;
    bool dot;
    int64_t outer, inner;
    if (!gemv_shape(A, TOMOS_NO_TRANSPOSE, &dot, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "backward_error: " + why);
    tomos_status s = workspace_check(ws, A->rows, A->cols);
    if (s) return s;
    if (!report) return fail(TOMOS_ERR_INVALID, "backward_error: null report");
    Elem ze;
    int32_t tier = (A->numeric == TOMOS_FP32) ? TOMOS_TIER_NATIVE : TOMOS_TIER_ACCURATE;
    if (!resolve_elem(A, tier, &ze, &why)) return fail(TOMOS_ERR_UNSUPPORTED, why);
    DensePass ops(ws, A, ze, ze);
    PassPlan pl = ops.plan(true);
    if (!pl.fused) {
        s = ensure_scratch(ws, dense_pass_scratch(A));
        if (s) return s;
    }
    cudaStream_t us = as_stream(stream), st = ws->stream;
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, us));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_fence, 0));
    const double coef_init[2] = {-1.0, 1.0};
    TOMOS_CUDA_TRY(cudaMemcpyAsync(ws->coef_init, coef_init, sizeof(coef_init),
                                   cudaMemcpyHostToDevice, st));
    s = ops.enqueue(pl, x, b, ws->coef_init, nullptr, st);
    if (s) return s;
    // beta = ||r|| and ||A^T r|| through N1 (no preconditioner, init mode).
    bool had = ws->has_precond;
    ws->has_precond = false;
    NSide S = make_nside(ws, pl, nullptr, true, nullptr, col_scale);
    ws->has_precond = had;
    nside_reduce_kernel<<<ws->nb1, 256, 0, st>>>(S);
    TOMOS_LAUNCH_CHECK("nside_reduce_kernel");
    sum_to_scalar_kernel<<<1, 256, 0, st>>>(ws->qnpart, ws->nb1, ws->scal + 4);
    sumsq_partial_kernel<<<ws->gs_max, 256, 0, st>>>(b, A->rows, nullptr, ws->bpart);
    sum_to_scalar_kernel<<<1, 256, 0, st>>>(ws->bpart, ws->gs_max, ws->scal + 2);
    scaled_sumsq_kernel<<<1, 256, 0, st>>>(x, col_scale, A->cols, ws->scal + 5);
    s = ops.fro2(ws->scal + 3, col_scale, st);
    if (s) return s;
    TOMOS_LAUNCH_CHECK("backward_error reductions");
    double h[6];
    TOMOS_CUDA_TRY(cudaMemcpyAsync(h, ws->scal, sizeof(h), cudaMemcpyDeviceToHost, st));
    TOMOS_CUDA_TRY(cudaStreamSynchronize(st));
    TOMOS_CUDA_TRY(cudaEventRecord(ws->ev_fence, st));
    TOMOS_CUDA_TRY(cudaStreamWaitEvent(us, ws->ev_fence, 0));
    LsqrDev L;
    std::memset(&L, 0, sizeof(L));
    L.beta = h[0];
    L.bnorm = std::sqrt(h[2]);
    L.anorm_fro = std::sqrt(h[3]);
    L.arnorm = std::sqrt(h[4]);
    L.xnorm = std::sqrt(h[5]);
    std::memset(report, 0, sizeof(*report));
    report->rnorm = L.beta;
    report->arnorm = L.arnorm;
    report->anorm_fro = L.anorm_fro;
    report->xnorm = L.xnorm;
    report->bnorm = L.bnorm;
    report->backward_error = eta_of(L);
    report->accurate_passes = 2;
    return TOMOS_OK;
}

}  // extern "C"
