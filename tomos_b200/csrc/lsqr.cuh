// lsqr.cuh -- internal interface of the LSQR driver (lsqr.cu): the device
// state of the recurrence, the workspace, and the "A pass" abstraction that
// lets dense and CSR storage share one driver.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace tomos_b200 {

// Device-resident LSQR state.  All scalars FP64.
struct LsqrDev {
    double alpha, beta, rho_bar, phi_bar;
    double rhsnorm;      // ||b|| (the reference's relres denominator)
    double beta_init;    // beta at the start of the current restart
    double xnorm;        // ||x|| after the last update
    double relres;       // |phi_bar| / ||b||
    double coef[2];      // [cp, cu] of the next A pass
    double arnorm;       // ||A^T r|| from the last restart pass
    double anorm_fro, bnorm;
    double tol, max_relres, inner_rtol;
    double inner_tol;    // BACKWARD rule: inner cycles end at eta1 <= this
    double* history;     // device, |phi_bar|/||b|| per iteration
    int iter;            // completed iterations, all restarts
    int iter_restart;    // completed iterations in this restart
    int max_iters;       // per restart
    int done;            // nonzero: kernels of an iteration return at once
    int converged;       // RELRES rule satisfied
    int breakdown;       // alpha or beta reached zero
    int stop_rule;
    int history_cap;
    int pipe_err;        // nonzero: a bounded pipeline wait expired in an A pass
    int pad_;
};

// How one pass over A is run.
// The BACKWARD tolerance from which the accurate passes sum FP32 runs.
constexpr double kRunsTolMin = 1e-6;

struct PassPlan {
    bool fused = false;
    Elem e = Elem::F32;
    bool acc64 = false;
    int grid = 0;    // fused CTAs
    int nch = 0;     // fused chunks per lane
    int g = 1;       // fused consumer warps per row
    int gq = 1;      // rows of A^T partials
    int gs = 1;      // ||ut||^2 partials
    int64_t qstride = 0;
    int tpw = 0;     // > 0: the tensor-core pass, k-tiles per consumer warp
    int src = 0;     // 1: the pass reads the refine copy of A (RefinePass)
    bool runs = false;  // FP64-summing fused pass: dots as FP32 runs (kRowBothRuns)
};

// One pass over A producing ut = cp*A p + cu*u_in in the workspace's u,
// ||ut||^2 partials (sspart, gs of them) and A^T ut partials (qpart, gq
// rows of stride qstride).
struct PassOps {
    virtual ~PassOps() = default;
    // accurate (init) passes may form their dots as FP32 runs (kRowBothRuns)
    bool runs = false;
    virtual PassPlan plan(bool init) = 0;
    virtual tomos_status enqueue(const PassPlan& pl, const float* p, const float* u_in,
                                 const double* coef, const int* skip, cudaStream_t st) = 0;
    // sum of squares of A's elements divided by d[column] (d may be NULL)
    virtual tomos_status fro2(double* out_dev, const double* d, cudaStream_t st) = 0;
    virtual uint64_t key() = 0;
    virtual int64_t rows() = 0;
    virtual int64_t cols() = 0;
    // Work done once per solve before the first pass (e.g. staging).
    virtual tomos_status prepare(cudaStream_t) { return TOMOS_OK; }
};

// Iterations over A, the initial and restart passes over a second copy of
// A at higher precision: the reference's mtx_refine_precision
// (--explicit-duplicates; lsqr.cpp:451-473 computes the restart residual
// u = b - A_refine x from it).  Here the whole restart pass, u and A^T u,
// streams the refine copy (one read of it instead of a read of each), and
// its ||A||_F feeds the backward-error rule.  Dense (lsqr.cu) and CSR
// (csr.cu) solves compose their passes with it.
struct RefinePass : PassOps {
    PassOps& it;
    PassOps& re;
    RefinePass(PassOps& a, PassOps& r) : it(a), re(r) {}
    PassPlan plan(bool init) override {
        re.runs = runs;
        it.runs = runs;
        PassPlan p = init ? re.plan(true) : it.plan(false);
        p.src = init ? 1 : 0;
        return p;
    }
    tomos_status enqueue(const PassPlan& pl, const float* p, const float* u_in, const double* coef,
                         const int* skip, cudaStream_t st) override {
        return pl.src ? re.enqueue(pl, p, u_in, coef, skip, st) : it.enqueue(pl, p, u_in, coef, skip, st);
    }
    tomos_status fro2(double* out, const double* d, cudaStream_t st) override { return re.fro2(out, d, st); }
    uint64_t key() override { return it.key() ^ (re.key() * 0x9E3779B97F4A7C15ull); }
    int64_t rows() override { return it.rows(); }
    int64_t cols() override { return it.cols(); }
    tomos_status prepare(cudaStream_t st) override {
        tomos_status s = it.prepare(st);
        return s ? s : re.prepare(st);
    }
};

// Block-wide sums (every thread gets the result), fixed order.
__device__ __forceinline__ double block_sum(double v, double* sm) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < nw ? sm[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) sm[0] = r;
    }
    __syncthreads();
    r = sm[0];
    __syncthreads();
    return r;
}

// Block-wide fixed-order sum of part[0..np).
__device__ __forceinline__ double block_sum_array(const double* part, int64_t np, double* sm) {
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < np; k += blockDim.x) s += part[k];
    return block_sum(s, sm);
}

// One pass over a dense A (the fused kernel when pl.fused, else the
// generic two-kernel path): ut = cp A p + cu u_in into ws->u, the
// partials of A^T ut into ws->qpart and of ||ut||^2 into ws->sspart.
PassPlan plan_dense_pass(tomos_workspace* ws, const tomos_dense* A, Elem e, bool acc64, bool runs = false);

// Options every solve entry accepts (stop rule, iteration counts).
bool opts_ok(const tomos_lsqr_opts* o, std::string* why);

// Row-sharded solves (comm.cu): fold a pass's partials into ws->shard and
// sum it across the communicator's ranks; sum any device doubles across them.
tomos_status enqueue_shard_reduce(tomos_workspace* ws, tomos_comm* c, const float* qpart, int gq,
                                  int64_t qstride, const double* sspart, int gs, const int* skip,
                                  cudaStream_t st);
tomos_status comm_allreduce(tomos_comm* c, double* buf, int64_t count, cudaStream_t st);
tomos_status enqueue_dense_pass(tomos_workspace* ws, const tomos_dense* A, const PassPlan& pl,
                                const float* p, const float* u_in, const double* coef,
                                const int* skip, cudaStream_t st);
size_t dense_pass_scratch(const tomos_dense* A);
// FP64 row- and column-major copies of the attached R^{-1} (Rrm, Rcm).
tomos_status refresh_precond(tomos_workspace* ws, cudaStream_t st);

tomos_status solve_driver(tomos_workspace* ws, PassOps& ops, const float* b, float* x,
                          const tomos_lsqr_opts* o, tomos_lsqr_report* rep, void* user_stream);
tomos_status workspace_check(tomos_workspace* ws, int64_t m, int64_t n);
tomos_status ensure_scratch(tomos_workspace* ws, size_t bytes);

}  // namespace tomos_b200

struct tomos_workspace {
    int64_t m = 0, n = 0;
    int32_t value_type = TOMOS_FP32, precond_type = TOMOS_FP32;
    int device = 0;
    int gmax = 0;          // max CTAs of the fused pass
    int64_t qstride = 0;   // row stride of the A^T partials
    int nb1 = 0, nb3 = 0;  // n-side block counts
    int gs_max = 0;        // sum-of-squares partial blocks

    float* u = nullptr;     // m: unnormalised u
    float* v = nullptr;     // n
    float* wt = nullptr;    // n: M w
    float* p = nullptr;     // n: M v, the right vector of the next pass
    float* qvec = nullptr;  // n
    double* t = nullptr;    // n: A^T u
    double* vhat = nullptr; // n
    float* qpart = nullptr;
    double* sspart = nullptr;
    double* vpart = nullptr;
    double* xpart = nullptr;
    double* qnpart = nullptr;
    double* scal = nullptr;
    double* coef_init = nullptr;
    double* bpart = nullptr;
    double* fro2 = nullptr;
    tomos_b200::LsqrDev* st = nullptr;
    double* Rcm = nullptr;  // FP64 copy of M, column-major
    double* Rrm = nullptr;  // FP64 copy of M, row-major
    double* hist = nullptr;
    int hist_cap = 0;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // fp16 copy of an FP32_16 wh plane for HALF-tier iterations (row-major,
    // ld a multiple of 8), allocated on the first solve that stages one.
    void* h16 = nullptr;
    size_t h16_bytes = 0;
    // adjoint solve (adjoint.cu): FP64 n-vectors and its device state,
    // allocated by the first adjoint call.
    void* adj = nullptr;
    // batched adjoint solves (adjoint_batch.cu): K columns of FP64 vectors,
    // the products' FP32 operands and split-K scratch, grown as needed.
    void* adjb = nullptr;
    size_t adjb_bytes = 0;
    // column-major copy of a CSR matrix for the CSR pass (csr.cu), rebuilt
    // by every CSR solve and grown as needed.
    void* csc = nullptr;
    size_t csc_bytes = 0;
    // row-sharded solves: the pass's partial sums folded to n + 1 doubles
    // (A^T u, ||u||^2), summed across ranks (comm.cu)
    double* shard = nullptr;
    // the solution the solve iterates on (copied from / to the caller's x),
    // so the iteration graph does not depend on the caller's buffer
    float* xg = nullptr;
    // the column scale of the backward-error rule (copied from the caller's)
    double* dscale = nullptr;
    tomos_comm* comm = nullptr;  // the running solve's communicator (or NULL)

    bool has_precond = false;
    tomos_dense precond{};

    tomos_b200::LsqrDev* st_host = nullptr;  // pinned mirror of *st
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_fence = nullptr;
    cudaEvent_t ev_pa = nullptr, ev_pb = nullptr;  // profiling: one pass over A

    cudaGraphExec_t graph = nullptr;
    int64_t launches = 0;        // kernels enqueued by the driver (graph replays included)
    int64_t graph_kernels = 0;   // kernels in one replay of `graph`'s iteration
    bool graph_loop = false;     // `graph` is a device-side while loop over the iteration
    std::vector<uint64_t> graph_key;
};
