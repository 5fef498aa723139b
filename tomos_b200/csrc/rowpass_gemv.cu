// rowpass_gemv.cu -- tomos_gemv through the row pass (rowpass.cuh).
//
// A strided product y = alpha op(A) x + beta y is, over the lines of A
// (rows of a row-major A, columns of a column-major one), either a dot per
// line or a sum of scaled lines (gemv.cu).  When the lines are 16-byte
// aligned and short enough for the consumer warps, both shapes stream every
// line through shared memory once with bulk asynchronous copies, as the
// LSQR pass does, and decode the storage in registers:
//   dot per line      kRowDot:  y_o = alpha (A_o . x) + beta y_o, one
//                     warp (or G warps) per line, written in place;
//   sum of lines      kRowAxpy: per-CTA partials of sum_o x_o A_o, then
//                     rowpass_reduce_kernel sums the partials of every
//                     column in CTA order (deterministic, no atomics; the
//                     reference adds with atomicAdd, mv_cuda_kernels.cu:529)
//                     into y = alpha sum + beta y.
// FP32 and HALF-tier products accumulate in FP32.  The exact tiers form
// FP32 products over short runs (a lane's part of a line, or 8 lines of a
// column) and sum the runs in FP64.  Other shapes take the generic
// kernels of gemv.cu.
#include <mutex>
#include <string>

#include "common.cuh"
#include "gemv.cuh"
#include "rowpass_launch.cuh"

namespace tomos_b200 {

namespace {

// y[j] = alpha * sum_c part[c][j] + beta * y[j], the partials in CTA order.
template <typename Acc>
__global__ void __launch_bounds__(256) rowpass_reduce_kernel(const Acc* __restrict__ part, int nparts,
                                                             int64_t stride, int64_t n, double alpha,
                                                             double beta, float* __restrict__ y) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int c = 0; c < nparts; ++c) s += (double)part[(size_t)c * stride + j];
    double r = alpha * s;
    if (beta != 0.0) r += beta * (double)y[j];
    y[j] = (float)r;
}

// The word a bounded pipeline wait of these launches records its expiry
// in (one per device; nothing reads it back: an expired wait leaves the
// product's y undefined, which the bounded waits make the only effect of
// a stalled copy).
__device__ int g_rowpass_gemv_err;
constexpr int kMaxDevices = 64;

int* err_word() {
    static std::mutex mu;
    static int* addr[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_rowpass_gemv_err) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        addr[dev] = static_cast<int*>(p);
    }
    return addr[dev];
}

template <int MODE>
tomos_status launch_mode(Elem e, bool acc64, const FusedParams& P, int* err, int nch, int g, int grid,
                         cudaStream_t st, double* qpart64) {
    switch (e) {
        case Elem::F32: return launch_fused_e<Elem::F32, false, MODE>(P, err, nch, g, grid, st, qpart64);
        case Elem::H16: return launch_fused_e<Elem::H16, false, MODE>(P, err, nch, g, grid, st, qpart64);
        case Elem::F16: return launch_fused_e<Elem::F16, false, MODE>(P, err, nch, g, grid, st, qpart64);
        case Elem::B16: return launch_fused_e<Elem::B16, false, MODE>(P, err, nch, g, grid, st, qpart64);
        case Elem::A16: return launch_fused_e<Elem::A16, true, MODE>(P, err, nch, g, grid, st, qpart64);
        case Elem::AB16: return launch_fused_e<Elem::AB16, true, MODE>(P, err, nch, g, grid, st, qpart64);
        case Elem::AB16R: return launch_fused_e<Elem::AB16R, true, MODE>(P, err, nch, g, grid, st, qpart64);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "gemv row pass: element type");
    }
}

}  // namespace

size_t rowpass_gemv_scratch_bytes(int64_t inner) {
    const int64_t qs = (inner + 31) / 32 * 32;
    return (size_t)sm_count() * (size_t)qs * sizeof(double);
}

tomos_status rowpass_gemv(const GemvLaunch& L, Elem e, cudaStream_t st, bool* used) {
    *used = false;
    const bool acc64 = elem_is_exact(e);
    if (e == Elem::F64 || L.coef || L.skip) return TOMOS_OK;
    int nch = 0, g = 1;
    if (!plan_row_lines(e, acc64, L.dot ? kRowDot : kRowAxpy, L.inner, L.ld, L.hi, L.lo, &nch, &g)) return TOMOS_OK;
    const int grid = row_pass_grid(L.outer);
    const int64_t qs = (L.inner + 31) / 32 * 32;
    if (!L.dot && (!L.scratch || L.scratch_bytes < (size_t)grid * qs * (acc64 ? 8 : 4))) return TOMOS_OK;
    int* err = err_word();
    if (!err) return TOMOS_OK;
    *used = true;
    FusedParams P;
    P.hi = L.hi;
    P.lo = L.lo;
    P.m = L.outer;
    P.n = L.inner;
    P.ld = L.ld;
    P.coef = nullptr;
    P.sspart = nullptr;
    P.skip = nullptr;
    P.qstride = qs;
    if (L.dot) {
        // y_o = alpha (A_o . x) + beta y_o, in place (y is not read when beta == 0)
        P.p = L.x;
        P.u_in = L.y;
        P.u_out = L.y;
        P.qpart = nullptr;
        P.cp = L.alpha;
        P.cu = L.beta;
        return launch_mode<kRowDot>(e, acc64, P, err, nch, g, grid, st, nullptr);
    }
    // partials of sum_o x_o A_o, then y = alpha sum + beta y
    P.p = nullptr;
    P.u_in = L.x;
    P.u_out = nullptr;
    P.cp = 0.0;
    P.cu = 1.0;
    P.qpart = acc64 ? nullptr : static_cast<float*>(L.scratch);
    double* q64 = acc64 ? static_cast<double*>(L.scratch) : nullptr;
    tomos_status s = launch_mode<kRowAxpy>(e, acc64, P, err, nch, g, grid, st, q64);
    if (s) return s;
    const unsigned rb = (unsigned)((L.inner + 255) / 256);
    if (acc64)
        rowpass_reduce_kernel<double><<<rb, 256, 0, st>>>(q64, grid, qs, L.inner, L.alpha, L.beta, L.y);
    else
        rowpass_reduce_kernel<float><<<rb, 256, 0, st>>>(P.qpart, grid, qs, L.inner, L.alpha, L.beta, L.y);
    TOMOS_LAUNCH_CHECK("rowpass_reduce_kernel");
    return TOMOS_OK;
}

}  // namespace tomos_b200
