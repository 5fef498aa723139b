// gemv.cu -- strided GEMV y = alpha * op(A) x + beta * y for every storage
// type, layout and leading dimension (tomos_gemv), and the same kernels
// with device-resident alpha/beta for the solver's unfused path.
//
// A strided matrix is `outer` lines of `inner` contiguous elements.  An
// op(A) product is then one of two shapes:
//   line dots  (row-major NO_TRANSPOSE, col-major TRANSPOSE):
//       y[o] = sum_i A[o, i] x[i]      -- one warp per line
//   line sums  (row-major TRANSPOSE, col-major NO_TRANSPOSE):
//       y[i] = sum_o A[o, i] x[o]      -- threads own i; blocks own a
//                                         chunk of lines and write partials
//                                         that a second kernel reduces in
//                                         a fixed order (deterministic, no
//                                         atomics; the reference uses
//                                         atomicAdd, mv_cuda_kernels.cu:529)
// HALF-tier and FP32 products accumulate in FP32, ACCURATE-tier in FP64.
// The LSQR iteration uses the fused row-major pass in fused.cuh instead;
// these kernels serve tomos_gemv and the shapes that pass does not cover.
#include <mutex>
#include <string>

#include "common.cuh"
#include "gemv.cuh"

namespace tomos_b200 {

template <bool ACC64>
struct AccT {
    using T = float;
};
template <>
struct AccT<true> {
    using T = double;
};

__device__ __forceinline__ void resolve_coef(const double* coef, double& alpha, double& beta) {
    if (coef) {
        alpha = coef[0];
        beta = coef[1];
    }
}

template <Elem E, bool ACC64>
__global__ void __launch_bounds__(256) line_dot_kernel(const void* __restrict__ hi,
                                                       const void* __restrict__ lo,
                                                       int64_t outer, int64_t inner, int64_t ld,
                                                       const float* __restrict__ x, double alpha,
                                                       double beta, const double* coef,
                                                       const int* skip, float* __restrict__ y) {
    if (skip && *skip) return;
    using Acc = typename AccT<ACC64>::T;
    resolve_coef(coef, alpha, beta);
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t o = warp; o < outer; o += nwarps) {
        const size_t base = (size_t)o * (size_t)ld;
        Acc a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        int64_t i = lane;
        for (; i + 96 < inner; i += 128) {
            a0 += (Acc)load_elem<E>(hi, lo, base + i) * (Acc)__ldg(x + i);
            a1 += (Acc)load_elem<E>(hi, lo, base + i + 32) * (Acc)__ldg(x + i + 32);
            a2 += (Acc)load_elem<E>(hi, lo, base + i + 64) * (Acc)__ldg(x + i + 64);
            a3 += (Acc)load_elem<E>(hi, lo, base + i + 96) * (Acc)__ldg(x + i + 96);
        }
        for (; i < inner; i += 32) a0 += (Acc)load_elem<E>(hi, lo, base + i) * (Acc)__ldg(x + i);
        Acc acc = warp_sum((a0 + a1) + (a2 + a3));
        if (lane == 0) {
            double r = alpha * (double)acc;
            if (beta != 0.0) r += beta * (double)y[o];
            y[o] = (float)r;
        }
    }
}

template <Elem E, bool ACC64>
__global__ void __launch_bounds__(256) line_sum_partial_kernel(
    const void* __restrict__ hi, const void* __restrict__ lo, int64_t outer, int64_t inner,
    int64_t ld, const float* __restrict__ x, int64_t lines_per_chunk, const int* skip,
    typename AccT<ACC64>::T* __restrict__ partial) {
    if (skip && *skip) return;
    using Acc = typename AccT<ACC64>::T;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (i >= inner) return;
    int64_t o0 = c * lines_per_chunk;
    int64_t o1 = o0 + lines_per_chunk;
    if (o1 > outer) o1 = outer;
    Acc a0 = 0, a1 = 0;
    int64_t o = o0;
    for (; o + 1 < o1; o += 2) {
        a0 += (Acc)load_elem<E>(hi, lo, (size_t)o * ld + i) * (Acc)__ldg(x + o);
        a1 += (Acc)load_elem<E>(hi, lo, (size_t)(o + 1) * ld + i) * (Acc)__ldg(x + o + 1);
    }
    if (o < o1) a0 += (Acc)load_elem<E>(hi, lo, (size_t)o * ld + i) * (Acc)__ldg(x + o);
    partial[(size_t)c * inner + i] = a0 + a1;
}

template <typename Acc>
__global__ void line_sum_reduce_kernel(const Acc* __restrict__ partial, int64_t nchunks,
                                       int64_t inner, double alpha, double beta,
                                       const double* coef, const int* skip,
                                       float* __restrict__ y) {
    if (skip && *skip) return;
    resolve_coef(coef, alpha, beta);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= inner) return;
    double acc = 0.0;
    for (int64_t c = 0; c < nchunks; ++c) acc += (double)partial[(size_t)c * inner + i];
    double r = alpha * acc;
    if (beta != 0.0) r += beta * (double)y[i];
    y[i] = (float)r;
}

int64_t line_sum_chunks(int64_t outer) {
    int64_t c = (outer + 127) / 128;
    if (c > 1184) c = 1184;
    return c < 1 ? 1 : c;
}

template <Elem E, bool ACC64>
static tomos_status run_gemv(const GemvLaunch& L, cudaStream_t st) {
    using Acc = typename AccT<ACC64>::T;
    if (L.dot) {
        int64_t blocks = (L.outer + 7) / 8;
        int64_t cap = (int64_t)sm_count() * 8;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        line_dot_kernel<E, ACC64><<<(unsigned)blocks, 256, 0, st>>>(
            L.hi, L.lo, L.outer, L.inner, L.ld, L.x, L.alpha, L.beta, L.coef, L.skip, L.y);
        TOMOS_LAUNCH_CHECK("line_dot_kernel");
        return TOMOS_OK;
    }
    int64_t nchunks = line_sum_chunks(L.outer);
    size_t need = (size_t)nchunks * (size_t)L.inner * sizeof(Acc);
    if (L.scratch_bytes < need || !L.scratch)
        return fail(TOMOS_ERR_INVALID,
                    "tomos_gemv: scratch too small (need " + std::to_string(need) + " bytes)");
    int64_t lpc = (L.outer + nchunks - 1) / nchunks;
    dim3 grid((unsigned)((L.inner + 255) / 256), (unsigned)nchunks);
    Acc* partial = static_cast<Acc*>(L.scratch);
    line_sum_partial_kernel<E, ACC64><<<grid, 256, 0, st>>>(L.hi, L.lo, L.outer, L.inner, L.ld,
                                                            L.x, lpc, L.skip, partial);
    TOMOS_LAUNCH_CHECK("line_sum_partial_kernel");
    line_sum_reduce_kernel<Acc><<<(unsigned)((L.inner + 255) / 256), 256, 0, st>>>(
        partial, nchunks, L.inner, L.alpha, L.beta, L.coef, L.skip, L.y);
    TOMOS_LAUNCH_CHECK("line_sum_reduce_kernel");
    return TOMOS_OK;
}

template <Elem E>
static tomos_status run_gemv_acc(const GemvLaunch& L, bool acc64, cudaStream_t st) {
    return acc64 ? run_gemv<E, true>(L, st) : run_gemv<E, false>(L, st);
}

tomos_status gemv_launch(const GemvLaunch& L, Elem e, bool acc64, cudaStream_t st) {
    switch (e) {
        case Elem::F32: return run_gemv_acc<Elem::F32>(L, acc64, st);
        case Elem::H16: return run_gemv_acc<Elem::H16>(L, acc64, st);
        case Elem::F16: return run_gemv_acc<Elem::F16>(L, acc64, st);
        case Elem::A16: return run_gemv<Elem::A16, true>(L, st);
        case Elem::B16: return run_gemv_acc<Elem::B16>(L, acc64, st);
        case Elem::AB16: return run_gemv<Elem::AB16, true>(L, st);
        case Elem::AB16R: return run_gemv<Elem::AB16R, true>(L, st);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "gemv: unsupported element type");
    }
}

bool elem_is_exact(Elem e) { return e == Elem::A16 || e == Elem::AB16 || e == Elem::AB16R; }

__global__ void scale_vec_kernel(float* y, int64_t n, double beta) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = beta != 0.0 ? (float)(beta * (double)y[i]) : 0.0f;
}

bool gemv_shape(const tomos_dense* A, int32_t trans, bool* dot, int64_t* outer, int64_t* inner,
                std::string* why) {
    if (!A) {
        *why = "null matrix";
        return false;
    }
    if (A->layout != TOMOS_ROW_MAJOR && A->layout != TOMOS_COL_MAJOR) {
        *why = "bad layout";
        return false;
    }
    if (trans != TOMOS_NO_TRANSPOSE && trans != TOMOS_TRANSPOSE) {
        *why = "bad transpose flag";
        return false;
    }
    if (A->rows < 0 || A->cols < 0) {
        *why = "negative dimension";
        return false;
    }
    bool row = A->layout == TOMOS_ROW_MAJOR;
    *outer = row ? A->rows : A->cols;
    *inner = row ? A->cols : A->rows;
    if (A->ld < *inner || A->ld < 1) {
        *why = "leading dimension smaller than the contiguous extent";
        return false;
    }
    *dot = (row == (trans == TOMOS_NO_TRANSPOSE));
    return true;
}

size_t gemv_scratch_bytes_max(const tomos_dense* A, int32_t trans) {
    bool dot;
    int64_t outer, inner;
    std::string why;
    if (!gemv_shape(A, trans, &dot, &outer, &inner, &why) || dot) return 0;
    const size_t generic = (size_t)line_sum_chunks(outer) * (size_t)inner * 8;
    const size_t rowpass = rowpass_gemv_scratch_bytes(inner);
    return generic > rowpass ? generic : rowpass;
}

tomos_status gemv_dispatch(int32_t trans, double alpha, const tomos_dense* A, int32_t tier,
                           const float* x, double beta, float* y, void* scratch,
                           size_t scratch_bytes, cudaStream_t st) {
    GemvLaunch L;
    std::string why;
    if (!gemv_shape(A, trans, &L.dot, &L.outer, &L.inner, &why))
        return fail(TOMOS_ERR_INVALID, "tomos_gemv: " + why);
    Elem e;
    if (!resolve_elem(A, tier, &e, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "tomos_gemv: " + why);
    int64_t ylen = (trans == TOMOS_NO_TRANSPOSE) ? A->rows : A->cols;
    if (ylen == 0) return TOMOS_OK;
    if (!y) return fail(TOMOS_ERR_INVALID, "tomos_gemv: null y");
    int64_t xlen = (trans == TOMOS_NO_TRANSPOSE) ? A->cols : A->rows;
    if (xlen == 0) {
        scale_vec_kernel<<<(unsigned)((ylen + 255) / 256), 256, 0, st>>>(y, ylen, beta);
        TOMOS_LAUNCH_CHECK("scale_vec_kernel");
        return TOMOS_OK;
    }
    if (!x || !A->values) return fail(TOMOS_ERR_INVALID, "tomos_gemv: null pointer");
    L.hi = A->values;
    L.lo = elem_is_exact(e) ? dense_lo_plane(A) : nullptr;
    L.ld = A->ld;
    L.x = x;
    L.y = y;
    L.alpha = alpha;
    L.beta = beta;
    L.scratch = scratch;
    L.scratch_bytes = scratch_bytes;
    bool used = false;
    tomos_status rs = rowpass_gemv(L, e, st, &used);
    if (used) return rs;
    return gemv_launch(L, e, elem_is_exact(e), st);
}

// Fixed scratch for tomos_gemv_no_alloc: the per-chunk partials of a
// line-sum product live in this module-scope buffer instead of caller
// memory.  The line-sum kernel writes every partial it later reduces, so
// nothing in it has to start at zero.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_gemv_static_scratch[kNoAllocScratchBytes / sizeof(double)];

// Device address of g_gemv_static_scratch on the current device, looked up
// on the first call made with that device current and cached afterwards.
static tomos_status no_alloc_scratch(void** out) {
    static std::mutex mu;
    static void* addr[kNoAllocMaxDevices] = {};
    int dev = 0;
    TOMOS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(TOMOS_ERR_UNSUPPORTED, "tomos_gemv_no_alloc: device ordinal " +
                                               std::to_string(dev) + " out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_gemv_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(gemv static scratch)");
        addr[dev] = p;
    }
    *out = addr[dev];
    return TOMOS_OK;
}

tomos_status gemv_no_alloc(int32_t trans, double alpha, const tomos_dense* A, int32_t tier,
                           const float* x, double beta, float* y, cudaStream_t st) {
    const size_t need = gemv_scratch_bytes_max(A, trans);
    if (need > kNoAllocScratchBytes)
        return fail(TOMOS_ERR_INVALID,
                    "tomos_gemv_no_alloc: this product needs " + std::to_string(need) +
                        " bytes of scratch; the fixed buffer holds " +
                        std::to_string(kNoAllocScratchBytes) + " (use tomos_gemv)");
    void* scratch = nullptr;
    tomos_status s = no_alloc_scratch(&scratch);
    if (s) return s;
    return gemv_dispatch(trans, alpha, A, tier, x, beta, y, scratch, kNoAllocScratchBytes, st);
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

tomos_status tomos_gemv_no_alloc(int32_t trans, double alpha, const tomos_dense* A, int32_t tier,
                                 const float* x, double beta, float* y, void* stream) {
    return gemv_no_alloc(trans, alpha, A, tier, x, beta, y, as_stream(stream));
}

size_t tomos_gemv_scratch_bytes(const tomos_dense* A, int32_t trans) {
    // Sized for the widest (FP64-accumulating) tier so one buffer serves all.
    return gemv_scratch_bytes_max(A, trans);
}

tomos_status tomos_gemv(int32_t trans, double alpha, const tomos_dense* A, int32_t tier,
                        const float* x, double beta, float* y, void* scratch,
                        size_t scratch_bytes, void* stream) {
    return gemv_dispatch(trans, alpha, A, tier, x, beta, y, scratch, scratch_bytes,
                         as_stream(stream));
}

}  // extern "C"
