// The CUDA GEMV launchers the reference's dispatch registries call, defined
// over this library's C ABI (tomos_gemv): the plug-in point for a build that
// keeps the reference's own src/dispatch.
//
// oracle/Makefile links this file with the reference's unmodified core and
// dispatch objects and with libtomos_b200 into _ref/libtomos_ref_b200.so.  A
// call of the reference's public mv_apply on Device::CUDA Dense objects then
// runs the reference's own registry lookup (dense_registries.cpp,
// fp32_16_registries.cpp) and reaches the sm_100a kernels through these
// definitions; every other CUDA launcher the reference references stays an
// aborting stub, so a lookup that went anywhere else would fail loudly.
// Test infrastructure: the product does not link or load it.
//
// Launchers defined here, with the reference registry slot that calls each:
//   cuda::mv_fp32_tiled                            FP32 A, FP32 compute
//       (dense_registries.cpp:326, mv_cuda_kernels.cuh:55)
//   cuda::mv_fp32_16_pure_half_no_transpose_flush256_swar
//   cuda::mv_fp32_16_pure_half_fast2_transpose_atomiconly_scaled_mblock_vec2_split
//   cuda::experimental::mv_fp32_16_pure_half_transpose_atomiconly_scaled_mblock_vec4_split_workspace_size
//                                                   FP32_16 A, FP16 compute
//       (fp32_16_registries.cpp:163, :256, :192; the HALF tier here)
//   cuda::experimental::mv_fp32_16_accurate_fast   FP32_16 A, FP32 compute
//       (fp32_16_registries.cpp:364; the ACCURATE tier here)
#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <mutex>
#include <stdexcept>
#include <string>

#include "blas.hpp"
#include "context.hpp"
#include "fp32_16_cuda_kernels.cuh"
#include "matrix.hpp"
#include "mv_cuda_kernels.cuh"
#include "tomos_b200.h"

using namespace tomos;

namespace {

// Scratch of the products that sum lines, grown and kept per process (the
// reference's own launchers keep a persistent buffer the same way).
void* gemv_scratch(size_t bytes) {
    static std::mutex mu;
    static void* buf = nullptr;
    static size_t cap = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (bytes > cap) {
        if (buf) cudaFree(buf);
        buf = nullptr;
        cap = 0;
        if (cudaMalloc(&buf, bytes) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("ref_launchers: cudaMalloc of the GEMV scratch failed");
        }
        cap = bytes;
    }
    return buf;
}

// y = alpha op(A) x + beta y for the reference's column-major A (wr may be
// NULL: the planar default after the wh plane).
void gemv(TransposeType trans, double alpha, int32_t numeric, int32_t tier, dim<2> size, const void* wh,
          const void* wr, size_t ld, const float* x, double beta, float* y, float* ws, size_t ws_floats) {
    tomos_dense d{numeric, TOMOS_COL_MAJOR, (int64_t)size[0], (int64_t)size[1], (int64_t)ld,
                  const_cast<void*>(wh), const_cast<void*>(wr), 0, 0};
    const int32_t t = trans == TransposeType::TRANSPOSE ? TOMOS_TRANSPOSE : TOMOS_NO_TRANSPOSE;
    const size_t need = tomos_gemv_scratch_bytes(&d, t);
    void* scratch = nullptr;
    if (need > 0) scratch = (ws && ws_floats * sizeof(float) >= need) ? (void*)ws : gemv_scratch(need);
    if (tomos_gemv(t, alpha, &d, tier, x, beta, y, scratch, need, nullptr) != TOMOS_OK)
        throw std::runtime_error(std::string("tomos_gemv: ") + tomos_last_error());
}

}  // namespace

namespace tomos {
namespace cuda {

void mv_fp32_tiled(TransposeType trans, double alpha, dim<2> size, const float* A, size_t ld_a,
                   const float* x, size_t, double beta, float* y, size_t) {
    gemv(trans, alpha, TOMOS_FP32, TOMOS_TIER_NATIVE, size, A, nullptr, ld_a, x, beta, y, nullptr, 0);
}

void mv_fp32_16_pure_half_no_transpose_flush256_swar(double alpha, dim<2> size, const uint16_t* wh,
                                                     size_t ld_a, const float* x, size_t, double beta,
                                                     float* y, size_t) {
    gemv(TransposeType::NO_TRANSPOSE, alpha, TOMOS_FP32_16, TOMOS_TIER_HALF, size, wh, nullptr, ld_a, x,
         beta, y, nullptr, 0);
}

void mv_fp32_16_pure_half_fast2_transpose_atomiconly_scaled_mblock_vec2_split(
    TransposeType trans, double alpha, dim<2> size, const uint16_t* wh, size_t ld_a, const float* x, size_t,
    double beta, float* y, size_t, float* workspace) {
    tomos_dense d{TOMOS_FP32_16, TOMOS_COL_MAJOR, (int64_t)size[0], (int64_t)size[1], (int64_t)ld_a,
                  const_cast<uint16_t*>(wh), nullptr, 0, 0};
    const size_t floats = (tomos_gemv_scratch_bytes(&d, TOMOS_TRANSPOSE) + 3) / 4;
    gemv(trans, alpha, TOMOS_FP32_16, TOMOS_TIER_HALF, size, wh, nullptr, ld_a, x, beta, y, workspace, floats);
}

namespace experimental {

// The registry sizes its persistent transpose workspace with this.
size_t mv_fp32_16_pure_half_transpose_atomiconly_scaled_mblock_vec4_split_workspace_size(dim<2> size) {
    tomos_dense d{TOMOS_FP32_16, TOMOS_COL_MAJOR, (int64_t)size[0], (int64_t)size[1], (int64_t)size[0],
                  nullptr, nullptr, 0, 0};
    const size_t bytes = tomos_gemv_scratch_bytes(&d, TOMOS_TRANSPOSE);
    return (bytes + 3) / 4 > 0 ? (bytes + 3) / 4 : 1;
}

void mv_fp32_16_accurate_fast(TransposeType trans, double alpha, dim<2> size, const uint16_t* wh,
                              const uint16_t* wr, size_t ld_a, const float* x, size_t, double beta, float* y,
                              size_t) {
    gemv(trans, alpha, TOMOS_FP32_16, TOMOS_TIER_ACCURATE, size, wh, wr, ld_a, x, beta, y, nullptr, 0);
}

}  // namespace experimental
}  // namespace cuda
}  // namespace tomos

extern "C" {

// The reference's mv_apply (blas.cpp:23-32, explicit compute type) on
// Device::CUDA Dense objects wrapping device buffers: A column-major m x n
// (numeric: the reference's NumericType value; FP32_16 as its planar
// [wh | wr] layout), x and y FP32 column vectors.  Returns 0, or -1 if the
// reference threw (the message to stderr).
int ref_b200_mv(int trans, double alpha, int numeric, int compute, size_t m, size_t n, void* A_dev,
                size_t ld, float* x_dev, double beta, float* y_dev) {
    try {
        Context ctx(Device::CUDA);
        Dense A = Dense::wrap_strided(ctx, Layout::COL_MAJOR, (NumericType)numeric, {m, n}, ld, A_dev);
        const size_t lx = trans ? m : n, ly = trans ? n : m;
        Dense X = Dense::wrap_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {lx, 1}, lx, x_dev);
        Dense Y = Dense::wrap_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {ly, 1}, ly, y_dev);
        mv_apply(Device::CUDA, trans ? TransposeType::TRANSPOSE : TransposeType::NO_TRANSPOSE, alpha, A, X,
                 beta, Y, (NumericType)compute, nullptr);
        if (cudaDeviceSynchronize() != cudaSuccess) return -1;
        return 0;
    } catch (const std::exception& e) {
        fprintf(stderr, "ref_b200_mv: %s\n", e.what());
        return -1;
    }
}

}  // extern "C"
