// gemv.cuh -- internal interface of the strided GEMV (gemv.cu).
#pragma once

#include <string>

#include "common.cuh"

namespace tomos_b200 {

// One strided product in line form (see gemv.cu).  When `coef` is set,
// alpha/beta are read from coef[0], coef[1] on the device; when `skip`
// points at a nonzero int the kernels return at once.
struct GemvLaunch {
    bool dot = true;
    int64_t outer = 0, inner = 0, ld = 0;
    const void* hi = nullptr;
    const void* lo = nullptr;
    const float* x = nullptr;
    float* y = nullptr;
    double alpha = 1.0, beta = 0.0;
    const double* coef = nullptr;
    const int* skip = nullptr;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
};

int64_t line_sum_chunks(int64_t outer);
bool elem_is_exact(Elem e);

bool gemv_shape(const tomos_dense* A, int32_t trans, bool* dot, int64_t* outer, int64_t* inner,
                std::string* why);

// Scratch that covers any tier of this product (0 for line dots).
size_t gemv_scratch_bytes_max(const tomos_dense* A, int32_t trans);

tomos_status gemv_launch(const GemvLaunch& L, Elem e, bool acc64, cudaStream_t st);

// The product through the row pass (rowpass_gemv.cu) when A's lines fit
// it; *used false (nothing launched) otherwise.
tomos_status rowpass_gemv(const GemvLaunch& L, Elem e, cudaStream_t st, bool* used);
size_t rowpass_gemv_scratch_bytes(int64_t inner);

tomos_status gemv_dispatch(int32_t trans, double alpha, const tomos_dense* A, int32_t tier,
                           const float* x, double beta, float* y, void* scratch,
                           size_t scratch_bytes, cudaStream_t st);

}  // namespace tomos_b200
