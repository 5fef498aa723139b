// runtime.cu -- C-ABI plumbing (errors, device info, tier resolution) and
// the pack/unpack kernels for the FP32_16 and FP32_BF16 formats.
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace tomos_b200 {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

tomos_status fail(tomos_status code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

tomos_status cuda_fail(cudaError_t err, const char* what) {
    g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(err);
    return TOMOS_ERR_CUDA;
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 1;
    }
    return cache[dev];
}

const void* dense_lo_plane(const tomos_dense* A) {
    if (A->values_lo) return A->values_lo;
    int64_t outer = (A->layout == TOMOS_COL_MAJOR) ? A->cols : A->rows;
    return static_cast<const uint16_t*>(A->values) + (size_t)A->ld * (size_t)outer;
}

static bool resolve_numeric(int32_t numeric, int32_t rounded, int32_t tier, Elem* out,
                            std::string* why) {
    switch (numeric) {
        case TOMOS_FP32:
            if (tier == TOMOS_TIER_AUTO || tier == TOMOS_TIER_NATIVE) {
                *out = Elem::F32;
                return true;
            }
            break;
        case TOMOS_FP16:
            // native IEEE fp16 storage (the reference's plain __half Dense,
            // --explicit-duplicates): products in FP32
            if (tier == TOMOS_TIER_AUTO || tier == TOMOS_TIER_NATIVE || tier == TOMOS_TIER_HALF) {
                *out = Elem::F16;
                return true;
            }
            break;
        case TOMOS_FP32_16:
            if (tier == TOMOS_TIER_AUTO || tier == TOMOS_TIER_HALF) {
                *out = Elem::H16;
                return true;
            }
            if (tier == TOMOS_TIER_ACCURATE) {
                *out = Elem::A16;
                return true;
            }
            break;
        case TOMOS_FP32_BF16:
            if (tier == TOMOS_TIER_AUTO || tier == TOMOS_TIER_HALF) {
                *out = Elem::B16;
                return true;
            }
            if (tier == TOMOS_TIER_ACCURATE) {
                *out = rounded ? Elem::AB16R : Elem::AB16;
                return true;
            }
            break;
        default:
            break;
    }
    *why = "no kernel registered for storage type " + std::to_string(numeric) +
           " with compute tier " + std::to_string(tier);
    return false;
}

bool resolve_elem(const tomos_dense* A, int32_t tier, Elem* out, std::string* why) {
    return resolve_numeric(A->numeric, A->rounded, tier, out, why);
}
bool resolve_elem_csr(const tomos_csr* A, int32_t tier, Elem* out, std::string* why) {
    return resolve_numeric(A->numeric, A->rounded, tier, out, why);
}

// ------------------------------------------------------------------ pack
//
// A strided matrix is `outer` lines of `inner` contiguous elements
// (col-major: lines are columns; row-major: rows).  One block walks a line
// at a time; threads stride the line, so loads and stores are coalesced
// for every layout and leading dimension.

__global__ void pack16_kernel(const float* __restrict__ src, int64_t outer, int64_t inner,
                              int64_t ld_src, uint16_t* __restrict__ wh,
                              uint16_t* __restrict__ wr, int64_t ld_dst,
                              unsigned long long* __restrict__ counts) {
    unsigned long long c[4] = {0, 0, 0, 0};
    for (int64_t o = blockIdx.x; o < outer; o += gridDim.x) {
        const float* s = src + (size_t)o * ld_src;
        uint16_t* h = wh + (size_t)o * ld_dst;
        uint16_t* r = wr + (size_t)o * ld_dst;
        for (int64_t i = threadIdx.x; i < inner; i += blockDim.x) {
            uint16_t a, b;
            int cls;
            encode_fp32_16(s[i], a, b, cls);
            h[i] = a;
            r[i] = b;
            c[cls] += 1;
        }
    }
    if (counts) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            unsigned long long v = c[k];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if ((threadIdx.x & 31) == 0 && v) atomicAdd(&counts[k], v);
        }
    }
}

__global__ void unpack16_kernel(const uint16_t* __restrict__ wh, const uint16_t* __restrict__ wr,
                                int64_t outer, int64_t inner, int64_t ld_src,
                                float* __restrict__ dst, int64_t ld_dst) {
    for (int64_t o = blockIdx.x; o < outer; o += gridDim.x) {
        const uint16_t* h = wh + (size_t)o * ld_src;
        const uint16_t* r = wr + (size_t)o * ld_src;
        float* d = dst + (size_t)o * ld_dst;
        for (int64_t i = threadIdx.x; i < inner; i += blockDim.x)
            d[i] = decode_fp32_16_exact(h[i], r[i]);
    }
}

__global__ void packbf16_kernel(const float* __restrict__ src, int64_t outer, int64_t inner,
                                int64_t ld_src, uint16_t* __restrict__ wh,
                                uint16_t* __restrict__ wr, int64_t ld_dst, int rounded) {
    for (int64_t o = blockIdx.x; o < outer; o += gridDim.x) {
        const float* s = src + (size_t)o * ld_src;
        uint16_t* h = wh + (size_t)o * ld_dst;
        uint16_t* r = wr + (size_t)o * ld_dst;
        for (int64_t i = threadIdx.x; i < inner; i += blockDim.x) {
            uint16_t a, b;
            encode_fp32_bf16(s[i], a, b, rounded != 0);
            h[i] = a;
            r[i] = b;
        }
    }
}

__global__ void unpackbf16_kernel(const uint16_t* __restrict__ wh, const uint16_t* __restrict__ wr,
                                  int64_t outer, int64_t inner, int64_t ld_src,
                                  float* __restrict__ dst, int64_t ld_dst, int rounded) {
    for (int64_t o = blockIdx.x; o < outer; o += gridDim.x) {
        const uint16_t* h = wh + (size_t)o * ld_src;
        const uint16_t* r = wr + (size_t)o * ld_src;
        float* d = dst + (size_t)o * ld_dst;
        for (int64_t i = threadIdx.x; i < inner; i += blockDim.x)
            d[i] = decode_fp32_bf16_exact(h[i], r[i], rounded != 0);
    }
}

static bool shape_ok(int32_t layout, int64_t rows, int64_t cols, int64_t ld_a, int64_t ld_b,
                     int64_t* outer, int64_t* inner, std::string* why) {
    if (layout != TOMOS_ROW_MAJOR && layout != TOMOS_COL_MAJOR) {
        *why = "layout must be ROW_MAJOR or COL_MAJOR";
        return false;
    }
    if (rows < 0 || cols < 0) {
        *why = "negative dimension";
        return false;
    }
    *outer = layout == TOMOS_COL_MAJOR ? cols : rows;
    *inner = layout == TOMOS_COL_MAJOR ? rows : cols;
    if (ld_a < *inner || ld_b < *inner) {
        *why = "leading dimension smaller than the contiguous extent";
        return false;
    }
    return true;
}

// FP32 -> IEEE fp16, round to nearest even (overflow to Inf, fp16
// subnormals kept): the reference's __half(value) when it fills a native
// FP16 Dense (fill_dense_from_host<__half>).
__global__ void packhalf_kernel(const float* __restrict__ src, int64_t outer, int64_t inner, int64_t ld_src,
                                uint16_t* __restrict__ dst, int64_t ld_dst) {
    for (int64_t o = blockIdx.x; o < outer; o += gridDim.x) {
        const float* s = src + (size_t)o * ld_src;
        uint16_t* d = dst + (size_t)o * ld_dst;
        for (int64_t i = threadIdx.x; i < inner; i += blockDim.x) d[i] = __half_as_ushort(__float2half_rn(s[i]));
    }
}

static int pack_grid(int64_t outer) {
    int64_t g = (int64_t)sm_count() * 16;
    if (outer < g) g = outer;
    return (int)(g > 0 ? g : 1);
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

const char* tomos_last_error(void) { return g_last_error.c_str(); }

const char* tomos_version(void) { return "tomos_b200 0.1 (sm_100a)"; }

tomos_status tomos_sync(void* stream) {
    TOMOS_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    return TOMOS_OK;
}

tomos_status tomos_pack_fp32_16(const float* src, int32_t layout, int64_t rows, int64_t cols,
                                int64_t ld_src, uint16_t* wh, uint16_t* wr, int64_t ld_dst,
                                unsigned long long* counts, void* stream) {
    int64_t outer, inner;
    std::string why;
    if (!shape_ok(layout, rows, cols, ld_src, ld_dst, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "tomos_pack_fp32_16: " + why);
    if (outer == 0 || inner == 0) return TOMOS_OK;
    if (!src || !wh || !wr) return fail(TOMOS_ERR_INVALID, "tomos_pack_fp32_16: null pointer");
    pack16_kernel<<<pack_grid(outer), 256, 0, as_stream(stream)>>>(src, outer, inner, ld_src, wh,
                                                                   wr, ld_dst, counts);
    TOMOS_LAUNCH_CHECK("pack16_kernel");
    return TOMOS_OK;
}

tomos_status tomos_unpack_fp32_16(const uint16_t* wh, const uint16_t* wr, int32_t layout,
                                  int64_t rows, int64_t cols, int64_t ld_src, float* dst,
                                  int64_t ld_dst, void* stream) {
    int64_t outer, inner;
    std::string why;
    if (!shape_ok(layout, rows, cols, ld_src, ld_dst, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "tomos_unpack_fp32_16: " + why);
    if (outer == 0 || inner == 0) return TOMOS_OK;
    if (!dst || !wh || !wr) return fail(TOMOS_ERR_INVALID, "tomos_unpack_fp32_16: null pointer");
    unpack16_kernel<<<pack_grid(outer), 256, 0, as_stream(stream)>>>(wh, wr, outer, inner, ld_src,
                                                                     dst, ld_dst);
    TOMOS_LAUNCH_CHECK("unpack16_kernel");
    return TOMOS_OK;
}

tomos_status tomos_pack_fp32_bf16(const float* src, int32_t layout, int64_t rows, int64_t cols,
                                  int64_t ld_src, uint16_t* wh, uint16_t* wr, int64_t ld_dst,
                                  int32_t rounded, void* stream) {
    int64_t outer, inner;
    std::string why;
    if (!shape_ok(layout, rows, cols, ld_src, ld_dst, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "tomos_pack_fp32_bf16: " + why);
    if (outer == 0 || inner == 0) return TOMOS_OK;
    if (!src || !wh || !wr) return fail(TOMOS_ERR_INVALID, "tomos_pack_fp32_bf16: null pointer");
    packbf16_kernel<<<pack_grid(outer), 256, 0, as_stream(stream)>>>(src, outer, inner, ld_src, wh,
                                                                     wr, ld_dst, rounded);
    TOMOS_LAUNCH_CHECK("packbf16_kernel");
    return TOMOS_OK;
}

tomos_status tomos_pack_fp16(const float* src, int32_t layout, int64_t rows, int64_t cols,
                             int64_t ld_src, uint16_t* dst, int64_t ld_dst, void* stream) {
    int64_t outer, inner;
    std::string why;
    if (!shape_ok(layout, rows, cols, ld_src, ld_dst, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "tomos_pack_fp16: " + why);
    if (outer == 0 || inner == 0) return TOMOS_OK;
    if (!src || !dst) return fail(TOMOS_ERR_INVALID, "tomos_pack_fp16: null pointer");
    packhalf_kernel<<<pack_grid(outer), 256, 0, as_stream(stream)>>>(src, outer, inner, ld_src, dst, ld_dst);
    TOMOS_LAUNCH_CHECK("packhalf_kernel");
    return TOMOS_OK;
}

tomos_status tomos_unpack_fp32_bf16(const uint16_t* wh, const uint16_t* wr, int32_t layout,
                                    int64_t rows, int64_t cols, int64_t ld_src, float* dst,
                                    int64_t ld_dst, int32_t rounded, void* stream) {
    int64_t outer, inner;
    std::string why;
    if (!shape_ok(layout, rows, cols, ld_src, ld_dst, &outer, &inner, &why))
        return fail(TOMOS_ERR_INVALID, "tomos_unpack_fp32_bf16: " + why);
    if (outer == 0 || inner == 0) return TOMOS_OK;
    if (!dst || !wh || !wr) return fail(TOMOS_ERR_INVALID, "tomos_unpack_fp32_bf16: null pointer");
    unpackbf16_kernel<<<pack_grid(outer), 256, 0, as_stream(stream)>>>(wh, wr, outer, inner,
                                                                       ld_src, dst, ld_dst, rounded);
    TOMOS_LAUNCH_CHECK("unpackbf16_kernel");
    return TOMOS_OK;
}

}  // extern "C"
