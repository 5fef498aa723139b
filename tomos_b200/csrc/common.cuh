// common.cuh -- shared device helpers for the sm_100a LSQR hot path:
// error plumbing for the C ABI, the FP32_16 / FP32_BF16 element codecs and
// warp reductions.
//
// Packed formats (both bit-compatible with the reference's encoders):
//   FP32_16   (src/core/matrix/fp32_16_pack.hpp)
//     wh = sign(1) | exponent field(5) | mant_hi(9) | control(1)
//     wr = mant_lo(14) | 0 | round_flag(1)
//     control 0: fp32 exponent 113..142 stored as exponent-112; wh is then a
//     valid fp16 bit pattern.  control 1: bit 14 is the direction (1 = above,
//     0 = below that range) and bits 13..10 hold steps-1 (steps 1..14 beyond
//     the range, bit-exact); steps field 14 marks saturation to signed
//     Inf / signed 0.  mant_hi is the round-to-nearest-even top 9 bits and
//     round_flag records the round-up.
//   FP32_BF16 (src/core/matrix/fp32_bf16_pack.hpp)
//     wh = top 16 bits of the float (a bf16), wr = low 16 bits; the rounded
//     variant rounds wh to nearest-even and keeps the round-up in wr bit 0.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "tomos_b200.h"

namespace tomos_b200 {

// ---------------------------------------------------------------- errors

void set_last_error(const std::string& msg);
tomos_status fail(tomos_status code, const std::string& msg);
tomos_status cuda_fail(cudaError_t err, const char* what);

#define TOMOS_CUDA_TRY(expr)                                  \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return ::tomos_b200::cuda_fail(_e, #expr); \
    } while (0)

#define TOMOS_LAUNCH_CHECK(what)                              \
    do {                                                      \
        cudaError_t _e = cudaGetLastError();                  \
        if (_e != cudaSuccess) return ::tomos_b200::cuda_fail(_e, what); \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

// ---------------------------------------------------------------- codecs

__host__ __device__ __forceinline__ uint32_t f2u(float v) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(v);
#else
    uint32_t u;
    __builtin_memcpy(&u, &v, 4);
    return u;
#endif
}
__host__ __device__ __forceinline__ float u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float v;
    __builtin_memcpy(&v, &u, 4);
    return v;
#endif
}

// FP32 -> (wh, wr), the full-carry encoder (fp32_16_pack.hpp:129-190).
__host__ __device__ __forceinline__ void encode_fp32_16(float value, uint16_t& wh,
                                                        uint16_t& wr, int& cls) {
    uint32_t bits = f2u(value);
    uint32_t sign = (bits >> 16) & 0x8000u;
    uint32_t e = (bits >> 23) & 0xFFu;
    uint32_t mant = bits & 0x7FFFFFu;
    if (e >= 99u && e <= 156u) {
        uint32_t hi = mant >> 14, lo = mant & 0x3FFFu;
        uint32_t up = (((lo >> 13) & 1u) != 0u) && (((lo & 0x1FFFu) != 0u) || ((hi & 1u) != 0u));
        uint32_t hr = hi + up;
        uint32_t carry = hr > 0x1FFu;
        uint32_t ee = e + carry;
        uint32_t hw = carry ? 0u : hr;
        if (ee >= 113u && ee <= 142u) {
            wh = (uint16_t)(sign | ((ee - 112u) << 10) | (hw << 1));
            wr = (uint16_t)((lo << 2) | up);
            cls = 0;
            return;
        }
        uint32_t dir = ee > 142u;
        uint32_t steps = dir ? ee - 142u : 113u - ee;
        if (steps >= 1u && steps <= 14u) {
            wh = (uint16_t)(sign | (dir << 14) | ((steps - 1u) << 10) | (hw << 1) | 1u);
            wr = (uint16_t)((lo << 2) | up);
            cls = dir ? 2 : 1;
            return;
        }
        wh = (uint16_t)(sign | (dir << 14) | (14u << 10) | 1u);
        wr = 0;
        cls = 3;
        return;
    }
    uint32_t dir = e > 142u;
    wh = (uint16_t)(sign | (dir << 14) | (14u << 10) | 1u);
    wr = 0;
    cls = 3;
}

// (wh, wr) -> FP32, exact inverse (fp32_16_pack.hpp:301-359).  The
// normal-range case is one integer expression: rebuilding the float with
// the ROUNDED mant_hi and then subtracting round_flag at bit 14 lets the
// borrow undo a carry into the exponent by itself.
__host__ __device__ __forceinline__ float decode_fp32_16_exact(uint32_t h, uint32_t r) {
    if (!(h & 1u)) {
        uint32_t mag = ((h & 0x7FFEu) << 13) + 0x38000000u + (r >> 2) - ((r & 1u) << 14);
        return u2f(((h & 0x8000u) << 16) | mag);
    }
    uint32_t sign = (h & 0x8000u) << 16;
    uint32_t s = (h >> 10) & 0xFu, dir = (h >> 14) & 1u;
    if (s == 14u) return u2f(dir ? (sign | 0x7F800000u) : sign);
    uint32_t e = dir ? 143u + s : 112u - s;
    uint32_t mag = (e << 23) + ((h & 0x3FEu) << 13) + (r >> 2) - ((r & 1u) << 14);
    return u2f(sign | mag);
}

// decode_fp32_16_exact without branches, equal to it for every (h, r)
// (checked over all 2^32 pairs): the exponent is 112 + e5 for control-0
// words and 112 + e5 + 15 (upward step) or 112 - e5 (downward step) for
// control-1 words, and the step field 14 stands for +-Inf / +-0.  A warp
// then never diverges on the rare control-1 elements.
__host__ __device__ __forceinline__ float decode_fp32_16_exact_nb(uint32_t hh, uint32_t rr) {
    const uint32_t e5 = (hh >> 10) & 0x1Fu;
    const uint32_t c = hh & 1u, dir = (hh >> 14) & 1u;
    const int32_t off = c ? (dir ? (int32_t)e5 + 15 : -(int32_t)e5) : (int32_t)e5;
    const uint32_t mag = ((uint32_t)(off + 112) << 23) + ((hh & 0x3FEu) << 13) + (rr >> 2) - ((rr & 1u) << 14);
    const uint32_t special = c & ((e5 & 0xFu) == 14u);
    const uint32_t res = special ? (dir ? 0x7F800000u : 0u) : mag;
    return u2f(((hh & 0x8000u) << 16) | res);
}

// wh -> the fp16 bit pattern fp32_16_half_only produces
// (fp32_16_pack.hpp:553-571): control-0 words are already fp16; overflow
// saturates to signed Inf; underflow steps become an fp16 subnormal by
// shifting the 10-bit significand right by the stored step field.
__host__ __device__ __forceinline__ uint32_t half_only_bits(uint32_t h) {
    if (!(h & 1u)) return h;
    uint32_t sign = h & 0x8000u;
    if ((h >> 14) & 1u) return sign | 0x7C00u;
    uint32_t s = (h >> 10) & 0xFu;
    uint32_t sig = 0x200u | ((h >> 1) & 0x1FFu);
    return sign | ((sig >> s) & 0x3FFu);
}

// IEEE binary16 bits -> float (exact; normal, subnormal, Inf).
__device__ __forceinline__ float half_bits_to_float(uint32_t hb) {
    return __half2float(__ushort_as_half((unsigned short)hb));
}

// FP32 -> FP32_BF16 (fp32_bf16_pack.hpp:68-73, :117-145).
__host__ __device__ __forceinline__ void encode_fp32_bf16(float value, uint16_t& wh,
                                                          uint16_t& wr, bool rounded) {
    uint32_t b = f2u(value);
    if (!rounded) {
        wh = (uint16_t)(b >> 16);
        wr = (uint16_t)(b & 0xFFFFu);
        return;
    }
    uint32_t t = b >> 16, lo = b & 0xFFFFu;
    uint32_t up = (((lo >> 15) & 1u) != 0u) && (((lo & 0x7FFFu) != 0u) || ((t & 1u) != 0u));
    wh = (uint16_t)(t + up);
    wr = (uint16_t)((lo & 0xFFFEu) | up);
}

// (wh, wr) -> FP32 (fp32_bf16_pack.hpp:78-81 and :180-186).
__host__ __device__ __forceinline__ float decode_fp32_bf16_exact(uint32_t h, uint32_t r,
                                                                 bool rounded) {
    if (!rounded) return u2f((h << 16) | r);
    uint32_t t = (h - (r & 1u)) & 0xFFFFu;
    return u2f((t << 16) | (r & 0xFFFEu));
}

// ------------------------------------------------------- warp reductions

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Element-type tags shared by the kernels.
enum class Elem : int {
    F32 = 0,       // FP32 storage
    F64 = 1,       // FP64 storage
    H16 = 2,       // FP32_16, wh plane only (half_only decode)
    A16 = 3,       // FP32_16, wh + wr exact
    B16 = 4,       // FP32_BF16, wh plane only (bf16 value)
    AB16 = 5,      // FP32_BF16 truncating, wh + wr exact
    AB16R = 6,     // FP32_BF16 rounded, wh + wr (combine_rounded)
    F16 = 7        // IEEE fp16 (the solver's staged copy of an FP32_16 wh
                   // plane, control words already decoded)
};

// Scalar element decode at flat index idx (generic kernels).
template <Elem E>
__device__ __forceinline__ float load_elem(const void* p, const void* q, size_t idx);

template <>
__device__ __forceinline__ float load_elem<Elem::F32>(const void* p, const void*, size_t idx) {
    return __ldg(reinterpret_cast<const float*>(p) + idx);
}
template <>
__device__ __forceinline__ float load_elem<Elem::H16>(const void* p, const void*, size_t idx) {
    uint32_t h = __ldg(reinterpret_cast<const unsigned short*>(p) + idx);
    return half_bits_to_float(half_only_bits(h));
}
template <>
__device__ __forceinline__ float load_elem<Elem::F16>(const void* p, const void*, size_t idx) {
    return half_bits_to_float(__ldg(reinterpret_cast<const unsigned short*>(p) + idx));
}
template <>
__device__ __forceinline__ float load_elem<Elem::A16>(const void* p, const void* q, size_t idx) {
    uint32_t h = __ldg(reinterpret_cast<const unsigned short*>(p) + idx);
    uint32_t r = __ldg(reinterpret_cast<const unsigned short*>(q) + idx);
    return decode_fp32_16_exact(h, r);
}
template <>
__device__ __forceinline__ float load_elem<Elem::B16>(const void* p, const void*, size_t idx) {
    uint32_t h = __ldg(reinterpret_cast<const unsigned short*>(p) + idx);
    return u2f(h << 16);
}
template <>
__device__ __forceinline__ float load_elem<Elem::AB16>(const void* p, const void* q, size_t idx) {
    uint32_t h = __ldg(reinterpret_cast<const unsigned short*>(p) + idx);
    uint32_t r = __ldg(reinterpret_cast<const unsigned short*>(q) + idx);
    return decode_fp32_bf16_exact(h, r, false);
}
template <>
__device__ __forceinline__ float load_elem<Elem::AB16R>(const void* p, const void* q, size_t idx) {
    uint32_t h = __ldg(reinterpret_cast<const unsigned short*>(p) + idx);
    uint32_t r = __ldg(reinterpret_cast<const unsigned short*>(q) + idx);
    return decode_fp32_bf16_exact(h, r, true);
}

// Resolves a tomos_dense + tier to the element tag it is read as.
// Returns false (with a message) if the combination has no kernel, the
// reference's "no kernel registered" contract.
bool resolve_elem(const tomos_dense* A, int32_t tier, Elem* out, std::string* why);
bool resolve_elem_csr(const tomos_csr* A, int32_t tier, Elem* out, std::string* why);

// wr plane of a packed dense matrix (planar default when values_lo is NULL).
const void* dense_lo_plane(const tomos_dense* A);

inline int elem_bytes(Elem e) {
    switch (e) {
        case Elem::F32: return 4;
        case Elem::F64: return 8;
        case Elem::H16: case Elem::B16: case Elem::F16: return 2;
        default: return 4;  // wh + wr
    }
}

}  // namespace tomos_b200
