// fused.cuh -- shared pieces of the fused Golub-Kahan pass over a
// row-major A (the kernel itself is in rowpass.cuh).
//
// One stream over A computes, for every row i,
//     ut_i = cp * (A p)_i + cu * u_i          (written back into u)
// and, while row i is still on chip,
//     q    += ut_i * A[i, :]                  (per-CTA partial of A^T ut)
//     ss   += ut_i^2                          (per-CTA partial, FP64)
// so LSQR's two products per iteration, u = A v - alpha u and
// v = A^T u - beta v (src/core/solver/lsqr.cpp:561-621, two passes over A
// in the reference), cost one read of A: A^T (ut / beta) = q / beta.
// cp and cu are read from device memory, so a captured iteration needs no
// host values.
//
// This header holds the launch parameters and the decoders of one 16-byte
// chunk of each storage type (also used by the CountSketch owner sums).
#pragma once

#include <cuda_fp16.h>

#include "common.cuh"

namespace tomos_b200 {

template <Elem E>
struct ChunkElems {
    static constexpr int value = 8;  // 16-bit planes: 8 elements per 16 B
};
template <>
struct ChunkElems<Elem::F32> {
    static constexpr int value = 4;
};

struct FusedParams {
    const void* hi;        // A (FP32) or its wh plane
    const void* lo;        // wr plane (exact tiers), else unused
    int64_t m, n, ld;      // ld in elements
    const float* p;        // n
    const float* u_in;     // m
    float* u_out;          // m (may alias u_in)
    const double* coef;    // device [cp, cu], or NULL: the host values cp, cu
    double cp, cu;
    float* qpart;          // gridDim.x x qstride
    double* sspart;        // gridDim.x
    int64_t qstride;
    const int* skip;       // nonzero: return at once (solver finished)
};

// Decodes one 16-byte chunk into VEC floats.
template <Elem E>
struct ChunkDecoder;

template <>
struct ChunkDecoder<Elem::F32> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4&) {
        h = __ldcs(reinterpret_cast<const uint4*>(static_cast<const float*>(P.hi) + off));
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4&, float* f) {
        f[0] = __uint_as_float(h.x);
        f[1] = __uint_as_float(h.y);
        f[2] = __uint_as_float(h.z);
        f[3] = __uint_as_float(h.w);
    }
};

__device__ __forceinline__ void half2_to_f32(uint32_t w, float& a, float& b) {
    __half2 h2 = *reinterpret_cast<const __half2*>(&w);
    float2 t = __half22float2(h2);
    a = t.x;
    b = t.y;
}

// half_only_bits without branches (selects only), for control-1 halves.
__device__ __forceinline__ uint32_t half_only_bits_flagged(uint32_t h) {
    const uint32_t sign = h & 0x8000u;
    const uint32_t sig = 0x200u | ((h >> 1) & 0x1FFu);
    const uint32_t sub = sign | ((sig >> ((h >> 10) & 0xFu)) & 0x3FFu);
    return (h & 0x4000u) ? (sign | 0x7C00u) : sub;
}

// fp32_16_half_only on both halves of a word (control-1 halves only),
// branch-free: a warp whose lanes disagree on which halves are flagged
// runs it once.
__device__ __forceinline__ uint32_t fix_half_pair(uint32_t w) {
    const uint32_t lo = w & 0xFFFFu, hi = w >> 16;
    const uint32_t flo = (lo & 1u) ? half_only_bits_flagged(lo) : lo;
    const uint32_t fhi = (hi & 1u) ? half_only_bits_flagged(hi) : hi;
    return flo | (fhi << 16);
}

// Fixes only the words of a chunk that hold a control-1 half (rare: the
// warp runs fix_half_pair for a word only when some lane's word needs it).
__device__ __forceinline__ void fix_half_chunk(uint4& h) {
    if (h.x & 0x00010001u) h.x = fix_half_pair(h.x);
    if (h.y & 0x00010001u) h.y = fix_half_pair(h.y);
    if (h.z & 0x00010001u) h.z = fix_half_pair(h.z);
    if (h.w & 0x00010001u) h.w = fix_half_pair(h.w);
}

__device__ __forceinline__ float2 h2f2(uint32_t w) {
    return __half22float2(*reinterpret_cast<const __half2*>(&w));
}

// FP32_16 wh only: the words are fp16 values unless their control bit is
// set; after the plain conversion, only elements whose control bit is set
// (rare) are redone with the exact fp32_16_half_only decode.
template <>
struct ChunkDecoder<Elem::H16> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4&) {
        h = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.hi) + off));
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4&, float* f) {
        half2_to_f32(h.x, f[0], f[1]);
        half2_to_f32(h.y, f[2], f[3]);
        half2_to_f32(h.z, f[4], f[5]);
        half2_to_f32(h.w, f[6], f[7]);
        if ((h.x | h.y | h.z | h.w) & 0x00010001u) {
            const uint32_t w[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t hb = (w[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
                if (hb & 1u) f[k] = half_bits_to_float(half_only_bits(hb));
            }
        }
    }
};

// IEEE fp16 (staged copy of a wh plane): plain conversion.
template <>
struct ChunkDecoder<Elem::F16> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4&) {
        h = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.hi) + off));
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4&, float* f) {
        half2_to_f32(h.x, f[0], f[1]);
        half2_to_f32(h.y, f[2], f[3]);
        half2_to_f32(h.z, f[4], f[5]);
        half2_to_f32(h.w, f[6], f[7]);
    }
};

// Both elements of one wh word and its wr word, exact for control-0
// words: for those wh is the fp16 value of the rounded top of the float,
// so its exact conversion to FP32 has zeros in bits 13..0, and the float's
// bits are those plus mant_lo (wr >> 2) minus the round flag (wr bit 0)
// at bit 14 -- the borrow undoes a carry of the rounding into the
// exponent, and never reaches the sign (the exponent is >= 113).
// Control-1 elements come out wrong and are redone by the caller.
__device__ __forceinline__ float2 decode_pair_fp32_16(uint32_t w, uint32_t r) {
    const float2 hv = h2f2(w);
    const uint32_t s = r >> 2;
    const uint32_t lo0 = s & 0x3FFFu, fl0 = (r << 14) & 0x4000u;
    const uint32_t lo1 = r >> 18, fl1 = s & 0x4000u;
    return make_float2(__uint_as_float(__float_as_uint(hv.x) + lo0 - fl0),
                       __uint_as_float(__float_as_uint(hv.y) + lo1 - fl1));
}

// Both elements of a word pair through the full exact decode.
__device__ __forceinline__ float2 decode_pair_fp32_16_exact(uint32_t w, uint32_t r) {
    return make_float2(decode_fp32_16_exact_nb(w & 0xFFFFu, r & 0xFFFFu),
                       decode_fp32_16_exact_nb(w >> 16, r >> 16));
}

// FP32_16 wh + wr, exact.
template <>
struct ChunkDecoder<Elem::A16> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4& r) {
        h = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.hi) + off));
        r = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.lo) + off));
    }
    // The branch-free exact decode for every element: control-1 words
    // are rare per element but common per warp, where a branch would make
    // the whole warp wait on them.
    static __device__ __forceinline__ void decode(const uint4& h, const uint4& r, float* f) {
        const uint32_t wh[4] = {h.x, h.y, h.z, h.w};
        const uint32_t wr[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t hh = (wh[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
            const uint32_t rr = (wr[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
            f[k] = decode_fp32_16_exact_nb(hh, rr);
        }
    }
};

// FP32_BF16 wh only: the bf16 value.
template <>
struct ChunkDecoder<Elem::B16> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4&) {
        h = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.hi) + off));
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4&, float* f) {
        const uint32_t w[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            f[2 * k] = __uint_as_float(w[k] << 16);
            f[2 * k + 1] = __uint_as_float(w[k] & 0xFFFF0000u);
        }
    }
};

// FP32_BF16 truncating, exact: the float is (wh << 16) | wr.
template <>
struct ChunkDecoder<Elem::AB16> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4& r) {
        ChunkDecoder<Elem::A16>::load(P, off, h, r);
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4& r, float* f) {
        const uint32_t wh[4] = {h.x, h.y, h.z, h.w};
        const uint32_t wr[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            f[2 * k] = __uint_as_float(__byte_perm(wr[k], wh[k], 0x5410));
            f[2 * k + 1] = __uint_as_float(__byte_perm(wr[k], wh[k], 0x7632));
        }
    }
};

// FP32_BF16 rounded: undo the round-up recorded in wr bit 0.
template <>
struct ChunkDecoder<Elem::AB16R> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4& r) {
        ChunkDecoder<Elem::A16>::load(P, off, h, r);
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4& r, float* f) {
        const uint32_t wh[4] = {h.x, h.y, h.z, h.w};
        const uint32_t wr[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            uint32_t hh = (wh[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
            uint32_t rr = (wr[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
            f[k] = decode_fp32_bf16_exact(hh, rr, true);
        }
    }
};

}  // namespace tomos_b200
