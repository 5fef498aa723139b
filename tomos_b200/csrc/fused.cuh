// fused.cuh -- the fused Golub-Kahan pass over a row-major A.
//
// One stream over A computes, for every row i,
//     ut_i = cp * (A p)_i + cu * u_i          (written back into u)
// and, while row i is still in registers,
//     q    += ut_i * A[i, :]                  (per-CTA partial of A^T ut)
//     ss   += ut_i^2                          (per-CTA partial, FP64)
// so LSQR's two products per iteration, u = A v - alpha u and
// v = A^T u - beta v (src/core/solver/lsqr.cpp:561-621, two passes over A
// in the reference), cost one read of A: A^T (ut / beta) = q / beta.
// cp and cu are read from device memory, so a captured iteration needs no
// host values.
//
// Work split: each CTA owns a contiguous block of rows; its warps take
// rows round-robin, two rows at a time.  Lane l of a warp owns the 16-byte
// column chunks l, l+32, l+64, ... of every row (NCH chunks), so p and the
// q accumulators live in registers and each row is one coalesced sweep.
// Partials are reduced across warps in shared memory (fixed order) and
// written per CTA; the n-side kernels reduce them across CTAs in a fixed
// order, so the result is deterministic for a given grid.
//
// Requirements (checked by the host): row-major, ld * element bytes a
// multiple of 16, 16-byte aligned planes, n <= 32 * NCH * VEC.
#pragma once

#include <cuda_fp16.h>

#include "common.cuh"

namespace tomos_b200 {

constexpr int kFusedWarps = 8;
constexpr int kFusedThreads = kFusedWarps * 32;

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
    const double* coef;    // [cp, cu]
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

// FP32_16 wh only: the words are fp16 values unless their control bit is
// set; a chunk with any control bit takes the exact fp32_16_half_only path
// for those elements only.
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
                uint32_t hb = (w[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
                if (hb & 1u) f[k] = half_bits_to_float(half_only_bits(hb));
            }
        }
    }
};

// FP32_16 wh + wr, exact.
template <>
struct ChunkDecoder<Elem::A16> {
    static __device__ __forceinline__ void load(const FusedParams& P, size_t off, uint4& h, uint4& r) {
        h = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.hi) + off));
        r = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(P.lo) + off));
    }
    static __device__ __forceinline__ void decode(const uint4& h, const uint4& r, float* f) {
        const uint32_t wh[4] = {h.x, h.y, h.z, h.w};
        const uint32_t wr[4] = {r.x, r.y, r.z, r.w};
        if (!((h.x | h.y | h.z | h.w) & 0x00010001u)) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                uint32_t hh = (wh[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
                uint32_t rr = (wr[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
                uint32_t mag = ((hh & 0x7FFEu) << 13) + 0x38000000u + (rr >> 2) - ((rr & 1u) << 14);
                f[k] = __uint_as_float(((hh & 0x8000u) << 16) | mag);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                uint32_t hh = (wh[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
                uint32_t rr = (wr[k >> 1] >> ((k & 1) * 16)) & 0xFFFFu;
                f[k] = decode_fp32_16_exact(hh, rr);
            }
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

template <Elem E, int NCH, bool ACC64>
__global__ void __launch_bounds__(kFusedThreads, 1) fused_pass_kernel(FusedParams P) {
    if (P.skip && *P.skip) return;
    constexpr int VEC = ChunkElems<E>::value;
    constexpr int WCOLS = NCH * 32 * VEC;  // columns covered by one warp
    using Dot = typename std::conditional<ACC64, double, float>::type;
    using Dec = ChunkDecoder<E>;

    __shared__ __align__(16) float red[kFusedWarps][WCOLS];
    __shared__ double ssw[kFusedWarps];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int64_t n = P.n;
    const int64_t nchunks = (n + VEC - 1) / VEC;
    const double cp = P.coef[0];
    const double cu = P.coef[1];

    float pv[NCH][VEC];
    float acc[NCH][VEC];
    bool live[NCH];
#pragma unroll
    for (int t = 0; t < NCH; ++t) {
        const int64_t c = (int64_t)t * 32 + lane;
        live[t] = c < nchunks;
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
            const int64_t col = c * VEC + e;
            pv[t][e] = (col < n) ? __ldg(P.p + col) : 0.0f;
            acc[t][e] = 0.0f;
        }
    }
    // Only the last chunk of a row can straddle n.
    const bool ragged = (n % VEC) != 0;

    const int64_t rows_per_cta = (P.m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    int64_t r1 = r0 + rows_per_cta;
    if (r1 > P.m) r1 = P.m;

    double ss = 0.0;
    for (int64_t i0 = r0 + warp; i0 < r1; i0 += 2 * kFusedWarps) {
        const int64_t i1 = i0 + kFusedWarps;
        const bool has1 = i1 < r1;
        uint4 h0[NCH], l0[NCH], h1[NCH], l1[NCH];
#pragma unroll
        for (int t = 0; t < NCH; ++t) {
            h0[t] = l0[t] = h1[t] = l1[t] = make_uint4(0, 0, 0, 0);
            const size_t coloff = ((size_t)t * 32 + lane) * VEC;
            if (live[t]) {
                Dec::load(P, (size_t)i0 * P.ld + coloff, h0[t], l0[t]);
                if (has1) Dec::load(P, (size_t)i1 * P.ld + coloff, h1[t], l1[t]);
            }
        }
        const float ui0 = __ldg(P.u_in + i0);
        const float ui1 = has1 ? __ldg(P.u_in + i1) : 0.0f;

        float a0[NCH][VEC], a1[NCH][VEC];
        Dot d0 = 0, d1 = 0;
#pragma unroll
        for (int t = 0; t < NCH; ++t) {
            Dec::decode(h0[t], l0[t], a0[t]);
            Dec::decode(h1[t], l1[t], a1[t]);
            if (!live[t]) {
#pragma unroll
                for (int e = 0; e < VEC; ++e) a0[t][e] = a1[t][e] = 0.0f;
            } else if (ragged) {
                const int64_t c = (int64_t)t * 32 + lane;
                if (c == nchunks - 1) {
#pragma unroll
                    for (int e = 0; e < VEC; ++e)
                        if (c * VEC + e >= n) a0[t][e] = a1[t][e] = 0.0f;
                }
            }
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                d0 += (Dot)a0[t][e] * (Dot)pv[t][e];
                d1 += (Dot)a1[t][e] * (Dot)pv[t][e];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d0 += __shfl_xor_sync(0xffffffffu, d0, o);
            d1 += __shfl_xor_sync(0xffffffffu, d1, o);
        }
        const float ut0 = (float)(cp * (double)d0 + cu * (double)ui0);
        const float ut1 = has1 ? (float)(cp * (double)d1 + cu * (double)ui1) : 0.0f;
        if (lane == 0) {
            P.u_out[i0] = ut0;
            ss += (double)ut0 * (double)ut0;
            if (has1) {
                P.u_out[i1] = ut1;
                ss += (double)ut1 * (double)ut1;
            }
        }
#pragma unroll
        for (int t = 0; t < NCH; ++t)
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[t][e] = fmaf(a1[t][e], ut1, fmaf(a0[t][e], ut0, acc[t][e]));
    }

    // Cross-warp reduction of the A^T partials, fixed order.
#pragma unroll
    for (int t = 0; t < NCH; ++t) {
        float* dst = &red[warp][(t * 32 + lane) * VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) dst[e] = acc[t][e];
    }
    if (lane == 0) ssw[warp] = ss;
    __syncthreads();
    float* qout = P.qpart + (size_t)blockIdx.x * P.qstride;
    for (int64_t j = threadIdx.x; j < n; j += kFusedThreads) {
        float s = 0.0f;
#pragma unroll
        for (int w = 0; w < kFusedWarps; ++w) s += red[w][j];
        qout[j] = s;
    }
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kFusedWarps; ++w) s += ssw[w];
        P.sspart[blockIdx.x] = s;
    }
}

}  // namespace tomos_b200
