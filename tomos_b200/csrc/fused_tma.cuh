// fused_tma.cuh -- the fused Golub-Kahan pass over a row-major A, staged
// through shared memory by bulk asynchronous copies (TMA, cp.async.bulk).
//
// Same arithmetic as fused.cuh (per row i: ut_i = cp (A p)_i + cu u_i,
// then q += ut_i A[i, :] and ss += ut_i^2 with the row still on chip), but
// the rows reach the SM through a ring of NSTAGE shared-memory stages of
// TR rows each, filled by one producer thread with one bulk copy per row
// and handed over with mbarriers:
//
//   producer (warp 8, lane 0)      consumers (warps 0..7)
//   wait empty[s]                  wait full[s]
//   expect_tx(full[s], bytes)      rows warp, warp+8 of the stage:
//   cp.async.bulk row -> stage s     LDS.128 chunks, decode, dot, shuffle
//                                    reduce, ut, q += ut * row
//                                  arrive empty[s]
//
// so the bytes in flight per SM are set by the ring (~190 KB), not by the
// registers of the warps -- the register-staged pass could keep only
// 2 rows per warp in flight.  One CTA per SM, grid = SM count.
//
// FP32_16 wh words whose control bit is set (values outside the fp16
// range, ~0.35% of a matrix with columns scaled over 1e-3..1e3) are fixed
// in shared memory in place, to the exact fp32_16_half_only bits, by the
// lane that owns the chunk; the work is proportional to the number of such
// words rather than to the warp's divergence.
//
// Every mbarrier wait is bounded (kSpinLimit polls); on expiry the kernel
// records the failure in *err, stops issuing copies, drains the copies it
// issued (bounded again) and returns, so a broken pipeline reports an
// error instead of hanging the GPU.
#pragma once

#include <cuda_fp16.h>

#include "common.cuh"
#include "fused.cuh"

namespace tomos_b200 {

constexpr int kTmaConsumers = 8;
constexpr int kTmaThreads = (kTmaConsumers + 1) * 32;
constexpr int kTmaRows = 16;          // rows per stage
constexpr int kTmaMaxStages = 8;
constexpr size_t kTmaSmemBudget = 200 * 1024;
constexpr long long kSpinLimit = 1ll << 24;

struct TmaParams {
    FusedParams f;
    int* err;            // set nonzero on a pipeline timeout
    int nstage;
    int copy_bytes;      // bytes copied per row and plane (16-byte multiple)
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false after kSpinLimit unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long long k = 0; k < kSpinLimit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// fp32_16_half_only on both halves of a word (control-1 halves only).
__device__ __forceinline__ uint32_t fix_half_pair(uint32_t w) {
    uint32_t lo = w & 0xFFFFu, hi = w >> 16;
    if (lo & 1u) lo = half_only_bits(lo);
    if (hi & 1u) hi = half_only_bits(hi);
    return lo | (hi << 16);
}

template <Elem E>
struct SmemChunk;

template <>
struct SmemChunk<Elem::F32> {
    static constexpr int planes = 1;
    static __device__ __forceinline__ void decode(const uint8_t* hrow, const uint8_t*, int c,
                                                  float* f) {
        const uint4 h = *reinterpret_cast<const uint4*>(hrow + (size_t)c * 16);
        f[0] = __uint_as_float(h.x);
        f[1] = __uint_as_float(h.y);
        f[2] = __uint_as_float(h.z);
        f[3] = __uint_as_float(h.w);
    }
};

template <>
struct SmemChunk<Elem::H16> {
    static constexpr int planes = 1;
    static __device__ __forceinline__ void decode(const uint8_t* hrow, const uint8_t*, int c,
                                                  float* f) {
        uint4* p = reinterpret_cast<uint4*>(const_cast<uint8_t*>(hrow) + (size_t)c * 16);
        uint4 h = *p;
        if ((h.x | h.y | h.z | h.w) & 0x00010001u) {
            // rare: rewrite the words that carry a control bit in place
            if (h.x & 0x00010001u) h.x = fix_half_pair(h.x);
            if (h.y & 0x00010001u) h.y = fix_half_pair(h.y);
            if (h.z & 0x00010001u) h.z = fix_half_pair(h.z);
            if (h.w & 0x00010001u) h.w = fix_half_pair(h.w);
            *p = h;
        }
        half2_to_f32(h.x, f[0], f[1]);
        half2_to_f32(h.y, f[2], f[3]);
        half2_to_f32(h.z, f[4], f[5]);
        half2_to_f32(h.w, f[6], f[7]);
    }
};

template <>
struct SmemChunk<Elem::B16> {
    static constexpr int planes = 1;
    static __device__ __forceinline__ void decode(const uint8_t* hrow, const uint8_t*, int c,
                                                  float* f) {
        const uint4 h = *reinterpret_cast<const uint4*>(hrow + (size_t)c * 16);
        ChunkDecoder<Elem::B16>::decode(h, h, f);
    }
};

template <Elem E>
struct SmemChunkExact {
    static constexpr int planes = 2;
    static __device__ __forceinline__ void decode(const uint8_t* hrow, const uint8_t* lrow, int c,
                                                  float* f) {
        const uint4 h = *reinterpret_cast<const uint4*>(hrow + (size_t)c * 16);
        const uint4 r = *reinterpret_cast<const uint4*>(lrow + (size_t)c * 16);
        ChunkDecoder<E>::decode(h, r, f);
    }
};
template <>
struct SmemChunk<Elem::A16> : SmemChunkExact<Elem::A16> {};
template <>
struct SmemChunk<Elem::AB16> : SmemChunkExact<Elem::AB16> {};
template <>
struct SmemChunk<Elem::AB16R> : SmemChunkExact<Elem::AB16R> {};

template <Elem E, int NCH, bool ACC64>
__global__ void __launch_bounds__(kTmaThreads, 1) fused_tma_kernel(TmaParams T) {
    const FusedParams& P = T.f;
    if (P.skip && *P.skip) return;
    constexpr int VEC = ChunkElems<E>::value;
    constexpr int WCOLS = NCH * 32 * VEC;
    constexpr int PLANES = SmemChunk<E>::planes;
    using Dot = typename std::conditional<ACC64, double, float>::type;

    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kTmaMaxStages];
    __shared__ __align__(8) uint64_t empty[kTmaMaxStages];
    __shared__ double ssw[kTmaConsumers];
    __shared__ int abort_flag;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nstage = T.nstage;
    const int cb = T.copy_bytes;
    const size_t row_stride = (size_t)cb;  // per plane
    const size_t stage_bytes = (size_t)kTmaRows * cb * PLANES;
    const int esz = (E == Elem::F32) ? 4 : 2;

    const int64_t rows_per_cta = (P.m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
    int64_t r1 = r0 + rows_per_cta;
    if (r1 > P.m) r1 = P.m;
    const int64_t nrows = r1 > r0 ? r1 - r0 : 0;
    const int ntiles = (int)((nrows + kTmaRows - 1) / kTmaRows);

    if (threadIdx.x == 0) {
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTmaConsumers);
        }
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();

    float acc[NCH][VEC];
#pragma unroll
    for (int k = 0; k < NCH; ++k)
#pragma unroll
        for (int e = 0; e < VEC; ++e) acc[k][e] = 0.0f;
    double ss = 0.0;

    if (warp == kTmaConsumers) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            int issued = 0;
            for (int t = 0; t < ntiles; ++t) {
                const int s = t % nstage;
                const uint32_t it = (uint32_t)(t / nstage);
                if (!mbar_wait(&empty[s], (it & 1u) ^ 1u)) {
                    atomicExch(T.err, 1);
                    break;
                }
                if (*(volatile int*)&abort_flag) break;
                const int64_t i0 = r0 + (int64_t)t * kTmaRows;
                const int rows = (int)((r1 - i0) < kTmaRows ? (r1 - i0) : kTmaRows);
                uint8_t* st = smem + (size_t)s * stage_bytes;
                mbar_expect_tx(&full[s], (uint32_t)(rows * cb * PLANES));
                for (int r = 0; r < rows; ++r) {
                    const size_t goff = (size_t)(i0 + r) * (size_t)P.ld * esz;
                    bulk_g2s(st + (size_t)r * row_stride, static_cast<const uint8_t*>(P.hi) + goff,
                             (uint32_t)cb, &full[s]);
                    if (PLANES == 2)
                        bulk_g2s(st + (size_t)(kTmaRows + r) * row_stride,
                                 static_cast<const uint8_t*>(P.lo) + goff, (uint32_t)cb, &full[s]);
                }
                issued = t + 1;
            }
            // Drain: every issued stage must land before the CTA may exit.
            for (int t = (issued > nstage ? issued - nstage : 0); t < issued; ++t) {
                if (!mbar_wait(&full[t % nstage], (uint32_t)(t / nstage) & 1u)) {
                    atomicExch(T.err, 2);
                    break;
                }
            }
        }
    } else {
        // --------------------------------------------------------- consumers
        const double cp = P.coef[0];
        const double cu = P.coef[1];
        const int64_t n = P.n;
        const int64_t nchunks = (n + VEC - 1) / VEC;
        float pv[NCH][VEC];
        bool live[NCH];
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            const int64_t c = (int64_t)k * 32 + lane;
            live[k] = c < nchunks;
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                const int64_t col = c * VEC + e;
                pv[k][e] = (col < n) ? __ldg(P.p + col) : 0.0f;
            }
        }
        const bool ragged = (n % VEC) != 0;
        // u of this warp's two rows, fetched one tile ahead
        float un0 = 0.f, un1 = 0.f;
        {
            const int64_t a = r0 + warp, b = r0 + warp + kTmaConsumers;
            if (a < r1) un0 = __ldg(P.u_in + a);
            if (b < r1) un1 = __ldg(P.u_in + b);
        }
        for (int t = 0; t < ntiles; ++t) {
            const int s = t % nstage;
            const int64_t i0 = r0 + (int64_t)t * kTmaRows;
            const int64_t ia = i0 + warp, ib = i0 + warp + kTmaConsumers;
            const bool hasa = ia < r1, hasb = ib < r1;
            const float ua = un0, ub = un1;
            {
                const int64_t na = ia + kTmaRows, nb = ib + kTmaRows;
                un0 = na < r1 ? __ldg(P.u_in + na) : 0.f;
                un1 = nb < r1 ? __ldg(P.u_in + nb) : 0.f;
            }
            if (!mbar_wait(&full[s], (uint32_t)(t / nstage) & 1u)) {
                atomicExch(T.err, 3);
                abort_flag = 1;
                break;
            }
            const uint8_t* st = smem + (size_t)s * stage_bytes;
            const uint8_t* ha = st + (size_t)warp * row_stride;
            const uint8_t* hb = st + (size_t)(warp + kTmaConsumers) * row_stride;
            const uint8_t* la = ha + (size_t)kTmaRows * row_stride;
            const uint8_t* lb = hb + (size_t)kTmaRows * row_stride;
            float a0[NCH][VEC], a1[NCH][VEC];
            Dot d0 = 0, d1 = 0;
#pragma unroll
            for (int k = 0; k < NCH; ++k) {
                const int c = k * 32 + lane;
                if (live[k] && hasa) {
                    SmemChunk<E>::decode(ha, la, c, a0[k]);
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) a0[k][e] = 0.f;
                }
                if (live[k] && hasb) {
                    SmemChunk<E>::decode(hb, lb, c, a1[k]);
                } else {
#pragma unroll
                    for (int e = 0; e < VEC; ++e) a1[k][e] = 0.f;
                }
                if (ragged && live[k] && c == nchunks - 1) {
#pragma unroll
                    for (int e = 0; e < VEC; ++e)
                        if ((int64_t)c * VEC + e >= n) a0[k][e] = a1[k][e] = 0.f;
                }
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    d0 += (Dot)a0[k][e] * (Dot)pv[k][e];
                    d1 += (Dot)a1[k][e] * (Dot)pv[k][e];
                }
            }
            // The stage may be refilled once every consumer warp has read it.
            // Words fixed in place were written by the generic proxy; order
            // them before the next asynchronous copy into the stage.
            if (E == Elem::H16) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                d0 += __shfl_xor_sync(0xffffffffu, d0, o);
                d1 += __shfl_xor_sync(0xffffffffu, d1, o);
            }
            const float ut0 = hasa ? (float)(cp * (double)d0 + cu * (double)ua) : 0.f;
            const float ut1 = hasb ? (float)(cp * (double)d1 + cu * (double)ub) : 0.f;
            if (lane == 0) {
                if (hasa) {
                    P.u_out[ia] = ut0;
                    ss += (double)ut0 * (double)ut0;
                }
                if (hasb) {
                    P.u_out[ib] = ut1;
                    ss += (double)ut1 * (double)ut1;
                }
            }
#pragma unroll
            for (int k = 0; k < NCH; ++k)
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                    acc[k][e] = fmaf(a1[k][e], ut1, fmaf(a0[k][e], ut0, acc[k][e]));
        }
    }

    // Epilogue: the pipeline is drained (the producer waited for every copy
    // it issued), so the stage memory holds the cross-warp reduction.
    __syncthreads();
    float* red = reinterpret_cast<float*>(smem);
    if (warp < kTmaConsumers) {
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            float* dst = &red[(size_t)warp * WCOLS + (k * 32 + lane) * VEC];
#pragma unroll
            for (int e = 0; e < VEC; ++e) dst[e] = acc[k][e];
        }
        if (lane == 0) ssw[warp] = ss;
    }
    __syncthreads();
    float* qout = P.qpart + (size_t)blockIdx.x * P.qstride;
    for (int64_t j = threadIdx.x; j < P.n; j += kTmaThreads) {
        float sum = 0.0f;
#pragma unroll
        for (int w = 0; w < kTmaConsumers; ++w) sum += red[(size_t)w * WCOLS + j];
        qout[j] = sum;
    }
    if (threadIdx.x == 0) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kTmaConsumers; ++w) sum += ssw[w];
        P.sspart[blockIdx.x] = sum;
    }
}

// Dynamic shared memory of one launch: the stage ring, at least the
// cross-warp reduction buffer.
template <Elem E, int NCH>
inline size_t fused_tma_smem(int nstage, int copy_bytes) {
    constexpr int VEC = ChunkElems<E>::value;
    const size_t ring = (size_t)nstage * kTmaRows * copy_bytes * SmemChunk<E>::planes;
    const size_t red = (size_t)kTmaConsumers * NCH * 32 * VEC * sizeof(float);
    return ring > red ? ring : red;
}

}  // namespace tomos_b200
