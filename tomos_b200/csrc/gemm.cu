// gemm.cu -- mm_apply: C = alpha op(A) op(B) + beta C on the 5th-generation
// tensor cores (tcgen05.mma, accumulators in tensor memory).
//
// The reference's dense GEMM (blas.cpp:98-106, mm_apply; the FP32_16
// tiers of blas.cpp:168-190 and fp32_16_registries.cpp:371-455) takes A in
// any storage and FP32 B and C.  Here one kernel serves every storage:
//
//   CTA tile      128 rows of op(A) x BN columns of op(B) (BN 16..128),
//                 the accumulator a 128-lane x BN-column FP32 tile of
//                 tensor memory (tcgen05.alloc), one CTA per tile.
//   producers     8 warps load op(A) and op(B) straight from global
//                 memory (16-byte vectors along K where the lines are
//                 K-contiguous, warp-coalesced scalar loads across lines
//                 otherwise), decode the storage in registers, split the
//                 values into tensor-core operands and write them as
//                 16-byte units to a ring of shared-memory stages in the
//                 UMMA canonical K-major layout (no swizzle).
//   MMA warp      one thread issues 4 K-steps x terms tcgen05.mma per
//                 stage and frees the stage with tcgen05.commit.
//   epilogue      the producer warps read the accumulator (tcgen05.ld
//                 32x32b) and write alpha acc + beta C.
//
// Operand precision per mode (the tier of the storage read):
//   kPure16   A's 16-bit values (FP32_16 HALF tier fp16, native fp16,
//             FP32_BF16 bf16) times B rounded to the same 16-bit type:
//             one kind::f16 product -- the operands of the reference's
//             pure_half tier (fp32_16_kernels.cpp:172-203), accumulated
//             in FP32 instead of fp16.
//   kTf32x2   the same 16-bit A values (exact in TF32) times B split as
//             B_big + B_small (two TF32 numbers): two kind::tf32 products,
//             B kept to about 22 bits -- the reference's "fast" tier
//             (half decode, wide accumulation, fp32_16_kernels.cpp:113-141).
//   kTf32x3   A exact (FP32 storage, or packed read exactly) split as
//             A_big + A_small, B likewise: A_big B_big + A_big B_small +
//             A_small B_big, three kind::tf32 products -- FP32-level
//             products for the accurate tier (fp32_16_kernels.cpp:57-85).
// Every product accumulates in FP32 in tensor memory; alpha and beta are
// applied in FP64 in the epilogue.  The error of an entry is a few units
// of 2^-22 times sum_l |op(A)_il| |op(B)_lj| plus FP32 summation over K.
//
// Every mbarrier wait is bounded (mbarrier.cuh): a wait that expires
// records an error word and the CTA stops work, drains its MMAs (bounded
// again), frees its tensor memory and exits; such a launch's C is
// undefined.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <mutex>
#include <string>
#include <utility>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "mbarrier.cuh"

namespace tomos_b200 {

namespace {

constexpr int kGemmM = 128;          // rows of op(A) per CTA (the MMA's M)
constexpr int kLineBytes = 128;      // K bytes of one operand line per stage
constexpr int kProducerWarps = 8;
constexpr int kProducers = kProducerWarps * 32;
constexpr int kGemmThreads = kProducers + 32;  // + the MMA warp
constexpr int kGemmSmemBudget = 200 * 1024;
constexpr int kMaxStages = 8;

enum GemmMode : int { kPure16 = 0, kTf32x2 = 1, kTf32x3 = 2 };

struct GemmArgs {
    const void* a_hi;
    const void* a_lo;
    int64_t a_si, a_sl;  // op(A)(i, l) is element i * a_si + l * a_sl
    const float* b;
    int64_t b_sl, b_sj;  // op(B)(l, j) is element l * b_sl + j * b_sj
    float* c;
    int64_t c_si, c_sj;  // C(i, j) is element i * c_si + j * c_sj
    int64_t M, N, K;
    double alpha, beta;
    int a_kc, b_kc;    // 1: the operand's lines run along K (else along M / N)
    int a_vec, b_vec;  // 1: 16-byte (or 8-byte) vector loads are aligned
    int bn;            // columns of op(B) per CTA: 16, 32, 64 or 128
    int stages;        // operand stages
    int raw_stages;    // raw (copied) stages of the TMA-fed pipeline
    int kt_per;        // K-tiles per split of K (blockIdx.z); all of them when unsplit
    int direct_a;      // TMA pipeline, 16-bit operands, K-contiguous A: the MMA reads A from the raw ring
    float* part;       // split K: FP32 partial sums [split][N][M] (NULL: write C)
    int* err;
};

template <int MODE>
struct ModeTraits {
    static constexpr int esz = MODE == kPure16 ? 2 : 4;  // operand bytes
    static constexpr int epu = 16 / esz;                  // elements per 16-byte unit
    static constexpr int kpl = kLineBytes / esz;          // K per stage
    static constexpr int na = MODE == kTf32x3 ? 2 : 1;    // A operand tiles
    static constexpr int nb = MODE == kPure16 ? 1 : 2;    // B operand tiles
};

// ---------------------------------------------------------------- PTX

__device__ __forceinline__ uint32_t tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// A value and its TF32 remainder: x = big + small up to 2^-22 |x|.
__device__ __forceinline__ void split_tf32(float x, uint32_t& big, uint32_t& small) {
    big = tf32_rn(x);
    small = tf32_rn(x - u2f(big));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // start address, leading (K-direction) and stride (MN-direction) core
    // matrix offsets in 16-byte units; version 1 (sm_100); no swizzle.
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_issue(int kind_tf32, uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                          uint32_t acc) {
    if (kind_tf32) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
    } else {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
    }
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    // the load and its wait in one statement: nothing reads r before the wait
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr)
        : "memory");
}

// ---------------------------------------------------------- element decode

// A 16-bit element (raw bits h, r of the two planes) as a float.
template <Elem E>
__device__ __forceinline__ float decode16(uint32_t h, uint32_t r) {
    if constexpr (E == Elem::H16) return half_bits_to_float(half_only_bits(h));
    else if constexpr (E == Elem::F16) return half_bits_to_float(h);
    else if constexpr (E == Elem::B16) return u2f(h << 16);
    else if constexpr (E == Elem::A16) return decode_fp32_16_exact(h, r);
    else if constexpr (E == Elem::AB16) return decode_fp32_bf16_exact(h, r, false);
    else return decode_fp32_bf16_exact(h, r, true);  // AB16R
}

// The 16-bit operand bits of a HALF-tier element (fp16, or bf16 for B16).
template <Elem E>
__device__ __forceinline__ uint32_t bits16(uint32_t h) {
    if constexpr (E == Elem::H16) return half_only_bits(h);
    else return h;  // F16, B16
}

template <Elem E>
__host__ __device__ constexpr bool two_planes() {
    return E == Elem::A16 || E == Elem::AB16 || E == Elem::AB16R;
}

// Scalar element of op(A) (0 outside) as a float / as 16-bit operand bits.
template <Elem E>
__device__ __forceinline__ float a_scalar(const GemmArgs& g, int64_t i, int64_t l) {
    if (i >= g.M || l >= g.K) return 0.0f;
    const size_t idx = (size_t)(i * g.a_si + l * g.a_sl);
    if constexpr (E == Elem::F32) return __ldg(static_cast<const float*>(g.a_hi) + idx);
    else {
        const uint32_t h = __ldg(static_cast<const unsigned short*>(g.a_hi) + idx);
        uint32_t r = 0;
        if constexpr (two_planes<E>()) r = __ldg(static_cast<const unsigned short*>(g.a_lo) + idx);
        return decode16<E>(h, r);
    }
}

template <Elem E>
__device__ __forceinline__ uint32_t a_scalar16(const GemmArgs& g, int64_t i, int64_t l) {
    if (i >= g.M || l >= g.K) return 0u;
    const size_t idx = (size_t)(i * g.a_si + l * g.a_sl);
    return bits16<E>(__ldg(static_cast<const unsigned short*>(g.a_hi) + idx));
}

__device__ __forceinline__ float b_scalar(const GemmArgs& g, int64_t l, int64_t j) {
    if (l >= g.K || j >= g.N) return 0.0f;
    return __ldg(g.b + (size_t)(l * g.b_sl + j * g.b_sj));
}

template <bool BF>
__device__ __forceinline__ uint32_t to16(float x) {
    if constexpr (BF) return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x));
    else return (uint32_t)__half_as_ushort(__float2half_rn(x));
}

// ---------------------------------------------------------- operand tiles
//
// A tile holds R lines (rows of op(A), or columns of op(B)) x 128 bytes of
// K, K-major, as 128-byte core matrices (8 lines x 16 bytes): unit (line
// r, K chunk u of 16 bytes) at ((u * R/8 + r/8) * 8 + r % 8) * 16 bytes.
// The MN-direction core stride (SBO) is 128 bytes, the K-direction one
// (LBO) R/8 core matrices.  Eight consecutive lanes always write eight
// consecutive lines of one chunk: one 128-byte shared-memory wavefront.
// (Operands are K-major whatever their global layout: the TF32 products
// are issued from K-major tiles only.)

__device__ __forceinline__ uint32_t kmajor_off(int r, int u, int R) {
    return (uint32_t)(((u * (R >> 3) + (r >> 3)) * 8 + (r & 7)) * 16);
}

// Writes op(A) rows [m0, m0 + 128) x K [k0, k0 + kpl) into tile(s) t0 (and
// t1: the TF32 remainders for kTf32x3).
template <Elem E, int MODE>
__device__ __forceinline__ void produce_a(const GemmArgs& g, uint8_t* t0, uint8_t* t1, int64_t m0, int64_t k0,
                                          int pt) {
    using T = ModeTraits<MODE>;
    constexpr int R = kGemmM;
    constexpr int items = R * 8;
    for (int it = pt; it < items; it += kProducers) {
        float v[8];
        uint32_t b16[8];
        int r, u;  // line, 16-byte K chunk
        uint32_t off;
        if (g.a_kc) {
            r = (it & 7) | ((it >> 6) << 3);
            u = (it >> 3) & 7;
            off = kmajor_off(r, u, R);
            const int64_t i = m0 + r, l = k0 + (int64_t)u * T::epu;
            const bool full = g.a_vec && i < g.M && l + T::epu <= g.K;
            const size_t idx = (size_t)(i * g.a_si + l);
            if constexpr (MODE == kPure16) {
                if (full) {
                    const uint4 h = __ldg(reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(g.a_hi) + idx));
                    const uint32_t w[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        b16[2 * e] = bits16<E>(w[e] & 0xFFFFu);
                        b16[2 * e + 1] = bits16<E>(w[e] >> 16);
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) b16[e] = a_scalar16<E>(g, i, l + e);
                }
            } else if constexpr (E == Elem::F32) {
                if (full) {
                    const float4 f = __ldg(reinterpret_cast<const float4*>(static_cast<const float*>(g.a_hi) + idx));
                    v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) v[e] = a_scalar<E>(g, i, l + e);
                }
            } else {
                if (full) {
                    const uint2 h = __ldg(reinterpret_cast<const uint2*>(static_cast<const uint16_t*>(g.a_hi) + idx));
                    uint2 q = make_uint2(0u, 0u);
                    if constexpr (two_planes<E>())
                        q = __ldg(reinterpret_cast<const uint2*>(static_cast<const uint16_t*>(g.a_lo) + idx));
                    v[0] = decode16<E>(h.x & 0xFFFFu, q.x & 0xFFFFu);
                    v[1] = decode16<E>(h.x >> 16, q.x >> 16);
                    v[2] = decode16<E>(h.y & 0xFFFFu, q.y & 0xFFFFu);
                    v[3] = decode16<E>(h.y >> 16, q.y >> 16);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) v[e] = a_scalar<E>(g, i, l + e);
                }
            }
        } else {
            // lines strided along K (op(A) contiguous along M): consecutive
            // lanes take consecutive lines, so each of the unit's scalar
            // loads is one coalesced access across the warp
            r = it % R;
            u = it / R;
            off = kmajor_off(r, u, R);
            const int64_t i = m0 + r, l = k0 + (int64_t)u * T::epu;
            if constexpr (MODE == kPure16) {
#pragma unroll
                for (int e = 0; e < 8; ++e) b16[e] = a_scalar16<E>(g, i, l + e);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) v[e] = a_scalar<E>(g, i, l + e);
            }
        }
        (void)r;
        (void)u;
        if constexpr (MODE == kPure16) {
            uint4 w;
            w.x = b16[0] | (b16[1] << 16);
            w.y = b16[2] | (b16[3] << 16);
            w.z = b16[4] | (b16[5] << 16);
            w.w = b16[6] | (b16[7] << 16);
            *reinterpret_cast<uint4*>(t0 + off) = w;
        } else if constexpr (MODE == kTf32x2) {
            // 16-bit values are exact in TF32
            *reinterpret_cast<uint4*>(t0 + off) = make_uint4(f2u(v[0]), f2u(v[1]), f2u(v[2]), f2u(v[3]));
        } else {
            uint32_t bg[4], sm[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) split_tf32(v[e], bg[e], sm[e]);
            *reinterpret_cast<uint4*>(t0 + off) = make_uint4(bg[0], bg[1], bg[2], bg[3]);
            *reinterpret_cast<uint4*>(t1 + off) = make_uint4(sm[0], sm[1], sm[2], sm[3]);
        }
    }
}

// Writes op(B) columns [n0, n0 + bn) x K [k0, k0 + kpl): t0 (the TF32 big
// parts, or the 16-bit values) and t1 (TF32 remainders).
template <int MODE, bool BF>
__device__ __forceinline__ void produce_b(const GemmArgs& g, uint8_t* t0, uint8_t* t1, int64_t n0, int64_t k0,
                                          int pt) {
    using T = ModeTraits<MODE>;
    const int R = g.bn;
    const int items = R * 8;
    for (int it = pt; it < items; it += kProducers) {
        float v[8];
        uint32_t off;
        if (g.b_kc) {
            const int r = (it & 7) | ((it >> 6) << 3);
            const int u = (it >> 3) & 7;
            off = kmajor_off(r, u, R);
            const int64_t j = n0 + r, l = k0 + (int64_t)u * T::epu;
            const bool full = g.b_vec && j < g.N && l + T::epu <= g.K;
            const float* p = g.b + (size_t)(j * g.b_sj + l);
            if (full) {
                const float4 f = __ldg(reinterpret_cast<const float4*>(p));
                v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
                if constexpr (T::epu == 8) {
                    const float4 f2 = __ldg(reinterpret_cast<const float4*>(p) + 1);
                    v[4] = f2.x; v[5] = f2.y; v[6] = f2.z; v[7] = f2.w;
                }
            } else {
#pragma unroll
                for (int e = 0; e < T::epu; ++e) v[e] = b_scalar(g, l + e, j);
            }
        } else {
            // lines strided along K: consecutive lanes, consecutive columns
            const int r = it % R, u = it / R;
            off = kmajor_off(r, u, R);
            const int64_t j = n0 + r, l = k0 + (int64_t)u * T::epu;
#pragma unroll
            for (int e = 0; e < T::epu; ++e) v[e] = b_scalar(g, l + e, j);
        }
        if constexpr (MODE == kPure16) {
            uint4 w;
            w.x = to16<BF>(v[0]) | (to16<BF>(v[1]) << 16);
            w.y = to16<BF>(v[2]) | (to16<BF>(v[3]) << 16);
            w.z = to16<BF>(v[4]) | (to16<BF>(v[5]) << 16);
            w.w = to16<BF>(v[6]) | (to16<BF>(v[7]) << 16);
            *reinterpret_cast<uint4*>(t0 + off) = w;
        } else {
            uint32_t bg[4], sm[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) split_tf32(v[e], bg[e], sm[e]);
            *reinterpret_cast<uint4*>(t0 + off) = make_uint4(bg[0], bg[1], bg[2], bg[3]);
            *reinterpret_cast<uint4*>(t1 + off) = make_uint4(sm[0], sm[1], sm[2], sm[3]);
        }
    }
}

// Descriptor of MMA K-step s (32 bytes of K: two 16-byte chunks) of a tile.
__device__ __forceinline__ uint64_t tile_desc(uint32_t base, int s, int R) {
    const uint32_t lbo = (uint32_t)(R >> 3) * 128u;
    return smem_desc(base + (uint32_t)(2 * s) * lbo, lbo, 128u);
}

// The MMA issuer (one thread): per stage, 4 K-steps x the mode's terms,
// then a commit that frees the stage; a final commit marks the
// accumulator complete (or the work stopped).
// A descriptor of K-step s (32 bytes of K) of a 128-byte-swizzled K-major
// tile as the copy engine writes it: 8-row atoms of 128-byte rows, atoms
// 1024 bytes apart (SBO), the step's 32 bytes at +32 s within each row
// (layout type 2 = 128-byte swizzle; LBO unused for swizzled K-major).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t base, int s) {
    return smem_desc(base + 32u * (uint32_t)s, 16u, 1024u) | (2ull << 61);
}

// The MMA issuer (one thread): per stage, 4 K-steps x the mode's terms,
// then a commit that frees the stage; a final commit marks the
// accumulator complete (or the work stopped).  raw != NULL (16-bit
// operands, K-contiguous A): A is read straight from the raw ring the copy
// engine filled (128-byte swizzle), and a second commit frees that raw
// stage.
template <int MODE, bool BF>
__device__ __forceinline__ void gemm_issue_mmas(const GemmArgs& g, uint8_t* ops, uint32_t stage_bytes,
                                                uint32_t a_bytes, uint32_t b_bytes, uint64_t* full, uint64_t* empty,
                                                uint64_t* done, uint32_t tmem, int nk, volatile int* abort_flag,
                                                const uint8_t* raw = nullptr, uint32_t raw_bytes = 0,
                                                uint64_t* rempty = nullptr) {
    using T = ModeTraits<MODE>;
    const int S = g.stages, BN = g.bn;
    uint32_t idesc = (1u << 4);  // FP32 accumulator
    const uint32_t fmt = MODE == kPure16 ? (BF ? 1u : 0u) : 2u;
    idesc |= fmt << 7;
    idesc |= fmt << 10;
    // bits 15, 16 (A, B major) stay 0: K-major operands
    idesc |= ((uint32_t)BN >> 3) << 17;
    idesc |= ((uint32_t)kGemmM >> 4) << 24;
    uint32_t acc = 0;
    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % S;
        if (!mbar_wait(&full[s], (uint32_t)((kt / S) & 1))) {
            atomicExch(g.err, 2);
            *abort_flag = 1;
        }
        if (*abort_flag) break;
        tc_fence_after();
        const uint32_t st = smem_addr(ops + (size_t)s * stage_bytes);
        const uint32_t a0 = st, a1 = st + a_bytes;
        const uint32_t b0 = raw ? st : st + T::na * a_bytes, b1 = b0 + b_bytes;
        const int rs = raw ? kt % g.raw_stages : 0;
        const uint32_t ra = raw ? smem_addr(raw + (size_t)rs * raw_bytes) : 0u;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const uint64_t da0 = raw ? sw128_desc(ra, ks) : tile_desc(a0, ks, kGemmM);
            const uint64_t db0 = tile_desc(b0, ks, BN);
            mma_issue(MODE != kPure16, tmem, da0, db0, idesc, acc);
            acc = 1;
            if constexpr (MODE != kPure16) {
                const uint64_t db1 = tile_desc(b1, ks, BN);
                mma_issue(1, tmem, da0, db1, idesc, 1);
            }
            if constexpr (MODE == kTf32x3) {
                const uint64_t da1 = tile_desc(a1, ks, kGemmM);
                mma_issue(1, tmem, da1, db0, idesc, 1);
            }
        }
        mma_commit(&empty[s]);  // frees the stage once these MMAs are done
        if (raw) mma_commit(&rempty[rs]);
    }
    mma_commit(done);
}

// Epilogue: worker warp w (of NW) reads TMEM lanes 32 (w % 4) .. + 31
// (rows of the tile) and every (NW / 4)-th 8-column chunk from chunk w / 4,
// and writes alpha acc + beta C; the MMA warp (warp NW) waits for its own
// MMAs before the memory is freed.
template <int NW>
__device__ __forceinline__ void gemm_epilogue(const GemmArgs& g, int warp, int lane, int64_t m0, int64_t n0,
                                              uint32_t tmem, uint64_t* done, volatile int* abort_flag) {
    float* part = g.part ? g.part + (size_t)blockIdx.z * (size_t)g.M * (size_t)g.N : nullptr;
    const int BN = g.bn;
    if (warp < NW) {
        if (!mbar_wait(done, 0u)) {
            if (lane == 0) atomicExch(g.err, 3);
            *abort_flag = 1;
        }
        tc_fence_after();
        const int q = warp & 3, h = warp >> 2;
        const int64_t i = m0 + q * 32 + lane;
        const bool ok = !*abort_flag;
        for (int c = h * 8; c < BN; c += (NW / 4) * 8) {
            uint32_t r[8];
            tmem_ld8(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c, r);
            if (!ok || i >= g.M) continue;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int64_t j = n0 + c + e;
                if (j >= g.N) break;
                if (part) {  // split K: this split's raw sum
                    part[(size_t)(j * g.M + i)] = u2f(r[e]);
                    continue;
                }
                float* cp = g.c + (size_t)(i * g.c_si + j * g.c_sj);
                double y = g.alpha * (double)u2f(r[e]);
                if (g.beta != 0.0) y += g.beta * (double)*cp;
                *cp = (float)y;
            }
        }
    } else if (warp == NW) {
        if (!mbar_wait(done, 0u) && lane == 0) atomicExch(g.err, 4);
    }
}

template <Elem E, int MODE>
__global__ void __launch_bounds__(kGemmThreads, 1) gemm_tc_kernel(GemmArgs g) {
    using T = ModeTraits<MODE>;
    constexpr bool BF = (E == Elem::B16);
    extern __shared__ __align__(1024) uint8_t smem[];
    const int S = g.stages, BN = g.bn;
    const uint32_t a_bytes = kGemmM * kLineBytes, b_bytes = (uint32_t)BN * kLineBytes;
    const uint32_t stage_bytes = T::na * a_bytes + T::nb * b_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * stage_bytes);
    uint64_t* empty = full + kMaxStages;
    uint64_t* done = empty + kMaxStages;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t m0 = (int64_t)blockIdx.x * kGemmM, n0 = (int64_t)blockIdx.y * BN;
    const int nk_all = (int)((g.K + T::kpl - 1) / T::kpl);
    const int kt0 = (int)blockIdx.z * g.kt_per;  // this split's first K-tile (the host gives each >= 1)
    const int nk = nk_all - kt0 < g.kt_per ? nk_all - kt0 : g.kt_per;
    const uint32_t ncols = BN <= 32 ? 32u : (uint32_t)BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], kProducerWarps);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == kProducerWarps) {  // the MMA warp owns the tensor memory
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp < kProducerWarps) {
        const int pt = threadIdx.x;
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % S;
            if (kt >= S && !mbar_wait(&empty[s], (uint32_t)((kt / S - 1) & 1))) {
                if (lane == 0) atomicExch(g.err, 1);
                *abort_flag = 1;
            }
            if (*abort_flag) break;
            uint8_t* st = smem + (size_t)s * stage_bytes;
            const int64_t k0 = (int64_t)(kt0 + kt) * T::kpl;
            produce_a<E, MODE>(g, st, st + a_bytes, m0, k0, pt);
            uint8_t* bt = st + T::na * a_bytes;
            produce_b<MODE, BF>(g, bt, bt + b_bytes, n0, k0, pt);
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&full[s]);
        }
    } else if (lane == 0) {
        gemm_issue_mmas<MODE, BF>(g, smem, stage_bytes, a_bytes, b_bytes, full, empty, done, tmem, nk, abort_flag);
    }
    gemm_epilogue<kProducerWarps>(g, warp, lane, m0, n0, tmem, done, abort_flag);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kProducerWarps)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// ------------------------------------------------------- TMA-fed pipeline
//
// When the operands' lines are 16-byte aligned (base and stride), one
// thread streams them with 2-D tensor copies (cp.async.bulk.tensor, zero
// fill past the edges) into a ring of raw stages, and the 8 producer warps
// become converters: raw shared memory -> decoded, split operand tiles.
// Raw tiles of K-contiguous lines are swizzled by the copy (128-byte rows:
// 16-byte chunk c of row r lands at chunk c ^ (r % 8); 64-byte rows: chunk
// c ^ ((r / 2) % 4)), so eight converter lanes reading one chunk of eight
// consecutive lines hit eight different bank groups; raw tiles of
// M- (N-) contiguous lines are stored k-row by k-row.

struct GemmMaps {
    CUtensorMap a_hi, a_lo, b;
};

constexpr int kConvWarps = 16;                   // converter warps
constexpr int kConv = kConvWarps * 32;
constexpr int kTmaThreads = kConv + 64;          // + the MMA warp + the copy warp
constexpr int kMmaWarp = kConvWarps, kCopyWarp = kConvWarps + 1;
constexpr int kConvItems = kGemmM * 8 / kConv;   // A units a converter thread owns (2)

__device__ __forceinline__ void tma2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

template <Elem E, int MODE>
struct RawTraits {
    using T = ModeTraits<MODE>;
    static constexpr int es = E == Elem::F32 ? 4 : 2;               // source bytes
    static constexpr int row = T::kpl * es;                           // bytes of a K-line
    static constexpr int a_plane = kGemmM * row;                      // one plane of A
    static constexpr int planes = two_planes<E>() ? 2 : 1;
    static constexpr int a_bytes = a_plane * planes;
};

// The 16-bit HALF-tier operand bits of 8 FP32_16 / FP16 / bf16 words:
// control-0 FP32_16 words are fp16 already, so only flagged words (bit 0,
// about 0.35 % of them) go through half_only_bits, one at a time.
template <Elem E>
__device__ __forceinline__ uint4 half_operands(uint4 h) {
    if constexpr (E == Elem::H16) {
        uint32_t m = (h.x & 0x10001u) | ((h.y & 0x10001u) << 1) | ((h.z & 0x10001u) << 2) | ((h.w & 0x10001u) << 3);
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            const int e = b & 3, sh = b & 16;
            uint32_t w = e == 0 ? h.x : e == 1 ? h.y : e == 2 ? h.z : h.w;
            const uint32_t fixed = half_only_bits((w >> sh) & 0xFFFFu);
            w = (w & ~(0xFFFFu << sh)) | (fixed << sh);
            if (e == 0) h.x = w;
            else if (e == 1) h.y = w;
            else if (e == 2) h.z = w;
            else h.w = w;
        }
    }
    return h;
}

template <bool BF>
__device__ __forceinline__ uint32_t pack16x2(float a, float b) {
    if constexpr (BF) {
        const __nv_bfloat162 t = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&t);
    } else {
        const __half2 t = __floats2half2_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&t);
    }
}

// Converts one raw stage into the operand tiles of one stage.  ra_off /
// rb_off: each owned unit's byte offset in the raw tiles (first element
// for lines strided along K), oa_off / ob_off: in the operand tiles.
template <Elem E, int MODE, bool BF>
__device__ __forceinline__ void convert_stage(const GemmArgs& g, const uint8_t* ra, const uint8_t* rb, uint8_t* oa0,
                                              uint8_t* oa1, uint8_t* ob0, uint8_t* ob1, const uint32_t* ra_off,
                                              const uint32_t* oa_off, const uint32_t* rb_off,
                                              const uint32_t* ob_off, int nb_items, bool direct) {
    using T = ModeTraits<MODE>;
    using RT = RawTraits<E, MODE>;
    constexpr int R = kGemmM;
#pragma unroll
    for (int j = 0; j < kConvItems; ++j) {
        if (direct) break;  // the MMA reads A from the raw ring
        const uint8_t* src = ra + ra_off[j];
        if constexpr (MODE == kPure16) {
            uint4 h;
            if (g.a_kc) {
                h = *reinterpret_cast<const uint4*>(src);
            } else {
                const uint16_t* c = reinterpret_cast<const uint16_t*>(src);
                h.x = (uint32_t)c[0] | ((uint32_t)c[R] << 16);
                h.y = (uint32_t)c[2 * R] | ((uint32_t)c[3 * R] << 16);
                h.z = (uint32_t)c[4 * R] | ((uint32_t)c[5 * R] << 16);
                h.w = (uint32_t)c[6 * R] | ((uint32_t)c[7 * R] << 16);
            }
            *reinterpret_cast<uint4*>(oa0 + oa_off[j]) = half_operands<E>(h);
        } else {
            float v[4];
            if constexpr (E == Elem::F32) {
                if (g.a_kc) {
                    const float4 f = *reinterpret_cast<const float4*>(src);
                    v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
                } else {
                    const float* c = reinterpret_cast<const float*>(src);
#pragma unroll
                    for (int e = 0; e < 4; ++e) v[e] = c[e * R];
                }
            } else {
                uint32_t hw[4], lw[4] = {0u, 0u, 0u, 0u};
                if (g.a_kc) {
                    const uint2 h = *reinterpret_cast<const uint2*>(src);
                    hw[0] = h.x & 0xFFFFu; hw[1] = h.x >> 16; hw[2] = h.y & 0xFFFFu; hw[3] = h.y >> 16;
                    if constexpr (RT::planes == 2) {
                        const uint2 q = *reinterpret_cast<const uint2*>(src + RT::a_plane);
                        lw[0] = q.x & 0xFFFFu; lw[1] = q.x >> 16; lw[2] = q.y & 0xFFFFu; lw[3] = q.y >> 16;
                    }
                } else {
                    const uint16_t* c = reinterpret_cast<const uint16_t*>(src);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        hw[e] = c[e * R];
                        if constexpr (RT::planes == 2) lw[e] = c[e * R + RT::a_plane / 2];
                    }
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if constexpr (E == Elem::A16) v[e] = decode_fp32_16_exact_nb(hw[e], lw[e]);
                    else v[e] = decode16<E>(hw[e], lw[e]);
                }
            }
            if constexpr (MODE == kTf32x2) {
                *reinterpret_cast<uint4*>(oa0 + oa_off[j]) = make_uint4(f2u(v[0]), f2u(v[1]), f2u(v[2]), f2u(v[3]));
            } else {
                uint32_t bg[4], sm[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) split_tf32(v[e], bg[e], sm[e]);
                *reinterpret_cast<uint4*>(oa0 + oa_off[j]) = make_uint4(bg[0], bg[1], bg[2], bg[3]);
                *reinterpret_cast<uint4*>(oa1 + oa_off[j]) = make_uint4(sm[0], sm[1], sm[2], sm[3]);
            }
        }
    }
    const int BN = g.bn;
#pragma unroll
    for (int j = 0; j < kConvItems; ++j) {
        if (j >= nb_items) break;
        const uint8_t* src = rb + rb_off[j];
        float v[8];
        if (g.b_kc) {
            if constexpr (T::epu == 8) {
                // two 16-byte chunks of a 128-byte swizzled row: rb_off holds the
                // first; the second is chunk c0 + 1 ^ (r % 8), kept in bits 16+
                const float4 f0 = *reinterpret_cast<const float4*>(rb + (rb_off[j] & 0xFFFFu));
                const float4 f1 = *reinterpret_cast<const float4*>(rb + (rb_off[j] >> 16));
                v[0] = f0.x; v[1] = f0.y; v[2] = f0.z; v[3] = f0.w;
                v[4] = f1.x; v[5] = f1.y; v[6] = f1.z; v[7] = f1.w;
            } else {
                const float4 f = *reinterpret_cast<const float4*>(src);
                v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
            }
        } else {
            const float* c = reinterpret_cast<const float*>(src);
#pragma unroll
            for (int e = 0; e < T::epu; ++e) v[e] = c[e * BN];
        }
        if constexpr (MODE == kPure16) {
            *reinterpret_cast<uint4*>(ob0 + ob_off[j]) =
                make_uint4(pack16x2<BF>(v[0], v[1]), pack16x2<BF>(v[2], v[3]), pack16x2<BF>(v[4], v[5]),
                           pack16x2<BF>(v[6], v[7]));
        } else {
            uint32_t bg[4], sm[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) split_tf32(v[e], bg[e], sm[e]);
            *reinterpret_cast<uint4*>(ob0 + ob_off[j]) = make_uint4(bg[0], bg[1], bg[2], bg[3]);
            *reinterpret_cast<uint4*>(ob1 + ob_off[j]) = make_uint4(sm[0], sm[1], sm[2], sm[3]);
        }
    }
}

// 16-bit operands read straight from the raw ring: only FP32_16's flagged
// control words need their fp16 value, fixed in place (the order of the
// 16-byte chunks does not matter for an elementwise fix).
template <Elem E>
__device__ __forceinline__ void fix_raw_a(uint8_t* ra, int pt) {
    if constexpr (E == Elem::H16) {
        for (int c = pt; c < kGemmM * 8; c += kConv) {
            uint4* p = reinterpret_cast<uint4*>(ra) + c;
            const uint4 h = *p;
            if (((h.x | h.y | h.z | h.w) & 0x10001u) != 0u) *p = half_operands<E>(h);
        }
    }
}

// Unit (line r, 16-byte operand chunk u) of converter item `it`: eight
// consecutive lanes take eight consecutive lines of one chunk.
__device__ __forceinline__ void unit_of(int it, int R, bool kc, int& r, int& u) {
    if (kc) {
        r = (it & 7) | ((it >> 6) << 3);
        u = (it >> 3) & 7;
    } else {
        r = it % R;
        u = it / R;
    }
}

template <Elem E, int MODE>
__global__ void __launch_bounds__(kTmaThreads, 2) gemm_tma_kernel(GemmArgs g, const __grid_constant__ GemmMaps maps) {
    using T = ModeTraits<MODE>;
    using RT = RawTraits<E, MODE>;
    constexpr bool BF = (E == Elem::B16);
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte alignment for the 128-byte swizzle of the raw tiles
    uint8_t* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
    const int S = g.stages, RS = g.raw_stages, BN = g.bn;
    const uint32_t rb_bytes = (uint32_t)BN * T::kpl * 4u;
    const uint32_t raw_bytes = RT::a_bytes + rb_bytes;
    const uint32_t a_bytes = kGemmM * kLineBytes, b_bytes = (uint32_t)BN * kLineBytes;
    const bool direct = g.direct_a != 0;
    const uint32_t a_ops = direct ? 0u : T::na * a_bytes;  // A operand tiles in a stage
    const uint32_t stage_bytes = a_ops + T::nb * b_bytes;
    uint8_t* ops = smem + (size_t)RS * raw_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(ops + (size_t)S * stage_bytes);
    uint64_t* empty = full + kMaxStages;
    uint64_t* rfull = empty + kMaxStages;
    uint64_t* rempty = rfull + kMaxStages;
    uint64_t* done = rempty + kMaxStages;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t m0 = (int64_t)blockIdx.x * kGemmM, n0 = (int64_t)blockIdx.y * BN;
    const int nk_all = (int)((g.K + T::kpl - 1) / T::kpl);
    const int kt0 = (int)blockIdx.z * g.kt_per;  // this split's first K-tile (the host gives each >= 1)
    const int nk = nk_all - kt0 < g.kt_per ? nk_all - kt0 : g.kt_per;
    const uint32_t ncols = BN <= 32 ? 32u : (uint32_t)BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], kConvWarps);
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < RS; ++s) {
            mbar_init(&rfull[s], 1);
            mbar_init(&rempty[s], direct ? 1 : kConvWarps);  // direct: the MMA commit frees it
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp < kConvWarps) {
        const int pt = threadIdx.x;
        // the stage-invariant offsets of this thread's units
        uint32_t ra_off[kConvItems], oa_off[kConvItems], rb_off[kConvItems], ob_off[kConvItems];
#pragma unroll
        for (int j = 0; j < kConvItems; ++j) {
            int r, u;
            unit_of(pt + kConv * j, kGemmM, g.a_kc, r, u);
            oa_off[j] = kmajor_off(r, u, kGemmM);
            if (!g.a_kc) ra_off[j] = (uint32_t)((u * T::epu * kGemmM + r) * RT::es);
            else if (RT::row == 128) ra_off[j] = (uint32_t)(r * 128 + ((u ^ (r & 7)) << 4));
            else ra_off[j] = (uint32_t)(r * 64 + ((((u >> 1) ^ ((r >> 1) & 3)) << 4) | ((u & 1) << 3)));
        }
        const int nb_items = (BN * 8 - pt + kConv - 1) / kConv;
#pragma unroll
        for (int j = 0; j < kConvItems; ++j) {
            int r, u;
            unit_of(pt + kConv * j, BN, g.b_kc, r, u);
            ob_off[j] = kmajor_off(r, u, BN);
            if (!g.b_kc) {
                rb_off[j] = (uint32_t)((u * T::epu * BN + r) * 4);
            } else if (T::epu == 8) {
                const uint32_t base = (uint32_t)((u >> 2) * BN * 128 + r * 128);
                const int c0 = 2 * (u & 3);
                rb_off[j] = (base + ((c0 ^ (r & 7)) << 4)) | ((base + (((c0 + 1) ^ (r & 7)) << 4)) << 16);
            } else {
                rb_off[j] = (uint32_t)(r * 128 + ((u ^ (r & 7)) << 4));
            }
        }
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % S, rs = kt % RS;
            bool ok = mbar_wait(&rfull[rs], (uint32_t)((kt / RS) & 1));
            if (ok && kt >= S) ok = mbar_wait(&empty[s], (uint32_t)((kt / S - 1) & 1));
            if (!ok) {
                if (lane == 0) atomicExch(g.err, 1);
                *abort_flag = 1;
            }
            if (*abort_flag) break;
            uint8_t* ra = smem + (size_t)rs * raw_bytes;
            uint8_t* st = ops + (size_t)s * stage_bytes;
            uint8_t* bt = st + a_ops;
            if (direct) fix_raw_a<E>(ra, pt);
            convert_stage<E, MODE, BF>(g, ra, ra + RT::a_bytes, st, st + a_bytes, bt, bt + b_bytes, ra_off, oa_off,
                                       rb_off, ob_off, nb_items, direct);
            fence_async_smem();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&full[s]);
                if (!direct) mbar_arrive(&rempty[rs]);
            }
        }
    } else if (warp == kCopyWarp) {
        if (lane == 0) {
            int issued = 0;
            for (int kt = 0; kt < nk; ++kt) {
                const int rs = kt % RS;
                if (kt >= RS && !mbar_wait(&rempty[rs], (uint32_t)((kt / RS - 1) & 1))) {
                    atomicExch(g.err, 5);
                    *abort_flag = 1;
                }
                if (*abort_flag) break;
                const uint32_t ra = smem_addr(smem + (size_t)rs * raw_bytes);
                const int k0 = (kt0 + kt) * T::kpl;
                mbar_expect_tx(&rfull[rs], raw_bytes);
                const int am = (int)m0, bn0 = (int)n0;
                if (g.a_kc) {
                    tma2d(ra, &maps.a_hi, k0, am, &rfull[rs]);
                    if constexpr (RT::planes == 2) tma2d(ra + RT::a_plane, &maps.a_lo, k0, am, &rfull[rs]);
                } else {
                    tma2d(ra, &maps.a_hi, am, k0, &rfull[rs]);
                    if constexpr (RT::planes == 2) tma2d(ra + RT::a_plane, &maps.a_lo, am, k0, &rfull[rs]);
                }
                const uint32_t rbs = ra + RT::a_bytes;
                if (g.b_kc) {
                    tma2d(rbs, &maps.b, k0, bn0, &rfull[rs]);
                    if constexpr (T::kpl == 64) tma2d(rbs + (uint32_t)BN * 128u, &maps.b, k0 + 32, bn0, &rfull[rs]);
                } else {
                    tma2d(rbs, &maps.b, bn0, k0, &rfull[rs]);
                }
                issued = kt + 1;
            }
            // no copy may still be writing this CTA's memory when it exits
            for (int kt = issued > RS ? issued - RS : 0; kt < issued; ++kt)
                if (!mbar_wait(&rfull[kt % RS], (uint32_t)((kt / RS) & 1))) atomicExch(g.err, 6);
        }
    } else if (lane == 0) {
        gemm_issue_mmas<MODE, BF>(g, ops, stage_bytes, a_bytes, b_bytes, full, empty, done, tmem, nk, abort_flag,
                                  direct ? smem : nullptr, raw_bytes, rempty);
    }
    gemm_epilogue<kConvWarps>(g, warp, lane, m0, n0, tmem, done, abort_flag);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// The word a bounded wait of these launches records its expiry in.
__device__ int g_gemm_err;
constexpr int kMaxDevices = 64;

int* gemm_err_word() {
    static std::mutex mu;
    static int* addr[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_gemm_err) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        addr[dev] = static_cast<int*>(p);
    }
    return addr[dev];
}

template <int MODE>
int stage_count(int bn) {
    using T = ModeTraits<MODE>;
    const int stage = T::na * kGemmM * kLineBytes + T::nb * bn * kLineBytes;
    int s = (kGemmSmemBudget - 1024) / stage;
    return s > kMaxStages ? kMaxStages : s;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// A 2-D map of `outer` lines of `inner` elements, line stride `stride`
// elements; false when the copy engine cannot address it (16-byte base and
// stride) or the driver refuses it.
bool encode_2d(CUtensorMap* map, CUtensorMapDataType dt, int es, const void* base, int64_t inner, int64_t outer,
               int64_t stride, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle sw) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || !base || reinterpret_cast<uintptr_t>(base) % 16 != 0 || (stride * es) % 16 != 0) return false;
    if (stride < inner) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)(stride * es)};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <Elem E, int MODE>
bool make_maps(const GemmArgs& g, GemmMaps* maps) {
    using T = ModeTraits<MODE>;
    using RT = RawTraits<E, MODE>;
    const CUtensorMapDataType adt = E == Elem::F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    const CUtensorMapSwizzle ksw = RT::row == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
    const void* planes[2] = {g.a_hi, g.a_lo};
    CUtensorMap* amaps[2] = {&maps->a_hi, &maps->a_lo};
    for (int p = 0; p < RT::planes; ++p) {
        const bool ok = g.a_kc ? encode_2d(amaps[p], adt, RT::es, planes[p], g.K, g.M, g.a_si, T::kpl, kGemmM, ksw)
                               : encode_2d(amaps[p], adt, RT::es, planes[p], g.M, g.K, g.a_sl, kGemmM, T::kpl,
                                           CU_TENSOR_MAP_SWIZZLE_NONE);
        if (!ok) return false;
    }
    if (RT::planes == 1) maps->a_lo = maps->a_hi;
    return g.b_kc ? encode_2d(&maps->b, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, g.b, g.K, g.N, g.b_sj, 32, (uint32_t)g.bn,
                              CU_TENSOR_MAP_SWIZZLE_128B)
                  : encode_2d(&maps->b, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, g.b, g.N, g.K, g.b_sl, (uint32_t)g.bn,
                              T::kpl, CU_TENSOR_MAP_SWIZZLE_NONE);
}

constexpr int kTmaSmemBudget = 224 * 1024;
constexpr int kTmaSmemTwo = 112 * 1024;  // two CTAs an SM (228 KB, 1 KB reserved a CTA)

template <Elem E, int MODE>
tomos_status launch_gemm(GemmArgs& g, cudaStream_t st) {
    using T = ModeTraits<MODE>;
    using RT = RawTraits<E, MODE>;
    const int nk_all = (int)((g.K + T::kpl - 1) / T::kpl);
    const dim3 grid((unsigned)((g.M + kGemmM - 1) / kGemmM), (unsigned)((g.N + g.bn - 1) / g.bn),
                    (unsigned)((nk_all + g.kt_per - 1) / g.kt_per));
    const size_t stage = (size_t)T::na * kGemmM * kLineBytes + (size_t)T::nb * g.bn * kLineBytes;
    const size_t bars = (5 * kMaxStages + 1) * sizeof(uint64_t) + 16;
    GemmMaps maps;
    if (make_maps<E, MODE>(g, &maps)) {
        const size_t raw = (size_t)RT::a_bytes + (size_t)g.bn * T::kpl * 4;
        // 16-bit operands with K-contiguous A: the copy's 128-byte-swizzled
        // tile is the MMA's A operand, no A tile in the operand stages
        g.direct_a = (MODE == kPure16 && g.a_kc && RT::row == 128) ? 1 : 0;
        const size_t tstage = g.direct_a ? (size_t)T::nb * g.bn * kLineBytes : stage;
        // operand and raw stages: the deepest rings that fit; with many
        // tiles, rings small enough for two CTAs an SM first, so that one
        // CTA's pipeline fill and epilogue overlap the other's main loop
        static const int pairs[][2] = {{2, 4}, {3, 3}, {2, 3}, {3, 2}, {2, 2}};
        const int64_t tiles = (int64_t)grid.x * grid.y * grid.z;
        const size_t budgets[2] = {tiles >= 2 * (int64_t)sm_count() ? (size_t)kTmaSmemTwo : 0,
                                   (size_t)kTmaSmemBudget};
        for (int pass = 0; pass < 2; ++pass)
        for (const auto& pr : pairs) {
            const size_t smem = (size_t)pr[0] * tstage + (size_t)pr[1] * raw + bars + 1024;
            if (smem > budgets[pass]) continue;
            g.stages = pr[0];
            g.raw_stages = pr[1];
            auto kern = gemm_tma_kernel<E, MODE>;
            TOMOS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            kern<<<grid, kTmaThreads, smem, st>>>(g, maps);
            TOMOS_LAUNCH_CHECK("gemm_tma_kernel");
            return TOMOS_OK;
        }
    }
    // direct loads (operands the copy engine cannot address)
    g.direct_a = 0;
    g.stages = stage_count<MODE>(g.bn);
    g.raw_stages = 0;
    if (g.stages < 2) return fail(TOMOS_ERR_UNSUPPORTED, "mm: shared memory");
    const size_t smem = (size_t)g.stages * stage + bars;
    auto kern = gemm_tc_kernel<E, MODE>;
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, kGemmThreads, smem, st>>>(g);
    TOMOS_LAUNCH_CHECK("gemm_tc_kernel");
    return TOMOS_OK;
}

template <int MODE>
tomos_status launch_mode(Elem e, GemmArgs& g, cudaStream_t st) {
    switch (e) {
        case Elem::H16: return launch_gemm<Elem::H16, MODE>(g, st);
        case Elem::F16: return launch_gemm<Elem::F16, MODE>(g, st);
        case Elem::B16: return launch_gemm<Elem::B16, MODE>(g, st);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "mm: element type");
    }
}

bool two_planes_elem(Elem e) { return e == Elem::A16 || e == Elem::AB16 || e == Elem::AB16R; }

// C = beta C (K == 0: op(A) op(B) is the zero matrix).
__global__ void gemm_scale_c_kernel(float* c, int64_t M, int64_t N, int64_t si, int64_t sj, double beta) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * N) return;
    const int64_t i = t % M, j = t / M;
    float* p = c + (size_t)(i * si + j * sj);
    *p = beta == 0.0 ? 0.0f : (float)(beta * (double)*p);
}

bool strides_of(const tomos_dense* D, int32_t trans, int64_t* s_row, int64_t* s_col) {
    // op(D)(r, c): element r * s_row + c * s_col
    int64_t sr = D->layout == TOMOS_COL_MAJOR ? 1 : D->ld;
    int64_t sc = D->layout == TOMOS_COL_MAJOR ? D->ld : 1;
    if (trans == TOMOS_TRANSPOSE) std::swap(sr, sc);
    *s_row = sr;
    *s_col = sc;
    return true;
}

}  // namespace

}  // namespace tomos_b200

using namespace tomos_b200;

namespace tomos_b200 {
namespace {

// C(i, j) = alpha sum_z part[z](i, j) + beta C(i, j), the splits summed in
// FP64 in split order (deterministic).
__global__ void gemm_split_reduce_kernel(const float* __restrict__ part, int splits, int64_t M, int64_t N,
                                         double alpha, double beta, float* c, int64_t si, int64_t sj) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * N) return;
    const int64_t i = t % M, j = t / M;
    double s = 0.0;
    for (int z = 0; z < splits; ++z) s += (double)part[(size_t)z * M * N + t];
    float* p = c + (size_t)(i * si + j * sj);
    double y = alpha * s;
    if (beta != 0.0) y += beta * (double)*p;
    *p = (float)y;
}

// Validates a product and fills the launch arguments (all but the split).
tomos_status mm_prepare(int32_t trans_a, int32_t trans_b, double alpha, const tomos_dense* A, int32_t tier,
                        const tomos_dense* B, double beta, const tomos_dense* C, GemmArgs* gp, Elem* ep, int* modep) {
    if (!A || !B || !C) return fail(TOMOS_ERR_INVALID, "mm: null matrix");
    if ((trans_a != TOMOS_NO_TRANSPOSE && trans_a != TOMOS_TRANSPOSE) ||
        (trans_b != TOMOS_NO_TRANSPOSE && trans_b != TOMOS_TRANSPOSE))
        return fail(TOMOS_ERR_INVALID, "mm: bad transpose");
    if (B->numeric != TOMOS_FP32 || C->numeric != TOMOS_FP32)
        return fail(TOMOS_ERR_UNSUPPORTED, "mm: B and C must be FP32 (dense_registries.cpp:396-405)");
    for (const tomos_dense* D : {A, B, C}) {
        if (D->rows < 0 || D->cols < 0) return fail(TOMOS_ERR_INVALID, "mm: negative size");
        if (D->layout != TOMOS_ROW_MAJOR && D->layout != TOMOS_COL_MAJOR)
            return fail(TOMOS_ERR_INVALID, "mm: bad layout");
        const int64_t inner = D->layout == TOMOS_ROW_MAJOR ? D->cols : D->rows;
        if (D->rows > 0 && D->cols > 0 && D->ld < inner)
            return fail(TOMOS_ERR_INVALID, "mm: leading dimension too small");
    }
    const int64_t M = trans_a == TOMOS_NO_TRANSPOSE ? A->rows : A->cols;
    const int64_t K = trans_a == TOMOS_NO_TRANSPOSE ? A->cols : A->rows;
    const int64_t Kb = trans_b == TOMOS_NO_TRANSPOSE ? B->rows : B->cols;
    const int64_t N = trans_b == TOMOS_NO_TRANSPOSE ? B->cols : B->rows;
    if (Kb != K || C->rows != M || C->cols != N) return fail(TOMOS_ERR_INVALID, "mm: size mismatch");
    // the operand tier: HALF_OPERANDS (16-bit A and B), HALF (16-bit A,
    // ~FP32 B), exact (FP32 or ACCURATE)
    const bool ops16 = tier == TOMOS_TIER_HALF_OPERANDS;
    int32_t rt = tier;
    if (ops16) rt = A->numeric == TOMOS_FP16 ? TOMOS_TIER_NATIVE : TOMOS_TIER_HALF;
    Elem e;
    std::string why;
    if (!resolve_elem(A, rt, &e, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "mm: " + why);
    const bool e16 = e == Elem::H16 || e == Elem::F16 || e == Elem::B16;
    if (ops16 && !e16) return fail(TOMOS_ERR_UNSUPPORTED, "mm: 16-bit operands need 16-bit A values");
    if (e == Elem::F64) return fail(TOMOS_ERR_UNSUPPORTED, "mm: FP64 A");
    GemmArgs& g = *gp;
    std::memset(&g, 0, sizeof(g));
    g.a_hi = A->values;
    g.a_lo = two_planes_elem(e) ? dense_lo_plane(A) : nullptr;
    strides_of(A, trans_a, &g.a_si, &g.a_sl);
    g.b = static_cast<const float*>(B->values);
    strides_of(B, trans_b, &g.b_sl, &g.b_sj);
    g.c = static_cast<float*>(C->values);
    strides_of(C, TOMOS_NO_TRANSPOSE, &g.c_si, &g.c_sj);
    g.M = M;
    g.N = N;
    g.K = K;
    g.alpha = alpha;
    g.beta = beta;
    g.bn = N <= 16 ? 16 : N <= 32 ? 32 : N <= 64 ? 64 : 128;
    // one of the two strides of a dense operand is 1: lines run along K
    // when the K stride is
    g.a_kc = g.a_sl == 1 ? 1 : 0;
    g.b_kc = g.b_sl == 1 ? 1 : 0;
    const int mode = ops16 ? kPure16 : (e16 ? kTf32x2 : kTf32x3);
    // vector loads: unit stride along the line, 16-byte aligned lines
    const int aes = e == Elem::F32 ? 4 : 2;
    const int aepu = mode == kPure16 ? 8 : 4;
    const int64_t a_lstride = g.a_kc ? g.a_si : g.a_sl;
    const uintptr_t ab = reinterpret_cast<uintptr_t>(A->values);
    const uintptr_t al = reinterpret_cast<uintptr_t>(g.a_lo);
    const int avb = aepu * aes;  // vector bytes
    g.a_vec = ((g.a_kc ? g.a_sl : g.a_si) == 1) && (a_lstride * aes) % avb == 0 && ab % avb == 0 &&
              (!g.a_lo || al % avb == 0);
    const int64_t b_lstride = g.b_kc ? g.b_sj : g.b_sl;
    const uintptr_t bb = reinterpret_cast<uintptr_t>(B->values);
    g.b_vec = ((g.b_kc ? g.b_sl : g.b_sj) == 1) && (b_lstride * 4) % 16 == 0 && bb % 16 == 0;
    g.kt_per = 1 << 30;
    *ep = e;
    *modep = mode;
    return TOMOS_OK;
}

// Splits of K for products with too few output tiles to fill the SMs
// (e.g. A^T Q with a tall K): at least one CTA an SM, and runs of at most 16
// K-tiles (512 TF32 / 1024 16-bit terms) in one FP32 accumulator -- a
// coherent sum such as the diagonal of A^T A loses ~u x run length
// relative in FP32, so long K is cut into short runs that are summed in
// FP64.  Each split has at least 4 K-tiles.
int split_count(const GemmArgs& g, int mode, int* kt_per) {
    const int kpl = mode == kPure16 ? 64 : 32;
    const int64_t nk_all = (g.K + kpl - 1) / kpl;
    const int64_t tiles = ((g.M + kGemmM - 1) / kGemmM) * ((g.N + g.bn - 1) / g.bn);
    int64_t splits = 1;
    if (tiles < sm_count() / 2 && nk_all >= 16) {
        splits = sm_count() / tiles;
        const int64_t runs = (nk_all + 15) / 16;
        if (splits < runs) splits = runs;
        if (splits > nk_all / 4) splits = nk_all / 4;
        if (splits < 1) splits = 1;
    }
    const int64_t per = (nk_all + splits - 1) / splits;
    *kt_per = (int)per;
    return (int)((nk_all + per - 1) / per);
}

}  // namespace
}  // namespace tomos_b200

extern "C" {

size_t tomos_mm_scratch_bytes(int32_t trans_a, int32_t trans_b, const tomos_dense* A, int32_t tier,
                              const tomos_dense* B) {
    if (!A || !B) return 0;
    tomos_dense C{TOMOS_FP32, TOMOS_COL_MAJOR, trans_a == TOMOS_NO_TRANSPOSE ? A->rows : A->cols,
                  trans_b == TOMOS_NO_TRANSPOSE ? B->cols : B->rows, 0, nullptr, nullptr, 0, 0};
    C.ld = C.rows > 0 ? C.rows : 1;
    GemmArgs g;
    Elem e;
    int mode;
    if (mm_prepare(trans_a, trans_b, 1.0, A, tier, B, 0.0, &C, &g, &e, &mode) != TOMOS_OK) return 0;
    if (g.M == 0 || g.N == 0 || g.K == 0) return 0;
    int per;
    const int splits = split_count(g, mode, &per);
    return splits > 1 ? (size_t)splits * (size_t)g.M * (size_t)g.N * sizeof(float) : 0;
}

tomos_status tomos_mm_ex(int32_t trans_a, int32_t trans_b, double alpha, const tomos_dense* A, int32_t tier,
                         const tomos_dense* B, double beta, tomos_dense* C, void* scratch, size_t scratch_bytes,
                         void* stream) {
    GemmArgs g;
    Elem e;
    int mode;
    tomos_status s = mm_prepare(trans_a, trans_b, alpha, A, tier, B, beta, C, &g, &e, &mode);
    if (s) return s;
    cudaStream_t st = as_stream(stream);
    if (g.M == 0 || g.N == 0) return TOMOS_OK;
    if ((!A->values && g.M * g.K > 0) || (!B->values && g.K * g.N > 0) || !C->values)
        return fail(TOMOS_ERR_INVALID, "mm: null values");
    g.err = gemm_err_word();
    if (!g.err) return fail(TOMOS_ERR_CUDA, "mm: error word");
    if (g.K == 0) {
        gemm_scale_c_kernel<<<(unsigned)((g.M * g.N + 255) / 256), 256, 0, st>>>(g.c, g.M, g.N, g.c_si, g.c_sj,
                                                                                 beta);
        TOMOS_LAUNCH_CHECK("gemm_scale_c_kernel");
        return TOMOS_OK;
    }
    int splits = split_count(g, mode, &g.kt_per);
    const size_t need = (size_t)splits * (size_t)g.M * (size_t)g.N * sizeof(float);
    if (splits > 1 && (!scratch || scratch_bytes < need)) {
        // no (or too little) scratch: one split
        splits = 1;
        g.kt_per = 1 << 30;
    }
    g.part = splits > 1 ? static_cast<float*>(scratch) : nullptr;
    switch (mode) {
        case kPure16: s = launch_mode<kPure16>(e, g, st); break;
        case kTf32x2: s = launch_mode<kTf32x2>(e, g, st); break;
        default:
            switch (e) {
                case Elem::F32: s = launch_gemm<Elem::F32, kTf32x3>(g, st); break;
                case Elem::A16: s = launch_gemm<Elem::A16, kTf32x3>(g, st); break;
                case Elem::AB16: s = launch_gemm<Elem::AB16, kTf32x3>(g, st); break;
                case Elem::AB16R: s = launch_gemm<Elem::AB16R, kTf32x3>(g, st); break;
                default: return fail(TOMOS_ERR_UNSUPPORTED, "mm: element type");
            }
    }
    if (s || splits == 1) return s;
    gemm_split_reduce_kernel<<<(unsigned)((g.M * g.N + 255) / 256), 256, 0, st>>>(g.part, splits, g.M, g.N, alpha,
                                                                                  beta, g.c, g.c_si, g.c_sj);
    TOMOS_LAUNCH_CHECK("gemm_split_reduce_kernel");
    return TOMOS_OK;
}

tomos_status tomos_mm(int32_t trans_a, int32_t trans_b, double alpha, const tomos_dense* A, int32_t tier,
                      const tomos_dense* B, double beta, tomos_dense* C, void* stream) {
    return tomos_mm_ex(trans_a, trans_b, alpha, A, tier, B, beta, C, nullptr, 0, stream);
}

}  // extern "C"
