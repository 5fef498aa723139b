// sketch.cu -- hash CountSketch SA = S A (tomos_countsketch_*).
//
// S is the reference's hash sketch (countsketch_kernels.cpp:59-85,
// countsketch_cuda_kernels.cu:267-286): row i of A is added, with sign
// +1 if bit 0 of splitmix64(i ^ sign_seed) is set and -1 otherwise, into
// row splitmix64(i ^ bucket_seed) mod s of SA.  Integer hashing is
// bit-exact with the reference.  Unlike the reference (atomicAdd scatter,
// order-dependent float sums), every bucket here is summed by one owner in
// increasing row order, in FP64, so SA is deterministic:
//   1. hash + bucket histogram       (integer atomics: order-free)
//   2. exclusive scan of the counts  (one block)
//   3. scatter row ids to buckets    (arbitrary order within a bucket)
//   4. sort each bucket's row ids    (one warp per bucket)
//   5. owner sums                    (row-major: a warp per bucket walks
//                                     whole rows; column-major: a warp
//                                     per (column, bucket) gathers down a
//                                     contiguous column)
// The sum of squares of the values read (||A||_F^2) falls out of step 5.
#include <string>

#include "common.cuh"
#include "fused.cuh"
#include "mbarrier.cuh"  // smem_addr
#include "sketch.cuh"

namespace tomos_b200 {

// Row i of this matrix is row row0 + i of the whole problem (a row shard);
// the hash takes the whole problem's row index.
__global__ void cs_hash_kernel(int64_t m, int64_t s, uint64_t bseed, uint64_t sseed, int64_t row0,
                               int32_t* __restrict__ bucket, int8_t* __restrict__ sign,
                               int32_t* __restrict__ counts) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t gi = (uint64_t)(row0 + i);
        const int32_t b = (int32_t)(splitmix64(gi ^ bseed) % (uint64_t)s);
        bucket[i] = b;
        sign[i] = (splitmix64(gi ^ sseed) & 1ull) ? (int8_t)1 : (int8_t)-1;
        if (counts) atomicAdd(&counts[b], 1);
    }
}

// Exclusive scan of counts[0..s) into offsets[0..s], one block.
__global__ void cs_scan_kernel(const int32_t* __restrict__ counts, int64_t s,
                               int32_t* __restrict__ offsets) {
    __shared__ int32_t carry;
    __shared__ int32_t wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t base = 0; base < s; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int32_t v = i < s ? counts[i] : 0;
        int32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            int32_t t = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            wsum[lane] = t;
        }
        __syncthreads();
        const int32_t before = carry + (w > 0 ? wsum[w - 1] : 0) + x - v;
        if (i < s) offsets[i] = before;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[s] = carry;
}

__global__ void cs_scatter_kernel(int64_t m, const int32_t* __restrict__ bucket,
                                  const int32_t* __restrict__ offsets, int32_t* __restrict__ cursor,
                                  int32_t* __restrict__ perm) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = bucket[i];
        perm[offsets[b] + atomicAdd(&cursor[b], 1)] = (int32_t)i;
    }
}

// Sorts each bucket's row ids ascending, a warp per bucket (buckets hold
// about m/s rows): a bitonic network in shared memory for buckets of up to
// kCsSortCap rows, odd-even transposition in place for longer ones.
constexpr int kCsSortCap = 1024;
constexpr int kCsSortWarps = 4;

__global__ void __launch_bounds__(kCsSortWarps * 32) cs_sort_kernel(int64_t s,
                                                                  const int32_t* __restrict__ offsets,
                                                                  int32_t* __restrict__ perm) {
    __shared__ int32_t buf[kCsSortWarps][kCsSortCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t b = (int64_t)blockIdx.x * kCsSortWarps + w;
    if (b >= s) return;
    const int32_t o0 = offsets[b], len = offsets[b + 1] - o0;
    int32_t* seg = perm + o0;
    if (len > kCsSortCap) {
        for (int32_t pass = 0; pass < len; ++pass) {
            const int32_t start = pass & 1;
            for (int32_t k = start + 2 * lane; k + 1 < len; k += 64) {
                int32_t x = seg[k], y = seg[k + 1];
                if (x > y) {
                    seg[k] = y;
                    seg[k + 1] = x;
                }
            }
            __syncwarp();
        }
        return;
    }
    int N = 1;
    while (N < len) N <<= 1;
    int32_t* v = buf[w];
    for (int e = lane; e < N; e += 32) v[e] = e < len ? seg[e] : 0x7fffffff;
    __syncwarp();
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            // pairs (i, i ^ j) with i < i ^ j are disjoint within a step
            for (int i = lane; i < N; i += 32) {
                const int p = i ^ j;
                if (p > i) {
                    const int32_t x = v[i], y = v[p];
                    if ((x > y) == ((i & k) == 0)) {
                        v[i] = y;
                        v[p] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
    for (int e = lane; e < len; e += 32) seg[e] = v[e];
}

// Row-major owner sums: warp per bucket, lanes over columns of a panel of
// 32 * KC columns (grid.y walks the panels).  Sums in FP32 with the rows
// of a bucket in increasing order: bit for bit the reference's
// countsketch_apply_impl<float> (countsketch_kernels.cpp:70-83).  The
// column sums of squares are FP32 per bucket and FP64 across buckets.
template <Elem E, int KC>
__global__ void __launch_bounds__(256) cs_rows_kernel(const void* hi, const void* lo, int64_t n,
                                                      int64_t ld, int64_t s,
                                                      const int32_t* __restrict__ offsets,
                                                      const int32_t* __restrict__ perm,
                                                      const int8_t* __restrict__ sign,
                                                      double* __restrict__ SA, int64_t ld_sa,
                                                      double* __restrict__ fro_part,
                                                      double* __restrict__ col_part) {
    __shared__ double smf[8];
    __shared__ float smc[8][32 * KC];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t b = (int64_t)blockIdx.x * 8 + w;
    const int64_t c0 = (int64_t)blockIdx.y * 32 * KC;
    float acc[KC], csq[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) acc[k] = csq[k] = 0.0f;
    double f2 = 0.0;
    if (b < s) {
        const int32_t o0 = offsets[b], o1 = offsets[b + 1];
        for (int32_t q = o0; q < o1; ++q) {
            const int32_t r = perm[q];
            const float sg = (float)sign[r];
            const size_t base = (size_t)r * ld;
#pragma unroll
            for (int k = 0; k < KC; ++k) {
                const int64_t j = c0 + k * 32 + lane;
                if (j < n) {
                    const float a = load_elem<E>(hi, lo, base + j);
                    acc[k] = fmaf(sg, a, acc[k]);
                    csq[k] = fmaf(a, a, csq[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < KC; ++k) {
            const int64_t j = c0 + k * 32 + lane;
            if (j < n) SA[(size_t)j * ld_sa + b] = (double)acc[k];
            f2 += (double)csq[k];
        }
    }
#pragma unroll
    for (int k = 0; k < KC; ++k) smc[w][k * 32 + lane] = csq[k];
    f2 = warp_sum(f2);
    if (lane == 0) smf[w] = f2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) t += smf[k];
        fro_part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
    if (col_part) {
        for (int e = threadIdx.x; e < 32 * KC; e += blockDim.x) {
            const int64_t j = c0 + e;
            if (j >= n) continue;
            double t = 0.0;
#pragma unroll
            for (int k = 0; k < 8; ++k) t += (double)smc[k][e];
            col_part[(size_t)blockIdx.x * n + j] = t;
        }
    }
}

// colsq[j] = sum over nparts rows of part[r][j] (fixed order).
__global__ void cs_col_reduce_kernel(const double* __restrict__ part, int64_t nparts, int64_t n,
                                     double* __restrict__ colsq) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double t = 0.0;
    for (int64_t r = 0; r < nparts; ++r) t += part[(size_t)r * n + j];
    colsq[j] = t;
}

// Row-major owner sums, gathered through shared memory by asynchronous
// copies.
//
// One CTA per SM of kCsWarps warps; each warp takes (bucket, panel) work
// items from a global counter (buckets hold ~m/s rows of uneven count, so
// items are handed out dynamically) and walks the bucket's rows in
// increasing order.  Lane l owns the 16-byte chunks l, l+32, ... (KCH of
// them) of the panel: it copies them of kCsStages batches of RB rows ahead
// into its slots of the warp's ring (cp.async, one commit group a batch)
// and sums a batch once its own group has landed -- no lane reads another
// lane's bytes, so no barrier is needed, and the rows being random, these
// per-thread 16-byte copies issue far faster than one bulk copy per row.
// Sums are FP32 in increasing row order (bit for bit the reference's
// countsketch_apply_impl<float>, countsketch_kernels.cpp:70-83; the packed
// FP32x2 FMAs round each element as fmaf does).  Each item writes its
// bucket's row of SA and its FP32 column sums of squares to col_part
// (s x n), which cs_colsq_chunk_kernel then reduces in bucket order, so the
// results do not depend on which warp took which item.
//
// STAGE (FP32_16 HALF tier only): the fp32_16_half_only words of every
// chunk read are also written to `plane` (row pitch ld_plane halves) -- the
// fixed fp16 copy of the wh plane the LSQR HALF-tier iterations read -- so
// a solve that follows the sketch needs no staging pass of its own.
constexpr int kCsWarps = 12;
constexpr int kCsStages = 4;
constexpr int kCsStageBytes = 4096;  // per warp and stage
constexpr int kCsPanelCols = 512;    // columns per work item
constexpr int kCsList = 512;         // a bucket's row ids kept in shared memory

struct CsRowsArgs {
    const void* hi;
    const void* lo;
    int64_t n, ld, s;
    int panels;
    const int32_t* offsets;
    const int32_t* perm;
    const int8_t* sign;
    double* SA;
    int64_t ld_sa;
    float* col_part;  // s x n
    uint16_t* plane;
    int64_t ld_plane;
    int* counter;     // zero at launch
};

template <Elem E>
struct CsRowsShape {
    static constexpr int VEC = ChunkElems<E>::value;
    static constexpr int ESZ = (E == Elem::F32) ? 4 : 2;
    static constexpr int PLANES = (E == Elem::A16 || E == Elem::AB16 || E == Elem::AB16R) ? 2 : 1;
    static constexpr int KCH = kCsPanelCols / (32 * VEC);  // chunks per lane
    static constexpr int PWB = kCsPanelCols * ESZ;         // panel bytes per row and plane
    static constexpr int RB = kCsStageBytes / (PWB * PLANES);  // rows per batch
    static_assert(RB >= 1, "a row's panel fits a stage");
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <Elem E, bool STAGE>
__global__ void __launch_bounds__(kCsWarps * 32, 1) cs_rows_tma_kernel(CsRowsArgs a) {
    using S = CsRowsShape<E>;
    constexpr int VEC = S::VEC, HV = VEC / 2, KCH = S::KCH, RB = S::RB, PLANES = S::PLANES;
    constexpr int ESZ = S::ESZ, PWB = S::PWB;
    static_assert(!STAGE || E == Elem::H16, "staging writes FP32_16 wh planes");
    extern __shared__ __align__(128) uint8_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint8_t* ring = smem + (size_t)warp * kCsStages * kCsStageBytes;
    // the bucket's first kCsList row ids, bit 31 set for sign -1
    uint32_t* list = reinterpret_cast<uint32_t*>(smem + (size_t)kCsWarps * kCsStages * kCsStageBytes) +
                     (size_t)warp * kCsList;
    const int64_t n = a.n, s = a.s;
    const int64_t nch = (n + VEC - 1) / VEC;
    const int64_t total = s * a.panels;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        const int64_t b = item % s;
        const int64_t c0 = (int64_t)(item / s) * kCsPanelCols;
        const int32_t o0 = a.offsets[b], len = a.offsets[b + 1] - o0;
        const int nbat = (len + RB - 1) / RB;
        // Row ids and signs of the bucket, gathered once (eight in flight
        // a lane) instead of two dependent loads per row.
        __syncwarp();  // the previous item's readers of the list are done
        {
            const int lim = len < kCsList ? len : kCsList;
            for (int e0 = 0; e0 < lim; e0 += 8 * 32) {
                int32_t rr[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int e = e0 + q * 32 + lane;
                    rr[q] = e < lim ? a.perm[o0 + e] : 0;
                }
                int8_t sq[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) sq[q] = (e0 + q * 32 + lane) < lim ? a.sign[rr[q]] : 1;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int e = e0 + q * 32 + lane;
                    if (e < lim) list[e] = (uint32_t)rr[q] | (sq[q] < 0 ? 0x80000000u : 0u);
                }
            }
            __syncwarp();
        }
        // row id and sign of the bucket's e-th row
        auto row_of = [&](int e, int32_t& r, float& sg) {
            if (e < kCsList) {
                const uint32_t v = list[e];
                r = (int32_t)(v & 0x7fffffffu);
                sg = (v >> 31) ? -1.0f : 1.0f;
            } else {
                r = a.perm[o0 + e];
                sg = (float)a.sign[r];
            }
        };
        bool live[KCH];
        int zero_from[KCH];  // elements of the chunk at or past column n
#pragma unroll
        for (int k = 0; k < KCH; ++k) {
            const int64_t c = c0 / VEC + k * 32 + lane;
            live[k] = c < nch;
            zero_from[k] = !live[k] ? 0 : ((c == nch - 1 && n % VEC != 0) ? (int)(n - c * VEC) : VEC);
        }
        // this lane's chunks of batch t into ring stage t % kCsStages (one
        // commit group, empty past the bucket's end)
        auto issue = [&](int t) {
            if (t < nbat) {
                uint8_t* st = ring + (size_t)(t % kCsStages) * kCsStageBytes;
                const int rows = (len - t * RB) < RB ? (len - t * RB) : RB;
                for (int u = 0; u < rows; ++u) {
                    int32_t r;
                    float sg;
                    row_of(t * RB + u, r, sg);
                    const uint8_t* src = static_cast<const uint8_t*>(a.hi) + ((size_t)r * a.ld + c0) * ESZ;
                    const uint8_t* srl = static_cast<const uint8_t*>(a.lo) + ((size_t)r * a.ld + c0) * ESZ;
#pragma unroll
                    for (int k = 0; k < KCH; ++k) {
                        if (!live[k]) continue;
                        const int coff = (k * 32 + lane) * 16;
                        cp_async16(st + (size_t)(u * PLANES) * PWB + coff, src + coff);
                        if (PLANES == 2) cp_async16(st + (size_t)(u * PLANES + 1) * PWB + coff, srl + coff);
                    }
                }
            }
            cp_async_commit();
        };
#pragma unroll
        for (int t = 0; t < kCsStages; ++t) issue(t);
        float2 acc[KCH][HV], csq[KCH][HV];
#pragma unroll
        for (int k = 0; k < KCH; ++k)
#pragma unroll
            for (int e = 0; e < HV; ++e) acc[k][e] = csq[k][e] = make_float2(0.0f, 0.0f);
        for (int t = 0; t < nbat; ++t) {
            cp_async_wait<kCsStages - 1>();  // this lane's copies of batch t landed
            const uint8_t* st = ring + (size_t)(t % kCsStages) * kCsStageBytes;
            const int rows = (len - t * RB) < RB ? (len - t * RB) : RB;
            for (int u = 0; u < rows; ++u) {
                int32_t r;
                float sgv;
                row_of(t * RB + u, r, sgv);
                const float2 sg2 = make_float2(sgv, sgv);
                const uint8_t* hrow = st + (size_t)(u * PLANES) * PWB;
#pragma unroll
                for (int k = 0; k < KCH; ++k) {
                    const int coff = (k * 32 + lane) * 16;
                    uint4 h = make_uint4(0, 0, 0, 0), l = make_uint4(0, 0, 0, 0);
                    if (live[k]) {
                        h = *reinterpret_cast<const uint4*>(hrow + coff);
                        if (PLANES == 2) l = *reinterpret_cast<const uint4*>(hrow + PWB + coff);
                    }
                    float2 v[HV];
                    if constexpr (E == Elem::H16) {
                        fix_half_chunk(h);
                        if constexpr (STAGE) {
                            if (live[k])
                                *reinterpret_cast<uint4*>(a.plane + (size_t)r * a.ld_plane + c0 +
                                                          (k * 32 + lane) * VEC) = h;
                        }
                        v[0] = h2f2(h.x);
                        v[1] = h2f2(h.y);
                        v[2] = h2f2(h.z);
                        v[3] = h2f2(h.w);
                    } else {
                        float f[VEC];
                        ChunkDecoder<E>::decode(h, l, f);
#pragma unroll
                        for (int e = 0; e < HV; ++e) v[e] = make_float2(f[2 * e], f[2 * e + 1]);
                    }
                    // chunks past the row's end and columns past n (the
                    // last chunk's padding) add nothing (a zero word need
                    // not decode to 0)
                    if (zero_from[k] < VEC) {
#pragma unroll
                        for (int e = 0; e < HV; ++e) {
                            if (2 * e >= zero_from[k]) v[e].x = 0.0f;
                            if (2 * e + 1 >= zero_from[k]) v[e].y = 0.0f;
                        }
                    }
#pragma unroll
                    for (int e = 0; e < HV; ++e) {
                        acc[k][e] = __ffma2_rn(v[e], sg2, acc[k][e]);
                        csq[k][e] = __ffma2_rn(v[e], v[e], csq[k][e]);
                    }
                }
            }
            // this lane read its slots of stage t: refill them
            issue(t + kCsStages);
        }
        cp_async_wait<0>();  // the trailing (empty) groups
#pragma unroll
        for (int k = 0; k < KCH; ++k) {
            const int64_t cb = c0 + (int64_t)(k * 32 + lane) * VEC;
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                if (!live[k] || cb + e >= n) continue;
                const float va = (e & 1) ? acc[k][e / 2].y : acc[k][e / 2].x;
                const float vq = (e & 1) ? csq[k][e / 2].y : csq[k][e / 2].x;
                a.SA[(size_t)(cb + e) * a.ld_sa + b] = (double)va;
                a.col_part[(size_t)b * n + cb + e] = vq;
            }
        }
    }
}

template <Elem E>
inline size_t cs_rows_tma_smem() {
    return (size_t)kCsWarps * (kCsStages * kCsStageBytes + kCsList * sizeof(uint32_t));
}

// Column sums of squares from the per-bucket FP32 partials: chunk q of the
// buckets sums its rows in bucket order into part[q][j] (FP64), then
// cs_colsq_final_kernel sums the chunks in order.
__global__ void cs_colsq_chunk_kernel(const float* __restrict__ col_part, int64_t s, int64_t n,
                                      int64_t per_chunk, double* __restrict__ part) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t q = blockIdx.y;
    if (j >= n) return;
    const int64_t b0 = q * per_chunk;
    const int64_t b1 = (b0 + per_chunk) < s ? (b0 + per_chunk) : s;
    double t = 0.0;
    for (int64_t b = b0; b < b1; ++b) t += (double)col_part[(size_t)b * n + j];
    part[(size_t)q * n + j] = t;
}

__global__ void cs_colsq_final_kernel(const double* __restrict__ part, int64_t chunks, int64_t n,
                                      double* __restrict__ colsq) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double t = 0.0;
    for (int64_t q = 0; q < chunks; ++q) t += part[(size_t)q * n + j];
    colsq[j] = t;
}

// Column-major owner sums: block per column, warps over buckets, lanes
// over the bucket's rows (gathered down the contiguous column).
template <Elem E>
__global__ void __launch_bounds__(256) cs_cols_kernel(const void* hi, const void* lo, int64_t n,
                                                      int64_t ld, int64_t s,
                                                      const int32_t* __restrict__ offsets,
                                                      const int32_t* __restrict__ perm,
                                                      const int8_t* __restrict__ sign,
                                                      double* __restrict__ SA, int64_t ld_sa,
                                                      double* __restrict__ fro_part,
                                                      double* __restrict__ colsq) {
    __shared__ double smf[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t j = blockIdx.x;
    const size_t cbase = (size_t)j * ld;
    double f2 = 0.0;
    for (int64_t b = w; b < s; b += 8) {
        const int32_t o0 = offsets[b], o1 = offsets[b + 1];
        double acc = 0.0;
        for (int32_t q = o0 + lane; q < o1; q += 32) {
            const int32_t r = perm[q];
            const double a = (double)load_elem<E>(hi, lo, cbase + r);
            acc += (double)sign[r] * a;
            f2 += a * a;
        }
        acc = warp_sum(acc);
        if (lane == 0) SA[(size_t)j * ld_sa + b] = acc;
    }
    f2 = warp_sum(f2);
    if (lane == 0) smf[w] = f2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) t += smf[k];
        fro_part[blockIdx.x] = t;
        if (colsq) colsq[blockIdx.x] = t;
    }
}

__global__ void cs_fro_reduce_kernel(const double* __restrict__ part, int64_t np,
                                     double* __restrict__ out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < np; k += blockDim.x) s += part[k];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) *out = t;
    }
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

CsScratch cs_layout(void* base, int64_t m, int64_t s, int64_t fro_parts, int64_t col_parts) {
    CsScratch c;
    size_t off = 0;
    char* p = static_cast<char*>(base);
    auto take = [&](size_t bytes) {
        char* q = p ? p + off : nullptr;
        off += align256(bytes);
        return q;
    };
    c.bucket = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (m > 0 ? m : 1)));
    c.sign = reinterpret_cast<int8_t*>(take(m > 0 ? m : 1));
    c.counts = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (s + 1)));
    c.offsets = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (s + 1)));
    c.cursor = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (s + 1)));
    c.perm = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (m > 0 ? m : 1)));
    c.fro_part = reinterpret_cast<double*>(take(sizeof(double) * (fro_parts > 0 ? fro_parts : 1)));
    c.col_part = reinterpret_cast<double*>(take(sizeof(double) * (col_parts > 0 ? col_parts : 1)));
    c.bytes = off;
    return c;
}

int64_t cs_col_part_rows(int64_t m, int64_t s) {
    // row-major: s x n FP32 per-bucket partials, then n FP64 column sums
    const int64_t rows = (s + 1) / 2 + 1;
    int64_t csr = (int64_t)sm_count() * 2;             // CSR row-chunk blocks
    const int64_t cm = (m + 63) / 64;
    if (csr > cm) csr = cm;
    return rows > csr ? rows : csr;
}

// Upper bound of the owner-sum partial count over both layouts and the
// CSR path, so one size query serves all callers.
int64_t cs_fro_parts(int64_t m, int64_t s) {
    (void)m;
    const int64_t rows = ((s + 7) / 8) * 64;  // row-major: blocks x panels (n <= 64 panels cap)
    const int64_t csr = (s + 7) / 8;
    int64_t v = rows > csr ? rows : csr;
    return v < 65536 ? 65536 : v;  // column-major: one per column (n <= 65536)
}

static bool cs_grid(int64_t m, int* g) {
    int64_t b = (m + 255) / 256;
    int64_t cap = (int64_t)sm_count() * 8;
    if (b > cap) b = cap;
    *g = (int)(b < 1 ? 1 : b);
    return true;
}

// Steps 1-4 (shared by the dense and CSR owner sums).
tomos_status cs_bucketize(int64_t m, int64_t s, uint64_t bseed, uint64_t sseed, const CsScratch& c,
                          cudaStream_t st, int64_t row0) {
    int g;
    cs_grid(m, &g);
    TOMOS_CUDA_TRY(cudaMemsetAsync(c.counts, 0, sizeof(int32_t) * (s + 1), st));
    TOMOS_CUDA_TRY(cudaMemsetAsync(c.cursor, 0, sizeof(int32_t) * (s + 1), st));
    cs_hash_kernel<<<g, 256, 0, st>>>(m, s, bseed, sseed, row0, c.bucket, c.sign, c.counts);
    TOMOS_LAUNCH_CHECK("cs_hash_kernel");
    cs_scan_kernel<<<1, 1024, 0, st>>>(c.counts, s, c.offsets);
    TOMOS_LAUNCH_CHECK("cs_scan_kernel");
    cs_scatter_kernel<<<g, 256, 0, st>>>(m, c.bucket, c.offsets, c.cursor, c.perm);
    TOMOS_LAUNCH_CHECK("cs_scatter_kernel");
    cs_sort_kernel<<<(unsigned)((s + kCsSortWarps - 1) / kCsSortWarps), kCsSortWarps * 32, 0, st>>>(
        s, c.offsets, c.perm);
    TOMOS_LAUNCH_CHECK("cs_sort_kernel");
    return TOMOS_OK;
}

// Whether the staged owner sums can read A (16-byte aligned rows).
static bool rows_vec_ok(const tomos_dense* A, const void* lo, int esz) {
    bool vec = ((A->ld * esz) % 16 == 0) && (reinterpret_cast<uintptr_t>(A->values) % 16 == 0);
    if (vec && lo) vec = reinterpret_cast<uintptr_t>(lo) % 16 == 0;
    return vec;
}

// The staged owner sums and the reductions behind them: SA, colsq and
// fro2 (both optional).  Returns nonzero with the error set on failure.
template <Elem E, bool STAGE>
static tomos_status launch_rows_tma(const tomos_dense* A, const void* lo, int64_t s, const CsScratch& c,
                                    double* SA, int64_t ld_sa, double* colsq, double* fro2,
                                    uint16_t* plane, int64_t ld_plane, cudaStream_t st) {
    const int64_t n = A->cols;
    const size_t smem = cs_rows_tma_smem<E>();
    TOMOS_CUDA_TRY(cudaFuncSetAttribute(cs_rows_tma_kernel<E, STAGE>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // the work counter: the first int of cursor (free after the scatter)
    TOMOS_CUDA_TRY(cudaMemsetAsync(c.cursor, 0, sizeof(int32_t), st));
    CsRowsArgs a;
    a.hi = A->values;
    a.lo = lo;
    a.n = n;
    a.ld = A->ld;
    a.s = s;
    a.panels = (int)((n + kCsPanelCols - 1) / kCsPanelCols);
    a.offsets = c.offsets;
    a.perm = c.perm;
    a.sign = c.sign;
    a.SA = SA;
    a.ld_sa = ld_sa;
    a.col_part = reinterpret_cast<float*>(c.col_part);
    a.plane = plane;
    a.ld_plane = ld_plane;
    a.counter = c.cursor;
    cs_rows_tma_kernel<E, STAGE><<<(unsigned)sm_count(), kCsWarps * 32, smem, st>>>(a);
    TOMOS_LAUNCH_CHECK("cs_rows_tma_kernel");
    // colsq (into the caller's buffer or the scratch after the partials),
    // then fro2 as their sum
    double* cs = colsq ? colsq : reinterpret_cast<double*>(a.col_part + s * n);
    int64_t chunks = (s + 63) / 64;
    const int64_t cap = cs_fro_parts(A->rows, s) / (n > 0 ? n : 1);
    if (chunks > cap) chunks = cap > 0 ? cap : 1;
    const int64_t per = (s + chunks - 1) / chunks;
    chunks = (s + per - 1) / per;
    cs_colsq_chunk_kernel<<<dim3((unsigned)((n + 255) / 256), (unsigned)chunks), 256, 0, st>>>(
        a.col_part, s, n, per, c.fro_part);
    TOMOS_LAUNCH_CHECK("cs_colsq_chunk_kernel");
    cs_colsq_final_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c.fro_part, chunks, n, cs);
    TOMOS_LAUNCH_CHECK("cs_colsq_final_kernel");
    if (fro2) {
        cs_fro_reduce_kernel<<<1, 256, 0, st>>>(cs, n, fro2);
        TOMOS_LAUNCH_CHECK("cs_fro_reduce_kernel");
    }
    return TOMOS_OK;
}

template <Elem E>
static unsigned launch_rows(const tomos_dense* A, const void* lo, int64_t s, const CsScratch& c,
                            double* SA, int64_t ld_sa, bool want_cols, unsigned gx,
                            cudaStream_t st) {
    const unsigned panels = (unsigned)((A->cols + 255) / 256);
    cs_rows_kernel<E, 8><<<dim3(gx, panels), 256, 0, st>>>(A->values, lo, A->cols, A->ld, s, c.offsets,
                                                           c.perm, c.sign, SA, ld_sa, c.fro_part,
                                                           want_cols ? c.col_part : nullptr);
    return panels;
}

template <Elem E>
static void launch_cols(const tomos_dense* A, const void* lo, int64_t s, const CsScratch& c,
                        double* SA, int64_t ld_sa, double* colsq, cudaStream_t st) {
    cs_cols_kernel<E><<<(unsigned)A->cols, 256, 0, st>>>(A->values, lo, A->cols, A->ld, s, c.offsets,
                                                         c.perm, c.sign, SA, ld_sa, c.fro_part, colsq);
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

tomos_status tomos_countsketch_hash(int64_t m, int64_t s, uint64_t bucket_seed, uint64_t sign_seed,
                                    int32_t* bucket, int8_t* sign, void* stream) {
    if (m < 0 || s <= 0) return fail(TOMOS_ERR_INVALID, "countsketch_hash: need m >= 0, s > 0");
    if (m == 0) return TOMOS_OK;
    if (m > 0x7fffffffLL) return fail(TOMOS_ERR_INVALID, "countsketch_hash: m exceeds int32");
    if (!bucket || !sign) return fail(TOMOS_ERR_INVALID, "countsketch_hash: null output");
    int g;
    cs_grid(m, &g);
    cs_hash_kernel<<<g, 256, 0, as_stream(stream)>>>(m, s, bucket_seed, sign_seed, 0, bucket, sign,
                                                     nullptr);
    TOMOS_LAUNCH_CHECK("cs_hash_kernel");
    return TOMOS_OK;
}

size_t tomos_countsketch_scratch_bytes(int64_t m, int64_t cols, int64_t s) {
    if (m < 0 || s <= 0 || cols < 0) return 0;
    return cs_layout(nullptr, m, s, cs_fro_parts(m, s), cs_col_part_rows(m, s) * cols).bytes;
}

}  // extern "C"

namespace tomos_b200 {

// tomos_countsketch_apply, and with `plane` the staged fp16 copy of an
// FP32_16 wh plane written by the same pass (tomos_countsketch_apply_stage).
static tomos_status countsketch_apply(const tomos_dense* A, int32_t tier, int64_t s,
                                      uint64_t bucket_seed, uint64_t sign_seed, double* SA,
                                      int64_t ld_sa, double* fro2, double* colsq, void* scratch,
                                      size_t scratch_bytes, void* stream, uint16_t* plane,
                                      int64_t ld_plane, int64_t row0 = 0) {
    if (!A || s <= 0) return fail(TOMOS_ERR_INVALID, "countsketch_apply: need A and s > 0");
    if (A->layout != TOMOS_ROW_MAJOR && A->layout != TOMOS_COL_MAJOR)
        return fail(TOMOS_ERR_INVALID, "countsketch_apply: bad layout");
    const int64_t m = A->rows, n = A->cols;
    if (m < 0 || n < 0) return fail(TOMOS_ERR_INVALID, "countsketch_apply: negative size");
    if (m > 0x7fffffffLL) return fail(TOMOS_ERR_INVALID, "countsketch_apply: m exceeds int32");
    if (ld_sa < s) return fail(TOMOS_ERR_INVALID, "countsketch_apply: ld_sa < s");
    const int64_t inner = A->layout == TOMOS_ROW_MAJOR ? n : m;
    if (A->ld < inner) return fail(TOMOS_ERR_INVALID, "countsketch_apply: bad leading dimension");
    if (A->layout == TOMOS_COL_MAJOR && n > 65536)
        return fail(TOMOS_ERR_INVALID, "countsketch_apply: column-major n > 65536");
    if (A->layout == TOMOS_ROW_MAJOR && n > 64 * 256)
        return fail(TOMOS_ERR_INVALID, "countsketch_apply: row-major n > 16384");
    Elem e;
    std::string why;
    if (!resolve_elem(A, tier, &e, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply: " + why);
    cudaStream_t st = as_stream(stream);
    if (n == 0) return TOMOS_OK;
    if (!SA) return fail(TOMOS_ERR_INVALID, "countsketch_apply: null SA");
    if (m == 0) {
        for (int64_t j = 0; j < n; ++j)
            TOMOS_CUDA_TRY(cudaMemsetAsync(SA + j * ld_sa, 0, sizeof(double) * s, st));
        if (fro2) TOMOS_CUDA_TRY(cudaMemsetAsync(fro2, 0, sizeof(double), st));
        if (colsq) TOMOS_CUDA_TRY(cudaMemsetAsync(colsq, 0, sizeof(double) * n, st));
        return TOMOS_OK;
    }
    const int64_t col_parts = cs_col_part_rows(m, s) * n;
    CsScratch need = cs_layout(nullptr, m, s, cs_fro_parts(m, s), col_parts);
    if (!scratch || scratch_bytes < need.bytes)
        return fail(TOMOS_ERR_INVALID, "countsketch_apply: scratch too small (need " +
                                           std::to_string(need.bytes) + " bytes)");
    CsScratch c = cs_layout(scratch, m, s, cs_fro_parts(m, s), col_parts);
    tomos_status rc = cs_bucketize(m, s, bucket_seed, sign_seed, c, st, row0);
    if (rc) return rc;
    const void* lo = (e == Elem::A16 || e == Elem::AB16 || e == Elem::AB16R) ? dense_lo_plane(A)
                                                                             : nullptr;
    int64_t nparts;
    if (A->layout == TOMOS_ROW_MAJOR && rows_vec_ok(A, lo, e == Elem::F32 ? 4 : 2)) {
        // staged owner sums: colsq and fro2 come with them
        tomos_status rs = TOMOS_OK;
        switch (e) {
            case Elem::F32: rs = launch_rows_tma<Elem::F32, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st); break;
            case Elem::H16:
                rs = plane ? launch_rows_tma<Elem::H16, true>(A, lo, s, c, SA, ld_sa, colsq, fro2, plane, ld_plane, st)
                           : launch_rows_tma<Elem::H16, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st);
                break;
            case Elem::A16: rs = launch_rows_tma<Elem::A16, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st); break;
            case Elem::F16: rs = launch_rows_tma<Elem::F16, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st); break;
            case Elem::B16: rs = launch_rows_tma<Elem::B16, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st); break;
            case Elem::AB16: rs = launch_rows_tma<Elem::AB16, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st); break;
            case Elem::AB16R: rs = launch_rows_tma<Elem::AB16R, false>(A, lo, s, c, SA, ld_sa, colsq, fro2, nullptr, 0, st); break;
            default: return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply: element type");
        }
        return rs;
    }
    if (plane) return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply_stage: rows of A not 16-byte aligned");
    if (A->layout == TOMOS_ROW_MAJOR) {
        const unsigned gx = (unsigned)((s + 7) / 8);
        unsigned panels = 0;
        switch (e) {
            case Elem::F32: panels = launch_rows<Elem::F32>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::H16: panels = launch_rows<Elem::H16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::A16: panels = launch_rows<Elem::A16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::F16: panels = launch_rows<Elem::F16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::B16: panels = launch_rows<Elem::B16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::AB16: panels = launch_rows<Elem::AB16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::AB16R: panels = launch_rows<Elem::AB16R>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            default: return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply: element type");
        }
        nparts = (int64_t)gx * panels;
        if (colsq) {
            TOMOS_LAUNCH_CHECK("countsketch owner sums");
            cs_col_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c.col_part, gx, n, colsq);
        }
    } else {
        switch (e) {
            case Elem::F32: launch_cols<Elem::F32>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            case Elem::H16: launch_cols<Elem::H16>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            case Elem::A16: launch_cols<Elem::A16>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            case Elem::F16: launch_cols<Elem::F16>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            case Elem::B16: launch_cols<Elem::B16>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            case Elem::AB16: launch_cols<Elem::AB16>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            case Elem::AB16R: launch_cols<Elem::AB16R>(A, lo, s, c, SA, ld_sa, colsq, st); break;
            default: return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply: element type");
        }
        nparts = n;
    }
    TOMOS_LAUNCH_CHECK("countsketch owner sums");
    if (fro2) {
        cs_fro_reduce_kernel<<<1, 256, 0, st>>>(c.fro_part, nparts, fro2);
        TOMOS_LAUNCH_CHECK("cs_fro_reduce_kernel");
    }
    return TOMOS_OK;
}

}  // namespace tomos_b200

extern "C" {

tomos_status tomos_countsketch_apply(const tomos_dense* A, int32_t tier, int64_t s,
                                     uint64_t bucket_seed, uint64_t sign_seed, double* SA,
                                     int64_t ld_sa, double* fro2, double* colsq, void* scratch,
                                     size_t scratch_bytes, void* stream) {
    return countsketch_apply(A, tier, s, bucket_seed, sign_seed, SA, ld_sa, fro2, colsq, scratch,
                             scratch_bytes, stream, nullptr, 0);
}

tomos_status tomos_countsketch_apply_shard(const tomos_dense* A, int32_t tier, int64_t s,
                                           uint64_t bucket_seed, uint64_t sign_seed, int64_t row0,
                                           double* SA, int64_t ld_sa, double* fro2, double* colsq,
                                           void* plane, int64_t ld_plane, void* scratch,
                                           size_t scratch_bytes, void* stream) {
    if (row0 < 0) return fail(TOMOS_ERR_INVALID, "countsketch_apply_shard: negative row0");
    if (plane) {
        if (!A || A->numeric != TOMOS_FP32_16 || A->layout != TOMOS_ROW_MAJOR || tier != TOMOS_TIER_HALF)
            return fail(TOMOS_ERR_INVALID,
                        "countsketch_apply_shard: a staged plane needs a row-major FP32_16 A at the HALF tier");
        if (reinterpret_cast<uintptr_t>(plane) % 16 != 0 || ld_plane < A->cols || ld_plane % 8 != 0)
            return fail(TOMOS_ERR_INVALID,
                        "countsketch_apply_shard: plane must be 16-byte aligned with ld_plane a multiple of 8 "
                        "and >= cols");
        if (!rows_vec_ok(A, nullptr, 2))
            return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply_shard: rows of A not 16-byte aligned");
    }
    return countsketch_apply(A, tier, s, bucket_seed, sign_seed, SA, ld_sa, fro2, colsq, scratch,
                             scratch_bytes, stream, static_cast<uint16_t*>(plane), ld_plane, row0);
}

tomos_status tomos_countsketch_apply_stage(const tomos_dense* A, int64_t s, uint64_t bucket_seed,
                                           uint64_t sign_seed, double* SA, int64_t ld_sa,
                                           double* fro2, double* colsq, void* plane,
                                           int64_t ld_plane, void* scratch, size_t scratch_bytes,
                                           void* stream) {
    if (!A || A->numeric != TOMOS_FP32_16 || A->layout != TOMOS_ROW_MAJOR)
        return fail(TOMOS_ERR_INVALID, "countsketch_apply_stage: A must be row-major FP32_16");
    if (!plane || reinterpret_cast<uintptr_t>(plane) % 16 != 0)
        return fail(TOMOS_ERR_INVALID, "countsketch_apply_stage: plane must be 16-byte aligned");
    if (ld_plane < A->cols || ld_plane % 8 != 0)
        return fail(TOMOS_ERR_INVALID,
                    "countsketch_apply_stage: ld_plane must be a multiple of 8 and >= cols");
    if (!rows_vec_ok(A, nullptr, 2))
        return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply_stage: rows of A not 16-byte aligned");
    return countsketch_apply(A, TOMOS_TIER_HALF, s, bucket_seed, sign_seed, SA, ld_sa, fro2, colsq,
                             scratch, scratch_bytes, stream, static_cast<uint16_t*>(plane), ld_plane);
}

}  // extern "C"
