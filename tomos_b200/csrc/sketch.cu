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
#include "sketch.cuh"

namespace tomos_b200 {

__global__ void cs_hash_kernel(int64_t m, int64_t s, uint64_t bseed, uint64_t sseed,
                               int32_t* __restrict__ bucket, int8_t* __restrict__ sign,
                               int32_t* __restrict__ counts) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = (int32_t)(splitmix64((uint64_t)i ^ bseed) % (uint64_t)s);
        bucket[i] = b;
        sign[i] = (splitmix64((uint64_t)i ^ sseed) & 1ull) ? (int8_t)1 : (int8_t)-1;
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

// Sorts each bucket's row ids ascending (odd-even transposition by a warp;
// buckets hold about m/s rows).
__global__ void cs_sort_kernel(int64_t s, const int32_t* __restrict__ offsets,
                               int32_t* __restrict__ perm) {
    const int lane = threadIdx.x & 31;
    const int64_t b = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= s) return;
    const int32_t o0 = offsets[b], o1 = offsets[b + 1];
    const int32_t len = o1 - o0;
    int32_t* seg = perm + o0;
    for (int32_t pass = 0; pass < len; ++pass) {
        const int32_t start = pass & 1;
        for (int32_t k = start + 2 * lane; k + 1 < len; k += 64) {
            int32_t a = seg[k], c = seg[k + 1];
            if (a > c) {
                seg[k] = c;
                seg[k + 1] = a;
            }
        }
        __syncwarp();
    }
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

// Row-major owner sums with 16-byte chunk loads: a warp per (bucket,
// panel); lane l owns chunks l, l+32, ... (KCH of them, VEC columns each)
// of the panel, and walks the bucket's rows four at a time, summing in
// FP32 in increasing row order (the reference's float path, as
// cs_rows_kernel).  Needs 16-byte aligned rows (ld * element bytes a
// multiple of 16).
template <Elem E, int KCH>
__global__ void __launch_bounds__(256) cs_rows_vec_kernel(const void* hi, const void* lo, int64_t n,
                                                          int64_t ld, int64_t s,
                                                          const int32_t* __restrict__ offsets,
                                                          const int32_t* __restrict__ perm,
                                                          const int8_t* __restrict__ sign,
                                                          double* __restrict__ SA, int64_t ld_sa,
                                                          double* __restrict__ fro_part,
                                                          double* __restrict__ col_part) {
    constexpr int VEC = ChunkElems<E>::value;
    constexpr int PW = 32 * KCH * VEC;  // columns per panel
    constexpr bool TWO = (E == Elem::A16 || E == Elem::AB16 || E == Elem::AB16R);
    constexpr int esz = (E == Elem::F32) ? 4 : 2;
    __shared__ double smf[8];
    __shared__ float smc[8][PW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t b = (int64_t)blockIdx.x * 8 + w;
    const int64_t c0 = (int64_t)blockIdx.y * PW;
    const int64_t nch = (n + VEC - 1) / VEC;
    float acc[KCH][VEC], csq[KCH][VEC];
#pragma unroll
    for (int k = 0; k < KCH; ++k)
#pragma unroll
        for (int e = 0; e < VEC; ++e) acc[k][e] = csq[k][e] = 0.0f;
    bool live[KCH];
#pragma unroll
    for (int k = 0; k < KCH; ++k) live[k] = (c0 / VEC + k * 32 + lane) < nch;
    const bool ragged = (n % VEC) != 0;
    if (b < s) {
        const int32_t o0 = offsets[b], o1 = offsets[b + 1];
        for (int32_t q = o0; q < o1; q += 4) {
            int32_t r[4];
            float sg[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                r[u] = q + u < o1 ? perm[q + u] : -1;
                sg[u] = r[u] >= 0 ? (float)sign[r[u]] : 0.0f;
            }
            uint4 h[4][KCH], l[4][KCH];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int k = 0; k < KCH; ++k) {
                    h[u][k] = l[u][k] = make_uint4(0, 0, 0, 0);
                    if (r[u] >= 0 && live[k]) {
                        const size_t off = (size_t)r[u] * ld * esz + (size_t)(c0 + (k * 32 + lane) * VEC) * esz;
                        h[u][k] = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint8_t*>(hi) + off));
                        if (TWO) l[u][k] = __ldcs(reinterpret_cast<const uint4*>(static_cast<const uint8_t*>(lo) + off));
                    }
                }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int k = 0; k < KCH; ++k) {
                    if (r[u] < 0 || !live[k]) continue;
                    float f[VEC];
                    ChunkDecoder<E>::decode(h[u][k], l[u][k], f);
                    const int64_t cbase = c0 + (int64_t)(k * 32 + lane) * VEC;
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        if (ragged && cbase + e >= n) continue;
                        const float a = f[e];
                        acc[k][e] = fmaf(sg[u], a, acc[k][e]);
                        csq[k][e] = fmaf(a, a, csq[k][e]);
                    }
                }
        }
#pragma unroll
        for (int k = 0; k < KCH; ++k) {
            const int64_t cbase = c0 + (int64_t)(k * 32 + lane) * VEC;
#pragma unroll
            for (int e = 0; e < VEC; ++e)
                if (live[k] && cbase + e < n) SA[(size_t)(cbase + e) * ld_sa + b] = (double)acc[k][e];
        }
    }
    double f2 = 0.0;
#pragma unroll
    for (int k = 0; k < KCH; ++k)
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
            smc[w][(k * 32 + lane) * VEC + e] = csq[k][e];
            f2 += (double)csq[k][e];
        }
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
        for (int e = threadIdx.x; e < PW; e += blockDim.x) {
            const int64_t j = c0 + e;
            if (j >= n) continue;
            double t = 0.0;
#pragma unroll
            for (int k = 0; k < 8; ++k) t += (double)smc[k][e];
            col_part[(size_t)blockIdx.x * n + j] = t;
        }
    }
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
    const int64_t rows = (s + 7) / 8;                  // row-major owner blocks
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
                          cudaStream_t st) {
    int g;
    cs_grid(m, &g);
    TOMOS_CUDA_TRY(cudaMemsetAsync(c.counts, 0, sizeof(int32_t) * (s + 1), st));
    TOMOS_CUDA_TRY(cudaMemsetAsync(c.cursor, 0, sizeof(int32_t) * (s + 1), st));
    cs_hash_kernel<<<g, 256, 0, st>>>(m, s, bseed, sseed, c.bucket, c.sign, c.counts);
    TOMOS_LAUNCH_CHECK("cs_hash_kernel");
    cs_scan_kernel<<<1, 1024, 0, st>>>(c.counts, s, c.offsets);
    TOMOS_LAUNCH_CHECK("cs_scan_kernel");
    cs_scatter_kernel<<<g, 256, 0, st>>>(m, c.bucket, c.offsets, c.cursor, c.perm);
    TOMOS_LAUNCH_CHECK("cs_scatter_kernel");
    cs_sort_kernel<<<(unsigned)((s + 7) / 8), 256, 0, st>>>(s, c.offsets, c.perm);
    TOMOS_LAUNCH_CHECK("cs_sort_kernel");
    return TOMOS_OK;
}

// Panel width of the row-major owner sums for an element type.
template <Elem E>
static int rows_vec_panel() {
    return 32 * 2 * ChunkElems<E>::value;
}

template <Elem E>
static unsigned launch_rows(const tomos_dense* A, const void* lo, int64_t s, const CsScratch& c,
                            double* SA, int64_t ld_sa, bool want_cols, unsigned gx,
                            cudaStream_t st) {
    const int esz = (E == Elem::F32) ? 4 : 2;
    bool vec = ((A->ld * esz) % 16 == 0) && (reinterpret_cast<uintptr_t>(A->values) % 16 == 0);
    if (vec && lo) vec = reinterpret_cast<uintptr_t>(lo) % 16 == 0;
    if (vec) {
        const unsigned panels = (unsigned)((A->cols + rows_vec_panel<E>() - 1) / rows_vec_panel<E>());
        cs_rows_vec_kernel<E, 2><<<dim3(gx, panels), 256, 0, st>>>(
            A->values, lo, A->cols, A->ld, s, c.offsets, c.perm, c.sign, SA, ld_sa, c.fro_part,
            want_cols ? c.col_part : nullptr);
        return panels;
    }
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
    cs_hash_kernel<<<g, 256, 0, as_stream(stream)>>>(m, s, bucket_seed, sign_seed, bucket, sign,
                                                     nullptr);
    TOMOS_LAUNCH_CHECK("cs_hash_kernel");
    return TOMOS_OK;
}

size_t tomos_countsketch_scratch_bytes(int64_t m, int64_t cols, int64_t s) {
    if (m < 0 || s <= 0 || cols < 0) return 0;
    return cs_layout(nullptr, m, s, cs_fro_parts(m, s), cs_col_part_rows(m, s) * cols).bytes;
}

tomos_status tomos_countsketch_apply(const tomos_dense* A, int32_t tier, int64_t s,
                                     uint64_t bucket_seed, uint64_t sign_seed, double* SA,
                                     int64_t ld_sa, double* fro2, double* colsq, void* scratch,
                                     size_t scratch_bytes, void* stream) {
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
    tomos_status rc = cs_bucketize(m, s, bucket_seed, sign_seed, c, st);
    if (rc) return rc;
    const void* lo = (e == Elem::A16 || e == Elem::AB16 || e == Elem::AB16R) ? dense_lo_plane(A)
                                                                             : nullptr;
    int64_t nparts;
    if (A->layout == TOMOS_ROW_MAJOR) {
        const unsigned gx = (unsigned)((s + 7) / 8);
        unsigned panels = 0;
        switch (e) {
            case Elem::F32: panels = launch_rows<Elem::F32>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::H16: panels = launch_rows<Elem::H16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
            case Elem::A16: panels = launch_rows<Elem::A16>(A, lo, s, c, SA, ld_sa, colsq, gx, st); break;
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

}  // extern "C"
