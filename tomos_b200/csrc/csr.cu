// csr.cu -- CSR products (tomos_csr_gemv), the CSR LSQR pass
// (tomos_lsqr_solve_csr) and the CSR CountSketch.
//
// The reference's CSR path (cuda::mv_csr, mv_cuda_kernels.cu:1964-2058)
// is one thread per row for A x and an atomicAdd scatter for A^T x; it has
// no packed (FP32_16) values (lsqr_registries.cpp:274-285).  Here values
// may be FP32, FP32_16 or FP32_BF16 (read at a tier like the dense path),
// indices int32, and both products are deterministic:
//   * a warp owns a row; lanes stride its nonzeros, reading p through L1;
//   * the transposed product accumulates into a warp-private FP32 vector
//     in shared memory.  A CSR row has distinct column indices, so the
//     lanes of one row never touch the same word and no atomics are
//     needed; the CTA sums its warps' vectors in a fixed order and writes
//     one partial row, reduced across CTAs in a fixed order later.
// The LSQR pass fuses both: ut_i = cp (A p)_i + cu u_i, then
// q += ut_i A[i, :] while row i is in registers -- one read of the index
// and value arrays per iteration.
#include <cstring>
#include <string>
#include <type_traits>

#include "common.cuh"
#include "gemv.cuh"
#include "lsqr.cuh"
#include "sketch.cuh"

namespace tomos_b200 {

constexpr int kCsrMaxWarps = 8;
constexpr size_t kCsrSmemBudget = 200 * 1024;

struct CsrPassParams {
    const void* hi;
    const void* lo;
    const int32_t* row_ptrs;
    const int32_t* col_idxs;
    int64_t m, n;
    const float* p;
    const float* u_in;
    float* u_out;
    const double* coef;     // device [cp, cu], or NULL: use cp_h / cu_h
    double cp_h, cu_h;
    float* qpart;           // gridDim.x x qstride (NULL: no transposed product)
    int64_t qstride;
    double* sspart;         // gridDim.x (NULL: skip)
    const int* skip;
    int write_u;            // 0: A p only feeds the transposed product
};

// One kernel, three uses: the fused LSQR pass (write_u, qpart, sspart),
// the plain product (write_u only: y = cp A p + cu y) and the transposed
// product (qpart only, with u_in as the input vector and cp = 0, cu = 1).
template <Elem E, bool ACC64>
__global__ void __launch_bounds__(256) csr_pass_kernel(CsrPassParams P) {
    if (P.skip && *P.skip) return;
    using Dot = typename std::conditional<ACC64, double, float>::type;
    extern __shared__ __align__(16) float qacc[];  // nw x n_pad
    __shared__ double ssw[kCsrMaxWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t npad = P.qstride;
    double cp = P.cp_h, cu = P.cu_h;
    if (P.coef) {
        cp = P.coef[0];
        cu = P.coef[1];
    }
    float* acc = qacc + (size_t)w * npad;
    if (P.qpart)
        for (int64_t j = lane; j < npad; j += 32) acc[j] = 0.0f;
    __syncwarp();
    const int64_t per = (P.m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * per;
    int64_t r1 = r0 + per;
    if (r1 > P.m) r1 = P.m;
    double ss = 0.0;
    for (int64_t i = r0 + w; i < r1; i += nw) {
        const int32_t k0 = P.row_ptrs[i], k1 = P.row_ptrs[i + 1];
        double ut;
        if (cp != 0.0) {
            Dot d = 0;
            for (int32_t k = k0 + lane; k < k1; k += 32)
                d += (Dot)load_elem<E>(P.hi, P.lo, k) * (Dot)__ldg(P.p + P.col_idxs[k]);
            d = warp_sum(d);
            ut = cp * (double)d + cu * (double)__ldg(P.u_in + i);
        } else {
            ut = cu * (double)__ldg(P.u_in + i);
        }
        const float uf = (float)ut;
        if (lane == 0) {
            if (P.write_u) P.u_out[i] = uf;
            ss += (double)uf * (double)uf;
        }
        if (P.qpart) {
            for (int32_t k = k0 + lane; k < k1; k += 32) {
                const int32_t c = P.col_idxs[k];
                acc[c] = fmaf(load_elem<E>(P.hi, P.lo, k), uf, acc[c]);
            }
            __syncwarp();
        }
    }
    if (lane == 0) ssw[w] = ss;
    __syncthreads();
    if (P.qpart) {
        float* out = P.qpart + (size_t)blockIdx.x * npad;
        for (int64_t j = threadIdx.x; j < P.n; j += blockDim.x) {
            float s = 0.0f;
            for (int k = 0; k < nw; ++k) s += qacc[(size_t)k * npad + j];
            out[j] = s;
        }
    }
    if (P.sspart && threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < nw; ++k) s += ssw[k];
        P.sspart[blockIdx.x] = s;
    }
}

// y[j] = alpha * sum_c part[c][j] + beta * y[j] (fixed order).
__global__ void csr_trans_reduce_kernel(const float* __restrict__ part, int g, int64_t stride,
                                        int64_t n, double alpha, double beta, float* __restrict__ y) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int c = 0; c < g; ++c) s += (double)part[(size_t)c * stride + j];
    double r = alpha * s;
    if (beta != 0.0) r += beta * (double)y[j];
    y[j] = (float)r;
}

static int csr_warps_for(int64_t n) {
    const int64_t npad = ((n + 31) / 32) * 32;
    int64_t w = (int64_t)(kCsrSmemBudget / (sizeof(float) * (npad > 0 ? npad : 32)));
    if (w > kCsrMaxWarps) w = kCsrMaxWarps;
    return (int)w;
}

template <Elem E, bool ACC64>
static tomos_status launch_csr_t(const CsrPassParams& P, int grid, int warps, cudaStream_t st) {
    const size_t smem = P.qpart ? (size_t)warps * P.qstride * sizeof(float) : 0;
    if (smem > 48 * 1024)
        TOMOS_CUDA_TRY(cudaFuncSetAttribute(csr_pass_kernel<E, ACC64>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    csr_pass_kernel<E, ACC64><<<grid, warps * 32, smem, st>>>(P);
    TOMOS_LAUNCH_CHECK("csr_pass_kernel");
    return TOMOS_OK;
}

static tomos_status launch_csr(Elem e, bool acc64, const CsrPassParams& P, int grid, int warps,
                               cudaStream_t st) {
    switch (e) {
        case Elem::F32: return acc64 ? launch_csr_t<Elem::F32, true>(P, grid, warps, st)
                                     : launch_csr_t<Elem::F32, false>(P, grid, warps, st);
        case Elem::H16: return acc64 ? launch_csr_t<Elem::H16, true>(P, grid, warps, st)
                                     : launch_csr_t<Elem::H16, false>(P, grid, warps, st);
        case Elem::F16: return acc64 ? launch_csr_t<Elem::F16, true>(P, grid, warps, st)
                                     : launch_csr_t<Elem::F16, false>(P, grid, warps, st);
        case Elem::B16: return acc64 ? launch_csr_t<Elem::B16, true>(P, grid, warps, st)
                                     : launch_csr_t<Elem::B16, false>(P, grid, warps, st);
        case Elem::A16: return launch_csr_t<Elem::A16, true>(P, grid, warps, st);
        case Elem::AB16: return launch_csr_t<Elem::AB16, true>(P, grid, warps, st);
        case Elem::AB16R: return launch_csr_t<Elem::AB16R, true>(P, grid, warps, st);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "csr: element type");
    }
}

static const void* csr_lo(const tomos_csr* A) {
    if (A->values_lo) return A->values_lo;
    return static_cast<const uint16_t*>(A->values) + A->nnz;
}

static bool csr_ok(const tomos_csr* A, std::string* why) {
    if (!A) {
        *why = "null matrix";
        return false;
    }
    if (A->rows < 0 || A->cols < 0 || A->nnz < 0) {
        *why = "negative size";
        return false;
    }
    if (A->index_type != 0) {
        *why = "only int32 indices are registered";
        return false;
    }
    if (A->rows > 0x7fffffffLL || A->nnz > 0x7fffffffLL) {
        *why = "size exceeds int32 indexing";
        return false;
    }
    if (csr_warps_for(A->cols) < 1) {
        *why = "n too large for the shared-memory accumulators";
        return false;
    }
    return true;
}

static int csr_grid(int64_t m) {
    int64_t g = (int64_t)sm_count() * 2;
    int64_t gr = (m + 63) / 64;
    if (g > gr) g = gr;
    return (int)(g < 1 ? 1 : g);
}

static int64_t csr_qstride(int64_t n) { return ((n + 31) / 32) * 32 < 32 ? 32 : ((n + 31) / 32) * 32; }

// ------------------------------------------------------------------
// The CSR LSQR pass as two gathers over a per-solve column-major copy.
//
// The fused row pass above keeps A^T ut deterministic with a private
// accumulator per warp (n floats of shared memory each), which caps a
// CTA at a few warps; a 20-nonzero row moves 120 bytes through a chain of
// dependent loads, so only a few KB are in flight per SM where the memory
// system needs tens.  The solver therefore runs each pass as two gathers:
//   csr_rows_kernel: ut_i = cp (A p)_i + cu u_i with G lanes per row and
//     two rows per lane group in flight, ||ut||^2 per CTA;
//   csc_cols_kernel: q_j = sum_i A[i, j] ut_i over a column-major (CSC)
//     copy of A, a warp per column, eight loads in flight per lane, ut
//     gathered from L2.
// Both sum in a fixed order.  The copy (row indices and both value planes,
// permuted) is built once per solve by a stable counting sort: entries per
// (row block, column), a scan over blocks and columns, then each row block
// scatters its rows in order.  Entries whose column lies outside [0, n)
// are skipped by every kernel here.

constexpr int kCscBlocksPerSm = 8;
constexpr int kRowsThreads = 256;

__device__ __forceinline__ void csc_block_rows(int64_t m, int nb, int b, int64_t* r0, int64_t* r1) {
    const int64_t per = (m + nb - 1) / nb;
    *r0 = (int64_t)b * per;
    if (*r0 > m) *r0 = m;
    *r1 = *r0 + per < m ? *r0 + per : m;
}

// cnt[b * n + j] = entries of column j in row block b.
__global__ void __launch_bounds__(256) csc_count_kernel(const int32_t* __restrict__ row_ptrs,
                                                        const int32_t* __restrict__ col_idxs, int64_t m,
                                                        int32_t n, int32_t* __restrict__ cnt) {
    extern __shared__ int32_t ccount[];
    for (int j = threadIdx.x; j < n; j += blockDim.x) ccount[j] = 0;
    __syncthreads();
    int64_t r0, r1;
    csc_block_rows(m, gridDim.x, blockIdx.x, &r0, &r1);
    if (r0 < r1) {
        const int32_t k1 = row_ptrs[r1];
        for (int32_t k = row_ptrs[r0] + (int32_t)threadIdx.x; k < k1; k += blockDim.x) {
            const int32_t c = __ldg(col_idxs + k);
            if ((uint32_t)c < (uint32_t)n) atomicAdd(&ccount[c], 1);
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) cnt[(size_t)blockIdx.x * n + j] = ccount[j];
}

// cnt[b][j] := entries of column j in the blocks before b; tot[j] := all.
// A CTA owns 32 columns; its 8 warps split the blocks into 8 runs.
__global__ void __launch_bounds__(256) csc_block_scan_kernel(int32_t* __restrict__ cnt, int nb, int32_t n,
                                                             int32_t* __restrict__ tot) {
    __shared__ int32_t part[8][33];
    const int jl = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * 32 + jl;
    const int per = (nb + 7) / 8;
    const int b0 = g * per < nb ? g * per : nb;
    const int b1 = b0 + per < nb ? b0 + per : nb;
    int32_t s = 0;
    if (j < n)
        for (int b = b0; b < b1; ++b) s += cnt[(size_t)b * n + j];
    part[g][jl] = s;
    __syncthreads();
    int32_t run = 0;
    for (int h = 0; h < g; ++h) run += part[h][jl];
    if (j < n) {
        for (int b = b0; b < b1; ++b) {
            const int32_t c = cnt[(size_t)b * n + j];
            cnt[(size_t)b * n + j] = run;
            run += c;
        }
        if (g == 7) tot[j] = run;
    }
}

// col_ptr[0..n] = exclusive scan of tot (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) csc_col_ptr_kernel(const int32_t* __restrict__ tot, int32_t n,
                                                           int32_t* __restrict__ col_ptr) {
    __shared__ int32_t wsum[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int per = (n + 1023) / 1024;
    const int j0 = t * per < n ? t * per : n;
    const int j1 = j0 + per < n ? j0 + per : n;
    int32_t s = 0;
    for (int j = j0; j < j1; ++j) s += tot[j];
    int32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int32_t v = wsum[lane];
        int32_t iv = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, iv, o);
            if (lane >= o) iv += y;
        }
        wsum[lane] = iv - v;
    }
    __syncthreads();
    int32_t run = wsum[w] + incl - s;
    for (int j = j0; j < j1; ++j) {
        col_ptr[j] = run;
        run += tot[j];
    }
    if (t == 1023) col_ptr[n] = run;
}

// The CSC copy: one warp per row block walks its rows in order, so each
// column keeps its entries in increasing row order.  Sixteen rows' first
// 32 entries are loaded before any is placed.  VB: bytes of a value in the
// first plane (4: FP32, 2: a packed wh plane); lo: the second 16-bit plane
// or NULL.
template <int VB>
__global__ void __launch_bounds__(32) csc_scatter_kernel(const int32_t* __restrict__ row_ptrs,
                                                         const int32_t* __restrict__ col_idxs,
                                                         const void* __restrict__ hi,
                                                         const uint16_t* __restrict__ lo, int64_t m,
                                                         int32_t n, const int32_t* __restrict__ cnt,
                                                         const int32_t* __restrict__ col_ptr,
                                                         int32_t* __restrict__ rows_out,
                                                         void* __restrict__ hi_out,
                                                         uint16_t* __restrict__ lo_out) {
    using V = typename std::conditional<VB == 4, uint32_t, uint16_t>::type;
    extern __shared__ int32_t cur[];
    const int lane = threadIdx.x;
    for (int j = lane; j < n; j += 32) cur[j] = col_ptr[j] + cnt[(size_t)blockIdx.x * n + j];
    __syncwarp();
    const V* h = static_cast<const V*>(hi);
    V* ho = static_cast<V*>(hi_out);
    int64_t r0, r1;
    csc_block_rows(m, gridDim.x, blockIdx.x, &r0, &r1);
    constexpr int R = 16;
    for (int64_t i0 = r0; i0 < r1; i0 += R) {
        const int nr = r1 - i0 < R ? (int)(r1 - i0) : R;
        const int32_t rp = lane <= nr ? __ldg(row_ptrs + i0 + lane) : 0;
        int32_t c[R];
        V hv[R];
        uint16_t lv[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
            const int32_t k0 = __shfl_sync(0xffffffffu, rp, t), k1 = __shfl_sync(0xffffffffu, rp, t + 1);
            const int32_t k = k0 + lane;
            const bool ok = t < nr && k < k1;
            c[t] = ok ? __ldg(col_idxs + k) : -1;
            hv[t] = ok ? h[k] : (V)0;
            lv[t] = (ok && lo) ? lo[k] : (uint16_t)0;
        }
#pragma unroll
        for (int t = 0; t < R; ++t) {
            const int32_t k0 = __shfl_sync(0xffffffffu, rp, t), k1 = __shfl_sync(0xffffffffu, rp, t + 1);
            if ((uint32_t)c[t] < (uint32_t)n) {
                const int32_t pos = atomicAdd(&cur[c[t]], 1);
                rows_out[pos] = (int32_t)(i0 + t);
                ho[pos] = hv[t];
                if (lo) lo_out[pos] = lv[t];
            }
            if (t < nr && k1 - k0 > 32) {  // the rest of a long row
                for (int32_t k = k0 + 32 + lane; k < k1; k += 32) {
                    const int32_t cc = __ldg(col_idxs + k);
                    if ((uint32_t)cc < (uint32_t)n) {
                        const int32_t pos = atomicAdd(&cur[cc], 1);
                        rows_out[pos] = (int32_t)(i0 + t);
                        ho[pos] = h[k];
                        if (lo) lo_out[pos] = lo[k];
                    }
                }
            }
            __syncwarp();
        }
    }
}

// ut_i = cp (A p)_i + cu u_i for every row (u_out, when write_u) and
// ||ut||^2 per CTA (sspart, when set).  2^lg lanes per row; a warp holds
// two rounds of 32 >> lg rows.  Each lane sums its entries in order, then
// the group sums by a fixed butterfly.
template <Elem E, bool ACC64>
__global__ void __launch_bounds__(kRowsThreads, 4) csr_rows_kernel(CsrPassParams P, int lg) {
    if (P.skip && *P.skip) return;
    using Dot = typename std::conditional<ACC64, double, float>::type;
    __shared__ double ssw[kRowsThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int G = 1 << lg, sub = lane & (G - 1), grp = lane >> lg, rpw = 32 >> lg;
    double cp = P.cp_h, cu = P.cu_h;
    if (P.coef) {
        cp = P.coef[0];
        cu = P.coef[1];
    }
    const bool dot = cp != 0.0;
    const uint32_t n = (uint32_t)P.n;
    const int64_t step = (int64_t)gridDim.x * nw * 2 * rpw;
    double ss = 0.0;
    for (int64_t base = ((int64_t)blockIdx.x * nw + w) * 2 * rpw; base < P.m; base += step) {
        const int64_t ia = base + grp, ib = base + rpw + grp;
        int32_t ka0 = 0, ka1 = 0, kb0 = 0, kb1 = 0;
        if (dot && ia < P.m) {
            ka0 = __ldg(P.row_ptrs + ia);
            ka1 = __ldg(P.row_ptrs + ia + 1);
        }
        if (dot && ib < P.m) {
            kb0 = __ldg(P.row_ptrs + ib);
            kb1 = __ldg(P.row_ptrs + ib + 1);
        }
        Dot da = 0, db = 0;
        {
            int32_t ca[4], cb[4];
            float va[4], vb[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int32_t k = ka0 + sub + t * G;
                ca[t] = k < ka1 ? __ldg(P.col_idxs + k) : -1;
                va[t] = k < ka1 ? load_elem<E>(P.hi, P.lo, k) : 0.0f;
                const int32_t kk = kb0 + sub + t * G;
                cb[t] = kk < kb1 ? __ldg(P.col_idxs + kk) : -1;
                vb[t] = kk < kb1 ? load_elem<E>(P.hi, P.lo, kk) : 0.0f;
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const float pa = (uint32_t)ca[t] < n ? __ldg(P.p + ca[t]) : 0.0f;
                const float pb = (uint32_t)cb[t] < n ? __ldg(P.p + cb[t]) : 0.0f;
                da += (Dot)va[t] * (Dot)pa;
                db += (Dot)vb[t] * (Dot)pb;
            }
        }
        for (int32_t k = ka0 + sub + 4 * G; k < ka1; k += G) {
            const int32_t c = __ldg(P.col_idxs + k);
            if ((uint32_t)c < n) da += (Dot)load_elem<E>(P.hi, P.lo, k) * (Dot)__ldg(P.p + c);
        }
        for (int32_t k = kb0 + sub + 4 * G; k < kb1; k += G) {
            const int32_t c = __ldg(P.col_idxs + k);
            if ((uint32_t)c < n) db += (Dot)load_elem<E>(P.hi, P.lo, k) * (Dot)__ldg(P.p + c);
        }
        for (int o = G >> 1; o > 0; o >>= 1) {
            da += __shfl_xor_sync(0xffffffffu, da, o);
            db += __shfl_xor_sync(0xffffffffu, db, o);
        }
        if (sub == 0) {
            if (ia < P.m) {
                const float uf = (float)(cp * (double)da + cu * (double)__ldg(P.u_in + ia));
                if (P.write_u) P.u_out[ia] = uf;
                ss += (double)uf * (double)uf;
            }
            if (ib < P.m) {
                const float uf = (float)(cp * (double)db + cu * (double)__ldg(P.u_in + ib));
                if (P.write_u) P.u_out[ib] = uf;
                ss += (double)uf * (double)uf;
            }
        }
    }
    if (!P.sspart) return;
    ss = warp_sum(ss);
    if (lane == 0) ssw[w] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < nw; ++k) s += ssw[k];
        P.sspart[blockIdx.x] = s;
    }
}

// q_j = sum_i A[i, j] u_i over the CSC copy: a warp per column, each lane
// summing its entries in order, then a fixed butterfly.
template <Elem E, bool ACC64>
__global__ void __launch_bounds__(256) csc_cols_kernel(const int32_t* __restrict__ col_ptr,
                                                       const int32_t* __restrict__ rows, const void* hi,
                                                       const void* lo, int64_t n,
                                                       const float* __restrict__ u, const int* skip,
                                                       float* __restrict__ q) {
    if (skip && *skip) return;
    using Dot = typename std::conditional<ACC64, double, float>::type;
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int64_t W = (int64_t)gridDim.x * nw;
    for (int64_t j = (int64_t)blockIdx.x * nw + (threadIdx.x >> 5); j < n; j += W) {
        const int32_t k0 = __ldg(col_ptr + j), k1 = __ldg(col_ptr + j + 1);
        Dot d = 0;
        int32_t k = k0 + lane;
        for (; k + 7 * 32 < k1; k += 8 * 32) {
            int32_t r[8];
            float v[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                r[t] = __ldg(rows + k + 32 * t);
                v[t] = load_elem<E>(hi, lo, k + 32 * t);
            }
#pragma unroll
            for (int t = 0; t < 8; ++t) d += (Dot)v[t] * (Dot)__ldg(u + r[t]);
        }
        for (; k < k1; k += 32) d += (Dot)load_elem<E>(hi, lo, k) * (Dot)__ldg(u + __ldg(rows + k));
        d = warp_sum(d);
        if (lane == 0) q[j] = (float)d;
    }
}

// Lanes per row for the row gather: 4 loads per lane cover a row of
// average length.
static int csr_rows_lg(const tomos_csr* A) {
    const double avg = A->rows > 0 ? (double)A->nnz / (double)A->rows : 0.0;
    if (avg <= 16.0) return 2;
    if (avg <= 32.0) return 3;
    if (avg <= 64.0) return 4;
    return 5;
}

static int csr_rows_grid(int64_t m, int lg, int cap) {
    const int64_t rows_cta = (int64_t)(kRowsThreads / 32) * 2 * (32 >> lg);
    int64_t g = (m + rows_cta - 1) / rows_cta;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

template <Elem E, bool ACC64>
static tomos_status launch_rows_t(const CsrPassParams& P, int lg, int grid, cudaStream_t st) {
    csr_rows_kernel<E, ACC64><<<grid, kRowsThreads, 0, st>>>(P, lg);
    TOMOS_LAUNCH_CHECK("csr_rows_kernel");
    return TOMOS_OK;
}

static tomos_status launch_rows(Elem e, bool acc64, const CsrPassParams& P, int lg, int grid,
                                cudaStream_t st) {
    switch (e) {
        case Elem::F32: return acc64 ? launch_rows_t<Elem::F32, true>(P, lg, grid, st)
                                     : launch_rows_t<Elem::F32, false>(P, lg, grid, st);
        case Elem::H16: return acc64 ? launch_rows_t<Elem::H16, true>(P, lg, grid, st)
                                     : launch_rows_t<Elem::H16, false>(P, lg, grid, st);
        case Elem::F16: return acc64 ? launch_rows_t<Elem::F16, true>(P, lg, grid, st)
                                     : launch_rows_t<Elem::F16, false>(P, lg, grid, st);
        case Elem::B16: return acc64 ? launch_rows_t<Elem::B16, true>(P, lg, grid, st)
                                     : launch_rows_t<Elem::B16, false>(P, lg, grid, st);
        case Elem::A16: return launch_rows_t<Elem::A16, true>(P, lg, grid, st);
        case Elem::AB16: return launch_rows_t<Elem::AB16, true>(P, lg, grid, st);
        case Elem::AB16R: return launch_rows_t<Elem::AB16R, true>(P, lg, grid, st);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "csr: element type");
    }
}

// The CSC copy of a CSR matrix inside one device buffer.
struct CscCopy {
    int32_t* col_ptr = nullptr;  // n + 1
    int32_t* tot = nullptr;      // n
    int32_t* cnt = nullptr;      // nb x n
    int32_t* rows = nullptr;     // nnz
    void* hi = nullptr;          // nnz x vb
    uint16_t* lo = nullptr;      // nnz (packed storage with an exact tier), else NULL
    int nb = 0;
    size_t bytes = 0;
};

static size_t csc_align(size_t b) { return (b + 255) / 256 * 256; }

static CscCopy csc_layout(void* base, const tomos_csr* A, bool with_lo) {
    CscCopy c;
    const int64_t n = A->cols, nnz = A->nnz;
    int64_t nb = (int64_t)sm_count() * kCscBlocksPerSm;
    if (nb > A->rows) nb = A->rows;
    const int64_t cap = ((int64_t)64 << 20) / (n > 0 ? n : 1);
    if (nb > cap) nb = cap;
    if (nb < 1) nb = 1;
    c.nb = (int)nb;
    const int vb = A->numeric == TOMOS_FP32 ? 4 : 2;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* q = p ? p + off : nullptr;
        off += csc_align(bytes);
        return q;
    };
    c.col_ptr = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (n + 1)));
    c.tot = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (n > 0 ? n : 1)));
    c.cnt = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * nb * n));
    c.rows = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * nnz));
    c.hi = take((size_t)vb * nnz);
    c.lo = with_lo ? reinterpret_cast<uint16_t*>(take(sizeof(uint16_t) * nnz)) : nullptr;
    c.bytes = off;
    return c;
}

// Builds the CSC copy (4 launches).
static tomos_status csc_build(const tomos_csr* A, const CscCopy& c, const void* lo_in, cudaStream_t st) {
    const int64_t m = A->rows;
    const int32_t n = (int32_t)A->cols;
    const int32_t* rp = static_cast<const int32_t*>(A->row_ptrs);
    const int32_t* ci = static_cast<const int32_t*>(A->col_idxs);
    const size_t smem = sizeof(int32_t) * (size_t)n;
    if (smem > 48 * 1024) {
        TOMOS_CUDA_TRY(cudaFuncSetAttribute(csc_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        TOMOS_CUDA_TRY(cudaFuncSetAttribute(csc_scatter_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        TOMOS_CUDA_TRY(cudaFuncSetAttribute(csc_scatter_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    csc_count_kernel<<<c.nb, 256, smem, st>>>(rp, ci, m, n, c.cnt);
    TOMOS_LAUNCH_CHECK("csc_count_kernel");
    csc_block_scan_kernel<<<(unsigned)((n + 31) / 32), 256, 0, st>>>(c.cnt, c.nb, n, c.tot);
    TOMOS_LAUNCH_CHECK("csc_block_scan_kernel");
    csc_col_ptr_kernel<<<1, 1024, 0, st>>>(c.tot, n, c.col_ptr);
    TOMOS_LAUNCH_CHECK("csc_col_ptr_kernel");
    const uint16_t* lo = c.lo ? static_cast<const uint16_t*>(lo_in) : nullptr;
    if (A->numeric == TOMOS_FP32)
        csc_scatter_kernel<4><<<c.nb, 32, smem, st>>>(rp, ci, A->values, nullptr, m, n, c.cnt, c.col_ptr,
                                                       c.rows, c.hi, nullptr);
    else
        csc_scatter_kernel<2><<<c.nb, 32, smem, st>>>(rp, ci, A->values, lo, m, n, c.cnt, c.col_ptr,
                                                       c.rows, c.hi, c.lo);
    TOMOS_LAUNCH_CHECK("csc_scatter_kernel");
    return TOMOS_OK;
}

template <Elem E, bool ACC64>
static tomos_status launch_cols_t(const CscCopy& c, int64_t n, const float* u, const int* skip, float* q,
                                  cudaStream_t st) {
    int64_t grid = (n + 7) / 8;
    const int64_t cap = (int64_t)sm_count() * 8;
    if (grid > cap) grid = cap;
    if (grid < 1) grid = 1;
    csc_cols_kernel<E, ACC64><<<(unsigned)grid, 256, 0, st>>>(c.col_ptr, c.rows, c.hi, c.lo, n, u, skip, q);
    TOMOS_LAUNCH_CHECK("csc_cols_kernel");
    return TOMOS_OK;
}

static tomos_status launch_cols(Elem e, bool acc64, const CscCopy& c, int64_t n, const float* u,
                                const int* skip, float* q, cudaStream_t st) {
    switch (e) {
        case Elem::F32: return acc64 ? launch_cols_t<Elem::F32, true>(c, n, u, skip, q, st)
                                     : launch_cols_t<Elem::F32, false>(c, n, u, skip, q, st);
        case Elem::H16: return acc64 ? launch_cols_t<Elem::H16, true>(c, n, u, skip, q, st)
                                     : launch_cols_t<Elem::H16, false>(c, n, u, skip, q, st);
        case Elem::F16: return acc64 ? launch_cols_t<Elem::F16, true>(c, n, u, skip, q, st)
                                     : launch_cols_t<Elem::F16, false>(c, n, u, skip, q, st);
        case Elem::B16: return acc64 ? launch_cols_t<Elem::B16, true>(c, n, u, skip, q, st)
                                     : launch_cols_t<Elem::B16, false>(c, n, u, skip, q, st);
        case Elem::A16: return launch_cols_t<Elem::A16, true>(c, n, u, skip, q, st);
        case Elem::AB16: return launch_cols_t<Elem::AB16, true>(c, n, u, skip, q, st);
        case Elem::AB16R: return launch_cols_t<Elem::AB16R, true>(c, n, u, skip, q, st);
        default: return fail(TOMOS_ERR_UNSUPPORTED, "csr: element type");
    }
}

// The CSR LSQR pass: the two gathers over the CSC copy, or the fused row
// pass when the copy does not fit in device memory.
struct CsrPass : PassOps {
    tomos_workspace* ws;
    const tomos_csr* A;
    Elem iter_e, init_e;
    bool csc = false;
    bool allow_csc = true;  // false: the row pass only (the workspace's CSC copy serves another pass)
    CscCopy cc;
    int lg = 3;
    CsrPass(tomos_workspace* w, const tomos_csr* a, Elem ie, Elem ze) : ws(w), A(a), iter_e(ie), init_e(ze) {}
    tomos_status prepare(cudaStream_t st) override {
        if (!allow_csc) return TOMOS_OK;
        const bool with_lo = A->numeric != TOMOS_FP32 && (elem_is_exact(iter_e) || elem_is_exact(init_e));
        const CscCopy need = csc_layout(nullptr, A, with_lo);
        if (need.bytes > ws->csc_bytes) {
            if (ws->csc) cudaFree(ws->csc);
            ws->csc = nullptr;
            ws->csc_bytes = 0;
            if (cudaMalloc(&ws->csc, need.bytes) != cudaSuccess) {
                cudaGetLastError();
                return TOMOS_OK;  // not enough memory: the fused row pass
            }
            ws->csc_bytes = need.bytes;
        }
        cc = csc_layout(ws->csc, A, with_lo);
        lg = csr_rows_lg(A);
        tomos_status s = csc_build(A, cc, with_lo ? csr_lo(A) : nullptr, st);
        if (s) return s;
        ws->launches += 4;
        csc = true;
        return TOMOS_OK;
    }
    PassPlan plan(bool init) override {
        PassPlan pl;
        pl.fused = true;
        pl.e = init ? init_e : iter_e;
        pl.acc64 = init || elem_is_exact(pl.e);
        pl.qstride = ws->qstride;
        if (csc) {
            pl.grid = csr_rows_grid(A->rows, lg, ws->gmax);
            pl.gq = 1;  // csc_cols_kernel writes A^T ut whole
            pl.gs = pl.grid;
            pl.nch = lg;
            pl.g = 2;
            return pl;
        }
        pl.grid = csr_grid(A->rows);
        if (pl.grid > ws->gmax) pl.grid = ws->gmax;
        pl.gq = pl.grid;
        pl.gs = pl.grid;
        pl.nch = csr_warps_for(A->cols);
        return pl;
    }
    tomos_status enqueue(const PassPlan& pl, const float* p, const float* u_in, const double* coef,
                         const int* skip, cudaStream_t st) override {
        CsrPassParams P;
        P.hi = A->values;
        P.lo = elem_is_exact(pl.e) ? csr_lo(A) : nullptr;
        P.row_ptrs = static_cast<const int32_t*>(A->row_ptrs);
        P.col_idxs = static_cast<const int32_t*>(A->col_idxs);
        P.m = A->rows;
        P.n = A->cols;
        P.p = p;
        P.u_in = u_in;
        P.u_out = ws->u;
        P.coef = coef;
        P.cp_h = 1.0;
        P.cu_h = 0.0;
        P.qpart = ws->qpart;
        P.qstride = pl.qstride;
        P.sspart = ws->sspart;
        P.skip = skip;
        P.write_u = 1;
        if (csc) {
            tomos_status s = launch_rows(pl.e, pl.acc64, P, pl.nch, pl.grid, st);
            if (s) return s;
            ws->launches += 2;
            return launch_cols(pl.e, pl.acc64, cc, A->cols, ws->u, skip, ws->qpart, st);
        }
        ws->launches += 1;
        return launch_csr(pl.e, pl.acc64, P, pl.grid, pl.nch, st);
    }
    tomos_status fro2(double* out, const double* d, cudaStream_t st) override;
    uint64_t key() override {
        return reinterpret_cast<uint64_t>(A->values) ^ (reinterpret_cast<uint64_t>(A->col_idxs) << 1) ^
               (reinterpret_cast<uint64_t>(cc.rows) << 3) ^ (uint64_t)csc;
    }
    int64_t rows() override { return A->rows; }
    int64_t cols() override { return A->cols; }
};

template <Elem E>
__global__ void csr_fro2_kernel(const void* hi, const void* lo, const int32_t* col_idxs,
                                const double* d, int64_t nnz, double* part) {
    __shared__ double sm[8];
    double s = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (int64_t)gridDim.x * blockDim.x) {
        double v = load_elem<E>(hi, lo, k);
        if (d) v /= d[col_idxs[k]];
        s += v * v;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sm[k];
        part[blockIdx.x] = t;
    }
}

__global__ void csr_sum_kernel(const double* part, int np, double* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < np; ++k) s += part[k];
        *out = s;
    }
}

tomos_status CsrPass::fro2(double* out, const double* d, cudaStream_t st) {
    const int g = ws->gs_max;
    const void* lo = elem_is_exact(init_e) ? csr_lo(A) : nullptr;
    const int32_t* ci = static_cast<const int32_t*>(A->col_idxs);
#define TOMOS_CFRO(EE) csr_fro2_kernel<EE><<<g, 256, 0, st>>>(A->values, lo, ci, d, A->nnz, ws->bpart)
    switch (init_e) {
        case Elem::F32: TOMOS_CFRO(Elem::F32); break;
        case Elem::H16: TOMOS_CFRO(Elem::H16); break;
        case Elem::F16: TOMOS_CFRO(Elem::F16); break;
        case Elem::A16: TOMOS_CFRO(Elem::A16); break;
        case Elem::B16: TOMOS_CFRO(Elem::B16); break;
        case Elem::AB16: TOMOS_CFRO(Elem::AB16); break;
        case Elem::AB16R: TOMOS_CFRO(Elem::AB16R); break;
        default: return fail(TOMOS_ERR_UNSUPPORTED, "csr fro2: element type");
    }
#undef TOMOS_CFRO
    TOMOS_LAUNCH_CHECK("csr_fro2_kernel");
    csr_sum_kernel<<<1, 32, 0, st>>>(ws->bpart, g, out);
    TOMOS_LAUNCH_CHECK("csr_sum_kernel");
    return TOMOS_OK;
}

// CSR CountSketch owner sums: a warp per bucket accumulates its rows into
// a warp-private dense row (shared memory, FP64; distinct columns within a
// row need no atomics) in increasing row order, then the CTA writes its
// buckets' rows of SA together.  The rows' metadata (row id, sign, extent)
// come 32 rows at a time, a row a lane, and the next row's values are
// loaded before the current one is added, so a row costs the shared-memory
// update rather than a chain of dependent global loads.  The CTA's nw
// buckets are consecutive rows of the column-major SA: for each column it
// writes them as one run of nw doubles (SA is s x n, so writing a row of it
// alone would touch one 8-byte word per 32-byte sector).
template <Elem E>
__global__ void cs_csr_kernel(const void* hi, const void* lo, const int32_t* row_ptrs,
                              const int32_t* col_idxs, int64_t n, int64_t s,
                              const int32_t* offsets, const int32_t* perm, const int8_t* sign,
                              double* SA, int64_t ld_sa, double* fro_part) {
    extern __shared__ __align__(16) double racc[];
    __shared__ double smf[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t b0 = (int64_t)blockIdx.x * nw;
    const int64_t b = b0 + w;
    double* acc = racc + (size_t)w * n;
    double f2 = 0.0;
    for (int64_t j = lane; j < n; j += 32) acc[j] = 0.0;
    __syncwarp();
    if (b < s) {
        const int32_t o0 = offsets[b], o1 = offsets[b + 1];
        for (int32_t base = o0; base < o1; base += 32) {
            // rows base .. base+31 of the bucket: a row a lane
            int32_t rs = 0, re = 0;
            double sgl = 0.0;
            if (base + lane < o1) {
                const int32_t r = perm[base + lane];
                rs = row_ptrs[r];
                re = row_ptrs[r + 1];
                sgl = (double)sign[r];
            }
            const int cnt = (o1 - base) < 32 ? (o1 - base) : 32;
            // the first 32 values of the next row, loaded ahead
            int32_t ks = __shfl_sync(0xffffffffu, rs, 0), ke = __shfl_sync(0xffffffffu, re, 0);
            double va = 0.0;
            int32_t ca = 0;
            if (ks + lane < ke) {
                va = load_elem<E>(hi, lo, ks + lane);
                ca = col_idxs[ks + lane];
            }
            for (int q = 0; q < cnt; ++q) {
                const double sg = __shfl_sync(0xffffffffu, sgl, q);
                const int32_t cs = ks, ce = ke;
                const double vcur = va;
                const int32_t ccur = ca;
                if (q + 1 < cnt) {
                    ks = __shfl_sync(0xffffffffu, rs, q + 1);
                    ke = __shfl_sync(0xffffffffu, re, q + 1);
                    va = 0.0;
                    if (ks + lane < ke) {
                        va = load_elem<E>(hi, lo, ks + lane);
                        ca = col_idxs[ks + lane];
                    }
                }
                if (cs + lane < ce) {
                    acc[ccur] += sg * vcur;
                    f2 += vcur * vcur;
                }
                // a row longer than a warp: the rest in order
                for (int32_t k = cs + 32 + lane; k < ce; k += 32) {
                    const double a = load_elem<E>(hi, lo, k);
                    acc[col_idxs[k]] += sg * a;
                    f2 += a * a;
                }
                __syncwarp();
            }
        }
    }
    __syncthreads();
    // the CTA's buckets b0 .. b0+nw-1 for every column j, as runs of nw doubles
    const int nb = (int)((s - b0) < nw ? (s - b0) : nw);
    const int tot = (int)n * nb;  // n * 8 doubles fit shared memory: no overflow
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int j = idx / nb, k = idx - j * nb;
        SA[(size_t)j * ld_sa + b0 + k] = racc[(size_t)k * n + j];
    }
    f2 = warp_sum(f2);
    if (lane == 0) smf[w] = f2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < nw; ++k) t += smf[k];
        fro_part[blockIdx.x] = t;
    }
}

// Column sums of squares of a CSR matrix: CTAs own row chunks, warps
// accumulate into private FP64 rows in shared memory (distinct columns per
// row, no atomics), the CTA writes one partial row.
template <Elem E>
__global__ void csr_colsq_kernel(const void* hi, const void* lo, const int32_t* row_ptrs,
                                 const int32_t* col_idxs, int64_t m, int64_t n, double* col_part) {
    extern __shared__ __align__(16) double cacc[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double* acc = cacc + (size_t)w * n;
    for (int64_t j = lane; j < n; j += 32) acc[j] = 0.0;
    __syncwarp();
    const int64_t per = (m + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * per;
    const int64_t r1 = r0 + per < m ? r0 + per : m;
    for (int64_t i = r0 + w; i < r1; i += nw) {
        for (int32_t k = row_ptrs[i] + lane; k < row_ptrs[i + 1]; k += 32) {
            const double a = load_elem<E>(hi, lo, k);
            acc[col_idxs[k]] += a * a;
        }
        __syncwarp();
    }
    __syncthreads();
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        double t = 0.0;
        for (int k = 0; k < nw; ++k) t += cacc[(size_t)k * n + j];
        col_part[(size_t)blockIdx.x * n + j] = t;
    }
}

__global__ void csr_col_reduce_kernel(const double* part, int64_t nparts, int64_t n, double* colsq) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double t = 0.0;
    for (int64_t r = 0; r < nparts; ++r) t += part[(size_t)r * n + j];
    colsq[j] = t;
}

__global__ void cs_csr_fro_reduce(const double* part, int64_t np, double* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int64_t k = 0; k < np; ++k) s += part[k];
        *out = s;
    }
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

size_t tomos_csr_gemv_scratch_bytes(const tomos_csr* A, int32_t trans) {
    std::string why;
    if (!csr_ok(A, &why) || trans != TOMOS_TRANSPOSE) return 0;
    return (size_t)csr_grid(A->rows) * csr_qstride(A->cols) * sizeof(float);
}

tomos_status tomos_csr_gemv(int32_t trans, double alpha, const tomos_csr* A, int32_t tier,
                            const float* x, double beta, float* y, void* scratch,
                            size_t scratch_bytes, void* stream) {
    std::string why;
    if (!csr_ok(A, &why)) return fail(TOMOS_ERR_INVALID, "tomos_csr_gemv: " + why);
    if (trans != TOMOS_NO_TRANSPOSE && trans != TOMOS_TRANSPOSE)
        return fail(TOMOS_ERR_INVALID, "tomos_csr_gemv: bad transpose flag");
    Elem e;
    if (!resolve_elem_csr(A, tier, &e, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "tomos_csr_gemv: " + why);
    cudaStream_t st = as_stream(stream);
    const int64_t ylen = trans == TOMOS_NO_TRANSPOSE ? A->rows : A->cols;
    if (ylen == 0) return TOMOS_OK;
    if (!y || (!x && (trans == TOMOS_NO_TRANSPOSE ? A->cols : A->rows) > 0))
        return fail(TOMOS_ERR_INVALID, "tomos_csr_gemv: null vector");
    CsrPassParams P;
    P.hi = A->values;
    P.lo = elem_is_exact(e) ? csr_lo(A) : nullptr;
    P.row_ptrs = static_cast<const int32_t*>(A->row_ptrs);
    P.col_idxs = static_cast<const int32_t*>(A->col_idxs);
    P.m = A->rows;
    P.n = A->cols;
    P.coef = nullptr;
    P.sspart = nullptr;
    P.skip = nullptr;
    P.qstride = csr_qstride(A->cols);
    const int grid = csr_grid(A->rows);
    if (trans == TOMOS_NO_TRANSPOSE) {
        if (A->rows > 0 && !A->row_ptrs) return fail(TOMOS_ERR_INVALID, "tomos_csr_gemv: null row_ptrs");
        P.p = x;
        P.u_in = y;
        P.u_out = y;
        P.cp_h = alpha;
        P.cu_h = beta;
        P.qpart = nullptr;
        P.write_u = 1;
        if (beta == 0.0) {
            // beta == 0 must not read y: run with cu = 0 on a zeroed y.
            TOMOS_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(float) * A->rows, st));
        }
        if (A->rows == 0) return TOMOS_OK;
        const int lg = csr_rows_lg(A);
        return launch_rows(e, elem_is_exact(e), P, lg, csr_rows_grid(A->rows, lg, sm_count() * 4), st);
    }
    const size_t need = (size_t)grid * P.qstride * sizeof(float);
    if (!scratch || scratch_bytes < need)
        return fail(TOMOS_ERR_INVALID, "tomos_csr_gemv: scratch too small (need " + std::to_string(need) + " bytes)");
    if (A->rows == 0) {
        csr_trans_reduce_kernel<<<(unsigned)((A->cols + 255) / 256), 256, 0, st>>>(
            static_cast<float*>(scratch), 0, P.qstride, A->cols, alpha, beta, y);
        TOMOS_LAUNCH_CHECK("csr_trans_reduce_kernel");
        return TOMOS_OK;
    }
    P.p = nullptr;
    P.u_in = x;
    P.u_out = nullptr;
    P.cp_h = 0.0;
    P.cu_h = 1.0;
    P.qpart = static_cast<float*>(scratch);
    P.write_u = 0;
    tomos_status s = launch_csr(e, elem_is_exact(e), P, grid, csr_warps_for(A->cols), st);
    if (s) return s;
    csr_trans_reduce_kernel<<<(unsigned)((A->cols + 255) / 256), 256, 0, st>>>(
        P.qpart, grid, P.qstride, A->cols, alpha, beta, y);
    TOMOS_LAUNCH_CHECK("csr_trans_reduce_kernel");
    return TOMOS_OK;
}

tomos_status tomos_lsqr_solve_csr(const tomos_csr* A, const float* b, float* x,
                                  tomos_workspace* ws, const tomos_lsqr_opts* opts,
                                  tomos_lsqr_report* report, void* stream) {
    std::string why;
    if (!csr_ok(A, &why)) return fail(TOMOS_ERR_INVALID, "lsqr_solve: " + why);
    if (!opts_ok(opts, &why)) return fail(TOMOS_ERR_INVALID, "lsqr_solve: " + why);
    if (opts->refine) return fail(TOMOS_ERR_INVALID, "lsqr_solve: a dense mtx_refine_precision for a sparse A");
    if (opts->staged_plane) return fail(TOMOS_ERR_INVALID, "lsqr_solve: staged_plane needs a dense A");
    tomos_status s = workspace_check(ws, A->rows, A->cols);
    if (s) return s;
    if (!b || !x) return fail(TOMOS_ERR_INVALID, "lsqr_solve: null pointer");
    if (opts->implicit_duplicate && A->numeric != TOMOS_FP32_16 && A->numeric != TOMOS_FP32_BF16)
        return fail(TOMOS_ERR_INVALID, "lsqr_solve: use_implicit_duplicate_ requires packed A");
    Elem ie, ze;
    if (!resolve_elem_csr(A, opts->iter_tier, &ie, &why))
        return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_solve: " + why);
    const bool packed = A->numeric == TOMOS_FP32_16 || A->numeric == TOMOS_FP32_BF16;
    int32_t it = opts->iter_tier == TOMOS_TIER_AUTO ? (packed ? TOMOS_TIER_HALF : TOMOS_TIER_NATIVE)
                                                    : opts->iter_tier;
    int32_t zt = (packed && (opts->implicit_duplicate || opts->stop_rule == TOMOS_STOP_BACKWARD))
                     ? TOMOS_TIER_ACCURATE : it;
    if (!resolve_elem_csr(A, zt, &ze, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_solve: " + why);
    if (A->rows == 0 || A->cols == 0) {
        if (A->cols > 0 && !opts->warm_start) cudaMemsetAsync(x, 0, sizeof(float) * A->cols, as_stream(stream));
        if (report) {
            std::memset(report, 0, sizeof(*report));
            report->converged = 1;
        }
        return TOMOS_OK;
    }
    // The explicit duplicate (lsqr_sparse_impl's mtx_refine_precision,
    // lsqr_registries.cpp:180-183): the initial and restart passes read it,
    // exactly (FP32 values, or packed ones at the ACCURATE tier), through
    // the row pass; the iterations keep the CSC copy of A.
    if (opts->refine_csr) {
        const tomos_csr* Rf = opts->refine_csr;
        if (!csr_ok(Rf, &why)) return fail(TOMOS_ERR_INVALID, "lsqr_solve: mtx_refine_precision: " + why);
        if (Rf->rows != A->rows || Rf->cols != A->cols)
            return fail(TOMOS_ERR_INVALID, "lsqr_solve: mtx_refine_precision must have A's size");
        if (Rf->nnz > 0 && (!Rf->values || !Rf->col_idxs))
            return fail(TOMOS_ERR_INVALID, "lsqr_solve: mtx_refine_precision: null pointer");
        Elem re;
        const int32_t rt = (Rf->numeric == TOMOS_FP32_16 || Rf->numeric == TOMOS_FP32_BF16) ? TOMOS_TIER_ACCURATE
                                                                                          : TOMOS_TIER_NATIVE;
        if (!resolve_elem_csr(Rf, rt, &re, &why))
            return fail(TOMOS_ERR_UNSUPPORTED, "lsqr_solve: mtx_refine_precision: " + why);
        CsrPass pa(ws, A, ie, ie), pr(ws, Rf, re, re);
        pr.allow_csc = false;
        RefinePass ops(pa, pr);
        return solve_driver(ws, ops, b, x, opts, report, stream);
    }
    CsrPass ops(ws, A, ie, ze);
    return solve_driver(ws, ops, b, x, opts, report, stream);
}

tomos_status tomos_countsketch_apply_csr(const tomos_csr* A, int32_t tier, int64_t s,
                                         uint64_t bucket_seed, uint64_t sign_seed, double* SA,
                                         int64_t ld_sa, double* fro2, double* colsq, void* scratch,
                                         size_t scratch_bytes, void* stream) {
    std::string why;
    if (!csr_ok(A, &why)) return fail(TOMOS_ERR_INVALID, "countsketch_apply_csr: " + why);
    if (s <= 0 || ld_sa < s) return fail(TOMOS_ERR_INVALID, "countsketch_apply_csr: bad s / ld_sa");
    Elem e;
    if (!resolve_elem_csr(A, tier, &e, &why)) return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply_csr: " + why);
    const int64_t m = A->rows, n = A->cols;
    cudaStream_t st = as_stream(stream);
    if (n == 0) return TOMOS_OK;
    if (!SA) return fail(TOMOS_ERR_INVALID, "countsketch_apply_csr: null SA");
    // A warp needs n doubles of shared memory.
    const int64_t wpb = (int64_t)(kCsrSmemBudget / (sizeof(double) * (size_t)n));
    if (wpb < 1) return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply_csr: n too large");
    const int nw = (int)(wpb > 8 ? 8 : wpb);
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
        return fail(TOMOS_ERR_INVALID, "countsketch_apply_csr: scratch too small (need " +
                                           std::to_string(need.bytes) + " bytes)");
    CsScratch c = cs_layout(scratch, m, s, cs_fro_parts(m, s), col_parts);
    tomos_status rc = cs_bucketize(m, s, bucket_seed, sign_seed, c, st);
    if (rc) return rc;
    const void* lo = elem_is_exact(e) ? csr_lo(A) : nullptr;
    const unsigned grid = (unsigned)((s + nw - 1) / nw);
    const size_t smem = (size_t)nw * n * sizeof(double);
    const int32_t* rp = static_cast<const int32_t*>(A->row_ptrs);
    const int32_t* ci = static_cast<const int32_t*>(A->col_idxs);
#define TOMOS_CS_CSR(EE)                                                                        \
    do {                                                                                        \
        if (smem > 48 * 1024)                                                                   \
            TOMOS_CUDA_TRY(cudaFuncSetAttribute(cs_csr_kernel<EE>,                              \
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                                (int)smem));                                    \
        cs_csr_kernel<EE><<<grid, nw * 32, smem, st>>>(A->values, lo, rp, ci, n, s, c.offsets,  \
                                                       c.perm, c.sign, SA, ld_sa, c.fro_part); \
    } while (0)
    switch (e) {
        case Elem::F32: TOMOS_CS_CSR(Elem::F32); break;
        case Elem::H16: TOMOS_CS_CSR(Elem::H16); break;
        case Elem::F16: TOMOS_CS_CSR(Elem::F16); break;
        case Elem::A16: TOMOS_CS_CSR(Elem::A16); break;
        case Elem::B16: TOMOS_CS_CSR(Elem::B16); break;
        case Elem::AB16: TOMOS_CS_CSR(Elem::AB16); break;
        case Elem::AB16R: TOMOS_CS_CSR(Elem::AB16R); break;
        default: return fail(TOMOS_ERR_UNSUPPORTED, "countsketch_apply_csr: element type");
    }
#undef TOMOS_CS_CSR
    TOMOS_LAUNCH_CHECK("cs_csr_kernel");
    if (fro2) {
        cs_csr_fro_reduce<<<1, 32, 0, st>>>(c.fro_part, grid, fro2);
        TOMOS_LAUNCH_CHECK("cs_csr_fro_reduce");
    }
    if (colsq) {
        const int cg = csr_grid(m);
        const int64_t cw = (int64_t)(kCsrSmemBudget / (sizeof(double) * (size_t)n));
        const int cnw = (int)(cw > 8 ? 8 : cw);
        const size_t csm = (size_t)cnw * n * sizeof(double);
#define TOMOS_CSR_COLSQ(EE)                                                                      \
    do {                                                                                         \
        if (csm > 48 * 1024)                                                                     \
            TOMOS_CUDA_TRY(cudaFuncSetAttribute(csr_colsq_kernel<EE>,                            \
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                                (int)csm));                                      \
        csr_colsq_kernel<EE><<<cg, cnw * 32, csm, st>>>(A->values, lo, rp, ci, m, n, c.col_part); \
    } while (0)
        switch (e) {
            case Elem::F32: TOMOS_CSR_COLSQ(Elem::F32); break;
            case Elem::H16: TOMOS_CSR_COLSQ(Elem::H16); break;
            case Elem::F16: TOMOS_CSR_COLSQ(Elem::F16); break;
            case Elem::A16: TOMOS_CSR_COLSQ(Elem::A16); break;
            case Elem::B16: TOMOS_CSR_COLSQ(Elem::B16); break;
            case Elem::AB16: TOMOS_CSR_COLSQ(Elem::AB16); break;
            case Elem::AB16R: TOMOS_CSR_COLSQ(Elem::AB16R); break;
            default: break;
        }
#undef TOMOS_CSR_COLSQ
        TOMOS_LAUNCH_CHECK("csr_colsq_kernel");
        csr_col_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c.col_part, cg, n, colsq);
        TOMOS_LAUNCH_CHECK("csr_col_reduce_kernel");
    }
    return TOMOS_OK;
}

}  // extern "C"
