// sketch.cuh -- internal interface of the hash CountSketch (sketch.cu),
// shared with the CSR owner sums (csr.cu).
#pragma once

#include "common.cuh"

namespace tomos_b200 {

// SplitMix64 finaliser (the reference's bucket/sign hash).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// Caller-scratch layout of one sketch application (256-byte aligned slices).
struct CsScratch {
    int32_t* bucket;    // m: bucket of row i
    int8_t* sign;       // m: +1 / -1
    int32_t* counts;    // s + 1
    int32_t* offsets;   // s + 1: bucket b holds perm[offsets[b] .. offsets[b+1])
    int32_t* cursor;    // s + 1
    int32_t* perm;      // m: row ids grouped by bucket, ascending within a bucket
    double* fro_part;   // owner-sum partials of sum(A_ij^2)
    double* col_part;   // per-block partial column sums of squares
    size_t bytes;
};

CsScratch cs_layout(void* base, int64_t m, int64_t s, int64_t fro_parts, int64_t col_parts);
// Rows of col_part any caller may need (times the column count).
int64_t cs_col_part_rows(int64_t m, int64_t s);
int64_t cs_fro_parts(int64_t m, int64_t s);
tomos_status cs_bucketize(int64_t m, int64_t s, uint64_t bseed, uint64_t sseed, const CsScratch& c,
                          cudaStream_t st, int64_t row0 = 0);

}  // namespace tomos_b200
