// comm.cu -- the communicator of a row-sharded solve (NCCL over NVLink /
// NVSwitch), and the partial-sum reduction every pass over a row shard ends
// with.
//
// Sharding: rank r of P holds rows [r0_r, r1_r) of A and of b.  A p is
// local; A^T u = sum_r A_r^T u_r and ||u||^2 = sum_r ||u_r||^2 are the only
// quantities that cross ranks (lsqr.cpp:561-621 splits into a local product
// and one sum over ranks).  After each pass, shard_reduce_kernel folds the
// pass's per-CTA partials into n + 1 doubles (A^T u, then ||u||^2) in a
// fixed order, and one ncclAllReduce sums them across ranks on the solver
// stream (captured into the iteration graph like the kernels around it;
// the solve destroys that graph before it returns, so no graph holding an
// NCCL call outlives the call that made it).
// Every rank then holds the same n-side inputs, runs the same
// deterministic n-side kernels, and keeps identical x, v, w and Givens
// state without further exchange.
#include <nccl.h>

#include <cstring>
#include <string>

#include "common.cuh"
#include "lsqr.cuh"

struct tomos_comm {
    ncclComm_t nccl = nullptr;
    int32_t nranks = 1, rank = 0, device = 0;
};

namespace tomos_b200 {

namespace {
tomos_status nccl_fail(ncclResult_t r, const char* what) {
    return fail(TOMOS_ERR_CUDA, std::string(what) + ": " + ncclGetErrorString(r));
}
}  // namespace

// out[j] = sum_c qpart[c][j] (j < n, c < gq, FP32 partials summed in FP64
// in CTA order), out[n] = sum_c sspart[c].
__global__ void shard_reduce_kernel(const float* __restrict__ qpart, int gq, int64_t qstride, int64_t n,
                                    const double* __restrict__ sspart, int gs, const int* skip,
                                    double* __restrict__ out) {
    if (skip && *skip) return;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        double q = 0.0;
        for (int c = 0; c < gq; ++c) q += (double)qpart[(size_t)c * qstride + j];
        out[j] = q;
    } else if (j == n) {
        double s = 0.0;
        for (int c = 0; c < gs; ++c) s += sspart[c];
        out[n] = s;
    }
}

tomos_status comm_allreduce(tomos_comm* c, double* buf, int64_t count, cudaStream_t st) {
    if (!c || count <= 0) return TOMOS_OK;  // one rank too: NCCL copies in place
    ncclResult_t r = ncclAllReduce(buf, buf, (size_t)count, ncclDouble, ncclSum, c->nccl, st);
    if (r != ncclSuccess) return nccl_fail(r, "ncclAllReduce");
    return TOMOS_OK;
}

tomos_status enqueue_shard_reduce(tomos_workspace* ws, tomos_comm* c, const float* qpart, int gq,
                                  int64_t qstride, const double* sspart, int gs, const int* skip,
                                  cudaStream_t st) {
    const int64_t n = ws->n;
    shard_reduce_kernel<<<(unsigned)((n + 1 + 255) / 256), 256, 0, st>>>(qpart, gq, qstride, n, sspart, gs,
                                                                         skip, ws->shard);
    TOMOS_LAUNCH_CHECK("shard_reduce_kernel");
    ws->launches += 1;
    return comm_allreduce(c, ws->shard, n + 1, st);
}

}  // namespace tomos_b200

using namespace tomos_b200;

extern "C" {

tomos_status tomos_comm_unique_id(void* id) {
    if (!id) return fail(TOMOS_ERR_INVALID, "comm_unique_id: null output");
    ncclUniqueId u;
    ncclResult_t r = ncclGetUniqueId(&u);
    if (r != ncclSuccess) return nccl_fail(r, "ncclGetUniqueId");
    static_assert(sizeof(ncclUniqueId) <= TOMOS_COMM_ID_BYTES, "unique id size");
    std::memset(id, 0, TOMOS_COMM_ID_BYTES);
    std::memcpy(id, &u, sizeof(u));
    return TOMOS_OK;
}

tomos_status tomos_comm_create(int32_t nranks, int32_t rank, const void* id, tomos_comm** out) {
    if (!out || !id) return fail(TOMOS_ERR_INVALID, "comm_create: null pointer");
    *out = nullptr;
    if (nranks < 1 || rank < 0 || rank >= nranks) return fail(TOMOS_ERR_INVALID, "comm_create: bad rank");
    tomos_comm* c = new tomos_comm();
    c->nranks = nranks;
    c->rank = rank;
    cudaGetDevice(&c->device);
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    ncclResult_t r = ncclCommInitRank(&c->nccl, nranks, u, rank);
    if (r != ncclSuccess) {
        delete c;
        return nccl_fail(r, "ncclCommInitRank");
    }
    *out = c;
    return TOMOS_OK;
}

tomos_status tomos_comm_destroy(tomos_comm* c) {
    if (!c) return TOMOS_OK;
    if (c->nccl) ncclCommDestroy(c->nccl);
    delete c;
    return TOMOS_OK;
}

tomos_status tomos_comm_allreduce_f64(tomos_comm* c, double* buf, int64_t count, void* stream) {
    if (!c) return fail(TOMOS_ERR_INVALID, "comm_allreduce_f64: null communicator");
    if (count > 0 && !buf) return fail(TOMOS_ERR_INVALID, "comm_allreduce_f64: null buffer");
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != c->device) return fail(TOMOS_ERR_INVALID, "comm_allreduce_f64: communicator of another device");
    return comm_allreduce(c, buf, count, as_stream(stream));
}

}  // extern "C"
