// tomos/b200.hpp -- the reference's C++ API (namespace tomos) over the C ABI
// of include/tomos_b200.h, header-only.
//
// A TOMOS caller switches by including this header instead of
// include/core/{solver,workspace,blas,matrix}.hpp and linking
// libtomos_b200.so + cudart.  Names, argument order and error behaviour
// follow the reference:
//   lsqr_solve, create_lsqr_workspace   include/core/solver.hpp:15-25,68-78
//   Workspace, add_precond              include/core/workspace.hpp:37-120
//   mv_apply, split_fp32_16,
//   combine_fp32_16                     include/core/blas.hpp
//   Dense::create_strided/wrap_strided  include/core/matrix.hpp:43-110
//   generate_sketch_qr_precond          src/core/precond/sketch_qr.hpp:19
// Invalid arguments throw std::invalid_argument and unregistered type
// combinations std::runtime_error, as the reference does.  Only
// Device::CUDA is registered (there is no CPU path).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tomos_b200.h"

namespace tomos {

enum class Device : std::size_t { CPU = 0, OMP = 1, CUDA = 2, Count };
enum class NumericType : std::size_t { FP64 = 0, FP32 = 1, FP16 = 2, FP32_16 = 3, BF16 = 4,
                                       FP32_BF16 = 5, Count };
enum class IntType : std::size_t { INT32 = 0, INT64 = 1, Count };
enum class Layout : std::size_t { ROW_MAJOR, COL_MAJOR };
enum TransposeType { NO_TRANSPOSE, TRANSPOSE };
enum Status { SUCCESS, FAILURE };

template <int len>
struct dim;
template <>
struct dim<2> {
    std::size_t nrows = 0, ncols = 0;
    dim(std::size_t r, std::size_t c) : nrows(r), ncols(c) {}
    std::size_t operator[](std::size_t i) const {
        if (i == 0) return nrows;
        if (i == 1) return ncols;
        throw std::invalid_argument("index should be either 0 or 1");
    }
};

namespace b200_detail {
inline void check(tomos_status s, const char* what) {
    if (s == TOMOS_OK) return;
    std::string msg = std::string(what) + ": " + tomos_last_error();
    if (s == TOMOS_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}
inline std::size_t elem_bytes(NumericType t) {
    switch (t) {
        case NumericType::FP64: return 8;
        case NumericType::FP32: return 4;
        case NumericType::FP16: return 2;  // native __half
        case NumericType::FP32_16:
        case NumericType::FP32_BF16: return 4;  // one uint32 slot: wh + wr planes
        default: throw std::runtime_error("no storage registered for this NumericType");
    }
}
inline int32_t tier_for(NumericType a, NumericType compute) {
    const bool packed = a == NumericType::FP32_16 || a == NumericType::FP32_BF16;
    if (packed && (compute == NumericType::FP16 || compute == NumericType::BF16))
        return TOMOS_TIER_HALF;
    if (packed && compute == NumericType::FP32) return TOMOS_TIER_ACCURATE;
    if (!packed && compute == a) return TOMOS_TIER_NATIVE;
    throw std::runtime_error("no mv kernel registered for this storage / compute type");
}
}  // namespace b200_detail

struct Context {
    explicit Context(Device d) : device_(d) {
        if (d != Device::CUDA)
            throw std::invalid_argument("Context: only Device::CUDA is registered");
    }
    Device get_device() const { return device_; }

private:
    Device device_;
};

// Strided dense matrix in device memory.
struct Dense {
    static Dense create_strided(Context& ctx, Layout layout, NumericType type, dim<2> size,
                                std::size_t lead_dim = 0) {
        (void)ctx;
        std::size_t outer = layout == Layout::COL_MAJOR ? size[1] : size[0];
        std::size_t inner = layout == Layout::COL_MAJOR ? size[0] : size[1];
        std::size_t ld = lead_dim ? lead_dim : inner;
        if (ld < inner) throw std::invalid_argument("create_strided: lead_dim too small");
        void* p = nullptr;
        std::size_t bytes = ld * outer * b200_detail::elem_bytes(type);
        if (cudaMalloc(&p, bytes ? bytes : 4) != cudaSuccess)
            throw std::runtime_error("create_strided: cudaMalloc failed");
        cudaMemset(p, 0, bytes ? bytes : 4);
        return Dense(layout, type, size, ld, p, true);
    }
    static Dense wrap_strided(Context&, Layout layout, NumericType type, dim<2> size,
                              std::size_t lead_dim, void* data) {
        return Dense(layout, type, size, lead_dim, data, false);
    }
    Dense(const Dense&) = delete;
    Dense& operator=(const Dense&) = delete;
    Dense(Dense&& o) noexcept { *this = std::move(o); }
    Dense& operator=(Dense&& o) noexcept {
        std::swap(d_, o.d_);
        std::swap(owns_, o.owns_);
        std::swap(size_, o.size_);
        return *this;
    }
    ~Dense() {
        if (owns_ && d_.values) cudaFree(d_.values);
    }
    dim<2> get_size() const { return size_; }
    NumericType get_value_type() const { return static_cast<NumericType>(d_.numeric); }
    Layout get_layout() const { return static_cast<Layout>(d_.layout); }
    std::size_t lead_dim() const { return static_cast<std::size_t>(d_.ld); }
    void* data() const { return d_.values; }
    const tomos_dense& desc() const { return d_; }
    // FP32_BF16 only: whether the pack rounds wh (fp32_bf16_split_rounded).
    void set_rounded(bool r) { d_.rounded = r ? 1 : 0; }

private:
    Dense(Layout layout, NumericType type, dim<2> size, std::size_t ld, void* p, bool owns)
        : size_(size) {
        d_.numeric = static_cast<int32_t>(type);
        d_.layout = layout == Layout::ROW_MAJOR ? TOMOS_ROW_MAJOR : TOMOS_COL_MAJOR;
        d_.rows = static_cast<int64_t>(size[0]);
        d_.cols = static_cast<int64_t>(size[1]);
        d_.ld = static_cast<int64_t>(ld);
        d_.values = p;
        d_.values_lo = nullptr;  // planar layout: wr follows wh
        d_.rounded = 0;
        d_.reserved = 0;
        owns_ = owns;
    }
    tomos_dense d_{};
    bool owns_ = false;
    dim<2> size_{0, 0};
};

// CSR matrix in device memory (non-owning view of caller buffers).
struct Sparse {
    static Sparse wrap_csr(Context&, NumericType type, IntType itype, dim<2> size, std::size_t nnz,
                           void* values, void* row_ptrs, void* col_idxs) {
        Sparse s;
        s.d_.numeric = static_cast<int32_t>(type);
        s.d_.index_type = static_cast<int32_t>(itype);
        s.d_.rows = static_cast<int64_t>(size[0]);
        s.d_.cols = static_cast<int64_t>(size[1]);
        s.d_.nnz = static_cast<int64_t>(nnz);
        s.d_.values = values;
        s.d_.row_ptrs = row_ptrs;
        s.d_.col_idxs = col_idxs;
        s.size_ = size;
        return s;
    }
    dim<2> get_size() const { return size_; }
    NumericType get_value_type() const { return static_cast<NumericType>(d_.numeric); }
    const tomos_csr& desc() const { return d_; }

private:
    tomos_csr d_{};
    dim<2> size_{0, 0};
};

enum class PrecondKind : std::size_t { None = 0, Dense = 1, Sparse = 2 };

struct Workspace {
    Device device_ = Device::CUDA;
    NumericType value_type_ = NumericType::FP32;
    NumericType precond_type_ = NumericType::FP32;
    PrecondKind precond_kind_ = PrecondKind::None;
    void* precond_ = nullptr;
    bool use_implicit_duplicate_ = false;
    NumericType mv_compute_type_ = NumericType::FP16;
    bool mv_compute_type_set_ = false;
    // The B200 solver's own options (defaults reproduce the reference).
    int32_t stop_rule = TOMOS_STOP_RELRES;
    double inner_rtol = 0.0;
    double anorm_fro = 0.0;
    tomos_lsqr_report last_report{};

    Workspace(std::size_t m, std::size_t n, NumericType value_type, NumericType precond_type)
        : value_type_(value_type), precond_type_(precond_type) {
        b200_detail::check(tomos_workspace_create(static_cast<int64_t>(m), static_cast<int64_t>(n),
                                                  static_cast<int32_t>(value_type),
                                                  static_cast<int32_t>(precond_type), &h_),
                           "create_lsqr_workspace");
    }
    Workspace(const Workspace&) = delete;
    Workspace& operator=(const Workspace&) = delete;
    Workspace(Workspace&& o) noexcept { *this = std::move(o); }
    Workspace& operator=(Workspace&& o) noexcept {
        std::swap(h_, o.h_);
        device_ = o.device_;
        value_type_ = o.value_type_;
        precond_type_ = o.precond_type_;
        precond_kind_ = o.precond_kind_;
        precond_ = o.precond_;
        use_implicit_duplicate_ = o.use_implicit_duplicate_;
        mv_compute_type_ = o.mv_compute_type_;
        mv_compute_type_set_ = o.mv_compute_type_set_;
        stop_rule = o.stop_rule;
        inner_rtol = o.inner_rtol;
        anorm_fro = o.anorm_fro;
        return *this;
    }
    ~Workspace() {
        if (h_) tomos_workspace_destroy(h_);
    }
    tomos_workspace* handle() const { return h_; }

private:
    tomos_workspace* h_ = nullptr;
};

inline Workspace create_lsqr_workspace(Context& ctx, dim<2> size, NumericType value_type,
                                       NumericType precond_type) {
    (void)ctx;
    return Workspace(size[0], size[1], value_type, precond_type);
}
inline Workspace create_lsqr_workspace(Context& ctx, dim<2> size, NumericType value_type) {
    return create_lsqr_workspace(ctx, size, value_type, value_type);
}

inline void add_precond(Dense& precond, Workspace& ws) {
    if (precond.get_value_type() != ws.precond_type_)
        throw std::invalid_argument(
            "add_precond: precond's NumericType doesn't match the precond_type the workspace "
            "was created with.");
    b200_detail::check(tomos_workspace_add_precond(ws.handle(), &precond.desc()), "add_precond");
    ws.precond_kind_ = PrecondKind::Dense;
    ws.precond_ = &precond;
}

namespace b200_detail {
inline tomos_lsqr_opts opts_for(const Workspace& ws, NumericType a, double tol, int max_iters,
                                double max_relres, int restarts,
                                std::vector<double>* hist, std::vector<double>& buf) {
    tomos_lsqr_opts o{};
    o.tol = tol;
    o.max_iters = max_iters;
    o.restarts = restarts;
    o.max_relres = max_relres;
    o.stop_rule = ws.stop_rule;
    o.iter_tier = ws.mv_compute_type_set_ ? tier_for(a, ws.mv_compute_type_) : TOMOS_TIER_AUTO;
    o.implicit_duplicate = ws.use_implicit_duplicate_ ? 1 : 0;
    o.inner_rtol = ws.inner_rtol;
    o.anorm_fro = ws.anorm_fro;
    if (hist) {
        buf.assign(static_cast<std::size_t>(max_iters > 0 ? max_iters : 0) * restarts + restarts + 1, 0.0);
        o.history = buf.data();
        o.history_cap = static_cast<int32_t>(buf.size());
    }
    return o;
}
}  // namespace b200_detail

// lsqr_solve (include/core/solver.hpp:68-78).  b and x are FP32 Dense
// vectors; x is overwritten.  mtx_refine_precision: a copy of A at higher
// precision (FP32, or packed read exactly), e.g. beside an FP16 A
// (--explicit-duplicates); the initial and restart passes read it.
inline void lsqr_solve(Context ctx, Dense& A, Dense& b, Dense& x, Workspace& ws, double tol,
                       int max_iters, double max_relres, int* iterations = nullptr,
                       std::vector<double>* residual_history = nullptr, int restarts = 1,
                       Dense* mtx_refine_precision = nullptr) {
    (void)ctx;
    if (b.get_value_type() != NumericType::FP32 || x.get_value_type() != NumericType::FP32)
        throw std::runtime_error("lsqr_solve: only FP32 b / x are registered");
    std::vector<double> buf;
    tomos_lsqr_opts o = b200_detail::opts_for(ws, A.get_value_type(), tol, max_iters, max_relres,
                                              restarts, residual_history, buf);
    if (mtx_refine_precision) o.refine = &mtx_refine_precision->desc();
    b200_detail::check(tomos_lsqr_solve_dense(&A.desc(), static_cast<const float*>(b.data()),
                                              static_cast<float*>(x.data()), ws.handle(), &o,
                                              &ws.last_report, nullptr),
                       "lsqr_solve");
    if (iterations) *iterations = ws.last_report.iterations;
    if (residual_history)
        residual_history->insert(residual_history->end(), buf.begin(),
                                 buf.begin() + ws.last_report.history_len);
}

inline void lsqr_solve(Context ctx, Sparse& A, Dense& b, Dense& x, Workspace& ws, double tol,
                       int max_iters, double max_relres, int* iterations = nullptr,
                       std::vector<double>* residual_history = nullptr, int restarts = 1,
                       Sparse* mtx_refine_precision = nullptr) {
    (void)ctx;
    std::vector<double> buf;
    tomos_lsqr_opts o = b200_detail::opts_for(ws, A.get_value_type(), tol, max_iters, max_relres,
                                              restarts, residual_history, buf);
    if (mtx_refine_precision) o.refine_csr = &mtx_refine_precision->desc();
    b200_detail::check(tomos_lsqr_solve_csr(&A.desc(), static_cast<const float*>(b.data()),
                                            static_cast<float*>(x.data()), ws.handle(), &o,
                                            &ws.last_report, nullptr),
                       "lsqr_solve");
    if (iterations) *iterations = ws.last_report.iterations;
    if (residual_history)
        residual_history->insert(residual_history->end(), buf.begin(),
                                 buf.begin() + ws.last_report.history_len);
}

// mv_apply (src/core/blas/blas.cpp:23-86).  `workspace` is the device
// scratch of the transposed product (tomos_gemv_scratch_bytes); when NULL
// a buffer is allocated for the call.
inline Status mv_apply(Device dev, TransposeType trans, double alpha, Dense& A, Dense& x,
                       double beta, Dense& y, NumericType compute_type,
                       float* workspace = nullptr) {
    if (dev != Device::CUDA) throw std::invalid_argument("mv_apply: Device::CUDA only");
    const int32_t tier = b200_detail::tier_for(A.get_value_type(), compute_type);
    const int32_t t = trans == TRANSPOSE ? TOMOS_TRANSPOSE : TOMOS_NO_TRANSPOSE;
    std::size_t nb = tomos_gemv_scratch_bytes(&A.desc(), t);
    void* scratch = workspace;
    bool own = false;
    if (!scratch && nb) {
        if (cudaMalloc(&scratch, nb) != cudaSuccess) throw std::runtime_error("mv_apply: scratch");
        own = true;
    }
    tomos_status s = tomos_gemv(t, alpha, &A.desc(), tier, static_cast<const float*>(x.data()),
                                beta, static_cast<float*>(y.data()), scratch,
                                workspace ? (std::size_t)-1 : nb, nullptr);
    if (own) {
        cudaStreamSynchronize(nullptr);
        cudaFree(scratch);
    }
    b200_detail::check(s, "mv_apply");
    return SUCCESS;
}
inline Status mv_apply(Device dev, TransposeType trans, double alpha, Dense& A, Dense& x,
                       double beta, Dense& y) {
    // blas.cpp:33-53: FP32_16 storage defaults to the FP16 ("pure_half") tier.
    NumericType a = A.get_value_type();
    NumericType c = a == NumericType::FP32_16 ? NumericType::FP16
                    : a == NumericType::FP32_BF16 ? NumericType::BF16 : a;
    return mv_apply(dev, trans, alpha, A, x, beta, y, c);
}

// split_fp32_16 / combine_fp32_16 (blas.hpp; fp32_16_registries.cpp:32-62).
inline Status split_fp32_16(Dense& source, Dense& target) {
    const tomos_dense& s = source.desc();
    const tomos_dense& t = target.desc();
    if (source.get_value_type() != NumericType::FP32 || target.get_value_type() != NumericType::FP32_16)
        throw std::invalid_argument("split_fp32_16: FP32 source and FP32_16 target required");
    std::size_t outer = t.layout == TOMOS_COL_MAJOR ? t.cols : t.rows;
    uint16_t* wh = static_cast<uint16_t*>(t.values);
    b200_detail::check(tomos_pack_fp32_16(static_cast<const float*>(s.values), s.layout, s.rows,
                                          s.cols, s.ld, wh, wh + t.ld * outer, t.ld, nullptr,
                                          nullptr),
                       "split_fp32_16");
    return SUCCESS;
}
inline Status combine_fp32_16(Dense& source, Dense& target) {
    const tomos_dense& s = source.desc();
    const tomos_dense& t = target.desc();
    std::size_t outer = s.layout == TOMOS_COL_MAJOR ? s.cols : s.rows;
    const uint16_t* wh = static_cast<const uint16_t*>(s.values);
    b200_detail::check(tomos_unpack_fp32_16(wh, wh + s.ld * outer, s.layout, s.rows, s.cols, s.ld,
                                            static_cast<float*>(t.values), t.ld, nullptr),
                       "combine_fp32_16");
    return SUCCESS;
}

// Hash CountSketch: target (s x n, FP64 column-major Dense) = S * source.
inline void apply_count_sketch_hashed(Dense& source, Dense& target,
                                      uint64_t bucket_seed = TOMOS_CS_BUCKET_SEED,
                                      uint64_t sign_seed = TOMOS_CS_SIGN_SEED) {
    const tomos_dense& t = target.desc();
    std::size_t nb = tomos_countsketch_scratch_bytes(source.desc().rows, source.desc().cols, t.rows);
    void* scratch = nullptr;
    if (cudaMalloc(&scratch, nb ? nb : 4) != cudaSuccess)
        throw std::runtime_error("apply_count_sketch: scratch allocation");
    tomos_status s = tomos_countsketch_apply(&source.desc(), TOMOS_TIER_AUTO, t.rows, bucket_seed,
                                             sign_seed, static_cast<double*>(t.values), t.ld,
                                             nullptr, nullptr, scratch, nb, nullptr);
    cudaStreamSynchronize(nullptr);
    cudaFree(scratch);
    b200_detail::check(s, "apply_count_sketch");
}

// generate_sketch_qr_precond (sketch_qr.hpp:19): on return the leading
// n x n block of the FP64 column-major sketched_mtx holds R^{-1}.
inline void generate_sketch_qr_precond(Dense& sketched_mtx) {
    const tomos_dense& d = sketched_mtx.desc();
    if (sketched_mtx.get_value_type() != NumericType::FP64 || d.layout != TOMOS_COL_MAJOR)
        throw std::runtime_error("generate_sketch_qr_precond: FP64 column-major only");
    std::size_t nb = tomos_sketch_qr_scratch_bytes(d.rows, d.cols);
    void* scratch = nullptr;
    if (cudaMalloc(&scratch, nb ? nb : 4) != cudaSuccess)
        throw std::runtime_error("generate_sketch_qr_precond: scratch allocation");
    tomos_status s = tomos_sketch_qr_precond_f64(d.rows, d.cols, static_cast<double*>(d.values),
                                                 d.ld, nullptr, scratch, nb, nullptr);
    cudaStreamSynchronize(nullptr);
    cudaFree(scratch);
    b200_detail::check(s, "generate_sketch_qr_precond");
}
inline void generate_sketch_qr_precond(Sparse& sketch, Dense& sketched_mtx) {
    (void)sketch;  // consulted only for its device, as in the reference
    generate_sketch_qr_precond(sketched_mtx);
}

}  // namespace tomos
