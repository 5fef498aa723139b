"""ctypes declarations of the C ABI in include/tomos_b200.h.

The shared library is built in-tree (python -m tomos_b200.build) and loaded
from tomos_b200/lib/.  There is no fallback: if the library is missing or
fails to load, importing this module raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtomos_b200.so")

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_u64 = ctypes.c_uint64
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_sz = ctypes.c_size_t

TOMOS_OK = 0
TOMOS_ERR_INVALID = -1
TOMOS_ERR_UNSUPPORTED = -2
TOMOS_ERR_CUDA = -3
TOMOS_ERR_ALLOC = -4
TOMOS_ERR_NUMERIC = -5

TOMOS_QR_ANY_SIGNS = 1  # tomos_sketch_qr_precond_ex_f64: R up to the signs of its rows

CS_BUCKET_SEED = 0x12345678ABCDEF00
CS_SIGN_SEED = 0xF00DD00D42BABE55


class DenseDesc(ctypes.Structure):
    _fields_ = [("numeric", c_i32), ("layout", c_i32), ("rows", c_i64), ("cols", c_i64),
                ("ld", c_i64), ("values", c_vp), ("values_lo", c_vp), ("rounded", c_i32),
                ("reserved", c_i32)]


class CsrDesc(ctypes.Structure):
    _fields_ = [("numeric", c_i32), ("index_type", c_i32), ("rows", c_i64), ("cols", c_i64),
                ("nnz", c_i64), ("values", c_vp), ("values_lo", c_vp), ("row_ptrs", c_vp),
                ("col_idxs", c_vp), ("rounded", c_i32), ("reserved", c_i32)]


class LsqrOpts(ctypes.Structure):
    _fields_ = [("tol", c_dbl), ("max_iters", c_i32), ("restarts", c_i32),
                ("max_relres", c_dbl), ("stop_rule", c_i32), ("iter_tier", c_i32),
                ("implicit_duplicate", c_i32), ("warm_start", c_i32), ("inner_rtol", c_dbl),
                ("anorm_fro", c_dbl), ("col_scale", c_vp), ("history", ctypes.POINTER(c_dbl)),
                ("history_cap", c_i32), ("profile", c_i32), ("staged_plane", c_vp),
                ("staged_ld", c_i64), ("anorm_fro_dev", c_vp), ("refine", c_vp),
                ("comm", c_vp), ("inner_eta_factor", c_dbl), ("refine_csr", c_vp)]


class LsqrReport(ctypes.Structure):
    _fields_ = [("iterations", c_i32), ("restarts_used", c_i32), ("converged", c_i32),
                ("history_len", c_i32), ("relres", c_dbl), ("rnorm", c_dbl), ("arnorm", c_dbl),
                ("anorm_fro", c_dbl), ("xnorm", c_dbl), ("bnorm", c_dbl),
                ("backward_error", c_dbl), ("elapsed_ms", c_dbl), ("accurate_passes", c_i32),
                ("half_passes", c_i32), ("iter_pass_ms", c_dbl), ("init_pass_ms", c_dbl),
                ("iter_pass_count", c_i32), ("init_pass_count", c_i32),
                ("kernel_launches", c_i32), ("reserved", c_i32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MtxInfo(ctypes.Structure):
    _fields_ = [("rows", c_i64), ("cols", c_i64), ("entries", c_i64), ("format", c_i32),
                ("field", c_i32), ("symmetry", c_i32), ("reserved", c_i32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# Every symbol the header declares, with (restype, argtypes).
SIGNATURES = {
    "tomos_pack_fp16": (c_i32, [c_vp, c_i32, c_i64, c_i64, c_i64, c_vp, c_i64, c_vp]),
    "tomos_mtx_read_info": (c_i32, [ctypes.c_char_p, ctypes.POINTER(MtxInfo)]),
    "tomos_mtx_read_dense": (c_i32, [ctypes.c_char_p, c_i32, c_vp, c_i64]),
    "tomos_mtx_read_coo": (c_i32, [ctypes.c_char_p, c_i64, c_vp, c_vp, c_vp, ctypes.POINTER(c_i64)]),
    "tomos_mtx_write_dense": (c_i32, [ctypes.c_char_p, c_i32, c_i64, c_i64, c_vp, c_i64]),
    "tomos_last_error": (ctypes.c_char_p, []),
    "tomos_version": (ctypes.c_char_p, []),
    "tomos_sync": (c_i32, [c_vp]),
    "tomos_pack_fp32_16": (c_i32, [c_vp, c_i32, c_i64, c_i64, c_i64, c_vp, c_vp, c_i64, c_vp,
                                   c_vp]),
    "tomos_unpack_fp32_16": (c_i32, [c_vp, c_vp, c_i32, c_i64, c_i64, c_i64, c_vp, c_i64, c_vp]),
    "tomos_pack_fp32_bf16": (c_i32, [c_vp, c_i32, c_i64, c_i64, c_i64, c_vp, c_vp, c_i64, c_i32,
                                     c_vp]),
    "tomos_unpack_fp32_bf16": (c_i32, [c_vp, c_vp, c_i32, c_i64, c_i64, c_i64, c_vp, c_i64,
                                       c_i32, c_vp]),
    "tomos_gemv_scratch_bytes": (c_sz, [ctypes.POINTER(DenseDesc), c_i32]),
    "tomos_mm": (c_i32, [c_i32, c_i32, c_dbl, ctypes.POINTER(DenseDesc), c_i32,
                         ctypes.POINTER(DenseDesc), c_dbl, ctypes.POINTER(DenseDesc), c_vp]),
    "tomos_mm_ex": (c_i32, [c_i32, c_i32, c_dbl, ctypes.POINTER(DenseDesc), c_i32,
                            ctypes.POINTER(DenseDesc), c_dbl, ctypes.POINTER(DenseDesc), c_vp,
                            ctypes.c_size_t, c_vp]),
    "tomos_lsqr_adjoint_batch_dense": (c_i32, [ctypes.POINTER(DenseDesc), c_i32, c_vp, c_i64, c_vp, c_i64,
                                               c_vp, ctypes.POINTER(LsqrOpts), c_vp, c_vp]),
    "tomos_mm_scratch_bytes": (ctypes.c_size_t, [c_i32, c_i32, ctypes.POINTER(DenseDesc), c_i32,
                                                 ctypes.POINTER(DenseDesc)]),
    "tomos_gemv": (c_i32, [c_i32, c_dbl, ctypes.POINTER(DenseDesc), c_i32, c_vp, c_dbl, c_vp,
                           c_vp, c_sz, c_vp]),
    "tomos_gemv_no_alloc": (c_i32, [c_i32, c_dbl, ctypes.POINTER(DenseDesc), c_i32, c_vp, c_dbl,
                                    c_vp, c_vp]),
    "tomos_csr_gemv_scratch_bytes": (c_sz, [ctypes.POINTER(CsrDesc), c_i32]),
    "tomos_csr_gemv": (c_i32, [c_i32, c_dbl, ctypes.POINTER(CsrDesc), c_i32, c_vp, c_dbl, c_vp,
                               c_vp, c_sz, c_vp]),
    "tomos_countsketch_hash": (c_i32, [c_i64, c_i64, c_u64, c_u64, c_vp, c_vp, c_vp]),
    "tomos_countsketch_scratch_bytes": (c_sz, [c_i64, c_i64, c_i64]),
    "tomos_countsketch_apply": (c_i32, [ctypes.POINTER(DenseDesc), c_i32, c_i64, c_u64, c_u64,
                                        c_vp, c_i64, c_vp, c_vp, c_vp, c_sz, c_vp]),
    "tomos_countsketch_apply_stage": (c_i32, [ctypes.POINTER(DenseDesc), c_i64, c_u64, c_u64,
                                              c_vp, c_i64, c_vp, c_vp, c_vp, c_i64, c_vp, c_sz,
                                              c_vp]),
    "tomos_countsketch_apply_csr": (c_i32, [ctypes.POINTER(CsrDesc), c_i32, c_i64, c_u64, c_u64,
                                            c_vp, c_i64, c_vp, c_vp, c_vp, c_sz, c_vp]),
    "tomos_sketch_qr_scratch_bytes": (c_sz, [c_i64, c_i64]),
    "tomos_sketch_qr_precond_f64": (c_i32, [c_i64, c_i64, c_vp, c_i64, c_vp, c_vp, c_sz, c_vp]),
    "tomos_sketch_qr_precond_ex_f64": (c_i32, [c_i64, c_i64, c_vp, c_i64, c_vp, c_i32, c_vp, c_sz, c_vp]),
    "tomos_column_scale": (c_i32, [c_vp, c_i64, c_vp, c_vp, c_vp]),
    "tomos_countsketch_apply_shard": (c_i32, [ctypes.POINTER(DenseDesc), c_i32, c_i64, c_u64, c_u64,
                                              c_i64, c_vp, c_i64, c_vp, c_vp, c_vp, c_i64, c_vp, c_sz,
                                              c_vp]),
    "tomos_comm_unique_id": (c_i32, [c_vp]),
    "tomos_comm_create": (c_i32, [c_i32, c_i32, c_vp, ctypes.POINTER(c_vp)]),
    "tomos_comm_destroy": (c_i32, [c_vp]),
    "tomos_comm_allreduce_f64": (c_i32, [c_vp, c_vp, c_i64, c_vp]),
    "tomos_workspace_create": (c_i32, [c_i64, c_i64, c_i32, c_i32, ctypes.POINTER(c_vp)]),
    "tomos_workspace_destroy": (c_i32, [c_vp]),
    "tomos_workspace_add_precond": (c_i32, [c_vp, ctypes.POINTER(DenseDesc)]),
    "tomos_lsqr_solve_dense": (c_i32, [ctypes.POINTER(DenseDesc), c_vp, c_vp, c_vp,
                                       ctypes.POINTER(LsqrOpts), ctypes.POINTER(LsqrReport),
                                       c_vp]),
    "tomos_lsqr_solve_csr": (c_i32, [ctypes.POINTER(CsrDesc), c_vp, c_vp, c_vp,
                                     ctypes.POINTER(LsqrOpts), ctypes.POINTER(LsqrReport), c_vp]),
    "tomos_backward_error_dense": (c_i32, [ctypes.POINTER(DenseDesc), c_vp, c_vp, c_vp, c_vp,
                                           ctypes.POINTER(LsqrReport), c_vp]),
    "tomos_lsqr_adjoint_dense": (c_i32, [ctypes.POINTER(DenseDesc), c_vp, c_vp, c_vp,
                                         ctypes.POINTER(LsqrOpts), ctypes.POINTER(LsqrReport),
                                         c_vp]),
    "tomos_lsqr_adjoint_grad_dense": (c_i32, [ctypes.POINTER(DenseDesc), c_i64, c_vp, c_i64, c_vp,
                                              c_i64, c_vp, c_i64, c_vp, c_i64, c_vp, c_i64, c_vp]),
}


class TomosError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded C ABI (raises if the library is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m tomos_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code, what=""):
    if code != TOMOS_OK:
        msg = lib().tomos_last_error().decode(errors="replace")
        raise TomosError(code, f"{what}: {msg}" if what else msg)
    return code
