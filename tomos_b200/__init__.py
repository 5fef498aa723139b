"""tomos_b200 -- the TOMOS LSQR hot path on NVIDIA B200 (sm_100a).

Python mirror of the reference's public API (include/core/*.hpp) over the
C ABI in include/tomos_b200.h.  Names, argument meaning and error behaviour
follow the reference: Dense / Workspace objects, create_lsqr_workspace,
add_precond, lsqr_solve, mv_apply, split_fp32_16 / combine_fp32_16,
apply_count_sketch, generate_sketch_qr_precond.  Device memory comes from
torch (CUDA tensors); every product runs in the sm_100a kernels of
libtomos_b200.so.  There is no CPU path: a CPU Context raises.
"""
import ctypes
import enum
import os

import torch

from . import _capi as C
from ._capi import TomosError, CS_BUCKET_SEED, CS_SIGN_SEED

__all__ = [
    "NumericType", "Layout", "TransposeType", "Device", "Tier", "StopRule", "Context", "Dense",
    "Csr", "Workspace", "create_lsqr_workspace", "add_precond", "lsqr_solve", "mv_apply",
    "split_fp32_16", "combine_fp32_16", "split_fp32_bf16", "combine_fp32_bf16",
    "countsketch_hash", "apply_count_sketch", "generate_sketch_qr_precond", "backward_error",
    "column_scale", "mtx_info", "read_mtx", "read_mtx_coo", "read_mtx_csr", "write_mtx",
    "dense_from_mtx", "csr_from_mtx", "sketch_lsqr", "shard_rows", "Comm", "apply_count_sketch_shard",
    "TomosError", "CS_BUCKET_SEED", "CS_SIGN_SEED", "NO_TRANSPOSE", "TRANSPOSE",
]


class NumericType(enum.IntEnum):
    """include/core/precision.hpp:43-50; FP32_BF16 takes the new slot 5."""
    FP64 = 0
    FP32 = 1
    FP16 = 2
    FP32_16 = 3
    BF16 = 4
    FP32_BF16 = 5


class Layout(enum.IntEnum):
    ROW_MAJOR = 0
    COL_MAJOR = 1


class TransposeType(enum.IntEnum):
    NO_TRANSPOSE = 0
    TRANSPOSE = 1


NO_TRANSPOSE = TransposeType.NO_TRANSPOSE
TRANSPOSE = TransposeType.TRANSPOSE


class Device(enum.IntEnum):
    CPU = 0
    OMP = 1
    CUDA = 2


class Tier(enum.IntEnum):
    AUTO = 0
    NATIVE = 1
    HALF = 2
    ACCURATE = 3
    HALF_OPERANDS = 4  # mm only: 16-bit A and B operands (the pure_half tier)


class StopRule(enum.IntEnum):
    RELRES = 0
    BACKWARD = 1


PACKED = (NumericType.FP32_16, NumericType.FP32_BF16)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Context:
    """include/core/context: only Device::CUDA is registered here."""

    def __init__(self, device=Device.CUDA):
        if Device(device) != Device.CUDA:
            raise ValueError("tomos_b200 runs on the GPU only: Context(Device.CUDA)")
        if not torch.cuda.is_available():
            raise RuntimeError("Context(Device.CUDA): no CUDA device available")
        self.device = Device.CUDA

    def get_device(self):
        return self.device


class Dense:
    """A strided dense matrix on the device (include/core/matrix.hpp Dense).

    FP32 / FP64 storage is one buffer of ld * outer elements; FP32_16 and
    FP32_BF16 use the reference's planar layout (fp32_16_pack.hpp:861-874):
    a uint16 buffer of 2 * ld * outer words, wh plane first, wr plane
    second.  outer = cols for COL_MAJOR, rows for ROW_MAJOR.
    """

    def __init__(self, numeric, layout, size, ld, storage, rounded=False):
        self.numeric = NumericType(numeric)
        self.layout = Layout(layout)
        self.size = (int(size[0]), int(size[1]))
        self.ld = int(ld)
        self.storage = storage
        self.rounded = bool(rounded)

    # -- construction ---------------------------------------------------
    @staticmethod
    def _outer_inner(layout, size):
        return (size[1], size[0]) if Layout(layout) == Layout.COL_MAJOR else (size[0], size[1])

    @classmethod
    def create_strided(cls, ctx, layout, store_type, size, lead_dim=None, rounded=False):
        outer, inner = cls._outer_inner(layout, size)
        ld = inner if lead_dim is None else int(lead_dim)
        if ld < inner:
            raise ValueError("lead_dim smaller than the contiguous extent")
        n = ld * outer
        st = NumericType(store_type)
        if st == NumericType.FP32:
            buf = torch.zeros(max(n, 1), dtype=torch.float32, device="cuda")
        elif st == NumericType.FP64:
            buf = torch.zeros(max(n, 1), dtype=torch.float64, device="cuda")
        elif st == NumericType.FP16:
            buf = torch.zeros(max(n, 1), dtype=torch.float16, device="cuda")
        elif st in PACKED:
            buf = torch.zeros(max(2 * n, 2), dtype=torch.int16, device="cuda")
        else:
            raise TomosError(C.TOMOS_ERR_UNSUPPORTED, f"no storage registered for {st.name}")
        return cls(st, layout, size, ld, buf, rounded)

    @classmethod
    def _empty_f64(cls, layout, size):
        """An FP64 Dense whose values the caller's kernel writes in full (no
        zero fill)."""
        outer, inner = cls._outer_inner(layout, size)
        buf = torch.empty(max(inner * outer, 1), dtype=torch.float64, device="cuda")
        return cls(NumericType.FP64, layout, size, inner, buf)

    @classmethod
    def from_tensor(cls, t, layout=Layout.COL_MAJOR, store_type=NumericType.FP32, lead_dim=None):
        """Copies a logical (rows x cols) tensor into a new Dense of this layout."""
        t = torch.as_tensor(t)
        if t.dim() == 1:
            t = t[:, None]
        rows, cols = t.shape
        st = NumericType(store_type)
        if st not in (NumericType.FP32, NumericType.FP64):
            raise ValueError("from_tensor builds FP32/FP64 storage; pack with split_fp32_16")
        d = cls.create_strided(None, layout, st, (rows, cols), lead_dim)
        d.view()[...] = t.to(device="cuda", dtype=d.storage.dtype)
        return d

    # -- views ----------------------------------------------------------
    @property
    def outer(self):
        return self._outer_inner(self.layout, self.size)[0]

    @property
    def inner(self):
        return self._outer_inner(self.layout, self.size)[1]

    def _plane(self, k):
        n = self.ld * self.outer
        return self.storage[k * n:(k + 1) * n]

    def view(self, plane=0):
        """The logical (rows x cols) view of the values (or of one packed plane)."""
        buf = self.storage if self.numeric not in PACKED else self._plane(plane)
        rows, cols = self.size
        if self.outer == 0 or self.inner == 0:
            return buf[:0].reshape(rows, cols) if rows * cols == 0 else buf
        m = buf[: self.ld * self.outer].view(self.outer, self.ld)[:, : self.inner]
        return m.t() if self.layout == Layout.COL_MAJOR else m

    def wh(self):
        return self.view(0)

    def wr(self):
        return self.view(1)

    def get_value_type(self):
        return self.numeric

    def get_size(self):
        return self.size

    def desc(self):
        d = C.DenseDesc()
        d.numeric = int(self.numeric)
        d.layout = int(self.layout)
        d.rows, d.cols = self.size
        d.ld = self.ld
        d.values = self.storage.data_ptr()
        d.values_lo = (self.storage.data_ptr() + 2 * self.ld * self.outer) if self.numeric in PACKED else None
        d.rounded = 1 if self.rounded else 0
        return d


class Csr:
    """A CSR matrix on the device (include/core/matrix.hpp Sparse)."""

    def __init__(self, numeric, size, row_ptrs, col_idxs, values, rounded=False):
        self.numeric = NumericType(numeric)
        self.size = (int(size[0]), int(size[1]))
        self.row_ptrs = row_ptrs
        self.col_idxs = col_idxs
        self.values = values
        self.rounded = bool(rounded)
        self.nnz = int(col_idxs.numel())

    def get_value_type(self):
        return self.numeric

    def desc(self):
        d = C.CsrDesc()
        d.numeric = int(self.numeric)
        d.index_type = 0 if self.col_idxs.dtype == torch.int32 else 1
        d.rows, d.cols = self.size
        d.nnz = self.nnz
        d.values = self.values.data_ptr()
        d.values_lo = (self.values.data_ptr() + 2 * self.nnz) if self.numeric in PACKED else None
        d.row_ptrs = self.row_ptrs.data_ptr()
        d.col_idxs = self.col_idxs.data_ptr()
        d.rounded = 1 if self.rounded else 0
        return d


# ------------------------------------------------------------ MatrixMarket

def _path(path):
    return os.fsencode(path)


def mtx_info(path):
    """Banner and sizes of a MatrixMarket file (mm_read_banner +
    mm_read_mtx_*_size, src/io/mmio.c): dict with rows, cols, entries,
    format (0 array, 1 coordinate), field (0 real, 1 integer, 2 pattern),
    symmetry (0 general, 1 symmetric, 2 skew-symmetric)."""
    info = C.MtxInfo()
    C.check(C.lib().tomos_mtx_read_info(_path(path), ctypes.byref(info)), "mtx_info")
    return info.as_dict()


def read_mtx(path, layout=None):
    """The whole matrix as a host FP64 numpy array (column-major, as the
    reference's read_mtx_host, lsqr_precision_runner.cu:101-125; Layout.
    ROW_MAJOR gives a C-ordered array)."""
    import numpy as np
    info = mtx_info(path)
    m, n = info["rows"], info["cols"]
    layout = Layout.COL_MAJOR if layout is None else Layout(layout)
    out = np.zeros((m, n), dtype=np.float64, order="F" if layout == Layout.COL_MAJOR else "C")
    ld = max(1, m if layout == Layout.COL_MAJOR else n)
    C.check(C.lib().tomos_mtx_read_dense(_path(path), int(layout), out.ctypes.data, ld), "read_mtx")
    return out


def read_mtx_coo(path):
    """(rows, cols, values) 0-based numpy triplets in file order, symmetric
    parts mirrored."""
    import numpy as np
    cnt = ctypes.c_int64(0)
    info = mtx_info(path)
    cap = info["entries"] * (2 if info["symmetry"] else 1)
    r = np.empty(max(cap, 1), np.int64)
    c = np.empty(max(cap, 1), np.int64)
    v = np.empty(max(cap, 1), np.float64)
    C.check(C.lib().tomos_mtx_read_coo(_path(path), cap, r.ctypes.data, c.ctypes.data, v.ctypes.data,
                                       ctypes.byref(cnt)), "read_mtx_coo")
    k = cnt.value
    return r[:k], c[:k], v[:k]


def read_mtx_csr(path):
    """(row_ptrs int32, col_idxs int32, values FP64, (m, n)) on the host:
    rows in order, columns increasing within a row, repeated positions
    summed."""
    import numpy as np
    info = mtx_info(path)
    m, n = info["rows"], info["cols"]
    r, c, v = read_mtx_coo(path)
    key = r * max(n, 1) + c
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    first = np.ones(key.size, bool)
    first[1:] = key[1:] != key[:-1]
    starts = np.flatnonzero(first)
    vals = np.add.reduceat(v, starts) if key.size else v
    ukey = key[starts]
    rows, cols = ukey // max(n, 1), ukey % max(n, 1)
    rp = np.zeros(m + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp)
    return rp.astype(np.int32), cols.astype(np.int32), vals, (m, n)


def write_mtx(path, a, layout=None):
    """Writes a 2-D array as `array real general` (17 significant digits,
    column by column)."""
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    if a.ndim != 2:
        raise TomosError(C.TOMOS_ERR_INVALID, "write_mtx: a 2-D array")
    if a.flags["C_CONTIGUOUS"] and not a.flags["F_CONTIGUOUS"]:
        buf, lay, ld = a, Layout.ROW_MAJOR, max(1, a.shape[1])  # no copy
    else:
        buf, lay, ld = np.asfortranarray(a), Layout.COL_MAJOR, max(1, a.shape[0])
    C.check(C.lib().tomos_mtx_write_dense(_path(path), int(lay), a.shape[0], a.shape[1],
                                          buf.ctypes.data, ld), "write_mtx")


def dense_from_mtx(path, store_type=NumericType.FP32, layout=Layout.COL_MAJOR):
    """A device Dense (FP32 or FP64, packed types through pack()) from a
    MatrixMarket file, values rounded from FP64 as the reference's
    fill_dense_from_host does."""
    st = NumericType(store_type)
    base = NumericType.FP64 if st == NumericType.FP64 else NumericType.FP32
    host = read_mtx(path, layout)
    dt = torch.float64 if base == NumericType.FP64 else torch.float32
    t = torch.from_numpy(host).to(dt)
    if Layout(layout) == Layout.COL_MAJOR:
        t = t.t().contiguous().t()
    D = Dense.from_tensor(t.cuda(), layout, base)
    return D if st == base else pack(D, st)


def csr_from_mtx(path, store_type=NumericType.FP32):
    """A device Csr (int32 indices; FP32 values, or packed FP32_16 /
    FP32_BF16) from a MatrixMarket file."""
    import numpy as np
    rp, ci, v, size = read_mtx_csr(path)
    st = NumericType(store_type)
    vals = torch.from_numpy(v.astype(np.float32)).cuda()
    if st != NumericType.FP32:
        vals = pack(Dense.from_tensor(vals[None, :], Layout.ROW_MAJOR), st).storage
    return Csr(st, size, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), vals)


# ------------------------------------------------------------------ packing

def split_fp32_16(source, target, counts=None, stream=None):
    """FP32 Dense -> FP32_16 Dense (blas.hpp split_fp32_16), bit-exact with
    the reference encoder.  counts (int64 cuda tensor of 4, optional) is
    accumulated with [normal, extended underflow, extended overflow,
    saturated] element counts."""
    if source.numeric != NumericType.FP32 or target.numeric != NumericType.FP32_16:
        raise TomosError(C.TOMOS_ERR_INVALID, "split_fp32_16: FP32 source, FP32_16 target")
    if source.size != target.size or source.layout != target.layout:
        raise TomosError(C.TOMOS_ERR_INVALID, "split_fp32_16: shape/layout mismatch")
    t = target.desc()
    C.check(C.lib().tomos_pack_fp32_16(_ptr(source.storage), int(source.layout), source.size[0],
                                       source.size[1], source.ld, t.values, t.values_lo, target.ld,
                                       _ptr(counts), _stream(stream)), "split_fp32_16")


def combine_fp32_16(source, target, stream=None):
    if source.numeric != NumericType.FP32_16 or target.numeric != NumericType.FP32:
        raise TomosError(C.TOMOS_ERR_INVALID, "combine_fp32_16: FP32_16 source, FP32 target")
    s = source.desc()
    C.check(C.lib().tomos_unpack_fp32_16(s.values, s.values_lo, int(source.layout), source.size[0],
                                         source.size[1], source.ld, _ptr(target.storage), target.ld,
                                         _stream(stream)), "combine_fp32_16")


def split_fp32_bf16(source, target, rounded=False, stream=None):
    if source.numeric != NumericType.FP32 or target.numeric != NumericType.FP32_BF16:
        raise TomosError(C.TOMOS_ERR_INVALID, "split_fp32_bf16: FP32 source, FP32_BF16 target")
    target.rounded = bool(rounded)
    t = target.desc()
    C.check(C.lib().tomos_pack_fp32_bf16(_ptr(source.storage), int(source.layout), source.size[0],
                                         source.size[1], source.ld, t.values, t.values_lo,
                                         target.ld, int(bool(rounded)), _stream(stream)),
            "split_fp32_bf16")


def combine_fp32_bf16(source, target, stream=None):
    s = source.desc()
    C.check(C.lib().tomos_unpack_fp32_bf16(s.values, s.values_lo, int(source.layout),
                                           source.size[0], source.size[1], source.ld,
                                           _ptr(target.storage), target.ld, s.rounded,
                                           _stream(stream)), "combine_fp32_bf16")


def pack_fp16(A_fp32, P, stream=None):
    """FP32 Dense -> native FP16 Dense of the same shape (round to nearest
    even; tomos_pack_fp16)."""
    C.check(C.lib().tomos_pack_fp16(_ptr(A_fp32.storage), int(A_fp32.layout), A_fp32.size[0],
                                    A_fp32.size[1], A_fp32.ld, _ptr(P.storage), P.ld, _stream(stream)),
            "pack_fp16")
    return P


def pack(A_fp32, store_type, rounded=False, stream=None):
    """Convenience: a packed (or native FP16) copy of an FP32 Dense with the
    same layout."""
    P = Dense.create_strided(None, A_fp32.layout, store_type, A_fp32.size, A_fp32.ld, rounded)
    if NumericType(store_type) == NumericType.FP16:
        return pack_fp16(A_fp32, P, stream=stream)
    if NumericType(store_type) == NumericType.FP32_16:
        split_fp32_16(A_fp32, P, stream=stream)
    else:
        split_fp32_bf16(A_fp32, P, rounded, stream=stream)
    return P


# ------------------------------------------------------------------ products

def _tier_of(A, compute_type):
    """The reference's compute_type rule (blas.cpp:33-53) as a tier."""
    if compute_type is None:
        return Tier.AUTO
    ct = NumericType(compute_type)
    if A.numeric in PACKED:
        if ct in (NumericType.FP16, NumericType.BF16):
            return Tier.HALF
        if ct == NumericType.FP32:
            return Tier.ACCURATE
    elif ct == A.numeric:
        return Tier.NATIVE
    raise TomosError(C.TOMOS_ERR_UNSUPPORTED,
                     f"no mv kernel registered for {A.numeric.name} with compute {ct.name}")


def _vec(v):
    if isinstance(v, Dense):
        return v.storage
    return v


def mv_apply(dev, transpose, alpha, A, x, beta, y, compute_type=None, tier=None, stream=None):
    """y = alpha * op(A) x + beta * y (src/core/blas/blas.cpp:23-86).

    A: Dense or Csr; x, y: FP32 Dense column vectors or float32 CUDA tensors.
    """
    if Device(dev) != Device.CUDA:
        raise ValueError("mv_apply: Device.CUDA only")
    t = _tier_of(A, compute_type) if tier is None else Tier(tier)
    xs, ys = _vec(x), _vec(y)
    if isinstance(A, Csr):
        d = A.desc()
        nb = C.lib().tomos_csr_gemv_scratch_bytes(ctypes.byref(d), int(transpose))
        scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
        C.check(C.lib().tomos_csr_gemv(int(transpose), float(alpha), ctypes.byref(d), int(t),
                                       _ptr(xs), float(beta), _ptr(ys), _ptr(scratch), nb,
                                       _stream(stream)), "mv_apply")
        return 0
    d = A.desc()
    nb = C.lib().tomos_gemv_scratch_bytes(ctypes.byref(d), int(transpose))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    C.check(C.lib().tomos_gemv(int(transpose), float(alpha), ctypes.byref(d), int(t), _ptr(xs),
                               float(beta), _ptr(ys), _ptr(scratch), nb, _stream(stream)),
            "mv_apply")
    return 0


def mm_apply(dev, transA, transB, alpha, A, B, beta, Cm, use_workspace=False, tier=None, stream=None):
    """C = alpha * op(A) op(B) + beta * C (include/core/blas.hpp:123-125,
    src/core/blas/blas.cpp:98-106) on the tcgen05 tensor cores.  A: a Dense
    (FP32, FP16 or packed); B, C (Cm): FP32 Dense.  Packed A is read
    exactly, as the reference's mm_apply routes it (dense_registries.cpp:
    396-405: the accurate tier, or its decode-into-scratch "workspace"
    variant, which yields the same exact values; use_workspace therefore
    changes nothing here).  `tier` overrides: Tier.HALF is the fast tier,
    Tier.HALF_OPERANDS the pure_half operands."""
    if Device(dev) != Device.CUDA:
        raise ValueError("mm_apply: Device.CUDA only")
    if tier is None:
        tier = Tier.ACCURATE if A.numeric in PACKED else Tier.AUTO
    da, db, dc = A.desc(), B.desc(), Cm.desc()
    nb = C.lib().tomos_mm_scratch_bytes(int(transA), int(transB), ctypes.byref(da), int(tier),
                                        ctypes.byref(db))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda") if nb else None
    C.check(C.lib().tomos_mm_ex(int(transA), int(transB), float(alpha), ctypes.byref(da), int(tier),
                                ctypes.byref(db), float(beta), ctypes.byref(dc), _ptr(scratch), nb,
                                _stream(stream)),
            "mm_apply")
    return 0


def mm_apply_fp32_16_pure_half(dev, transA, transB, alpha, A, B, beta, Cm, stream=None):
    """blas.hpp:185-187: 16-bit A values and B rounded to fp16 (bf16 for
    FP32_BF16 storage), FP32 accumulation."""
    return mm_apply(dev, transA, transB, alpha, A, B, beta, Cm, tier=Tier.HALF_OPERANDS, stream=stream)


def mm_apply_fp32_16_fast(dev, transA, transB, alpha, A, B, beta, Cm, stream=None):
    """blas.hpp:189-191: 16-bit A values, B to ~22 bits, FP32 accumulation."""
    return mm_apply(dev, transA, transB, alpha, A, B, beta, Cm, tier=Tier.HALF, stream=stream)


def mm_apply_fp32_16_ext(dev, transA, transB, alpha, A, B, beta, Cm, stream=None):
    """blas.hpp:193-195: A exact (wh + wr), products to ~22 bits."""
    return mm_apply(dev, transA, transB, alpha, A, B, beta, Cm, tier=Tier.ACCURATE, stream=stream)


# ------------------------------------------------------------------ sketch

def countsketch_hash(m, s, bucket_seed=CS_BUCKET_SEED, sign_seed=CS_SIGN_SEED, stream=None):
    """Per-row bucket and sign of the hash CountSketch (device tensors)."""
    bucket = torch.empty(max(m, 1), dtype=torch.int32, device="cuda")
    sign = torch.empty(max(m, 1), dtype=torch.int8, device="cuda")
    C.check(C.lib().tomos_countsketch_hash(m, s, bucket_seed, sign_seed, _ptr(bucket), _ptr(sign),
                                           _stream(stream)), "countsketch_hash")
    return bucket[:m], sign[:m]


def apply_count_sketch(A, s, tier=Tier.AUTO, bucket_seed=CS_BUCKET_SEED, sign_seed=CS_SIGN_SEED,
                       with_colsq=False, stage=False, stream=None):
    """SA = S A (s x n, column-major FP64 Dense) and ||A||_F^2 of the values
    read; with_colsq also returns the column sums of squares (same pass).
    stage (row-major FP32_16 A, HALF tier): the same pass also writes the
    fixed fp16 copy of A's wh plane, returned last (an m x ld int16 tensor
    for lsqr_solve's staged_plane)."""
    if stage:
        return _count_sketch_stage(A, s, bucket_seed, sign_seed, with_colsq, stream)
    n = A.size[1]
    # every output is written in full by the sketch
    SA = Dense._empty_f64(Layout.COL_MAJOR, (s, n))
    fro2 = torch.empty(1, dtype=torch.float64, device="cuda")
    colsq = torch.empty(max(n, 1), dtype=torch.float64, device="cuda") if with_colsq else None
    m = A.size[0]
    nb = C.lib().tomos_countsketch_scratch_bytes(m, n, s)
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    d = A.desc()
    fn = C.lib().tomos_countsketch_apply_csr if isinstance(A, Csr) else C.lib().tomos_countsketch_apply
    C.check(fn(ctypes.byref(d), int(tier), s, bucket_seed, sign_seed, _ptr(SA.storage), s,
               _ptr(fro2), _ptr(colsq), _ptr(scratch), nb, _stream(stream)), "apply_count_sketch")
    if with_colsq:
        return SA, fro2, colsq[:n]
    return SA, fro2


def _count_sketch_stage(A, s, bucket_seed, sign_seed, with_colsq, stream):
    if isinstance(A, Csr) or A.numeric != NumericType.FP32_16 or A.layout != Layout.ROW_MAJOR:
        raise TomosError(C.TOMOS_ERR_INVALID, "apply_count_sketch: stage needs a row-major FP32_16 A")
    m, n = A.size
    ldp = (n + 7) // 8 * 8
    plane = torch.empty((max(m, 1), ldp), dtype=torch.int16, device="cuda")
    SA = Dense._empty_f64(Layout.COL_MAJOR, (s, n))
    fro2 = torch.empty(1, dtype=torch.float64, device="cuda")
    colsq = torch.empty(max(n, 1), dtype=torch.float64, device="cuda") if with_colsq else None
    nb = C.lib().tomos_countsketch_scratch_bytes(m, n, s)
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    d = A.desc()
    C.check(C.lib().tomos_countsketch_apply_stage(ctypes.byref(d), s, bucket_seed, sign_seed,
                                                  _ptr(SA.storage), s, _ptr(fro2), _ptr(colsq),
                                                  _ptr(plane), ldp, _ptr(scratch), nb,
                                                  _stream(stream)), "apply_count_sketch")
    if with_colsq:
        return SA, fro2, colsq[:n], plane
    return SA, fro2, plane


def generate_sketch_qr_precond(sketched, R_out=None, copy=True, any_signs=False, stream=None):
    """FP64 Householder QR of the k x n column-major sketched matrix; on
    return its leading n x n block holds R^{-1} (sketch_qr.hpp:19).
    Returns R^{-1} as an n x n Dense: a copy of that block, or with
    copy=False a view of it (leading dimension k, no device copy; it
    shares the sketched matrix's storage).  any_signs: R's rows may carry
    other signs than LAPACK's (TOMOS_QR_ANY_SIGNS), which a preconditioned
    LSQR does not see and which saves the sign reconstruction."""
    if sketched.numeric != NumericType.FP64 or sketched.layout != Layout.COL_MAJOR:
        raise TomosError(C.TOMOS_ERR_INVALID, "generate_sketch_qr_precond: FP64 column-major input")
    k, n = sketched.size
    if k < n:
        raise TomosError(C.TOMOS_ERR_INVALID,
                         "generate_sketch_qr_precond: sketched_mtx must have at least as many "
                         "rows as columns (k >= n).")
    nb = C.lib().tomos_sketch_qr_scratch_bytes(k, n)
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    C.check(C.lib().tomos_sketch_qr_precond_ex_f64(k, n, _ptr(sketched.storage), sketched.ld, _ptr(R_out),
                                                   C.TOMOS_QR_ANY_SIGNS if any_signs else 0, _ptr(scratch),
                                                   nb, _stream(stream)),
            "generate_sketch_qr_precond")
    if not copy:
        return Dense(NumericType.FP64, Layout.COL_MAJOR, (n, n), sketched.ld, sketched.storage)
    Rinv = Dense.create_strided(None, Layout.COL_MAJOR, NumericType.FP64, (n, n))
    Rinv.view()[...] = sketched.view()[:n, :n]
    return Rinv


# ------------------------------------------------------------------ LSQR

class Workspace:
    """include/core/workspace.hpp Workspace over a tomos_workspace*."""

    def __init__(self, m, n, value_type=NumericType.FP32, precond_type=None):
        self.size = (int(m), int(n))
        self.value_type_ = NumericType(value_type)
        self.precond_type_ = NumericType(value_type if precond_type is None else precond_type)
        h = ctypes.c_void_p()
        C.check(C.lib().tomos_workspace_create(m, n, int(self.value_type_),
                                               int(self.precond_type_), ctypes.byref(h)),
                "create_lsqr_workspace")
        self._h = h
        self.precond_ = None
        self.use_implicit_duplicate_ = False
        self.mv_compute_type_ = NumericType.FP16
        self.mv_compute_type_set_ = False

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            C.lib().tomos_workspace_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_lsqr_workspace(ctx, size, value_type, precond_type=None):
    return Workspace(size[0], size[1], value_type, precond_type)


def add_precond(precond, workspace):
    """Attaches a non-owning R^{-1} (include/core/workspace.hpp:112-120)."""
    if precond.get_value_type() != workspace.precond_type_:
        raise TomosError(C.TOMOS_ERR_INVALID,
                         "add_precond: precond's NumericType doesn't match the precond_type the "
                         "workspace was created with.")
    d = precond.desc()
    C.check(C.lib().tomos_workspace_add_precond(workspace.handle, ctypes.byref(d)), "add_precond")
    workspace.precond_ = precond


def lsqr_solve(ctx, A, b, x, workspace, tol, max_iters, max_relres, iterations=None,
               residual_history=None, restarts=1, stop_rule=StopRule.RELRES, inner_rtol=0.0,
               anorm_fro=0.0, warm_start=False, tier=None, profile=False, col_scale=None,
               staged_plane=None, mtx_refine_precision=None, inner_eta_factor=0.0, comm=None,
               stream=None):
    """include/core/solver.hpp:68-78.  A: Dense or Csr on the device; b, x:
    FP32 Dense column vectors or float32 CUDA tensors.  iterations and
    residual_history, when lists, receive the reference's out-parameters.
    staged_plane: the (m x ld) int16 tensor apply_count_sketch(..., stage=True)
    filled for this A (HALF-tier iterations then skip their staging pass).
    mtx_refine_precision: a copy of A at higher precision (FP32, or packed
    read exactly; a Dense beside a Dense A, a Csr beside a Csr A) for the
    initial and restart passes, e.g. beside an FP16 A (the reference's
    --explicit-duplicates).
    Returns the solver report as a dict."""
    opts = C.LsqrOpts()
    opts.tol = float(tol)
    opts.max_iters = int(max_iters)
    opts.restarts = int(restarts)
    opts.max_relres = float(max_relres)
    opts.stop_rule = int(stop_rule)
    if tier is not None:
        opts.iter_tier = int(tier)
    elif workspace.mv_compute_type_set_:
        opts.iter_tier = int(_tier_of(A, workspace.mv_compute_type_))
    else:
        opts.iter_tier = int(Tier.AUTO)
    opts.implicit_duplicate = 1 if workspace.use_implicit_duplicate_ else 0
    opts.warm_start = 1 if warm_start else 0
    opts.inner_rtol = float(inner_rtol)
    opts.inner_eta_factor = float(inner_eta_factor)
    opts.comm = comm.handle if comm is not None else None
    if isinstance(anorm_fro, torch.Tensor):  # a device value (column_scale)
        opts.anorm_fro_dev = anorm_fro.data_ptr()
        opts.anorm_fro = 0.0
    else:
        opts.anorm_fro = float(anorm_fro)
    refine_desc = None
    if mtx_refine_precision is not None:
        refine_desc = mtx_refine_precision.desc()
        if isinstance(mtx_refine_precision, Csr):
            opts.refine_csr = ctypes.addressof(refine_desc)
        else:
            opts.refine = ctypes.addressof(refine_desc)
    opts.profile = 1 if profile else 0
    opts.col_scale = col_scale.data_ptr() if col_scale is not None else None
    if staged_plane is not None:
        opts.staged_plane = staged_plane.data_ptr()
        opts.staged_ld = staged_plane.stride(0)
    cap = max(1, int(max_iters) * int(restarts) + int(restarts))
    hist = (ctypes.c_double * cap)()
    opts.history = hist
    opts.history_cap = cap
    rep = C.LsqrReport()
    d = A.desc()
    fn = C.lib().tomos_lsqr_solve_csr if isinstance(A, Csr) else C.lib().tomos_lsqr_solve_dense
    C.check(fn(ctypes.byref(d), _ptr(_vec(b)), _ptr(_vec(x)), workspace.handle, ctypes.byref(opts),
               ctypes.byref(rep), _stream(stream)), "lsqr_solve")
    out = rep.as_dict()
    out["history"] = [hist[i] for i in range(rep.history_len)]
    if isinstance(iterations, list):
        iterations.append(rep.iterations)
    if isinstance(residual_history, list):
        residual_history.extend(out["history"])
    return out


def backward_error(A, b, x, workspace, col_scale=None, stream=None):
    """Normwise backward error of x (FP64, accurate tier); with col_scale D
    (float64 CUDA tensor) the backward error of the column-scaled problem."""
    rep = C.LsqrReport()
    d = A.desc()
    C.check(C.lib().tomos_backward_error_dense(ctypes.byref(d), _ptr(_vec(b)), _ptr(_vec(x)),
                                               _ptr(col_scale), workspace.handle,
                                               ctypes.byref(rep), _stream(stream)),
            "backward_error")
    return rep.as_dict()


def lsqr_adjoint(A, g, workspace, tol=1e-7, max_iters=500, tier=None, stream=None):
    """lambda = (A^T A)^{-1} g by preconditioned CG with the workspace's
    R^{-1} (tomos_lsqr_adjoint_dense).  g: float32 CUDA tensor (n).
    Returns (lambda, report)."""
    opts = C.LsqrOpts()
    opts.tol = float(tol)
    opts.max_iters = int(max_iters)
    opts.restarts = 1
    opts.iter_tier = int(Tier.AUTO if tier is None else Tier(tier))
    lam = torch.empty(A.size[1], dtype=torch.float32, device="cuda")
    rep = C.LsqrReport()
    d = A.desc()
    C.check(C.lib().tomos_lsqr_adjoint_dense(ctypes.byref(d), _ptr(_vec(g)), _ptr(lam),
                                             workspace.handle, ctypes.byref(opts),
                                             ctypes.byref(rep), _stream(stream)),
            "lsqr_adjoint")
    return lam, rep.as_dict()


def lsqr_adjoint_batch(A, G, workspace, tol=1e-7, max_iters=500, tier=None, stream=None):
    """Lambda = (A^T A)^{-1} G for the K columns of G (n x K float32 CUDA
    tensor) at once (tomos_lsqr_adjoint_batch_dense: one CG recurrence per
    column, the products with A shared, two tensor-core products an
    iteration).  Returns (Lambda (n x K), list of K reports)."""
    n = A.size[1]
    K = G.shape[1]
    opts = C.LsqrOpts()
    opts.tol = float(tol)
    opts.max_iters = int(max_iters)
    opts.restarts = 1
    opts.iter_tier = int(Tier.AUTO if tier is None else Tier(tier))
    Gc = G.t().contiguous().float()  # column-major n x K
    Lc = torch.empty((K, n), dtype=torch.float32, device="cuda")
    reps = (C.LsqrReport * max(K, 1))()
    d = A.desc()
    C.check(C.lib().tomos_lsqr_adjoint_batch_dense(ctypes.byref(d), K, _ptr(Gc), n, _ptr(Lc), n,
                                                   workspace.handle, ctypes.byref(opts), reps,
                                                   _stream(stream)),
            "lsqr_adjoint_batch")
    return Lc.t(), [reps[k].as_dict() for k in range(K)]


def lsqr_adjoint_grad(A, B, X, Lam, want_grad_a=True, stream=None):
    """dL/dB = A Lam and dL/dA = (B - A X) Lam^T - (A Lam) X^T in one pass
    over the row-major A (tomos_lsqr_adjoint_grad_dense).  B: (m, K), X and
    Lam: (n, K) float32 CUDA tensors.  Returns (gradA or None, gradB)."""
    m, n = A.size
    K = B.shape[1]
    Bc = B.t().contiguous()  # column-major (m x K)
    Xc = X.t().contiguous()
    Lc = Lam.t().contiguous()
    gB = torch.empty((K, m), dtype=torch.float32, device="cuda")
    gA = torch.empty((m, n), dtype=torch.float32, device="cuda") if want_grad_a else None
    d = A.desc()
    C.check(C.lib().tomos_lsqr_adjoint_grad_dense(ctypes.byref(d), K, _ptr(Bc), m, _ptr(Xc), n,
                                                  _ptr(Lc), n, _ptr(gB), m, _ptr(gA), n,
                                                  _stream(stream)),
            "lsqr_adjoint_grad")
    return gA, gB.t()


def column_scale(colsq, stream=None):
    """D = column norms from column sums of squares (zero columns -> 1), and
    ||A D^{-1}||_F for it, both computed on the device (tomos_column_scale):
    returns (d, anorm) with anorm a one-element float64 CUDA tensor, which
    lsqr_solve takes as anorm_fro without a host round trip."""
    n = colsq.numel()
    d = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
    an = torch.empty(1, dtype=torch.float64, device="cuda")
    C.check(C.lib().tomos_column_scale(_ptr(colsq), n, _ptr(d), _ptr(an), _stream(stream)),
            "column_scale")
    return d[:n], an


def sketch_lsqr(A, b, s, tol=1e-6, max_iters=200, restarts=8, inner_rtol=None, workspace=None,
                x=None, profile=False, events=None, comm=None, row0=0, stream=None):
    """The sketch-preconditioned LSQR pipeline of the reference's runner
    (lsqr_precision_runner.cu:588-656: sketch, generate_sketch_qr_precond,
    add_precond, lsqr_solve) with the BACKWARD stopping rule on the
    column-scaled problem:

      hash CountSketch SA = S A (s rows) with the column sums of squares --
      for a row-major FP32_16 A the same pass writes the fp16 plane its
      HALF-tier iterations read -- then the FP64 sketch QR and R^{-1}, the
      column scale D on the device, and LSQR until eta_D <= tol, packed
      storage refined by exact restart passes.

    Returns (x, report, d).  workspace: an (m, n) FP32/FP64 workspace to
    reuse (created when None).  inner_rtol: the refinement cycles' residual
    reduction (default 2e-3 for packed storage, none for FP32).  events:
    four torch.cuda.Event recorded at the start, after the sketch, after
    the QR and after the solve (phase timing).  comm (a Comm): A and b are
    this rank's rows of one problem, starting at row row0 of it; the
    sketches are summed over the ranks (one all-reduce of SA and the column
    sums), the QR is repeated on every rank, and the solve sums its
    per-pass partials over the ranks (x, returned on every rank, is the
    whole solution)."""
    m, n = A.size
    packed = A.numeric in PACKED
    plane = None
    if events:
        events[0].record()
    stage = (isinstance(A, Dense) and A.numeric == NumericType.FP32_16 and A.layout == Layout.ROW_MAJOR
             and (A.ld * 2) % 16 == 0)
    if comm is not None:
        if not isinstance(A, Dense):
            raise TomosError(C.TOMOS_ERR_UNSUPPORTED, "sketch_lsqr: sharded solves take a Dense A")
        SA, _, colsq, plane = apply_count_sketch_shard(A, s, row0, tier=Tier.HALF if packed else Tier.AUTO,
                                                       stage=stage, stream=stream)
        comm.allreduce_f64(SA.storage, stream=stream)
        comm.allreduce_f64(colsq, stream=stream)
    elif stage:
        SA, _, colsq, plane = apply_count_sketch(A, s, tier=Tier.HALF, with_colsq=True, stage=True,
                                                 stream=stream)
    else:
        SA, _, colsq = apply_count_sketch(A, s, tier=Tier.HALF if packed else Tier.AUTO,
                                          with_colsq=True, stream=stream)
    if events:
        events[1].record()
    # R up to row signs: LSQR preconditioned by R^-1 S iterates as with R^-1
    Rinv = generate_sketch_qr_precond(SA, copy=False, any_signs=True, stream=stream)
    if events:
        events[2].record()
    d, anorm = column_scale(colsq, stream=stream)
    ws = workspace
    if ws is None:
        ws = create_lsqr_workspace(None, (m, n), NumericType.FP32, NumericType.FP64)
    add_precond(Rinv, ws)
    if x is None:
        x = torch.empty(n, dtype=torch.float32, device="cuda")  # the solve zeroes x
    if inner_rtol is None:
        inner_rtol = 2e-3 if packed else 0.0
    rep = lsqr_solve(None, A, b, x, ws, tol, max_iters, 0.0, restarts=restarts,
                     stop_rule=StopRule.BACKWARD, inner_rtol=inner_rtol, anorm_fro=anorm,
                     col_scale=d, staged_plane=plane, profile=profile, comm=comm, stream=stream)
    if events:
        events[3].record()
    return x, rep, d


# ------------------------------------------------------------------ row-sharded solves

def shard_rows(m, rank, world):
    """Rows [r0, r1) of an m-row problem that rank `rank` of `world` holds:
    contiguous blocks, the first m % world ranks one row longer."""
    base, extra = divmod(int(m), int(world))
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


class Comm:
    """The ranks of a row-sharded solve (tomos_comm_create; NCCL over
    NVLink / NVSwitch).  Comm(group) takes the ranks of a torch.distributed
    process group (rank 0's id reaches the others by a broadcast over the
    group); Comm.single() is a one-rank communicator."""

    @staticmethod
    def exchange_id(group=None):
        """Rank 0's communicator id (tomos_comm_unique_id), broadcast over the
        process group; returns (id bytes, rank, world size)."""
        import torch.distributed as dist
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        idbuf = (ctypes.c_char * 128)()
        if rank == 0:
            C.check(C.lib().tomos_comm_unique_id(idbuf), "comm_unique_id")
        obj = [bytes(idbuf) if rank == 0 else None]
        src = 0 if group is None else dist.get_global_rank(group, 0)
        dist.broadcast_object_list(obj, src=src, group=group)
        return obj[0], rank, world

    def __init__(self, group=None, _single=False):
        if _single:
            rank, world = 0, 1
            idbuf = (ctypes.c_char * 128)()
            C.check(C.lib().tomos_comm_unique_id(idbuf), "comm_unique_id")
        else:
            idb, rank, world = Comm.exchange_id(group)
            idbuf = (ctypes.c_char * 128).from_buffer_copy(idb)
        h = ctypes.c_void_p()
        C.check(C.lib().tomos_comm_create(world, rank, idbuf, ctypes.byref(h)), "comm_create")
        self._h = h
        self.rank, self.size = rank, world

    @classmethod
    def single(cls):
        return cls(_single=True)

    @property
    def handle(self):
        return self._h

    def allreduce_f64(self, t, stream=None):
        """Sum a float64 CUDA tensor across the ranks, in place."""
        C.check(C.lib().tomos_comm_allreduce_f64(self._h, _ptr(t), t.numel(), _stream(stream)),
                "comm_allreduce_f64")
        return t

    def close(self):
        if self._h:
            C.lib().tomos_comm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def apply_count_sketch_shard(A, s, row0, tier=Tier.AUTO, bucket_seed=CS_BUCKET_SEED,
                             sign_seed=CS_SIGN_SEED, stage=False, stream=None):
    """The CountSketch of a row shard whose row i is row row0 + i of the
    whole problem (tomos_countsketch_apply_shard): returns (SA, fro2, colsq,
    plane or None); summed over the ranks they are the whole problem's."""
    m, n = A.size
    plane = None
    if stage:
        ldp = (n + 7) // 8 * 8
        plane = torch.empty((max(m, 1), ldp), dtype=torch.int16, device="cuda")
    SA = Dense._empty_f64(Layout.COL_MAJOR, (s, n))
    fro2 = torch.empty(1, dtype=torch.float64, device="cuda")
    colsq = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
    nb = C.lib().tomos_countsketch_scratch_bytes(m, n, s)
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    d = A.desc()
    C.check(C.lib().tomos_countsketch_apply_shard(
        ctypes.byref(d), int(tier), s, bucket_seed, sign_seed, int(row0), _ptr(SA.storage), s, _ptr(fro2),
        _ptr(colsq), _ptr(plane), plane.stride(0) if plane is not None else 0, _ptr(scratch), nb,
        _stream(stream)), "apply_count_sketch_shard")
    return SA, fro2, colsq[:n], plane
