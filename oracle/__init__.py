"""CPU checkers for the tests (TEST INFRASTRUCTURE ONLY).

Two libraries, both built by oracle/Makefile:
  * liboracle.so      -- our C restatement of the reference's algorithms
                         (oracle.c), always available;
  * _ref/libtomos_ref.so -- the reference's own CPU path compiled from its
                         sources (only where the reference tree exists).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
use this package; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtomos_ref.so")

_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_dbl = ctypes.c_double
_i32 = ctypes.c_int
_u64 = ctypes.c_uint64

BUCKET_SEED = 0x12345678ABCDEF00
SIGN_SEED = 0xF00DD00D42BABE55


# Where the reference's sources are looked for: TOMOS_REF_SRC, else the
# checkout this build recipe was written against.
REF_SRC_DEFAULT = "/root/reference"


def ref_src():
    """The reference source tree, or None when it is not on this machine."""
    d = os.environ.get("TOMOS_REF_SRC") or REF_SRC_DEFAULT
    return d if os.path.isdir(os.path.join(d, "src")) else None


def build(ref=None):
    """Builds liboracle.so, and the reference CPU library when its sources
    exist (ref=None: when found; ref=True: required; ref=False: never)."""
    src = ref_src()
    if ref and not src:
        raise FileNotFoundError("reference sources not found (set TOMOS_REF_SRC)")
    target = ["oracle", "ref", "ref_b200"] if (src and ref is not False) else ["oracle"]
    args = [f"REF={src}"] if src else []
    subprocess.run(["make", "-s", "-j8", *args, *target], cwd=HERE, check=True)


def _P(a):
    return a.ctypes.data_as(_vp)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.or_splitmix64.restype = _u64
        L.or_splitmix64.argtypes = [_u64]
        L.or_countsketch_hash.argtypes = [_sz, _sz, _u64, _u64, _vp, _vp]
        L.or_countsketch_apply_f64.argtypes = [_sz, _sz, _vp, _sz, _i32, _sz, _u64, _u64, _vp]
        L.or_countsketch_apply_f32.argtypes = [_sz, _sz, _vp, _sz, _i32, _sz, _u64, _u64, _vp]
        L.or_householder_qr_f64.argtypes = [_sz, _sz, _vp, _sz, _vp]
        L.or_trtri_upper_f64.argtypes = [_sz, _vp, _sz, _vp, _sz]
        L.or_lsqr_f32.argtypes = [_sz, _sz, _vp, _sz, _vp, _vp, _vp, _dbl, _i32, _dbl, _i32, _vp, _vp]
        for f in ("or_fp32_16_split", "or_fp32_bf16_split", "or_fp32_bf16_split_rounded"):
            getattr(L, f).argtypes = [_vp, _sz, _vp, _vp]
        for f in ("or_fp32_16_combine", "or_fp32_bf16_combine", "or_fp32_bf16_combine_rounded"):
            getattr(L, f).argtypes = [_vp, _vp, _sz, _vp]
        L.or_fp32_16_half_only.argtypes = [_vp, _sz, _vp]
        L.or_fp32_16_half_only_f32.argtypes = [_vp, _sz, _vp]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    """The reference's own CPU build (raises if it was not built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        R = ctypes.CDLL(REF_SO)
        for f in ("ref_fp32_16_split", "ref_fp32_bf16_split", "ref_fp32_bf16_split_rounded"):
            getattr(R, f).argtypes = [_vp, _sz, _vp, _vp]
        for f in ("ref_fp32_16_combine", "ref_fp32_bf16_combine", "ref_fp32_bf16_combine_rounded"):
            getattr(R, f).argtypes = [_vp, _vp, _sz, _vp]
        R.ref_fp32_16_half_only.argtypes = [_vp, _sz, _vp]
        R.ref_countsketch_apply_f32.argtypes = [_sz, _sz, _vp, _sz, _sz, _vp, _sz]
        R.ref_countsketch_apply_f64.argtypes = [_sz, _sz, _vp, _sz, _sz, _vp, _sz]
        R.ref_mv_fp32_16.argtypes = [_i32, _i32, _dbl, _sz, _sz, _vp, _vp, _sz, _vp, _dbl, _vp]
        R.ref_mv_f32.argtypes = [_i32, _dbl, _sz, _sz, _vp, _vp, _dbl, _vp]
        R.ref_sketch_qr_f64.argtypes = [_sz, _sz, _vp]
        R.ref_lsqr_solve_f32.argtypes = [_sz, _sz, _vp, _vp, _vp, _vp, _dbl, _i32, _dbl, _i32, _vp, _vp]
        R.ref_lsqr_solve_f32_timed.argtypes = [_sz, _sz, _vp, _vp, _vp, _vp, _dbl, _i32, _dbl, _i32,
                                               _vp, _vp]
        R.ref_sketch_qr_f64_timed.argtypes = [_sz, _sz, _vp, _vp]
        R.ref_lsqr_iterate_f32.argtypes = [_sz, _sz, _vp, _vp, _vp, _vp, _i32]
        _ref = R
    return _ref


# ------------------------------------------------------------------ packs

def _pack(fn, x):
    x = np.ascontiguousarray(x, dtype=np.float32).ravel()
    wh = np.empty(x.size, np.uint16)
    wr = np.empty(x.size, np.uint16)
    fn(_P(x), x.size, _P(wh), _P(wr))
    return wh, wr


def _unpack(fn, wh, wr):
    wh = np.ascontiguousarray(wh, dtype=np.uint16).ravel()
    wr = np.ascontiguousarray(wr, dtype=np.uint16).ravel()
    out = np.empty(wh.size, np.float32)
    fn(_P(wh), _P(wr), wh.size, _P(out))
    return out


def fp32_16_split(x):
    return _pack(lib().or_fp32_16_split, x)


def fp32_16_combine(wh, wr):
    return _unpack(lib().or_fp32_16_combine, wh, wr)


def fp32_16_half_only(wh):
    wh = np.ascontiguousarray(wh, dtype=np.uint16).ravel()
    out = np.empty(wh.size, np.uint16)
    lib().or_fp32_16_half_only(_P(wh), wh.size, _P(out))
    return out


def fp32_16_half_only_f32(wh):
    wh = np.ascontiguousarray(wh, dtype=np.uint16).ravel()
    out = np.empty(wh.size, np.float32)
    lib().or_fp32_16_half_only_f32(_P(wh), wh.size, _P(out))
    return out


def fp32_bf16_split(x, rounded=False):
    return _pack(lib().or_fp32_bf16_split_rounded if rounded else lib().or_fp32_bf16_split, x)


def fp32_bf16_combine(wh, wr, rounded=False):
    f = lib().or_fp32_bf16_combine_rounded if rounded else lib().or_fp32_bf16_combine
    return _unpack(f, wh, wr)


def bf16_value(wh):
    return (np.asarray(wh, np.uint16).astype(np.uint32) << 16).view(np.float32)


def decode(numeric, wh, wr=None, tier="half", rounded=False):
    """Values a packed matrix is read as at a tier ('half' or 'accurate')."""
    shape = np.shape(wh)
    if numeric == "fp32_16":
        v = fp32_16_half_only_f32(wh) if tier == "half" else fp32_16_combine(wh, wr)
    else:
        v = bf16_value(np.ravel(wh)) if tier == "half" else fp32_bf16_combine(wh, wr, rounded)
    return v.reshape(shape)


# ------------------------------------------------------------------ sketch

def splitmix64(x):
    return lib().or_splitmix64(x)


def countsketch_hash(m, s, bucket_seed=BUCKET_SEED, sign_seed=SIGN_SEED):
    b = np.empty(m, np.int32)
    g = np.empty(m, np.int8)
    lib().or_countsketch_hash(m, s, bucket_seed, sign_seed, _P(b), _P(g))
    return b, g


def countsketch_apply(A, s, row_major=True, bucket_seed=BUCKET_SEED, sign_seed=SIGN_SEED,
                      acc="f64"):
    """SA (s x n, returned as FP64) = S A for a float32 (m x n) array,
    accumulated in FP64 (acc="f64") or, as the reference's float path, in
    FP32 in increasing row order (acc="f32")."""
    A = np.asarray(A, np.float32)
    m, n = A.shape
    src = np.ascontiguousarray(A) if row_major else np.asfortranarray(A)
    ld = n if row_major else m
    SA = np.zeros((s, n), np.float64, order="F")
    fn = lib().or_countsketch_apply_f32 if acc == "f32" else lib().or_countsketch_apply_f64
    fn(m, n, _P(src), ld, 1 if row_major else 0, s, bucket_seed, sign_seed, _P(SA))
    return SA


# ------------------------------------------------------------------ QR / LSQR

def householder_qr(A):
    """(R, tau) of the FP64 Householder QR (LAPACK dgeqr2 convention)."""
    A = np.array(A, np.float64, order="F")
    m, n = A.shape
    tau = np.zeros(n)
    rc = lib().or_householder_qr_f64(m, n, _P(A), m, _P(tau))
    if rc != 0:
        raise ValueError("householder_qr: need m >= n")
    return np.triu(A[:n, :n]), tau


def trtri_upper(R):
    R = np.asfortranarray(R, np.float64)
    n = R.shape[0]
    X = np.zeros((n, n), np.float64, order="F")
    if lib().or_trtri_upper_f64(n, _P(R), n, _P(X), n) != 0:
        raise ZeroDivisionError("singular R")
    return X


def sketch_qr_precond(SA):
    """R^{-1} of the sketch, as the reference's generate_sketch_qr_precond."""
    R, _ = householder_qr(SA)
    return trtri_upper(R)


def lstsq_f64(A, b):
    """FP64 least-squares solution by Householder QR (the solution oracle)."""
    A = np.asarray(A, np.float64)
    b = np.asarray(b, np.float64)
    Q, R = np.linalg.qr(A)
    return np.linalg.solve(R, Q.T @ b)


def lstsq_f64_blocks(blocks, n):
    """FP64 least-squares solution of a tall problem given as row blocks
    (A_k, b_k), by Householder QR of [A b] one block at a time (TSQR): the
    R of [R_prev; A_k b_k] is carried, so only one block is in memory.
    Returns (x, ||r||) with ||r|| = |R[n, n]|, the least-squares residual.
    Same solution as lstsq_f64 on the stacked rows."""
    R = np.zeros((0, n + 1))
    for A, b in blocks:
        blk = np.empty((A.shape[0], n + 1))
        blk[:, :n] = A
        blk[:, n] = b
        R = np.linalg.qr(np.vstack([R, blk]), mode="r")
        R = R[: n + 1]
    x = np.linalg.solve(np.triu(R[:n, :n]), R[:n, n])
    rn = abs(R[n, n]) if R.shape[0] > n else 0.0
    return x, rn


def residual_norms_blocks(blocks, x, d=None):
    """FP64 ||b - A x||, ||D^{-1} A^T (b - A x)||, ||A D^{-1}||_F^2 and ||b||
    over row blocks (the pieces of eta and eta_D, accumulated exactly in
    FP64 without holding A)."""
    x = np.asarray(x, np.float64)
    r2 = b2 = 0.0
    atr = None
    fro = None
    for A, b in blocks:
        A = np.asarray(A, np.float64)
        r = np.asarray(b, np.float64) - A @ x
        r2 += float(r @ r)
        b2 += float(np.asarray(b, np.float64) @ np.asarray(b, np.float64))
        t = A.T @ r
        atr = t if atr is None else atr + t
        c = (A * A).sum(axis=0)
        fro = c if fro is None else fro + c
    if d is None:
        d = np.ones_like(fro)
    return np.sqrt(r2), float(np.linalg.norm(atr / d)), float((fro / d ** 2).sum()), np.sqrt(b2)


def backward_error(A, b, x):
    """eta = min(||r|| / (||A||_F ||x|| + ||b||), ||A^T r|| / (||A||_F ||r||)), FP64."""
    A = np.asarray(A, np.float64)
    b = np.asarray(b, np.float64)
    x = np.asarray(x, np.float64)
    r = b - A @ x
    an = np.linalg.norm(A)
    rn = np.linalg.norm(r)
    e1 = rn / (an * np.linalg.norm(x) + np.linalg.norm(b))
    e2 = np.linalg.norm(A.T @ r) / (an * rn) if rn > 0 else 0.0
    return min(e1, e2)


def backward_error_scaled(A, b, x, d=None):
    """eta_D: the backward error of the column-scaled problem (A D^{-1}, b,
    D x), D = column norms of A by default (FP64)."""
    A = np.asarray(A, np.float64)
    if d is None:
        d = np.linalg.norm(A, axis=0)
        d = np.where(d > 0, d, 1.0)
    return backward_error(A / d, b, np.asarray(x, np.float64) * d)


def lstsq_grads_f64(A, B, G):
    """FP64 normal-equations reference for the adjoint of X = argmin
    ||A X - B|| (columnwise) and the loss sum_k <G_k, X_k>:
    Lam = (A^T A)^{-1} G, dL/dB = A Lam, dL/dA = R Lam^T - (A Lam) X^T with
    R = B - A X.  Returns (X, Lam, gradA, gradB)."""
    A = np.asarray(A, np.float64)
    B = np.asarray(B, np.float64).reshape(A.shape[0], -1)
    G = np.asarray(G, np.float64).reshape(A.shape[1], -1)
    N = A.T @ A
    X = np.linalg.solve(N, A.T @ B)
    Lam = np.linalg.solve(N, G)
    R = B - A @ X
    W = A @ Lam
    return X, Lam, R @ Lam.T - W @ X.T, W


def lstsq_loss_f64(A, B, G):
    """sum_k <G_k, argmin ||A x - B_k||> in FP64 (Householder QR)."""
    A = np.asarray(A, np.float64)
    B = np.asarray(B, np.float64).reshape(A.shape[0], -1)
    G = np.asarray(G, np.float64).reshape(A.shape[1], -1)
    Q, R = np.linalg.qr(A)
    X = np.linalg.solve(R, Q.T @ B)
    return float(np.sum(G * X))


def lstsq_fd_f64(A, B, G, entries_A, entries_B, h=1e-6):
    """Central finite differences of lstsq_loss_f64 at the given (i, j)
    entries of A and of B, step h."""
    A = np.array(A, np.float64)
    B = np.array(B, np.float64).reshape(A.shape[0], -1)
    dA, dB = [], []
    for (i, j) in entries_A:
        a0 = A[i, j]
        A[i, j] = a0 + h
        lp = lstsq_loss_f64(A, B, G)
        A[i, j] = a0 - h
        lm = lstsq_loss_f64(A, B, G)
        A[i, j] = a0
        dA.append((lp - lm) / (2 * h))
    for (i, k) in entries_B:
        b0 = B[i, k]
        B[i, k] = b0 + h
        lp = lstsq_loss_f64(A, B, G)
        B[i, k] = b0 - h
        lm = lstsq_loss_f64(A, B, G)
        B[i, k] = b0
        dB.append((lp - lm) / (2 * h))
    return np.array(dA), np.array(dB)


def lsqr_f32(A, b, Rinv=None, tol=1e-6, max_iters=400, max_relres=1e-6, restarts=1):
    """Plain FP32 LSQR restated from the reference (oracle.c or_lsqr_f32).
    Returns (x, iterations, history)."""
    A = np.asfortranarray(A, np.float32)
    m, n = A.shape
    b = np.ascontiguousarray(b, np.float32)
    x = np.zeros(n, np.float32)
    it = ctypes.c_int(0)
    hist = np.zeros(max(1, max_iters * restarts + restarts), np.float64)
    Rp = None
    if Rinv is not None:
        Rf = np.asfortranarray(Rinv, np.float32)
        Rp = _P(Rf)
    nh = lib().or_lsqr_f32(m, n, _P(A), m, _P(b), _P(x), Rp, tol, max_iters, max_relres, restarts,
                           ctypes.byref(it), _P(hist))
    return x, it.value, hist[:nh].copy()


def ref_lsqr_f32(A, b, Rinv=None, tol=1e-6, max_iters=400, max_relres=1e-6, restarts=1):
    """The reference's own lsqr_solve on the CPU (oracle/_ref)."""
    A = np.asfortranarray(A, np.float32)
    m, n = A.shape
    b = np.ascontiguousarray(b, np.float32)
    x = np.zeros(n, np.float32)
    it = ctypes.c_int(0)
    hist = np.zeros(max(1, max_iters * restarts + restarts), np.float64)
    Rp = None
    if Rinv is not None:
        Rf = np.asfortranarray(Rinv, np.float32)
        Rp = _P(Rf)
    rc = ref().ref_lsqr_solve_f32(m, n, _P(A), _P(b), _P(x), Rp, tol, max_iters, max_relres,
                                  restarts, ctypes.byref(it), _P(hist))
    if rc != 0:
        raise RuntimeError("reference lsqr_solve threw")
    k = int(np.count_nonzero(hist))
    return x, it.value, hist[:k].copy()
