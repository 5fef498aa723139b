"""The oracle (oracle.c, a C restatement of the reference's algorithms) is
pinned against the golden vectors the reference's own CPU build produced
(tests/golden/make_golden.py) and, where that build exists here, against
the reference library directly."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def test_fp32_16_split_combine_golden(orc):
    g = load("pack_fp32_16.npz")
    wh, wr = orc.fp32_16_split(g["x"])
    assert np.array_equal(wh, g["wh"]) and np.array_equal(wr, g["wr"])
    assert np.array_equal(bits(orc.fp32_16_combine(wh, wr)), bits(g["combine"]))


def test_fp32_16_half_only_all_words_golden(orc):
    g = load("pack_fp32_16.npz")
    assert np.array_equal(orc.fp32_16_half_only(np.arange(65536, dtype=np.uint16)), g["half_only"])


@pytest.mark.parametrize("rounded", [0, 1])
def test_fp32_bf16_golden(orc, rounded):
    g = load("pack_fp32_bf16.npz")
    wh, wr = orc.fp32_bf16_split(g["x"], rounded=bool(rounded))
    assert np.array_equal(wh, g[f"wh{rounded}"]) and np.array_equal(wr, g[f"wr{rounded}"])
    c = orc.fp32_bf16_combine(wh, wr, rounded=bool(rounded))
    assert np.array_equal(bits(c), bits(g[f"combine{rounded}"]))


def test_exponent_sweep_contract(orc):
    """test_fp32_16.cpp:285-331: exact in the normal and extended ranges,
    signed Inf / 0 in the saturated one."""
    rng = np.random.default_rng(7)
    e = np.repeat(np.arange(256, dtype=np.uint32), 40)
    mant = rng.integers(0, 1 << 23, e.size, dtype=np.uint64).astype(np.uint32)
    sign = rng.integers(0, 2, e.size, dtype=np.uint64).astype(np.uint32)
    b = (sign << 31) | (e << 23) | mant
    x = b.view(np.float32)
    keep = ~np.isnan(x)
    x, b = x[keep], b[keep]
    wh, wr = orc.fp32_16_split(x)
    rec = bits(orc.fp32_16_combine(wh, wr))
    sat = ((wh & 1) == 1) & (((wh >> 10) & 0xF) == 14)
    assert np.array_equal(rec[~sat], b[~sat])
    direction = (wh[sat] >> 14) & 1
    expect = np.where(direction == 1, np.float32(np.inf), np.float32(0.0))
    expect = np.where((b[sat] >> 31) == 1, -expect, expect).astype(np.float32)
    assert np.array_equal(rec[sat], bits(expect))


def test_half_only_matches_ieee_half(orc):
    """test_fp32_16.cpp:438-500: underflow steps 1..10 reconstruct real fp16
    subnormals (a truncation of the fp32 value); steps 11+ flush to signed
    zero, overflow is signed Inf."""
    rng = np.random.default_rng(11)
    for steps in range(1, 11):
        e = 113 - steps
        mant = rng.integers(0, 1 << 23, 20, dtype=np.uint64).astype(np.uint32)
        sign = rng.integers(0, 2, 20, dtype=np.uint64).astype(np.uint32)
        x = ((sign << 31) | (np.uint32(e) << 23) | mant).view(np.float32)
        wh, _ = orc.fp32_16_split(x)
        got = orc.fp32_16_half_only_f32(wh)
        # fp32_16_half_only truncates the rounded 10-bit significand onto
        # the fp16 subnormal grid.
        mag = np.abs(orc.fp32_16_combine(wh, np.zeros_like(wh)).astype(np.float64))
        expect = np.floor(mag / 2.0 ** -24) * 2.0 ** -24 * np.sign(x)
        assert np.array_equal(got.astype(np.float64), expect)
    x = np.float32([2.0 ** 16, -2.0 ** 20, 1e9])
    wh, _ = orc.fp32_16_split(x)
    assert np.array_equal(orc.fp32_16_half_only_f32(wh), np.float32([np.inf, -np.inf, np.inf]))
    x = np.float32([2.0 ** -25 * 1.5, -(2.0 ** -28)])
    wh, _ = orc.fp32_16_split(x)
    out = orc.fp32_16_half_only_f32(wh)
    assert np.all(out == 0) and np.signbit(out[1])


def test_countsketch_hash_golden(orc):
    g = load("countsketch.npz")
    for s in (64, 4000):
        b, sg = orc.countsketch_hash(4096, s)
        assert np.array_equal(b, g[f"bucket_s{s}"]) and np.array_equal(sg, g[f"sign_s{s}"])
    SA = orc.countsketch_apply(g["X"], 64, row_major=False)
    np.testing.assert_allclose(SA, g["Y"], rtol=1e-5, atol=1e-5)
    # the float restatement is the reference's float path bit for bit
    SA32 = orc.countsketch_apply(g["X"], 64, row_major=False, acc="f32")
    assert np.array_equal(SA32.astype(np.float32), g["Y"])


def test_countsketch_f32_matches_reference_build(orc):
    if not orc.ref_available():
        pytest.skip("reference CPU build not present")
    import ctypes
    rng = np.random.default_rng(12)
    X = np.asfortranarray((rng.standard_normal((3001, 17)) * np.logspace(-3, 3, 17)).astype(np.float32))
    Y = np.zeros((97, 17), np.float32, order="F")
    sz = ctypes.c_size_t
    orc.ref().ref_countsketch_apply_f32(sz(3001), sz(17), X.ctypes.data_as(ctypes.c_void_p), sz(3001),
                                       sz(97), Y.ctypes.data_as(ctypes.c_void_p), sz(97))
    SA = orc.countsketch_apply(X, 97, row_major=False, acc="f32")
    assert np.array_equal(SA.astype(np.float32), Y)


def test_countsketch_linear_and_norm_unbiased(orc):
    """test_countsketch_cpu_kernels.cpp:80-179: linearity and
    E||Sx||^2 = ||x||^2 within 0.05 over 200 trials."""
    rng = np.random.default_rng(42)
    X = rng.uniform(-1, 1, (128, 4)).astype(np.float32)
    np.testing.assert_allclose(orc.countsketch_apply(2.5 * X, 32), 2.5 * orc.countsketch_apply(X, 32),
                               rtol=1e-6, atol=1e-6)
    ratios = []
    for t in range(200):
        X = rng.uniform(-1, 1, (128, 4)).astype(np.float32)
        # a different sketch per trial: new seeds, same hash family
        Y = orc.countsketch_apply(X, 32, bucket_seed=0x12345678ABCDEF00 + 977 * t,
                                  sign_seed=0xF00DD00D42BABE55 + 131 * t)
        ratios += list((Y ** 2).sum(0) / (X.astype(np.float64) ** 2).sum(0))
    assert abs(np.mean(ratios) - 1.0) < 0.05


def test_sketch_qr_golden_and_property(orc):
    """test_sketch_qr.cpp:20-71 (4x2 known matrix, R^-T A^T A R^-1 = I) and
    the reference's R^{-1} of a 300x40 matrix."""
    A = np.array([[1.0, 2.0], [3.0, 4.0], [5.0, 6.0], [7.0, 8.0]])
    Ri = orc.sketch_qr_precond(A)
    assert np.allclose(np.tril(Ri, -1), 0)
    np.testing.assert_allclose(Ri.T @ A.T @ A @ Ri, np.eye(2), atol=1e-10)
    g = load("sketch_qr.npz")
    Ri = orc.sketch_qr_precond(g["SA"])
    np.testing.assert_allclose(Ri, g["Rinv"], rtol=1e-10, atol=1e-12 * np.abs(g["Rinv"]).max())
    with pytest.raises(ValueError):
        orc.householder_qr(np.ones((2, 3)))


def test_lsqr_known_system(orc):
    """test_lsqr.cpp:203-247: a 6x3 consistent system, x = (1, -1, 2)."""
    A = np.array([[4, 1, 0], [0, 3, 1], [1, 0, 5], [2, 1, 1], [0, 2, 3], [1, 1, 2]], np.float32)
    xt = np.array([1, -1, 2], np.float32)
    x, it, _ = orc.lsqr_f32(A, A @ xt, tol=1e-7, max_iters=200, max_relres=1e-7)
    np.testing.assert_allclose(x, xt, atol=1e-5)


@pytest.mark.parametrize("precond", [False, True])
def test_lsqr_matches_reference_golden(orc, precond):
    """Plain FP32 LSQR restated in C vs the reference's lsqr_solve: x within
    1e-5 relative, iterations within +-1, histories within 1e-3 relative."""
    g = load("lsqr_small.npz")
    key = "precond" if precond else "plain"
    Rinv = g["Rinv"].astype(np.float32) if precond else None
    x, it, h = orc.lsqr_f32(g["A"], g["b"], Rinv, 1e-6, 400, 1e-6, 1)
    assert abs(it - int(g[f"it_{key}"])) <= 1
    xr = g[f"x_{key}"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-5
    k = min(len(h), len(g[f"hist_{key}"])) - 1
    # relres near 1e-6 sits at the FP32 rounding floor of the recurrence
    np.testing.assert_allclose(h[:k], g[f"hist_{key}"][:k], rtol=2e-3, atol=1e-7)


def test_oracle_against_reference_library(orc):
    """Direct cross-check with the reference's CPU build when it exists
    here (it is built from the reference sources by oracle/Makefile)."""
    if not orc.ref_available():
        pytest.skip("reference CPU build not present")
    import ctypes
    R = orc.ref()
    rng = np.random.default_rng(3)
    x = rng.integers(0, 1 << 32, 1 << 20, dtype=np.uint64).astype(np.uint32).view(np.float32)
    wh = np.empty(x.size, np.uint16)
    wr = np.empty(x.size, np.uint16)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    R.ref_fp32_16_split(P(x), x.size, P(wh), P(wr))
    a, b = orc.fp32_16_split(x)
    assert np.array_equal(a, wh) and np.array_equal(b, wr)
    m, n = 20000, 200
    rng = np.random.default_rng(0)
    A = rng.standard_normal((m, n)).astype(np.float32)
    xt = rng.standard_normal(n).astype(np.float32)
    bb = (A.astype(np.float64) @ xt + 1e-6 * rng.standard_normal(m)).astype(np.float32)
    x1, i1, _ = orc.lsqr_f32(A, bb)
    x2, i2, _ = orc.ref_lsqr_f32(A, bb)
    assert abs(i1 - i2) <= 1
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x2) < 1e-5


def test_blocked_lstsq_and_residuals_match_dense(orc):
    """The row-block oracle (TSQR of [A b] by Householder QR, FP64 residual
    pieces) agrees with the dense oracle on a problem held whole."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((4000, 30)) * 10.0 ** rng.uniform(-3, 3, 30)
    b = rng.standard_normal(4000)
    blocks = [(A[i:i + 650], b[i:i + 650]) for i in range(0, 4000, 650)]
    x, rn = orc.lstsq_f64_blocks(blocks, 30)
    xo = orc.lstsq_f64(A, b)
    assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)
    assert abs(rn - np.linalg.norm(b - A @ xo)) <= 1e-10 * rn
    d = np.linalg.norm(A, axis=0)
    r2, atr, fro, bn = orc.residual_norms_blocks(blocks, xo, d)
    an = np.sqrt(fro)
    eta = min(r2 / (an * np.linalg.norm(d * xo) + bn), atr / (an * r2))
    assert abs(eta - orc.backward_error_scaled(A, b, xo)) <= 1e-10 * max(eta, 1e-300) + 1e-15
