"""CSR products, CSR CountSketch and CSR LSQR against FP64 oracles."""
import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import cuda

pytestmark = pytest.mark.gpu
NT = tb.NumericType


def random_csr(m, n, k, seed, decades=1.0):
    rng = np.random.default_rng(seed)
    cols = np.stack([np.sort(rng.choice(n, k, replace=False)) for _ in range(m)])
    vals = rng.standard_normal((m, k)) * 10.0 ** rng.uniform(-decades, decades, (m, 1))
    D = np.zeros((m, n))
    np.put_along_axis(D, cols, vals, axis=1)
    rp = np.arange(0, (m + 1) * k, k, dtype=np.int32)
    return rp, cols.astype(np.int32).ravel(), vals.astype(np.float32).ravel(), D.astype(np.float32)


def make(rp, ci, v, m, n, numeric=NT.FP32, rounded=False):
    vals = cuda(v)
    if numeric != NT.FP32:
        t = tb.Dense.from_tensor(vals[None, :], tb.Layout.ROW_MAJOR)
        P = tb.pack(t, numeric, rounded=rounded)
        vals = P.storage  # [wh | wr] planar, nnz each
    return tb.Csr(numeric, (m, n), cuda(rp, torch.int32), cuda(ci, torch.int32), vals, rounded)


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.HALF),
                                          (NT.FP32_16, tb.Tier.ACCURATE), (NT.FP32_BF16, tb.Tier.HALF)])
def test_csr_gemv(orc, numeric, tier):
    m, n = 3001, 517
    rp, ci, v, D = random_csr(m, n, 9, 1)
    A = make(rp, ci, v, m, n, numeric)
    if numeric == NT.FP32:
        Dd = D.astype(np.float64)
    else:
        wh, wr = (orc.fp32_16_split(v) if numeric == NT.FP32_16 else orc.fp32_bf16_split(v))
        kind = "fp32_16" if numeric == NT.FP32_16 else "fp32_bf16"
        vv = orc.decode(kind, wh, wr, "half" if tier == tb.Tier.HALF else "accurate")
        Dd = np.zeros((m, n))
        np.put_along_axis(Dd, ci.reshape(m, -1).astype(np.int64), vv.reshape(m, -1), axis=1)
    rng = np.random.default_rng(2)
    for trans, M in ((tb.NO_TRANSPOSE, Dd), (tb.TRANSPOSE, Dd.T)):
        x = rng.standard_normal(M.shape[1]).astype(np.float32)
        y0 = rng.standard_normal(M.shape[0]).astype(np.float32)
        for beta in (0.0, -0.25):
            yy = y0.copy()
            if beta == 0.0:
                yy[:] = np.nan
            y = cuda(yy)
            tb.mv_apply(tb.Device.CUDA, trans, 2.0, A, cuda(x), beta, y, tier=tier)
            ref = 2.0 * (M @ x) + (beta * y0 if beta else 0.0)
            scale = 2.0 * (np.abs(M) @ np.abs(x)) + abs(beta) * np.abs(y0)
            assert np.all(np.abs(y.cpu().numpy() - ref) <= 2e-5 * scale + 1e-6 * np.abs(ref) + 1e-30)


def test_csr_countsketch(orc):
    m, n, s = 4000, 300, 211
    rp, ci, v, D = random_csr(m, n, 12, 5)
    A = make(rp, ci, v, m, n)
    SA, fro2, colsq = tb.apply_count_sketch(A, s, with_colsq=True)
    np.testing.assert_allclose(colsq.cpu().numpy(), (D.astype(np.float64) ** 2).sum(0), rtol=1e-12)
    ref = orc.countsketch_apply(D, s)
    np.testing.assert_allclose(SA.view().cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_allclose(fro2.item(), (v.astype(np.float64) ** 2).sum(), rtol=1e-12)


@pytest.mark.parametrize("numeric", [NT.FP32, NT.FP32_16])
def test_csr_lsqr_preconditioned(orc, numeric):
    m, n = 20000, 400
    rp, ci, v, D = random_csr(m, n, 20, 7, decades=2.0)
    rng = np.random.default_rng(8)
    xt = rng.standard_normal(n)
    b = (D.astype(np.float64) @ xt + 1e-8 * rng.standard_normal(m)).astype(np.float32)
    A = make(rp, ci, v, m, n, numeric)
    SA, fro2, colsq = tb.apply_count_sketch(A, 4 * n, tier=tb.Tier.AUTO, with_colsq=True)
    Rinv = tb.generate_sketch_qr_precond(SA)
    d, an = tb.column_scale(colsq)
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32, NT.FP64)
    tb.add_precond(Rinv, ws)
    x = torch.zeros(n, device="cuda")
    rep = tb.lsqr_solve(None, A, cuda(b), x, ws, 1e-6, 200, 0.0, restarts=6,
                        stop_rule=tb.StopRule.BACKWARD, inner_rtol=1e-3 if numeric != NT.FP32 else 0.0,
                        col_scale=d, anorm_fro=an)
    xx = x.cpu().numpy()
    eta = orc.backward_error_scaled(D, b, xx)
    assert rep["converged"] == 1 and eta <= 1.05e-6, (eta, rep)
    assert orc.backward_error(D, b, xx) <= eta * 1.01


def ragged_csr(m, n, seed):
    """Row lengths 0..96, 5% empty rows, eight rows of 300 entries (longer
    than any lane group's first loads), the last 7 columns empty."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 97, m)
    lens[rng.random(m) < 0.05] = 0
    lens[rng.choice(m, 8, replace=False)] = 300
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n - 7, k, replace=False)) for k in lens]).astype(np.int32)
    v = (rng.standard_normal(rp[-1]) * 10.0 ** rng.uniform(-1, 1, rp[-1])).astype(np.float32)
    return rp.astype(np.int32), ci, v


def decoded_dense(orc, rp, ci, v, m, n, numeric, tier):
    """The values a tier reads, scattered into a dense FP64 matrix."""
    if numeric == NT.FP32:
        vv = v.astype(np.float64)
    else:
        wh, wr = orc.fp32_16_split(v) if numeric == NT.FP32_16 else orc.fp32_bf16_split(v)
        kind = "fp32_16" if numeric == NT.FP32_16 else "fp32_bf16"
        vv = orc.decode(kind, wh, wr, "half" if tier == tb.Tier.HALF else "accurate").astype(np.float64)
    D = np.zeros((m, n))
    rows = np.repeat(np.arange(m), np.diff(rp))
    D[rows, ci] = vv
    return D


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.HALF),
                                          (NT.FP32_16, tb.Tier.ACCURATE)])
def test_csr_ragged_products(orc, numeric, tier):
    """Both products on ragged rows (empty, short and long) and empty columns."""
    m, n = 5000, 700
    rp, ci, v = ragged_csr(m, n, 3)
    A = make(rp, ci, v, m, n, numeric)
    Dd = decoded_dense(orc, rp, ci, v, m, n, numeric, tier)
    rng = np.random.default_rng(4)
    for trans, M in ((tb.NO_TRANSPOSE, Dd), (tb.TRANSPOSE, Dd.T)):
        x = rng.standard_normal(M.shape[1]).astype(np.float32)
        y0 = rng.standard_normal(M.shape[0]).astype(np.float32)
        y = cuda(y0)
        tb.mv_apply(tb.Device.CUDA, trans, 1.5, A, cuda(x), 0.5, y, tier=tier)
        ref = 1.5 * (M @ x) + 0.5 * y0
        scale = 1.5 * (np.abs(M) @ np.abs(x)) + 0.5 * np.abs(y0)
        assert np.all(np.abs(y.cpu().numpy() - ref) <= 2e-5 * scale + 1e-30)


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.HALF),
                                          (NT.FP32_16, tb.Tier.ACCURATE)])
def test_csr_ragged_lsqr_iterations(orc, numeric, tier):
    """Six LSQR iterations over ragged CSR storage against the oracle's LSQR
    on the values the tier reads (FP32 arithmetic in both, different
    summation order); a second solve gives a bit-identical x."""
    m, n = 5000, 700
    rp, ci, v = ragged_csr(m, n, 5)
    A = make(rp, ci, v, m, n, numeric)
    Dd = decoded_dense(orc, rp, ci, v, m, n, numeric, tier)
    b = np.random.default_rng(6).standard_normal(m).astype(np.float32)
    x_ref, it_ref, h_ref = orc.lsqr_f32(Dd.astype(np.float32), b, None, 0.0, 6, 0.0, 1)
    xs = []
    for _ in range(2):
        ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
        x = torch.zeros(n, device="cuda")
        rep = tb.lsqr_solve(None, A, cuda(b), x, ws, 0.0, 6, 0.0, tier=tier)
        xs.append(x)
    assert rep["iterations"] == it_ref == 6
    np.testing.assert_allclose(rep["history"][:6], h_ref[:6], rtol=1e-4)
    xx = xs[0].cpu().numpy()
    assert np.linalg.norm(xx - x_ref) / np.linalg.norm(x_ref) < 1e-4
    assert np.all(xx[n - 7:] == 0.0)
    assert torch.equal(xs[0], xs[1])


# ------------------------------------------------- FP16 values, explicit duplicates

def make_fp16(rp, ci, v, m, n):
    """A CSR of native IEEE fp16 values (the reference's __half Sparse)."""
    return tb.Csr(NT.FP16, (m, n), cuda(rp, torch.int32), cuda(ci, torch.int32), cuda(v, torch.float16))


def fp16_values_dense(ci, v, m, n):
    D = np.zeros((m, n))
    np.put_along_axis(D, ci.reshape(m, -1).astype(np.int64),
                      v.astype(np.float16).astype(np.float64).reshape(m, -1), axis=1)
    return D


def test_csr_fp16_gemv():
    """Both products over fp16 CSR values against the FP64 product of the
    fp16 values (FP32 accumulation)."""
    m, n = 3001, 517
    rp, ci, v, _ = random_csr(m, n, 9, 21)
    A = make_fp16(rp, ci, v, m, n)
    Dd = fp16_values_dense(ci, v, m, n)
    rng = np.random.default_rng(22)
    for trans, M in ((tb.NO_TRANSPOSE, Dd), (tb.TRANSPOSE, Dd.T)):
        x = rng.standard_normal(M.shape[1]).astype(np.float32)
        y0 = rng.standard_normal(M.shape[0]).astype(np.float32)
        y = cuda(y0)
        tb.mv_apply(tb.Device.CUDA, trans, 1.5, A, cuda(x), 0.5, y)
        ref = 1.5 * (M @ x) + 0.5 * y0
        scale = 1.5 * (np.abs(M) @ np.abs(x)) + 0.5 * np.abs(y0)
        assert np.all(np.abs(y.cpu().numpy() - ref) <= 2e-5 * scale + 1e-30)


def test_csr_explicit_duplicates_backward_error(orc):
    """lsqr_solve(Sparse&, ..., mtx_refine_precision): fp16 iterations (the
    CSC gathers) with the FP32 CSR duplicate for the initial and restart
    passes reach backward error 1e-6 of the column-scaled FP32 problem,
    checked in FP64 on the FP32 values."""
    m, n = 20000, 300
    rp, ci, v, D = random_csr(m, n, 20, 23, decades=2.0)
    rng = np.random.default_rng(24)
    b = (D.astype(np.float64) @ rng.standard_normal(n) + 1e-8 * rng.standard_normal(m)).astype(np.float32)
    A32 = make(rp, ci, v, m, n)
    A16 = make_fp16(rp, ci, v, m, n)
    SA, _, colsq = tb.apply_count_sketch(A32, 4 * n, with_colsq=True)
    Rinv = tb.generate_sketch_qr_precond(SA)
    d, an = tb.column_scale(colsq)
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32, NT.FP64)
    tb.add_precond(Rinv, ws)
    xd = torch.zeros(n, device="cuda")
    rep = tb.lsqr_solve(None, A16, cuda(b), xd, ws, 1e-6, 100, 0.0, restarts=6,
                        stop_rule=tb.StopRule.BACKWARD, inner_rtol=1e-3, col_scale=d, anorm_fro=an,
                        mtx_refine_precision=A32)
    x = xd.cpu().numpy()
    eta = orc.backward_error_scaled(D, b, x)
    assert rep["converged"] == 1 and rep["restarts_used"] >= 2, rep
    assert eta <= 1.05e-6, (eta, rep)
    assert abs(rep["backward_error"] - eta) <= 0.05 * eta + 1e-9  # measured on the FP32 copy
    xs = orc.lstsq_f64(D.astype(np.float64), b.astype(np.float64))
    dn = np.sqrt((D.astype(np.float64) ** 2).sum(0))
    assert np.linalg.norm(dn * (x - xs)) / np.linalg.norm(dn * xs) < 1e-4


def test_csr_explicit_duplicates_relres_restarts(orc):
    """Under the reference's RELRES rule the restart residual b - A_refine x
    drives x to the FP32 system's least-squares solution; fp16 iterations
    alone stop far from it."""
    m, n = 20000, 200
    rp, ci, v, D = random_csr(m, n, 16, 25, decades=0.0)
    rng = np.random.default_rng(26)
    b = (D.astype(np.float64) @ rng.standard_normal(n)).astype(np.float32)
    A32 = make(rp, ci, v, m, n)
    A16 = make_fp16(rp, ci, v, m, n)
    xs = orc.lstsq_f64(D.astype(np.float64), b.astype(np.float64))
    err = {}
    for dup in (False, True):
        ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
        x = torch.zeros(n, device="cuda")
        tb.lsqr_solve(None, A16, cuda(b), x, ws, 1e-7, 60, 1e-7, restarts=5,
                      mtx_refine_precision=A32 if dup else None)
        err[dup] = np.linalg.norm(x.cpu().numpy() - xs) / np.linalg.norm(xs)
    assert err[True] < 1e-5, err
    assert err[False] > 10 * err[True], err


def test_csr_explicit_duplicates_errors():
    m, n = 100, 10
    rp, ci, v, _ = random_csr(m, n, 3, 27)
    A16 = make_fp16(rp, ci, v, m, n)
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
    x = torch.zeros(n, device="cuda")
    b = torch.ones(m, device="cuda")
    rp2, ci2, v2, _ = random_csr(m, n - 1, 3, 28)
    with pytest.raises(tb.TomosError) as e:  # another size
        tb.lsqr_solve(None, A16, b, x, ws, 1e-6, 10, 1e-6, mtx_refine_precision=make(rp2, ci2, v2, m, n - 1))
    assert "size" in str(e.value)
    dense = tb.Dense.from_tensor(torch.ones((m, n), device="cuda"), tb.Layout.ROW_MAJOR)
    with pytest.raises(tb.TomosError):  # a dense copy beside a CSR A
        tb.lsqr_solve(None, A16, b, x, ws, 1e-6, 10, 1e-6, mtx_refine_precision=dense)
    with pytest.raises(tb.TomosError):  # a CSR copy beside a dense A
        tb.lsqr_solve(None, dense, b, x, ws, 1e-6, 10, 1e-6, mtx_refine_precision=make(rp, ci, v, m, n))
