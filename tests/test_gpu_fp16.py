"""Native FP16 storage and LSQR's explicit duplicates: A stored as plain
__half (the reference's --explicit-duplicates storage, whose products it
runs in mv_fp16_native, dense_registries.cpp:73-92, 329-333), plus an FP32
copy (mtx_refine_precision) for the restart residual (lsqr.cpp:451-473)."""
import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import cuda, to_dense
from test_gpu_lsqr import gpu_precond, scaled_problem

pytestmark = pytest.mark.gpu
NT = tb.NumericType
L = tb.Layout


def fp16_dense(A, layout, pad=0):
    return to_dense(A, layout, NT.FP16, pad=pad)


def values(D):
    """The fp16 values of a native FP16 Dense as float64 (m x n)."""
    return D.view().double().cpu().numpy()


@pytest.mark.parametrize("layout,pad", [(L.ROW_MAJOR, 0), (L.COL_MAJOR, 0), (L.ROW_MAJOR, 5), (L.COL_MAJOR, 3)])
def test_pack_fp16_bit_exact(layout, pad):
    """Round to nearest even as numpy's float16 (overflow to Inf, fp16
    subnormals and signed zeros kept)."""
    rng = np.random.default_rng(1)
    A = (rng.standard_normal((300, 77)) * 10.0 ** rng.uniform(-9, 5, (300, 77))).astype(np.float32)
    specials = np.array([65504, 65519.996, 65520, 7e4, -7e4, 6e-8, 5.9e-8, 2.9e-8, 3.0e-8, -0.0, 1e-30,
                         0.1, 1.0 / 3.0, np.inf, -np.inf], np.float32)
    A.ravel()[: specials.size] = specials
    D = fp16_dense(A, layout, pad)
    got = D.view().cpu().numpy().view(np.uint16)
    want = A.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, want)
    # NaN stays NaN
    An = A.copy()
    An[3, 4] = np.nan
    assert np.isnan(fp16_dense(An, layout).view()[3, 4].item())


@pytest.mark.parametrize("layout", [L.ROW_MAJOR, L.COL_MAJOR])
def test_gemv_fp16(layout):
    """Both products over FP16 storage against an FP64 product of the fp16
    values: FP32 accumulation, 2e-5 of sum |a||x|; beta = 0 never reads y."""
    rng = np.random.default_rng(2)
    A = (rng.standard_normal((2001, 333)) * 10.0 ** rng.uniform(-2, 2, 333)).astype(np.float32)
    D = fp16_dense(A, layout, pad=2)
    M = values(D)
    for trans, Mt in ((tb.NO_TRANSPOSE, M), (tb.TRANSPOSE, M.T)):
        x = rng.standard_normal(Mt.shape[1]).astype(np.float32)
        y0 = rng.standard_normal(Mt.shape[0]).astype(np.float32)
        for beta in (0.0, 0.5):
            yy = y0.copy()
            if beta == 0.0:
                yy[:] = np.nan
            y = cuda(yy)
            tb.mv_apply(tb.Device.CUDA, trans, 1.5, D, cuda(x), beta, y)
            ref = 1.5 * (Mt @ x) + (beta * y0 if beta else 0.0)
            scale = 1.5 * (np.abs(Mt) @ np.abs(x)) + abs(beta) * np.abs(y0)
            assert np.all(np.abs(y.cpu().numpy() - ref) <= 2e-5 * scale + 1e-30)


def test_countsketch_fp16(orc):
    """The CountSketch of FP16 storage is the sketch of its fp16 values."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((5000, 120)).astype(np.float32)
    for layout in (L.ROW_MAJOR, L.COL_MAJOR):
        D = fp16_dense(A, layout)
        SA, fro2, colsq = tb.apply_count_sketch(D, 480, with_colsq=True)
        M = values(D)
        ref = orc.countsketch_apply(M, 480)
        np.testing.assert_allclose(SA.view().cpu().numpy(), ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())
        np.testing.assert_allclose(colsq.cpu().numpy(), (M ** 2).sum(0), rtol=1e-6)


@pytest.mark.parametrize("layout,n,pad", [(L.ROW_MAJOR, 300, 4), (L.ROW_MAJOR, 1500, 4), (L.COL_MAJOR, 300, 0)])
def test_lsqr_fp16_iterations(orc, layout, n, pad):
    """Six LSQR iterations over FP16 storage against the oracle's FP32 LSQR
    on the fp16 values (row-major n <= 1152 takes the tensor-core pass)."""
    m = 6000
    rng = np.random.default_rng(n)
    A = rng.standard_normal((m, n)).astype(np.float32)
    b = rng.standard_normal(m).astype(np.float32)
    D = fp16_dense(A, layout, pad)
    x_ref, it_ref, h_ref = orc.lsqr_f32(values(D).astype(np.float32), b, None, 0.0, 6, 0.0, 1)
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
    x = torch.zeros(n, device="cuda")
    rep = tb.lsqr_solve(None, D, cuda(b), x, ws, 0.0, 6, 0.0)
    assert rep["iterations"] == it_ref == 6
    np.testing.assert_allclose(rep["history"][:6], h_ref[:6], rtol=1e-4)
    xx = x.cpu().numpy()
    assert np.linalg.norm(xx - x_ref) / np.linalg.norm(x_ref) < 1e-4


@pytest.mark.parametrize("layout", [L.ROW_MAJOR, L.COL_MAJOR])
def test_explicit_duplicates_backward_error(orc, layout):
    """FP16 iterations with the FP32 duplicate for the restart residuals
    reach backward error 1e-6 of the column-scaled FP32 problem (FP64
    oracle on the FP32 values)."""
    A0, b = scaled_problem(30000, 250, 5)
    A32 = to_dense(A0, layout)
    A16 = tb.pack(A32, NT.FP16)
    Rinv, d, an = gpu_precond(A32, 1000)
    ws = tb.create_lsqr_workspace(None, A0.shape, NT.FP32, NT.FP64)
    tb.add_precond(Rinv, ws)
    xd = torch.zeros(A0.shape[1], device="cuda")
    rep = tb.lsqr_solve(None, A16, cuda(b), xd, ws, 1e-6, 100, 0.0, restarts=6,
                        stop_rule=tb.StopRule.BACKWARD, inner_rtol=1e-3, col_scale=d,
                        anorm_fro=an, mtx_refine_precision=A32)
    x = xd.cpu().numpy()
    eta = orc.backward_error_scaled(A0, b, x)
    assert rep["converged"] == 1, rep
    assert eta <= 1.05e-6, (eta, rep)
    assert abs(rep["backward_error"] - eta) <= 0.05 * eta + 1e-9  # measured on the FP32 copy
    xs = orc.lstsq_f64(A0, b)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-2


def test_explicit_duplicates_relres_restarts(orc):
    """Under the reference's RELRES rule the restart residual b - A_refine x
    drives the solution to the FP32 system's: after restarts x is far closer
    to the FP32 least-squares solution than FP16 iterations alone get."""
    rng = np.random.default_rng(7)
    m, n = 20000, 200
    A0 = rng.standard_normal((m, n)).astype(np.float32)
    b = (A0.astype(np.float64) @ rng.standard_normal(n)).astype(np.float32)
    A32 = to_dense(A0, L.COL_MAJOR)
    A16 = tb.pack(A32, NT.FP16)
    xs = orc.lstsq_f64(A0.astype(np.float64), b.astype(np.float64))
    err = {}
    for dup in (False, True):
        ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
        x = torch.zeros(n, device="cuda")
        tb.lsqr_solve(None, A16, cuda(b), x, ws, 1e-7, 60, 1e-7, restarts=5,
                      mtx_refine_precision=A32 if dup else None)
        err[dup] = np.linalg.norm(x.cpu().numpy() - xs) / np.linalg.norm(xs)
    assert err[True] < 1e-5, err
    assert err[False] > 10 * err[True], err


def test_explicit_duplicate_takes_precedence_over_implicit():
    """With both an explicit FP32 copy and the workspace's implicit duplicate
    set, the restart residual reads the explicit copy (lsqr.cpp:459-473
    tests it first): the solve is the explicit-duplicate solve, bit for bit,
    and differs from the implicit-duplicate one."""
    rng = np.random.default_rng(11)
    m, n = 20000, 120
    A0 = rng.standard_normal((m, n)).astype(np.float32)
    b = cuda((A0.astype(np.float64) @ rng.standard_normal(n)).astype(np.float32))
    A32 = to_dense(A0, L.COL_MAJOR)
    P = tb.pack(A32, NT.FP32_16)
    # a refine copy that is not A: the explicit and implicit residuals differ
    R32 = to_dense((A0 * np.float32(1.001)).astype(np.float32), L.COL_MAJOR)
    xs = {}
    for name, implicit, refine in (("both", True, R32), ("explicit", False, R32), ("implicit", True, None)):
        ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
        ws.use_implicit_duplicate_ = implicit
        x = torch.zeros(n, device="cuda")
        tb.lsqr_solve(None, P, b, x, ws, 1e-7, 40, 1e-7, restarts=3, mtx_refine_precision=refine)
        xs[name] = x.cpu().numpy()
    assert np.array_equal(xs["both"], xs["explicit"])
    assert not np.array_equal(xs["both"], xs["implicit"])


def test_explicit_duplicates_errors():
    A = np.ones((100, 10), np.float32)
    A32 = to_dense(A, L.COL_MAJOR)
    A16 = tb.pack(A32, NT.FP16)
    ws = tb.create_lsqr_workspace(None, (100, 10), NT.FP32)
    x = torch.zeros(10, device="cuda")
    b = torch.ones(100, device="cuda")
    wrong = to_dense(np.ones((100, 9), np.float32), L.COL_MAJOR)
    with pytest.raises(tb.TomosError) as e:
        tb.lsqr_solve(None, A16, b, x, ws, 1e-6, 10, 1e-6, mtx_refine_precision=wrong)
    assert "size" in str(e.value)
