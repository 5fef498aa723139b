"""lsqr_solve on the device against the reference's own LSQR (golden
fixtures and the oracle restatement) and against the FP64 least-squares
oracle, for FP32 and packed storage, plain and sketch-preconditioned."""
import os

import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, cuda, decoded

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu
L = tb.Layout
NT = tb.NumericType
CTX = None


def solve(A, b, Rinv=None, tol=1e-6, max_iters=400, max_relres=1e-6, restarts=1, **kw):
    m, n = A.size if hasattr(A, "size") and isinstance(A.size, tuple) else A.size
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32,
                                  None if Rinv is None else Rinv.numeric)
    if Rinv is not None:
        tb.add_precond(Rinv, ws)
    for k in ("implicit_duplicate",):
        if kw.pop(k, False):
            ws.use_implicit_duplicate_ = True
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    rep = tb.lsqr_solve(CTX, A, cuda(b), x, ws, tol, max_iters, max_relres, restarts=restarts, **kw)
    return x.cpu().numpy(), rep


def config1(m=20000, n=200, seed=0):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((m, n)).astype(np.float32)
    xt = rng.standard_normal(n).astype(np.float32)
    b = (A.astype(np.float64) @ xt + 1e-6 * rng.standard_normal(m)).astype(np.float32)
    return A, b


@pytest.mark.parametrize("layout", [L.COL_MAJOR, L.ROW_MAJOR])
def test_plain_fp32_matches_reference_config1(orc, layout):
    """Plain FP32 LSQR on 20000 x 200: x within 1e-5 of the reference's,
    iteration count within +-1, residual history close."""
    A0, b = config1()
    x_ref, it_ref, h_ref = orc.lsqr_f32(A0, b, None, 1e-6, 400, 1e-6, 1)
    if orc.ref_available():
        x_ref2, it_ref2, _ = orc.ref_lsqr_f32(A0, b, None, 1e-6, 400, 1e-6, 1)
        assert abs(it_ref2 - it_ref) <= 1
    x, rep = solve(to_dense(A0, layout), b)
    assert abs(rep["iterations"] - it_ref) <= 1
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-5
    k = min(len(h_ref), len(rep["history"])) - 1
    np.testing.assert_allclose(rep["history"][:k], h_ref[:k], rtol=2e-3, atol=1e-7)
    assert rep["converged"] == 1


@pytest.mark.parametrize("precond", [False, True])
@pytest.mark.parametrize("layout", [L.COL_MAJOR, L.ROW_MAJOR])
def test_matches_reference_golden(precond, layout):
    g = np.load(os.path.join(GOLD, "lsqr_small.npz"))
    key = "precond" if precond else "plain"
    R = None
    if precond:
        R = tb.Dense.from_tensor(torch.from_numpy(g["Rinv"].astype(np.float32)), L.COL_MAJOR)
    x, rep = solve(to_dense(g["A"], layout), g["b"], R)
    assert abs(rep["iterations"] - int(g[f"it_{key}"])) <= 1
    xr = g[f"x_{key}"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-5


def test_known_systems():
    """test_lsqr.cpp: 6x3 consistent (x = (1,-1,2)), identity, diagonal and
    an inconsistent 4x2 (x = (3.5, 1.4))."""
    A = np.array([[4, 1, 0], [0, 3, 1], [1, 0, 5], [2, 1, 1], [0, 2, 3], [1, 1, 2]], np.float32)
    x, _ = solve(to_dense(A, L.COL_MAJOR), A @ np.float32([1, -1, 2]), tol=1e-7, max_relres=1e-7,
                 max_iters=200)
    np.testing.assert_allclose(x, [1, -1, 2], atol=2e-5)
    x, _ = solve(to_dense(np.eye(3, dtype=np.float32), L.ROW_MAJOR), np.float32([1, 2, 3]),
                 tol=1e-10, max_iters=50, max_relres=1e-10)
    np.testing.assert_allclose(x, [1, 2, 3], atol=1e-6)
    x, _ = solve(to_dense(np.diag(np.float32([1, 2, 4])), L.COL_MAJOR), np.float32([1, 4, 8]),
                 tol=1e-10, max_iters=50, max_relres=1e-10)
    np.testing.assert_allclose(x, [1, 2, 2], atol=1e-6)
    A = np.array([[1, 1], [1, 2], [1, 3], [1, 4]], np.float32)
    x, _ = solve(to_dense(A, L.ROW_MAJOR), np.float32([6, 5, 7, 10]), tol=1e-10, max_iters=200,
                 max_relres=1e-10)
    np.testing.assert_allclose(x, [3.5, 1.4], atol=1e-5)


def gpu_precond(A, s):
    SA, fro2, colsq = tb.apply_count_sketch(A, s, tier=tb.Tier.AUTO, with_colsq=True)
    d, an = tb.column_scale(colsq)
    return tb.generate_sketch_qr_precond(SA), d, an


def scaled_problem(m, n, seed, decades=2.0):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-decades, decades, n)).astype(np.float32)
    xt = rng.standard_normal(n)
    b = (A.astype(np.float64) @ xt + 1e-8 * rng.standard_normal(m)).astype(np.float32)
    return A, b


@pytest.mark.parametrize("numeric", [NT.FP32, NT.FP32_16, NT.FP32_BF16])
@pytest.mark.parametrize("layout", [L.ROW_MAJOR, L.COL_MAJOR])
def test_preconditioned_backward_error(orc, numeric, layout):
    """Sketch-preconditioned LSQR to backward error 1e-6 of the
    column-scaled problem (FP64 oracle check), with FP32 residual
    refinement for packed storage; the plain normwise backward error is
    then below it too."""
    A0, b = scaled_problem(30000, 250, 3)
    A = to_dense(A0, layout, numeric)
    Rinv, d, an = gpu_precond(A, 1000)
    x, rep = solve(A, b, Rinv, tol=1e-6, max_iters=100, restarts=6,
                   stop_rule=tb.StopRule.BACKWARD, inner_rtol=1e-3 if numeric != NT.FP32 else 0.0,
                   col_scale=d, anorm_fro=an)
    eta = orc.backward_error_scaled(A0, b, x)
    assert rep["converged"] == 1, rep
    assert eta <= 1.05e-6, (eta, rep)
    assert abs(rep["backward_error"] - eta) <= 0.05 * eta + 1e-9
    assert orc.backward_error(A0, b, x) <= eta * 1.01
    xs = orc.lstsq_f64(A0, b)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-2


@pytest.mark.parametrize("tier", [tb.Tier.AUTO, tb.Tier.ACCURATE])
@pytest.mark.parametrize("numeric", [NT.FP32, NT.FP32_16, NT.FP32_BF16])
@pytest.mark.parametrize("n,ld", [(257, 264), (1000, 1000), (1001, 1008), (500, 512),
                                  (1500, 1504), (2000, 2000), (3001, 3008)])
def test_fused_pass_matches_oracle_lsqr(orc, numeric, n, ld, tier):
    """The staged fused pass (row-major, one CTA per SM; one warp per row
    up to 1024 columns, 2 or 4 beyond) against the oracle's LSQR on the
    values the tier reads: the same 6 iterations give the same x (FP32
    arithmetic in both, different summation order).  ACCURATE runs the
    iterations on the exact (wh + wr) values with FP64 chunk sums."""
    if tier == tb.Tier.ACCURATE and numeric == NT.FP32:
        pytest.skip("FP32 storage has one tier")
    m = 6000
    rng = np.random.default_rng(n)
    A0 = (rng.standard_normal((m, n)) * np.where(rng.random((m, n)) < 0.02, 1e-6, 1.0)).astype(np.float32)
    b = rng.standard_normal(m).astype(np.float32)
    A = to_dense(A0, L.ROW_MAJOR, numeric, pad=ld - n)
    read = tb.Tier.AUTO if numeric == NT.FP32 else (tb.Tier.HALF if tier == tb.Tier.AUTO else tier)
    Ad = decoded(orc, A, read).astype(np.float32)
    x_ref, it_ref, h_ref = orc.lsqr_f32(Ad, b, None, 0.0, 6, 0.0, 1)
    x, rep = solve(A, b, tol=0.0, max_iters=6, max_relres=0.0, tier=tier)
    assert rep["iterations"] == it_ref == 6
    np.testing.assert_allclose(rep["history"][:6], h_ref[:6], rtol=1e-4)
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-4


def test_prestaged_plane_same_solve():
    """A solve handed the plane the staging sketch wrote runs the same passes
    as one that stages its own copy: bit-identical x and reports."""
    A0, b = scaled_problem(20000, 300, 11)
    A = to_dense(A0, L.ROW_MAJOR, NT.FP32_16, pad=4)  # 16-byte aligned rows
    SA, _, colsq, plane = tb.apply_count_sketch(A, 1200, tier=tb.Tier.HALF, with_colsq=True,
                                                stage=True)
    Rinv = tb.generate_sketch_qr_precond(SA)
    d, anorm = tb.column_scale(colsq)
    out = []
    for staged in (None, plane):
        ws = tb.create_lsqr_workspace(None, A.size, NT.FP32, NT.FP64)
        tb.add_precond(Rinv, ws)
        x = torch.zeros(300, device="cuda")
        rep = tb.lsqr_solve(None, A, cuda(b), x, ws, 1e-6, 100, 0.0, restarts=6,
                            stop_rule=tb.StopRule.BACKWARD, inner_rtol=2e-3, anorm_fro=anorm,
                            col_scale=d, staged_plane=staged)
        out.append((x.cpu().numpy(), rep))
    (x0, r0), (x1, r1) = out
    assert r0["converged"] == 1 and r0["backward_error"] <= 1e-6
    assert np.array_equal(x0, x1)
    assert r0["iterations"] == r1["iterations"] and r0["backward_error"] == r1["backward_error"]
    ws = tb.create_lsqr_workspace(None, A.size, NT.FP32)
    with pytest.raises(tb.TomosError):
        tb.lsqr_solve(None, A, cuda(b), torch.zeros(300, device="cuda"), ws, 1e-6, 10, 0.0,
                      staged_plane=plane[:, 1:])


@pytest.mark.parametrize("zeros", [False, True])
@pytest.mark.parametrize("numeric,rounded", [(NT.FP32, False), (NT.FP32_16, False),
                                             (NT.FP32_BF16, False), (NT.FP32_BF16, True)])
@pytest.mark.parametrize("n", [1000, 300])
def test_exact_pass_residual(orc, numeric, rounded, zeros, n):
    """The exact (FP64-summing) pass behind the restart residuals and the
    backward-error entry: with b = fl32(A x) for the exactly decoded A, the
    residual is the rounding of b alone, so one element decoded one unit
    off at any bit would swamp it.  Covers FP32_16 control words below and
    above the fp16 range and, with zeros, the saturated words (signed
    zeros) that take the conversion-pipe path."""
    rng = np.random.default_rng(n + (7 if zeros else 0))
    m = 6000
    A0 = rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-3, 3, n)
    pick = rng.random((m, n))
    A0 = np.where(pick < 0.01, A0 * 1e-6, A0)                 # control words below fp16 range
    A0 = np.where((pick >= 0.01) & (pick < 0.015), A0 * 1e4, A0)  # and above it
    if zeros:
        A0 = np.where((pick >= 0.015) & (pick < 0.017), 0.0, A0)
    A0 = A0.astype(np.float32)
    A = to_dense(A0, L.ROW_MAJOR, numeric, pad=(-n) % 8, rounded=rounded)
    Ae = decoded(orc, A, tb.Tier.ACCURATE)
    x = rng.standard_normal(n).astype(np.float32)
    b = (Ae @ x.astype(np.float64)).astype(np.float32)
    r = b.astype(np.float64) - Ae @ x.astype(np.float64)
    ws = tb.create_lsqr_workspace(None, A.size, NT.FP32)
    rep = tb.backward_error(A, cuda(b), cuda(x), ws)
    np.testing.assert_allclose(rep["rnorm"], np.linalg.norm(r), rtol=1e-6)
    np.testing.assert_allclose(rep["arnorm"], np.linalg.norm(Ae.T @ r), rtol=2e-3)


def test_backward_error_entry(orc):
    A0, b = scaled_problem(5000, 60, 8)
    A = to_dense(A0, L.ROW_MAJOR)
    x = orc.lstsq_f64(A0, b).astype(np.float32) * np.float32(1.0001)
    ws = tb.create_lsqr_workspace(None, A.size, NT.FP32)
    rep = tb.backward_error(A, cuda(b), cuda(x), ws)
    np.testing.assert_allclose(rep["backward_error"], orc.backward_error(A0, b, x), rtol=1e-6)
    d = np.linalg.norm(A0.astype(np.float64), axis=0)
    rep = tb.backward_error(A, cuda(b), cuda(x), ws, col_scale=cuda(d, torch.float64))
    np.testing.assert_allclose(rep["backward_error"], orc.backward_error_scaled(A0, b, x), rtol=1e-6)


def test_errors():
    A = to_dense(np.ones((10, 3), np.float32), L.COL_MAJOR)
    ws = tb.create_lsqr_workspace(None, (10, 4), NT.FP32)
    x = torch.zeros(3, device="cuda")
    with pytest.raises(tb.TomosError):
        tb.lsqr_solve(None, A, cuda(np.ones(10)), x, ws, 1e-6, 10, 1e-6)
    ws = tb.create_lsqr_workspace(None, (10, 3), NT.FP32, NT.FP64)
    R32 = tb.Dense.from_tensor(torch.eye(3), L.COL_MAJOR)
    with pytest.raises(tb.TomosError):
        tb.add_precond(R32, ws)
    ws.use_implicit_duplicate_ = True
    with pytest.raises(tb.TomosError):
        tb.lsqr_solve(None, A, cuda(np.ones(10)), x, ws, 1e-6, 10, 1e-6)


def test_zero_rhs_and_restarts():
    A0, _ = config1(500, 20, 1)
    x, rep = solve(to_dense(A0, L.ROW_MAJOR), np.zeros(500, np.float32))
    assert np.all(x == 0) and rep["converged"] == 1
    A0, b = config1(2000, 40, 2)
    x1, r1 = solve(to_dense(A0, L.ROW_MAJOR), b, max_iters=3, restarts=4)
    assert r1["iterations"] <= 12


def test_repeated_solves_on_one_workspace():
    """Solves that reuse a workspace (and its captured iteration graph) read
    the column scale and x of the current call: the caller's buffers of an
    earlier call are freed and overwritten in between (NaN-filled tensors of
    their size take their memory), and every solve still converges with the
    same iterations and the same x."""
    A0, b = scaled_problem(30000, 300, 21)
    A = to_dense(A0, L.ROW_MAJOR, NT.FP32_16, pad=4)
    ws = tb.create_lsqr_workspace(None, A.size, NT.FP32, NT.FP64)
    bd = cuda(b)
    out = []
    for _ in range(4):
        x, rep, d = tb.sketch_lsqr(A, bd, 1200, workspace=ws)
        out.append((x.cpu().numpy(), rep["iterations"], rep["converged"], rep["backward_error"]))
        del x, d
        junk = [torch.full((300,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(8)]
        junk += [torch.full((300,), float("nan"), dtype=torch.float32, device="cuda") for _ in range(8)]
        del junk
    x0, it0, c0, e0 = out[0]
    assert c0 == 1 and e0 <= 1e-6
    for x, it, c, e in out[1:]:
        assert c == 1 and it == it0 and e == e0
        assert np.array_equal(x, x0)
