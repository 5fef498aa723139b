"""The adjoint of x* = argmin ||A x - b|| (no reference counterpart):
lambda from preconditioned CG on the normal equations, dL/dB and dL/dA in
one pass over A, and the torch.autograd wrapper, against the FP64
normal-equations gradient and FP64 central finite differences (step 1e-6).
The bar is 1e-4 relative."""
import numpy as np
import pytest
import torch

import tomos_b200 as tb
from tomos_b200.adjoint import lstsq
from gpu_util import to_dense, cuda

pytestmark = pytest.mark.gpu
NT = tb.NumericType
L = tb.Layout


def problem(m, n, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((m, n)).astype(np.float32)
    B = rng.standard_normal((m, K)).astype(np.float32)
    G = rng.standard_normal((n, K)).astype(np.float32)
    return A, B, G


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)


def gpu_grads(A0, B0, G0, numeric=NT.FP32, precond=True, tol=1e-7, batch=False):
    """Forward solves, adjoint solves (one CG per column, or all columns at
    once with shared products when batch) and the gradient pass through the
    C ABI; returns (X, Lam, gradA, gradB, adjoint reports)."""
    m, n = A0.shape
    K = B0.shape[1]
    A = to_dense(A0, L.ROW_MAJOR, numeric)
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32, NT.FP64 if precond else None)
    if precond:
        SA, _, colsq = tb.apply_count_sketch(A, 4 * n, tier=tb.Tier.AUTO, with_colsq=True)
        Rinv = tb.generate_sketch_qr_precond(SA)
        tb.add_precond(Rinv, ws)
    X = torch.zeros((n, K), device="cuda")
    Lam = torch.zeros((n, K), device="cuda")
    reps = []
    for k in range(K):
        x = torch.zeros(n, device="cuda")
        tb.lsqr_solve(None, A, cuda(B0[:, k]), x, ws, 1e-7, 400, 1e-7, restarts=4,
                      stop_rule=tb.StopRule.BACKWARD,
                      tier=tb.Tier.ACCURATE if numeric != NT.FP32 else None)
        X[:, k] = x
        if not batch:
            lam, rep = tb.lsqr_adjoint(A, cuda(G0[:, k]), ws, tol=tol, max_iters=1000)
            Lam[:, k] = lam
            reps.append(rep)
    if batch:
        Lam, reps = tb.lsqr_adjoint_batch(A, cuda(G0), ws, tol=tol, max_iters=1000)
    gA, gB = tb.lsqr_adjoint_grad(A, cuda(B0), X, Lam)
    return (X.cpu().numpy(), Lam.cpu().numpy(), gA.cpu().numpy(), gB.cpu().numpy(), reps)


def test_adjoint_vs_fp64_and_finite_differences(orc):
    A0, B0, G0 = problem(2000, 50, 3, 1)
    X, Lam, gA, gB, reps = gpu_grads(A0, B0, G0)
    assert all(r["converged"] for r in reps), reps
    Xr, Lr, gAr, gBr = orc.lstsq_grads_f64(A0, B0, G0)
    assert rel(X, Xr) < 1e-5
    assert rel(Lam, Lr) < 1e-5
    assert rel(gA, gAr) < 1e-4
    assert rel(gB, gBr) < 1e-4
    rng = np.random.default_rng(2)
    ea = [(int(i), int(j)) for i, j in zip(rng.integers(0, 2000, 12), rng.integers(0, 50, 12))]
    eb = [(int(i), int(k)) for i, k in zip(rng.integers(0, 2000, 12), rng.integers(0, 3, 12))]
    fa, fb = orc.lstsq_fd_f64(A0, B0, G0, ea, eb, h=1e-6)
    ga = np.array([gA[i, j] for i, j in ea])
    gb = np.array([gB[i, k] for i, k in eb])
    assert np.all(np.abs(ga - fa) <= 1e-4 * np.abs(gAr).max()), (ga, fa)
    assert np.all(np.abs(gb - fb) <= 1e-4 * np.abs(gBr).max()), (gb, fb)


def test_adjoint_config5_size(orc):
    """200,000 x 500, 8 right-hand sides: dL/dB in full and dL/dA on 2000
    sampled rows against the FP64 normal-equations gradient."""
    A0, B0, G0 = problem(200_000, 500, 8, 3)
    X, Lam, gA, gB, reps = gpu_grads(A0, B0, G0)
    assert all(r["converged"] for r in reps)
    assert max(r["iterations"] for r in reps) < 60
    Xr, Lr, gAr, gBr = orc.lstsq_grads_f64(A0, B0, G0)
    assert rel(Lam, Lr) < 1e-5
    assert rel(gB, gBr) < 1e-4
    rows = np.random.default_rng(4).choice(200_000, 2000, replace=False)
    assert rel(gA[rows], gAr[rows]) < 1e-4


def test_autograd_function(orc):
    A0, B0, G0 = problem(3000, 40, 2, 5)
    A = torch.from_numpy(A0).cuda().requires_grad_(True)
    B = torch.from_numpy(B0).cuda().requires_grad_(True)
    X = lstsq(A, B, tol=1e-7)
    loss = (torch.from_numpy(G0).cuda() * X).sum()
    loss.backward()
    Xr, _, gAr, gBr = orc.lstsq_grads_f64(A0, B0, G0)
    assert rel(X.detach().cpu().numpy(), Xr) < 1e-5
    assert rel(A.grad.cpu().numpy(), gAr) < 1e-4
    assert rel(B.grad.cpu().numpy(), gBr) < 1e-4


@pytest.mark.parametrize("numeric", [NT.FP32_16, NT.FP32_BF16])
def test_adjoint_packed_exact_values(orc, numeric):
    """Packed A: the adjoint and the gradient pass read the exact (wh + wr)
    values, which equal the FP32 matrix."""
    A0, B0, G0 = problem(4000, 60, 2, 6)
    A0 = (A0 * 10.0 ** np.random.default_rng(7).uniform(-2, 2, 60)).astype(np.float32)
    X, Lam, gA, gB, reps = gpu_grads(A0, B0, G0, numeric=numeric)
    assert all(r["converged"] for r in reps)
    _, Lr, gAr, gBr = orc.lstsq_grads_f64(A0, B0, G0)
    assert rel(Lam, Lr) < 1e-5
    assert rel(gA, gAr) < 1e-4
    assert rel(gB, gBr) < 1e-4


def test_adjoint_without_preconditioner(orc):
    A0, B0, G0 = problem(3000, 30, 1, 8)
    _, Lam, _, _, reps = gpu_grads(A0, B0, G0, precond=False)
    assert reps[0]["converged"] == 1
    _, Lr, _, _ = orc.lstsq_grads_f64(A0, B0, G0)
    assert rel(Lam, Lr) < 1e-5


def test_adjoint_zero_gradient_and_errors():
    A0, B0, _ = problem(500, 20, 1, 9)
    A = to_dense(A0, L.ROW_MAJOR)
    ws = tb.create_lsqr_workspace(None, (500, 20), NT.FP32)
    lam, rep = tb.lsqr_adjoint(A, torch.zeros(20, device="cuda"), ws)
    assert rep["converged"] == 1 and rep["iterations"] == 0
    assert torch.count_nonzero(lam).item() == 0
    ws2 = tb.create_lsqr_workspace(None, (500, 21), NT.FP32)
    with pytest.raises(tb.TomosError):
        tb.lsqr_adjoint(A, torch.zeros(20, device="cuda"), ws2)
    Ac = to_dense(A0, L.COL_MAJOR)
    with pytest.raises(tb.TomosError):
        tb.lsqr_adjoint_grad(Ac, cuda(B0), torch.zeros((20, 1), device="cuda"),
                             torch.zeros((20, 1), device="cuda"))


@pytest.mark.parametrize("m,n,K", [(200_000, 500, 8), (5000, 64, 1), (3000, 40, 3)])
def test_adjoint_batch(orc, m, n, K):
    """All K adjoints at once (two tensor-core products over A an iteration
    shared by the K recurrences) against the FP64 normal equations, and
    against the one-column CG solves."""
    A0, B0, G0 = problem(m, n, K, 11 + K)
    X, Lam, gA, gB, reps = gpu_grads(A0, B0, G0, batch=True)
    assert len(reps) == K and all(r["converged"] for r in reps), reps
    assert max(r["iterations"] for r in reps) < 60
    _, Lr, gAr, gBr = orc.lstsq_grads_f64(A0, B0, G0)
    assert rel(Lam, Lr) < 1e-5
    assert rel(gB, gBr) < 1e-4
    rows = np.random.default_rng(4).choice(m, min(m, 2000), replace=False)
    assert rel(gA[rows], gAr[rows]) < 1e-4
    _, Lam1, _, _, reps1 = gpu_grads(A0, B0, G0)
    assert rel(Lam, Lam1) < 1e-5
    assert all(abs(r["iterations"] - q["iterations"]) <= 2 for r, q in zip(reps, reps1))


@pytest.mark.parametrize("numeric", [NT.FP32_16, NT.FP32_BF16])
def test_adjoint_batch_packed_and_plain(orc, numeric):
    """Packed A (exact values through the accurate tensor-core tier), no
    preconditioner, and a zero column: that column stops at once while the
    others iterate."""
    A0, B0, G0 = problem(4000, 60, 3, 12)
    A0 = (A0 * 10.0 ** np.random.default_rng(7).uniform(-1, 1, 60)).astype(np.float32)
    G0[:, 1] = 0.0
    _, Lam, _, _, reps = gpu_grads(A0, B0, G0, numeric=numeric, batch=True)
    _, Lr, _, _ = orc.lstsq_grads_f64(A0, B0, G0)
    assert reps[1]["iterations"] == 0 and reps[1]["converged"] == 1
    assert np.count_nonzero(Lam[:, 1]) == 0
    assert rel(Lam[:, [0, 2]], Lr[:, [0, 2]]) < 1e-5
    _, Lam_np, _, _, reps_np = gpu_grads(A0, B0, G0, precond=False, batch=True)
    assert all(r["converged"] for r in reps_np)
    assert rel(Lam_np[:, [0, 2]], Lr[:, [0, 2]]) < 1e-5
