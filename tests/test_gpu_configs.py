"""The full-size parity configurations besides the benchmark's own:

* 4,000,000 x 2000 in FP32_BF16 storage (32 GB packed): bf16 iterations with
  FP32 accumulation and exact restarts as the residual refinement (at most
  three after the first cycle) to a column-scaled backward error of 1e-6,
  checked in FP64 on the device; and the FP64 host oracle on the first
  200,000 rows of the same counter-based matrix, solved by the same pipeline;
* sparse CSR 2,000,000 x 5000, 20 distinct columns a row, FP32_16 values,
  CountSketch s = 20000 + sketch QR, tol 1e-6, checked with an independent
  FP64 residual (torch sparse) on the device.
"""
import numpy as np
import pytest
import torch

import tomos_b200 as tb
from tomos_b200 import _capi as C
from tomos_b200 import problems

pytestmark = pytest.mark.gpu
NT = tb.NumericType
L = tb.Layout


def packed_ctr(m, n, seed, block=32768):
    """A (FP32_BF16, row-major, packed block by block from the counter-based
    generator) and b."""
    P = tb.Dense.create_strided(None, L.ROW_MAJOR, NT.FP32_BF16, (m, n))
    b = torch.empty(m, dtype=torch.float32, device="cuda")
    params = problems.ctr_scaled_params(n, seed)
    base = P.storage.data_ptr()
    plane = P.ld * m * 2  # bytes of the wh plane
    for r0 in range(0, m, block):
        r1 = min(m, r0 + block)
        Ab, bb = problems.ctr_scaled_rows(r0, r1, n, seed, params=params)
        b[r0:r1] = bb
        off = r0 * P.ld * 2
        C.check(C.lib().tomos_pack_fp32_bf16(Ab.data_ptr(), int(L.ROW_MAJOR), r1 - r0, n, n,
                                             base + off, base + plane + off, P.ld, 0, None),
                "pack block")
        del Ab
    return P, b, params


def solve(A, b, s, restarts, inner_rtol, sketch_tier=tb.Tier.AUTO):
    m, n = A.size
    SA, _, colsq = tb.apply_count_sketch(A, s, tier=sketch_tier, with_colsq=True)
    Rinv = tb.generate_sketch_qr_precond(SA)
    del SA
    d, an = tb.column_scale(colsq)
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32, NT.FP64)
    tb.add_precond(Rinv, ws)
    x = torch.zeros(n, device="cuda")
    rep = tb.lsqr_solve(None, A, b, x, ws, 1e-6, 400, 0.0, restarts=restarts,
                        stop_rule=tb.StopRule.BACKWARD, inner_rtol=inner_rtol, anorm_fro=an,
                        col_scale=d)
    return x, rep, d


def test_config3_bf16_refinement_4e6x2000(orc):
    m, n, s, seed = 4_000_000, 2000, 8000, 3
    A, b, _ = packed_ctr(m, n, seed)
    x, rep, d = solve(A, b, s, restarts=4, inner_rtol=1e-2, sketch_tier=tb.Tier.HALF)
    assert rep["converged"] == 1, rep
    assert rep["restarts_used"] <= 4  # the first cycle + at most three refinements
    ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32)
    eta = tb.backward_error(A, b, x, ws, col_scale=d)["backward_error"]  # FP64, exact values
    assert eta <= 1e-6, eta
    del A
    torch.cuda.empty_cache()

    # the FP64 oracle on the first 200,000 rows of the same matrix
    ms = 200_000
    As, bs, _ = packed_ctr(ms, n, seed)
    xs, reps, ds = solve(As, bs, s, restarts=4, inner_rtol=1e-2, sketch_tier=tb.Tier.HALF)
    assert reps["converged"] == 1
    # the same rows again from the generator (entrywise functions of
    # (seed, row, column)), to the host in FP64
    A64 = np.empty((ms, n), np.float64)
    params = problems.ctr_scaled_params(n, seed)
    for r0 in range(0, ms, 32768):
        r1 = min(ms, r0 + 32768)
        A64[r0:r1] = problems.ctr_scaled_rows(r0, r1, n, seed, params=params)[0].double().cpu().numpy()
    b64 = bs.cpu().numpy().astype(np.float64)
    xo = orc.lstsq_f64(A64, b64)
    xg = xs.cpu().numpy().astype(np.float64)
    dn = np.linalg.norm(A64, axis=0)
    assert np.linalg.norm(dn * (xg - xo)) / np.linalg.norm(dn * xo) < 1e-4
    assert orc.backward_error_scaled(A64, b64, xg) <= 1.05e-6


def test_config4_csr_fp32_16_2e6x5000():
    m, n, k, s = 2_000_000, 5000, 20, 20000
    rp, ci, v, xt, b = problems.csr_scaled(m, n, k, seed=4)
    t = tb.Dense.from_tensor(v[None, :], L.ROW_MAJOR)
    P = tb.pack(t, NT.FP32_16)
    A = tb.Csr(NT.FP32_16, (m, n), rp, ci, P.storage)
    x, rep, d = solve(A, b, s, restarts=6, inner_rtol=1e-3)
    assert rep["converged"] == 1, rep
    # independent FP64 eta_D (FP32_16 values are the FP32 values exactly)
    rows = torch.repeat_interleave(torch.arange(m, device="cuda"), k)
    S = torch.sparse_coo_tensor(torch.stack([rows, ci.long()]), v.double(), (m, n)).coalesce()
    xd = x.double()
    r = b.double() - torch.sparse.mm(S, xd[:, None])[:, 0]
    atr = torch.sparse.mm(S.t(), r[:, None])[:, 0]
    an = torch.sqrt(((v.double() ** 2) / d[ci.long()] ** 2).sum())
    e1 = r.norm() / (an * (d * xd).norm() + b.double().norm())
    e2 = (atr / d).norm() / (an * r.norm())
    eta = float(torch.minimum(e1, e2))
    assert eta <= 1.05e-6, (eta, rep)
