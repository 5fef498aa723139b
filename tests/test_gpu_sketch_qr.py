"""CountSketch (bit-exact hash, deterministic FP64 owner sums) and the FP64
Householder sketch QR against the oracle and the reference's outputs."""
import os

import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, decoded

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu
L = tb.Layout
NT = tb.NumericType


@pytest.mark.parametrize("s", [1, 64, 4000])
def test_hash_bit_exact(orc, s):
    m = 100_003
    b, g = tb.countsketch_hash(m, s)
    eb, eg = orc.countsketch_hash(m, s)
    assert np.array_equal(b.cpu().numpy(), eb) and np.array_equal(g.cpu().numpy(), eg)
    gold = np.load(os.path.join(GOLD, "countsketch.npz"))
    if s in (64, 4000):
        assert np.array_equal(b[:4096].cpu().numpy(), gold[f"bucket_s{s}"])


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.HALF),
                                          (NT.FP32_16, tb.Tier.ACCURATE), (NT.FP32_BF16, tb.Tier.HALF)])
@pytest.mark.parametrize("layout", [L.ROW_MAJOR, L.COL_MAJOR])
def test_apply_vs_oracle(orc, numeric, tier, layout):
    rng = np.random.default_rng(4)
    m, n, s = 5003, 301, 97
    A0 = (rng.standard_normal((m, n)) * np.logspace(-2, 2, n)).astype(np.float32)
    A = to_dense(A0, layout, numeric, pad=3)
    SA, fro2, colsq = tb.apply_count_sketch(A, s, tier=tier, with_colsq=True)
    Ad = decoded(orc, A, tier).astype(np.float32)
    got = SA.view().cpu().numpy()
    if layout == L.ROW_MAJOR:
        # one owner per bucket, rows in increasing order, FP32: the
        # reference's float path (countsketch_apply_impl<float>) bit for bit
        assert np.array_equal(got, orc.countsketch_apply(Ad, s, row_major=True, acc="f32"))
        tol = 1e-6  # column sums of squares: FP32 per bucket, FP64 across
    else:
        ref = orc.countsketch_apply(Ad, s, row_major=True)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        tol = 1e-12
    np.testing.assert_allclose(colsq.cpu().numpy(), (Ad.astype(np.float64) ** 2).sum(0), rtol=tol)
    np.testing.assert_allclose(fro2.item(), (Ad.astype(np.float64) ** 2).sum(), rtol=tol)


@pytest.mark.parametrize("n,pad,s", [(301, 3, 113), (1000, 0, 113), (1100, 4, 5)])
def test_apply_stage(orc, n, pad, s):
    """The staging sketch: SA bit for bit the HALF-tier sketch, and the plane
    it writes holds fp32_16_half_only of every wh word (values outside the
    fp16 range included: the columns span 1e-9 .. 1e9).  s = 5 gives
    buckets of ~1400 rows (past the in-shared-memory row list and sort)
    and n = 1100 two column panels."""
    rng = np.random.default_rng(n)
    m = 7001
    A0 = (rng.standard_normal((m, n)) * np.logspace(-9, 9, n)).astype(np.float32)
    A = to_dense(A0, L.ROW_MAJOR, NT.FP32_16, pad=pad)
    SA0, f0, c0 = tb.apply_count_sketch(A, s, tier=tb.Tier.HALF, with_colsq=True)
    SA, f1, c1, plane = tb.apply_count_sketch(A, s, tier=tb.Tier.HALF, with_colsq=True, stage=True)
    # bitwise (columns past the fp16 range decode to +-Inf, so sums hold NaN)
    assert torch.equal(SA.storage.view(torch.int64), SA0.storage.view(torch.int64))
    assert torch.equal(f0.view(torch.int64), f1.view(torch.int64))
    assert torch.equal(c0.view(torch.int64), c1.view(torch.int64))
    got = plane[:, :n].view(torch.float16).float().cpu().numpy()
    want = decoded(orc, A, tb.Tier.HALF).astype(np.float32)
    assert np.array_equal(got, want)
    ref = orc.countsketch_apply(want, s, row_major=True, acc="f32")
    assert np.array_equal(SA.view().cpu().numpy(), ref, equal_nan=True)
    with pytest.raises(tb.TomosError):
        tb.apply_count_sketch(to_dense(A0, L.COL_MAJOR, NT.FP32_16), s, tier=tb.Tier.HALF, stage=True)


def test_apply_reference_golden(orc):
    g = np.load(os.path.join(GOLD, "countsketch.npz"))
    A = to_dense(g["X"], L.COL_MAJOR)
    SA, _ = tb.apply_count_sketch(A, 64)
    np.testing.assert_allclose(SA.view().cpu().numpy(), g["Y"], rtol=1e-5, atol=1e-5)


def test_apply_deterministic():
    rng = np.random.default_rng(9)
    A = to_dense(rng.standard_normal((20000, 64)).astype(np.float32), L.COL_MAJOR)
    a, _ = tb.apply_count_sketch(A, 128)
    b, _ = tb.apply_count_sketch(A, 128)
    assert torch.equal(a.storage, b.storage)


def qr_on_gpu(SA):
    D = tb.Dense.create_strided(None, L.COL_MAJOR, NT.FP64, SA.shape)
    D.view()[...] = torch.from_numpy(np.asarray(SA, np.float64)).cuda()
    R = torch.zeros(SA.shape[1] * SA.shape[1], dtype=torch.float64, device="cuda")
    Rinv = tb.generate_sketch_qr_precond(D, R_out=R)
    return Rinv.view().cpu().numpy(), R.view(SA.shape[1], SA.shape[1]).t().cpu().numpy()


def test_qr_reference_golden(orc):
    g = np.load(os.path.join(GOLD, "sketch_qr.npz"))
    Rinv, R = qr_on_gpu(g["SA"])
    np.testing.assert_allclose(Rinv, g["Rinv"], rtol=1e-9, atol=1e-12 * np.abs(g["Rinv"]).max())
    Ro, _ = orc.householder_qr(g["SA"])
    np.testing.assert_allclose(R, Ro, rtol=1e-10, atol=1e-10 * np.abs(Ro).max())


def test_qr_known_4x2():
    A = np.array([[1.0, 2.0], [3.0, 4.0], [5.0, 6.0], [7.0, 8.0]])
    Rinv, _ = qr_on_gpu(A)
    assert np.allclose(np.tril(Rinv, -1), 0)
    np.testing.assert_allclose(Rinv.T @ A.T @ A @ Rinv, np.eye(2), atol=1e-10)


@pytest.mark.parametrize("k,n", [(64, 64), (97, 33), (700, 100), (4000, 1000), (4001, 1777), (3000, 1537)])
def test_qr_property_and_vs_lapack(k, n):
    """From 1536 columns the QR is blocked (256-column blocks, the rest of
    the matrix updated by FP64 tensor-core products); 1537 leaves a last
    block of one column, 1777 a ragged one."""
    rng = np.random.default_rng(k + n)
    SA = rng.standard_normal((k, n)) * np.logspace(0, 4, n)
    Rinv, R = qr_on_gpu(SA)
    Rl = np.linalg.qr(SA, mode="r")
    # same Householder sign convention as LAPACK: R agrees entry-wise
    np.testing.assert_allclose(R, Rl, rtol=1e-8, atol=1e-9 * np.abs(Rl).max())
    Q = SA @ Rinv
    np.testing.assert_allclose(Q.T @ Q, np.eye(n), atol=1e-8)


@pytest.mark.parametrize("k,n", [(20000, 96), (9000, 300)])
def test_qr_tall_sketch(k, n):
    """Sketches taller than one CTA's shared memory (the panel passes read
    their rows from global memory)."""
    rng = np.random.default_rng(k)
    SA = rng.standard_normal((k, n)) * np.logspace(0, 3, n)
    Rinv, R = qr_on_gpu(SA)
    Rl = np.linalg.qr(SA, mode="r")
    np.testing.assert_allclose(R, Rl, rtol=1e-8, atol=1e-9 * np.abs(Rl).max())
    Q = SA @ Rinv
    np.testing.assert_allclose(Q.T @ Q, np.eye(n), atol=1e-8)


def test_qr_ill_conditioned_panel():
    """Two nearly equal columns inside one 32-column panel (cond ~ 1e10):
    Cholesky QR breaks down there and that panel takes Householder column
    steps.  R is backward stable (R^T R = SA^T SA to rounding), agrees with
    LAPACK's on the columns before the near-duplicate, and keeps its
    diagonal signs; past it two correct Householder QRs may differ by
    eps * cond."""
    rng = np.random.default_rng(5)
    SA = rng.standard_normal((600, 80))
    SA[:, 41] = SA[:, 37] * (1.0 + 1e-10) + 1e-11 * rng.standard_normal(600)
    Rinv, R = qr_on_gpu(SA)
    Rl = np.linalg.qr(SA, mode="r")
    np.testing.assert_allclose(R[:, :41], Rl[:, :41], rtol=1e-8, atol=1e-9 * np.abs(Rl).max())
    assert np.array_equal(np.sign(np.diag(R))[:41], np.sign(np.diag(Rl))[:41])
    G = SA.T @ SA
    assert np.abs(R.T @ R - G).max() <= 1e-12 * np.abs(G).max()
    assert np.allclose(np.tril(Rinv, -1), 0) and np.all(np.isfinite(Rinv))


@pytest.mark.parametrize("k,n", [(3000, 1600), (1700, 1700)])
def test_qr_blocked_ill_conditioned_panel_and_square(k, n):
    """The blocked QR (256-column blocks) with a near-duplicate column pair
    inside its third block (one 32-column panel), which takes the Householder
    column steps
    and hands its T to the block's merge; square at 1700.  R is backward
    stable and keeps LAPACK's diagonal signs before the near-duplicate."""
    rng = np.random.default_rng(k + n)
    SA = rng.standard_normal((k, n)) * np.logspace(0, 2, n)
    # columns 705 and 709 share the 32-column panel at 704
    SA[:, 709] = SA[:, 705] * (1.0 + 1e-10) + 1e-11 * np.abs(SA[:, 705]).max() * rng.standard_normal(k)
    Rinv, R = qr_on_gpu(SA)
    Rl = np.linalg.qr(SA, mode="r")
    np.testing.assert_allclose(R[:, :709], Rl[:, :709], rtol=1e-8, atol=1e-9 * np.abs(Rl).max())
    assert np.array_equal(np.sign(np.diag(R))[:709], np.sign(np.diag(Rl))[:709])
    G = SA.T @ SA
    assert np.abs(R.T @ R - G).max() <= 1e-12 * np.abs(G).max()
    assert np.allclose(np.tril(Rinv, -1), 0) and np.all(np.isfinite(Rinv))


@pytest.mark.timeout(300)
@pytest.mark.parametrize("wide", ["0", "3"])
def test_qr_panel_and_wide_paths(wide):
    """Up to 2048 columns a well-conditioned sketch is factored at once
    (Gram on the tensor cores, blocked Cholesky, Householder reconstruction
    of the signs; TOMOS_QR_WIDE=3 requires that path from one column, so a
    fallback would fail the test); TOMOS_QR_WIDE=0 keeps the 32-column panel
    path.  Both give LAPACK's R.  Run in a child process, as the switch is
    read once per process."""
    import subprocess
    import sys
    code = (
        "import numpy as np, sys\n"
        "sys.path.insert(0, %r)\n"
        "from test_gpu_sketch_qr import qr_on_gpu\n"
        "for k, n in ((4000, 1000), (300, 37), (64, 64), (8000, 2000), (5000, 1537)):\n"
        "    rng = np.random.default_rng(k)\n"
        "    SA = rng.standard_normal((k, n)) * np.logspace(0, 4, n)\n"
        "    Rinv, R = qr_on_gpu(SA)\n"
        "    Rl = np.linalg.qr(SA, mode='r')\n"
        "    np.testing.assert_allclose(R, Rl, rtol=1e-8, atol=1e-9 * np.abs(Rl).max())\n"
        "    Q = SA @ Rinv\n"
        "    np.testing.assert_allclose(Q.T @ Q, np.eye(n), atol=1e-8)\n"
        "print('ok')\n" % os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, TOMOS_QR_WIDE=wide)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=280)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-3000:]


def test_qr_rejects_wide_and_singular():
    with pytest.raises(tb.TomosError):
        qr_on_gpu(np.ones((3, 5)))
    with pytest.raises(tb.TomosError):
        qr_on_gpu(np.zeros((10, 4)))


def test_qr_any_signs():
    """TOMOS_QR_ANY_SIGNS: R equals LAPACK's up to the signs of its rows, so
    R^{-1} = R_lapack^{-1} S; the preconditioned LSQR solve (sketch_lsqr
    uses it) reaches the same solution."""
    for k, n in ((4000, 1000), (300, 64)):
        rng = np.random.default_rng(k + 1)
        SA0 = rng.standard_normal((k, n)) * np.logspace(0, 4, n)
        Rinv_l, R_l = qr_on_gpu(SA0)
        D = tb.Dense.create_strided(None, tb.Layout.COL_MAJOR, tb.NumericType.FP64, (k, n))
        D.view()[...] = torch.from_numpy(SA0).cuda()
        Rout = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        Rinv = tb.generate_sketch_qr_precond(D, R_out=Rout, any_signs=True).view().cpu().numpy()
        R = Rout.t().cpu().numpy()  # column-major n x n
        S = np.sign(np.diag(R)) * np.sign(np.diag(R_l))
        np.testing.assert_allclose(R, S[:, None] * R_l, rtol=1e-8, atol=1e-9 * np.abs(R_l).max())
        np.testing.assert_allclose(Rinv, Rinv_l * S[None, :], rtol=1e-8, atol=1e-9 * np.abs(Rinv_l).max())
        assert np.all(np.diag(R) > 0)
