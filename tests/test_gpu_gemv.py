"""tomos_gemv (every storage type, tier, layout, transpose, beta) against
an FP64 product of the values the tier reads (oracle decode), and against
the reference's own CPU FP32_16 tiers."""
import os

import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, decoded, cuda

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu

L = tb.Layout
NT = tb.NumericType
CASES = [(NT.FP32, tb.Tier.AUTO, False), (NT.FP32_16, tb.Tier.HALF, False),
         (NT.FP32_16, tb.Tier.ACCURATE, False), (NT.FP32_BF16, tb.Tier.HALF, False),
         (NT.FP32_BF16, tb.Tier.ACCURATE, False), (NT.FP32_BF16, tb.Tier.ACCURATE, True)]


def run(A, trans, tier, x, alpha, beta, y0):
    y = cuda(y0)
    tb.mv_apply(tb.Device.CUDA, trans, alpha, A, cuda(x), beta, y, tier=tier)
    return y.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("numeric,tier,rounded", CASES)
@pytest.mark.parametrize("layout", [L.ROW_MAJOR, L.COL_MAJOR])
@pytest.mark.parametrize("shape", [(1, 1), (7, 5), (33, 257), (1000, 37), (4097, 300)])
def test_gemv_vs_fp64(orc, numeric, tier, rounded, layout, shape):
    rng = np.random.default_rng(hash((shape, int(layout))) % 2 ** 32)
    m, n = shape
    A0 = (rng.standard_normal((m, n)) * np.where(rng.random((m, n)) < 0.05, 1e-6, 1.0)).astype(np.float32)
    A = to_dense(A0, layout, numeric, pad=2, rounded=rounded)
    Ad = decoded(orc, A, tier)
    acc64 = tier == tb.Tier.ACCURATE
    for trans in (tb.NO_TRANSPOSE, tb.TRANSPOSE):
        M = Ad if trans == tb.NO_TRANSPOSE else Ad.T
        x = rng.standard_normal(M.shape[1]).astype(np.float32)
        for beta in (0.0, 0.5):
            y0 = rng.standard_normal(M.shape[0]).astype(np.float32)
            if beta == 0.0:
                y0[:] = np.nan  # beta == 0 must not read y
            ref = 1.5 * (M @ x.astype(np.float64)) + (beta * y0.astype(np.float64) if beta else 0.0)
            scale = 1.5 * (np.abs(M) @ np.abs(x.astype(np.float64))) + abs(beta) * np.abs(np.nan_to_num(y0))
            got = run(A, trans, tier, x, 1.5, beta, y0)
            tol = (2e-6 if acc64 else 2e-5) * scale + 1e-30
            assert np.all(np.abs(got - ref) <= tol + 1e-7 * np.abs(ref)), (trans, beta)


def test_fp32_16_tiers_vs_reference_cpu(orc):
    """The reference's CPU tiers (fp32_16_kernels.cpp): our HALF tier is its
    'fast' tier (fp32_16_half_only decode, wide accumulation), ACCURATE its
    exact tier.  Reference tolerances (test_fp32_16.cpp:178-182) plus a
    tight FP32-rounding bound."""
    g = np.load(os.path.join(GOLD, "mv_fp32_16.npz"))
    A = to_dense(g["A"], L.COL_MAJOR, NT.FP32_16)
    for trans, x, key in ((tb.NO_TRANSPOSE, g["x"], "y"), (tb.TRANSPOSE, g["xt"], "yt")):
        half = run(A, trans, tb.Tier.HALF, x, 1.0, 0.0, np.zeros(len(g[key + "1"]), np.float32))
        acc = run(A, trans, tb.Tier.ACCURATE, x, 1.0, 0.0, np.zeros(len(g[key + "2"]), np.float32))
        fast_ref, acc_ref = g[key + "1"].astype(np.float64), g[key + "2"].astype(np.float64)
        assert np.all(np.abs(half - fast_ref) <= 0.05 * np.abs(fast_ref) + 0.05)
        assert np.all(np.abs(acc - acc_ref) <= 1e-3 * np.abs(acc_ref) + 1e-4)
        np.testing.assert_allclose(half, fast_ref, rtol=1e-5, atol=1e-4)
        np.testing.assert_allclose(acc, acc_ref, rtol=1e-6, atol=1e-5)


def test_unregistered_compute_type_raises():
    A = to_dense(np.ones((4, 4), np.float32), L.COL_MAJOR)
    y = cuda(np.zeros(4, np.float32))
    with pytest.raises(tb.TomosError):
        tb.mv_apply(tb.Device.CUDA, tb.NO_TRANSPOSE, 1.0, A, cuda(np.ones(4)), 0.0, y,
                    compute_type=NT.FP16)
