"""FP32 -> FP32_16 / FP32_BF16 pack kernels against the oracle and the
reference's golden vectors: bit-exact, every layout and leading dimension."""
import os

import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, planes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", [tb.Layout.ROW_MAJOR, tb.Layout.COL_MAJOR])
@pytest.mark.parametrize("pad", [0, 3])
def test_split_fp32_16_bit_exact(orc, layout, pad):
    g = np.load(os.path.join(GOLD, "pack_fp32_16.npz"))
    x = g["x"][: 97 * 251].reshape(97, 251)
    A = to_dense(x, layout, pad=pad)
    P = tb.Dense.create_strided(None, layout, tb.NumericType.FP32_16, A.size, A.ld)
    counts = torch.zeros(4, dtype=torch.int64, device="cuda")
    tb.split_fp32_16(A, P, counts=counts)
    wh, wr = planes(P)
    ewh, ewr = g["wh"][: x.size].reshape(x.shape), g["wr"][: x.size].reshape(x.shape)
    assert np.array_equal(wh, ewh) and np.array_equal(wr, ewr)
    # classes: control bit 0 = normal; steps field 14 = saturated
    ctrl = (ewh & 1) == 1
    sat = ctrl & (((ewh >> 10) & 0xF) == 14)
    over = ctrl & ~sat & (((ewh >> 14) & 1) == 1)
    under = ctrl & ~sat & ~over
    assert counts.tolist() == [int((~ctrl).sum()), int(under.sum()), int(over.sum()), int(sat.sum())]
    B = tb.Dense.create_strided(None, layout, tb.NumericType.FP32, A.size, A.ld + 1)
    tb.combine_fp32_16(P, B)
    got = B.view().cpu().numpy().view(np.uint32)
    assert np.array_equal(got, g["combine"][: x.size].reshape(x.shape).view(np.uint32))


@pytest.mark.parametrize("rounded", [False, True])
@pytest.mark.parametrize("layout", [tb.Layout.ROW_MAJOR, tb.Layout.COL_MAJOR])
def test_split_fp32_bf16_bit_exact(orc, rounded, layout):
    g = np.load(os.path.join(GOLD, "pack_fp32_bf16.npz"))
    x = g["x"][: 64 * 300].reshape(64, 300)
    A = to_dense(x, layout, pad=5)
    P = tb.pack(A, tb.NumericType.FP32_BF16, rounded=rounded)
    wh, wr = planes(P)
    k = int(rounded)
    assert np.array_equal(wh, g[f"wh{k}"][: x.size].reshape(x.shape))
    assert np.array_equal(wr, g[f"wr{k}"][: x.size].reshape(x.shape))
    B = tb.Dense.create_strided(None, layout, tb.NumericType.FP32, A.size)
    tb.combine_fp32_bf16(P, B)
    assert np.array_equal(B.view().cpu().numpy().view(np.uint32),
                          g[f"combine{k}"][: x.size].reshape(x.shape).view(np.uint32))


def test_split_random_bits_large(orc):
    rng = np.random.default_rng(1)
    x = rng.integers(0, 1 << 32, (1024, 4096), dtype=np.uint64).astype(np.uint32).view(np.float32)
    A = to_dense(x, tb.Layout.ROW_MAJOR)
    P = tb.pack(A, tb.NumericType.FP32_16)
    wh, wr = planes(P)
    ewh, ewr = orc.fp32_16_split(x)
    assert np.array_equal(wh.ravel(), ewh) and np.array_equal(wr.ravel(), ewr)


def test_empty_and_invalid():
    A = tb.Dense.create_strided(None, tb.Layout.COL_MAJOR, tb.NumericType.FP32, (0, 5))
    P = tb.Dense.create_strided(None, tb.Layout.COL_MAJOR, tb.NumericType.FP32_16, (0, 5))
    tb.split_fp32_16(A, P)  # no-op
    B = tb.Dense.create_strided(None, tb.Layout.ROW_MAJOR, tb.NumericType.FP32_16, (3, 5))
    C = tb.Dense.create_strided(None, tb.Layout.ROW_MAJOR, tb.NumericType.FP32, (3, 4))
    with pytest.raises(tb.TomosError):
        tb.split_fp32_16(C, B)
