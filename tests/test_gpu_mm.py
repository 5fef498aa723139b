"""mm_apply on the tcgen05 tensor cores (tomos_mm) against FP64 products of
the operand values each tier reads: FP32, native FP16 and packed A, every
transpose and layout of A, B and C, ragged sizes (M, N, K not multiples of
the 128 x BN x K-stage tiles), beta = 0 (C never read) and beta != 0, K = 0.

Tolerances, per entry, relative to S = sum_l |op(A)_il| |op(B)_lj|:
  HALF_OPERANDS  the exact product of the 16-bit operands (B rounded to
                 fp16 / bf16 first) to 1e-5 S (FP32 accumulation);
  HALF           A's 16-bit values times B to 1e-5 S (B split in two TF32
                 parts, ~2^-22);
  ACCURATE / FP32  the exact values to 1e-5 S (A and B split, ~2^-21)."""
import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, decoded

pytestmark = pytest.mark.gpu
NT = tb.NumericType
L = tb.Layout
T = tb.TransposeType


def dense_f32(M, layout, pad=0):
    return to_dense(np.ascontiguousarray(M, np.float32), layout, pad=pad)


def values(D):
    return D.view().double().cpu().numpy()


def check(orc, A, A0, tier, ta, tb_, shape_b, layouts, beta, rng, bf16_ops=False, bpad=None):
    """One product against FP64; returns the max error / bound ratio."""
    lb, lc = layouts
    if A.numeric == NT.FP32:
        Av = A0.astype(np.float64)
    elif A.numeric == NT.FP16:
        Av = A.view().double().cpu().numpy()
    else:
        Av = decoded(orc, A, tb.Tier.HALF if tier in (tb.Tier.HALF, tb.Tier.HALF_OPERANDS) else tier)
    opA = Av.T if ta == T.TRANSPOSE else Av
    M, K = opA.shape
    B0 = rng.standard_normal(shape_b).astype(np.float32)
    if bpad is None:
        bpad = 3 if beta else 0  # strided and aligned B
    B = dense_f32(B0, lb, pad=bpad)
    Bv = B0.astype(np.float64)
    if tier == tb.Tier.HALF_OPERANDS:
        Bv = (torch.from_numpy(B0).to(torch.bfloat16 if bf16_ops else torch.float16)).double().numpy()
    opB = Bv.T if tb_ == T.TRANSPOSE else Bv
    assert opB.shape[0] == K
    N = opB.shape[1]
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    Cd = dense_f32(C0 if beta else np.full((M, N), np.nan, np.float32), lc, pad=1)
    tb.mm_apply(tb.Device.CUDA, ta, tb_, 1.25, A, B, beta, Cd, tier=tier)
    got = values(Cd)
    ref = 1.25 * (opA @ opB) + (beta * C0.astype(np.float64) if beta else 0.0)
    S = 1.25 * (np.abs(opA) @ np.abs(opB)) + (abs(beta) * np.abs(C0) if beta else 0.0)
    err = np.abs(got - ref)
    bound = 1e-5 * S + 1e-30
    assert np.all(np.isfinite(got))
    assert np.all(err <= bound), float((err / bound).max())
    return float((err / bound).max())


SHAPES = [(300, 17, 129), (1000, 130, 500), (128, 16, 64), (257, 1, 33), (77, 200, 1000), (5, 3, 2)]


@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("ta", [T.NO_TRANSPOSE, T.TRANSPOSE])
@pytest.mark.parametrize("tb_", [T.NO_TRANSPOSE, T.TRANSPOSE])
def test_mm_fp32(M, N, K, ta, tb_):
    """FP32 A (the accurate TF32x3 products), column- and row-major."""
    rng = np.random.default_rng(M * 7 + N + K)
    A0 = (rng.standard_normal((M, K) if ta == T.NO_TRANSPOSE else (K, M)) *
          10.0 ** rng.uniform(-2, 2, (1, K if ta == T.NO_TRANSPOSE else M))).astype(np.float32)
    for la, lb, lc in ((L.COL_MAJOR, L.COL_MAJOR, L.COL_MAJOR), (L.ROW_MAJOR, L.ROW_MAJOR, L.ROW_MAJOR),
                       (L.ROW_MAJOR, L.COL_MAJOR, L.ROW_MAJOR)):
        A = dense_f32(A0, la, pad=2)
        shape_b = (K, N) if tb_ == T.NO_TRANSPOSE else (N, K)
        for beta in (0.0, -0.5):
            check(None, A, A0, tb.Tier.AUTO, ta, tb_, shape_b, (lb, lc), beta, rng)


@pytest.mark.parametrize("numeric", [NT.FP32_16, NT.FP32_BF16])
@pytest.mark.parametrize("tier", [tb.Tier.ACCURATE, tb.Tier.HALF, tb.Tier.HALF_OPERANDS])
@pytest.mark.parametrize("layout", [L.COL_MAJOR, L.ROW_MAJOR])
@pytest.mark.parametrize("ta", [T.NO_TRANSPOSE, T.TRANSPOSE])
def test_mm_packed(orc, numeric, tier, layout, ta):
    """Packed A at each tier (values outside fp16 range included for the
    exact tiers' control words)."""
    M, N, K = 600, 70, 333
    rng = np.random.default_rng(int(numeric) * 10 + int(tier))
    shape_a = (M, K) if ta == T.NO_TRANSPOSE else (K, M)
    A0 = (rng.standard_normal(shape_a) * np.where(rng.random(shape_a) < 0.02, 1e-6, 1.0)).astype(np.float32)
    A = to_dense(A0, layout, numeric, pad=8)
    for tb_ in (T.NO_TRANSPOSE, T.TRANSPOSE):
        shape_b = (K, N) if tb_ == T.NO_TRANSPOSE else (N, K)
        check(orc, A, A0, tier, ta, tb_, shape_b, (L.COL_MAJOR, L.COL_MAJOR), 0.5, rng,
              bf16_ops=numeric == NT.FP32_BF16)


@pytest.mark.parametrize("tier", [tb.Tier.AUTO, tb.Tier.HALF_OPERANDS])
def test_mm_fp16(tier):
    rng = np.random.default_rng(9)
    A0 = rng.standard_normal((513, 250)).astype(np.float32)
    A = to_dense(A0, L.ROW_MAJOR, NT.FP16, pad=6)
    check(None, A, A0, tier, T.NO_TRANSPOSE, T.NO_TRANSPOSE, (250, 40), (L.COL_MAJOR, L.COL_MAJOR), 0.0, rng)


def test_mm_reference_routing_and_errors(orc):
    """mm_apply's default for packed A is the accurate tier (the reference's
    mm_apply routing), use_workspace gives the same values; K = 0 scales C;
    wrong shapes and FP32 A at HALF_OPERANDS are refused."""
    rng = np.random.default_rng(3)
    A0 = rng.standard_normal((200, 64)).astype(np.float32)
    A = to_dense(A0, L.COL_MAJOR, NT.FP32_16)
    B = dense_f32(rng.standard_normal((64, 20)), L.COL_MAJOR)
    C1 = dense_f32(np.zeros((200, 20)), L.COL_MAJOR)
    C2 = dense_f32(np.zeros((200, 20)), L.COL_MAJOR)
    C3 = dense_f32(np.zeros((200, 20)), L.COL_MAJOR)
    tb.mm_apply(tb.Device.CUDA, T.NO_TRANSPOSE, T.NO_TRANSPOSE, 1.0, A, B, 0.0, C1)
    tb.mm_apply(tb.Device.CUDA, T.NO_TRANSPOSE, T.NO_TRANSPOSE, 1.0, A, B, 0.0, C2, use_workspace=True)
    tb.mm_apply_fp32_16_ext(tb.Device.CUDA, T.NO_TRANSPOSE, T.NO_TRANSPOSE, 1.0, A, B, 0.0, C3)
    assert torch.equal(C1.view(), C2.view()) and torch.equal(C1.view(), C3.view())
    # K = 0
    Z = dense_f32(np.zeros((200, 0)), L.COL_MAJOR)
    Bz = dense_f32(np.zeros((0, 20)), L.COL_MAJOR, pad=1)
    C0 = rng.standard_normal((200, 20)).astype(np.float32)
    Cz = dense_f32(C0, L.COL_MAJOR)
    tb.mm_apply(tb.Device.CUDA, T.NO_TRANSPOSE, T.NO_TRANSPOSE, 1.0, Z, Bz, 2.0, Cz)
    np.testing.assert_array_equal(Cz.view().cpu().numpy(), (2.0 * C0.astype(np.float64)).astype(np.float32))
    with pytest.raises(tb.TomosError):
        tb.mm_apply(tb.Device.CUDA, T.TRANSPOSE, T.NO_TRANSPOSE, 1.0, A, B, 0.0, C1)
    A32 = dense_f32(A0, L.COL_MAJOR)
    with pytest.raises(tb.TomosError):
        tb.mm_apply(tb.Device.CUDA, T.NO_TRANSPOSE, T.NO_TRANSPOSE, 1.0, A32, B, 0.0, C1,
                    tier=tb.Tier.HALF_OPERANDS)


def aligned_pad(inner, mult=8):
    return (-inner) % mult


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP16, tb.Tier.AUTO),
                                          (NT.FP16, tb.Tier.HALF_OPERANDS), (NT.FP32_16, tb.Tier.ACCURATE),
                                          (NT.FP32_16, tb.Tier.HALF), (NT.FP32_16, tb.Tier.HALF_OPERANDS),
                                          (NT.FP32_BF16, tb.Tier.ACCURATE), (NT.FP32_BF16, tb.Tier.HALF_OPERANDS)])
@pytest.mark.parametrize("la", [L.COL_MAJOR, L.ROW_MAJOR])
@pytest.mark.parametrize("lb", [L.COL_MAJOR, L.ROW_MAJOR])
@pytest.mark.parametrize("M,N,K", [(300, 50, 200), (256, 128, 256), (130, 16, 1000)])
def test_mm_tma_pipeline(orc, numeric, tier, la, lb, M, N, K):
    """Operands whose lines are 16-byte aligned take the TMA-fed pipeline
    (tensor copies with zero fill at the ragged edges, converter warps)."""
    rng = np.random.default_rng(M + N + K + int(numeric) * 3 + int(tier))
    A0 = (rng.standard_normal((M, K)) * np.where(rng.random((M, K)) < 0.02, 1e-6, 1.0)).astype(np.float32)
    pad = aligned_pad(K if la == L.ROW_MAJOR else M)
    A = to_dense(A0, la, numeric, pad=pad)
    bpad = aligned_pad(N if lb == L.ROW_MAJOR else K)
    for beta in (0.0, 0.5):
        check(orc, A, A0, tier, T.NO_TRANSPOSE, T.NO_TRANSPOSE, (K, N), (lb, L.COL_MAJOR), beta, rng,
              bf16_ops=numeric == NT.FP32_BF16, bpad=bpad)


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.ACCURATE),
                                          (NT.FP32_16, tb.Tier.HALF)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_mm_split_k(orc, numeric, tier, beta):
    """A^T Q with a tall K (the transposed multi-right-hand-side product):
    few output tiles, so K is split over CTAs and the FP32 partials are summed
    in FP64 in split order; without scratch (tomos_mm) the same product runs
    unsplit."""
    import ctypes
    from tomos_b200 import _capi as C
    rng = np.random.default_rng(int(numeric) + int(tier) * 7)
    m, n, k = 100_000, 300, 8
    A0 = (rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-1, 1, n)).astype(np.float32)
    A = to_dense(A0, L.ROW_MAJOR, numeric)
    da, db = A.desc(), None
    Q = dense_f32(rng.standard_normal((m, k)), L.COL_MAJOR)
    db = Q.desc()
    nb = C.lib().tomos_mm_scratch_bytes(int(T.TRANSPOSE), int(T.NO_TRANSPOSE), ctypes.byref(da), int(tier),
                                        ctypes.byref(db))
    assert nb > 0  # the split is taken
    check(orc, A, A0, tier, T.TRANSPOSE, T.NO_TRANSPOSE, (m, k), (L.COL_MAJOR, L.COL_MAJOR), beta, rng)
    # unsplit (no scratch) against split: equal up to summation order
    C0 = rng.standard_normal((n, k)).astype(np.float32)
    Cs, Cu = dense_f32(C0, L.COL_MAJOR), dense_f32(C0, L.COL_MAJOR)
    tb.mm_apply(tb.Device.CUDA, T.TRANSPOSE, T.NO_TRANSPOSE, 1.0, A, Q, beta, Cs, tier=tier)
    dc = Cu.desc()
    C.check(C.lib().tomos_mm(int(T.TRANSPOSE), int(T.NO_TRANSPOSE), 1.0, ctypes.byref(da), int(tier),
                             ctypes.byref(db), float(beta), ctypes.byref(dc), None), "mm")
    a, b = values(Cs), values(Cu)
    # both within the product bound; the unsplit one sums all m rows of a
    # column in FP32 in one accumulator, so it sits further from FP64
    Av = A0.astype(np.float64) if numeric == NT.FP32 else decoded(
        orc, A, tb.Tier.HALF if tier == tb.Tier.HALF else tier)
    Qv = Q.view().double().cpu().numpy()
    ref = Av.T @ Qv + beta * C0.astype(np.float64)
    S = np.abs(Av.T) @ np.abs(Qv) + abs(beta) * np.abs(C0)
    assert np.all(np.abs(a - ref) <= 1e-5 * S)
    # unsplit: 100,000 terms in one FP32 accumulator (tomos_mm's documented
    # summation error grows with K)
    assert np.all(np.abs(b - ref) <= 1e-4 * S)
    assert np.abs(a - ref).max() <= np.abs(b - ref).max()
