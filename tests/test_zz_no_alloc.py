"""tomos_gemv_no_alloc: the GEMV entry that takes no scratch and allocates
nothing (its scratch is a fixed 16 MiB buffer inside the library).  Called
through the C ABI twice in a row and compared with tomos_gemv on the same
inputs.  Collected last so it also runs after every other test has used the
device; it passes alone in a fresh process too."""
import ctypes

import numpy as np
import pytest
import torch

import tomos_b200 as tb
from tomos_b200 import _capi as C

L = tb.Layout
NT = tb.NumericType
LIMIT = 16 << 20


def _gemv(A, trans, tier, x, alpha, beta, y0):
    d = A.desc()
    nb = C.lib().tomos_gemv_scratch_bytes(ctypes.byref(d), int(trans))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    y = y0.clone()
    C.check(C.lib().tomos_gemv(int(trans), alpha, ctypes.byref(d), int(tier), x.data_ptr(), beta,
                               y.data_ptr(), scratch.data_ptr(), nb, None), "tomos_gemv")
    return y


def _no_alloc(A, trans, tier, x, alpha, beta, y0):
    d = A.desc()
    y = y0.clone()
    C.check(C.lib().tomos_gemv_no_alloc(int(trans), alpha, ctypes.byref(d), int(tier),
                                        x.data_ptr(), beta, y.data_ptr(), None),
            "tomos_gemv_no_alloc")
    return y


@pytest.mark.gpu
@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.HALF),
                                          (NT.FP32_16, tb.Tier.ACCURATE)])
@pytest.mark.parametrize("layout,shape", [(L.ROW_MAJOR, (4097, 300)), (L.COL_MAJOR, (300, 4097)),
                                          (L.ROW_MAJOR, (200000, 1000))])
def test_no_alloc_matches_gemv(numeric, tier, layout, shape):
    rng = np.random.default_rng(7)
    m, n = shape
    A0 = torch.from_numpy(rng.standard_normal((m, n)).astype(np.float32)).cuda()
    Af = tb.Dense.create_strided(None, layout, NT.FP32, (m, n))
    Af.view()[...] = A0
    A = Af if numeric == NT.FP32 else tb.pack(Af, numeric)
    for trans in (tb.NO_TRANSPOSE, tb.TRANSPOSE):
        xl, yl = (n, m) if trans == tb.NO_TRANSPOSE else (m, n)
        x = torch.from_numpy(rng.standard_normal(xl).astype(np.float32)).cuda()
        y0 = torch.from_numpy(rng.standard_normal(yl).astype(np.float32)).cuda()
        ref = _gemv(A, trans, tier, x, 1.5, 0.5, y0).double()
        M = A0.double() if trans == tb.NO_TRANSPOSE else A0.double().T
        scale = 1.5 * (M.abs() @ x.double().abs()) + 0.5 * y0.double().abs()
        tol = 2e-5 * scale + 1e-7 * ref.abs() + 1e-30
        exact = None
        if numeric == NT.FP32 and shape == (4097, 300):
            # and against the FP64 product on the host for one small case
            Mh = M.cpu().numpy()
            exact = torch.from_numpy(1.5 * (Mh @ x.double().cpu().numpy()) +
                                     0.5 * y0.double().cpu().numpy()).cuda()
        for _ in range(2):  # two calls in a row reuse the same fixed buffer
            got = _no_alloc(A, trans, tier, x, 1.5, 0.5, y0).double()
            torch.cuda.synchronize()
            assert bool(((got - ref).abs() <= tol).all()), (trans, float((got - ref).abs().max()))
            if exact is not None:
                assert bool(((got - exact).abs() <= tol).all()), (trans, float((got - exact).abs().max()))


def test_no_alloc_rejects_products_beyond_the_fixed_buffer():
    """Checked on the host before any device work: 1184 line chunks x 4096
    columns x 8 bytes = 38.8 MB of partials exceed the 16 MiB buffer."""
    d = C.DenseDesc()
    d.numeric = int(NT.FP32)
    d.layout = int(L.ROW_MAJOR)
    d.rows, d.cols, d.ld = 1_000_000, 4096, 4096
    d.values = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    need = C.lib().tomos_gemv_scratch_bytes(ctypes.byref(d), int(tb.TRANSPOSE))
    assert need > LIMIT
    rc = C.lib().tomos_gemv_no_alloc(int(tb.TRANSPOSE), 1.0, ctypes.byref(d), int(tb.Tier.AUTO),
                                     ctypes.c_void_p(256), 0.0, ctypes.c_void_p(256), None)
    assert rc == C.TOMOS_ERR_INVALID
    msg = C.lib().tomos_last_error().decode()
    assert "16777216" in msg and "tomos_gemv_no_alloc" in msg
