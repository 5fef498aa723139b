"""The reference's own dispatch as the caller: its core/blas mv_apply and
its src/dispatch registries, compiled unmodified (oracle/Makefile ->
oracle/_ref/libtomos_ref_b200.so), with the CUDA GEMV launchers those
registries call defined over this library's C ABI (oracle/ref_launchers.cpp).
mv_apply on Device::CUDA Dense objects then runs the reference's registry
lookup (dense_registries.cpp: FP32 -> mv_fp32_tiled; fp32_16_registries.cpp:
FP32_16 with FP16 compute -> pure_half, with FP32 compute -> accurate) and
lands in the sm_100a kernels; any other launcher would abort.  Checked
against the FP64 product of the values each tier reads."""
import ctypes
import os

import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, decoded, cuda

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libtomos_ref_b200.so")
NT = tb.NumericType


def ref_dispatch():
    if not os.path.exists(LIB):
        pytest.skip("the reference dispatch build (oracle/_ref) is absent")
    L = ctypes.CDLL(LIB)
    v, sz, d, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int
    L.ref_b200_mv.argtypes = [i, d, i, i, sz, sz, v, sz, v, d, v]
    L.ref_b200_mv.restype = i
    return L


# (storage, the reference's compute type, the tier it resolves to here)
CASES = [(NT.FP32, NT.FP32, tb.Tier.AUTO), (NT.FP32_16, NT.FP16, tb.Tier.HALF),
         (NT.FP32_16, NT.FP32, tb.Tier.ACCURATE)]


@pytest.mark.parametrize("numeric,compute,tier", CASES)
@pytest.mark.parametrize("shape", [(4097, 300), (200000, 64), (33, 257)])
def test_reference_mv_apply_through_its_registry(orc, numeric, compute, tier, shape):
    L = ref_dispatch()
    rng = np.random.default_rng(shape[0] + int(compute))
    m, n = shape
    A0 = (rng.standard_normal((m, n)) * np.where(rng.random((m, n)) < 0.05, 1e-6, 1.0)).astype(np.float32)
    A = to_dense(A0, tb.Layout.COL_MAJOR, numeric)  # the reference is column-major
    Ad = decoded(orc, A, tier)
    for trans in (0, 1):
        M = Ad if trans == 0 else Ad.T
        x = rng.standard_normal(M.shape[1]).astype(np.float32)
        y0 = rng.standard_normal(M.shape[0]).astype(np.float32)
        xd, yd = cuda(x), cuda(y0)
        rc = L.ref_b200_mv(trans, 1.5, int(numeric), int(compute), m, n, A.storage.data_ptr(), A.ld,
                           xd.data_ptr(), 0.5, yd.data_ptr())
        assert rc == 0
        got = yd.cpu().numpy().astype(np.float64)
        ref = 1.5 * (M @ x.astype(np.float64)) + 0.5 * y0.astype(np.float64)
        scale = 1.5 * (np.abs(M) @ np.abs(x.astype(np.float64))) + 0.5 * np.abs(y0)
        tol = (2e-6 if tier == tb.Tier.ACCURATE else 2e-5) * scale + 1e-7 * np.abs(ref) + 1e-30
        assert np.all(np.abs(got - ref) <= tol), (trans, float(np.abs(got - ref).max()))


def test_reference_registry_refuses_unregistered_compute():
    """The reference's own 'no kernel registered' contract still holds
    around the plugged launchers (FP32 storage with FP16 compute)."""
    L = ref_dispatch()
    A = to_dense(np.ones((8, 4), np.float32), tb.Layout.COL_MAJOR)
    x, y = cuda(np.ones(4, np.float32)), cuda(np.zeros(8, np.float32))
    assert L.ref_b200_mv(0, 1.0, int(NT.FP32), int(NT.FP16), 8, 4, A.storage.data_ptr(), A.ld,
                         x.data_ptr(), 0.0, y.data_ptr()) == -1
