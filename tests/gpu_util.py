"""Helpers shared by the GPU tests: numpy <-> device Dense, decoded oracle values."""
import numpy as np
import torch

import tomos_b200 as tb


def to_dense(A, layout, numeric=tb.NumericType.FP32, pad=0, rounded=False):
    """A float32 (m x n) numpy array as a device Dense of the given layout,
    leading dimension padded by `pad`, optionally packed."""
    m, n = A.shape
    inner = m if layout == tb.Layout.COL_MAJOR else n
    D = tb.Dense.create_strided(None, layout, tb.NumericType.FP32, (m, n), lead_dim=inner + pad)
    # poison the padding so a kernel reading it shows up
    D.storage.fill_(float("nan"))
    D.view()[...] = torch.from_numpy(np.ascontiguousarray(A, np.float32)).cuda()
    if numeric == tb.NumericType.FP32:
        return D
    return tb.pack(D, numeric, rounded=rounded)


def planes(D):
    """(wh, wr) of a packed Dense as uint16 numpy (m x n) arrays."""
    wh = D.view(0).cpu().numpy().view(np.uint16)
    wr = D.view(1).cpu().numpy().view(np.uint16)
    return wh, wr


def decoded(orc, D, tier):
    """The values the kernels read A as, in float64."""
    if D.numeric == tb.NumericType.FP32:
        return D.view().double().cpu().numpy()
    wh, wr = planes(D)
    kind = "fp32_16" if D.numeric == tb.NumericType.FP32_16 else "fp32_bf16"
    t = "half" if tier == tb.Tier.HALF else "accurate"
    return orc.decode(kind, wh, wr, t, D.rounded).astype(np.float64)


def cuda(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)
