"""Row-sharded solves on one GPU: the shard-aware CountSketch (rows hashed
by their row in the whole problem, so the shards' sketches sum to the whole
sketch), and the sharded LSQR path -- each pass's partials folded to n + 1
doubles and all-reduced through NCCL (one rank here), the n-side kernels
reading the summed values -- against the unsharded solve of the same rows.
Several ranks need several GPUs; the host side of the decomposition with
two ranks is tests/test_sharding.py (gloo, CPU)."""
import numpy as np
import pytest
import torch

import tomos_b200 as tb
from gpu_util import to_dense, cuda

pytestmark = pytest.mark.gpu
NT = tb.NumericType
L = tb.Layout


def scaled_problem(m, n, seed, decades=2.0):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-decades, decades, n)).astype(np.float32)
    x = rng.standard_normal(n)
    b = (A.astype(np.float64) @ x + 1e-6 * rng.standard_normal(m)).astype(np.float32)
    return A, b


@pytest.mark.parametrize("numeric,tier", [(NT.FP32, tb.Tier.AUTO), (NT.FP32_16, tb.Tier.HALF)])
@pytest.mark.parametrize("world", [1, 3])
def test_shard_sketches_sum_to_whole(numeric, tier, world):
    m, n, s = 30001, 200, 800
    A0, _ = scaled_problem(m, n, 5)
    stage = numeric == NT.FP32_16  # rows of 400 bytes: 16-byte aligned for the staging copies
    A = to_dense(A0, L.ROW_MAJOR, numeric)
    if stage:
        SA1, f1, c1, plane1 = tb.apply_count_sketch(A, s, tier=tier, with_colsq=True, stage=True)
    else:
        SA1, f1, c1 = tb.apply_count_sketch(A, s, tier=tier, with_colsq=True)
    SA = torch.zeros(s, n, dtype=torch.float64, device="cuda")
    fro2 = torch.zeros(1, dtype=torch.float64, device="cuda")
    colsq = torch.zeros(n, dtype=torch.float64, device="cuda")
    planes = []
    for r in range(world):
        r0, r1 = tb.shard_rows(m, r, world)
        Ar = to_dense(A0[r0:r1], L.ROW_MAJOR, numeric)
        S, f, c, p = tb.apply_count_sketch_shard(Ar, s, r0, tier=tier, stage=stage)
        SA += S.view()
        fro2 += f
        colsq += c
        if stage:
            planes.append(p[: r1 - r0, :n])
    ref = SA1.view()
    scale = float(ref.abs().max())
    # the FP32 sketch sums a bucket's rows in FP32 (as the reference's
    # countsketch_apply_impl<float>): shards round their partial sums apart
    assert float((SA - ref).abs().max()) <= 2e-6 * scale
    assert abs(float(fro2[0]) - float(f1.reshape(-1)[0])) <= 1e-6 * float(f1.reshape(-1)[0])
    assert torch.allclose(colsq, c1, rtol=1e-6, atol=0.0)
    if stage:
        # the staged fp16 plane of every shard is the whole plane's rows
        assert torch.equal(torch.cat(planes), plane1[:m, :n])
    if world == 1:
        assert torch.equal(SA, ref)


@pytest.mark.parametrize("numeric", [NT.FP32, NT.FP32_16])
def test_single_rank_sharded_solve_matches_unsharded(numeric):
    """The sharded path with one rank (every pass's partials through
    shard_reduce_kernel and an NCCL all-reduce) reaches the unsharded
    solve's solution in as many iterations."""
    m, n, s = 40000, 300, 1200
    A0, b0 = scaled_problem(m, n, 7)
    A = to_dense(A0, L.ROW_MAJOR, numeric, pad=4)
    b = cuda(b0)
    x0, r0, _ = tb.sketch_lsqr(A, b, s)
    comm = tb.Comm.single()
    try:
        ws = tb.create_lsqr_workspace(None, (m, n), NT.FP32, NT.FP64)
        for _ in range(2):  # the workspace is reused: the solve's graph went with it
            x1, r1, _ = tb.sketch_lsqr(A, b, s, workspace=ws, comm=comm, row0=0)
            assert r1["converged"] == 1 and r1["backward_error"] <= 1e-6
            assert abs(r1["iterations"] - r0["iterations"]) <= 1
            assert float((x1 - x0).norm() / x0.norm()) <= 1e-6
    finally:
        comm.close()
    # the workspace serves an unsharded solve after the communicator is gone
    x2, r2, _ = tb.sketch_lsqr(A, b, s, workspace=ws)
    assert r2["converged"] == 1 and torch.equal(x2, x0)


def test_comm_api():
    comm = tb.Comm.single()
    try:
        assert (comm.rank, comm.size) == (0, 1)
        t = torch.arange(1000, dtype=torch.float64, device="cuda")
        comm.allreduce_f64(t)
        assert torch.equal(t.cpu(), torch.arange(1000, dtype=torch.float64))
        comm.allreduce_f64(torch.empty(0, dtype=torch.float64, device="cuda"))
    finally:
        comm.close()
    import ctypes
    from tomos_b200 import _capi as C
    idbuf, h = (ctypes.c_char * 128)(), ctypes.c_void_p()
    assert C.lib().tomos_comm_create(2, 5, idbuf, ctypes.byref(h)) != 0 and not h.value
    closed = tb.Comm.single()
    closed.close()
    with pytest.raises(tb.TomosError):
        closed.allreduce_f64(torch.zeros(4, dtype=torch.float64, device="cuda"))
