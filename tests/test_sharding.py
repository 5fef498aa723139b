"""Row-sharded LSQR, the host side on CPU (two gloo ranks): the row
partition, the communicator id every rank receives, and the sharded
algorithm itself -- each rank's products over its rows, the n + 1 partial
sums (A^T u, ||u||^2) all-reduced once a pass, the sketch summed over the
ranks with the whole problem's row indices hashed -- giving the single-rank
solve's iterations and solution.  The product runs the same decomposition
on the GPU (comm.cu, lsqr.cu), exercised by tests/test_gpu_shard.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import tomos_b200 as tb


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_rows_partition():
    for m in (0, 1, 7, 1000, 1_000_003):
        for world in (1, 2, 3, 8):
            spans = [tb.shard_rows(m, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == m
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def problem(m=6000, n=40, seed=3):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-2, 2, n)
    x = rng.standard_normal(n)
    b = A @ x + 1e-6 * rng.standard_normal(m)
    return A, b


def sketch(orc, A, s, row0):
    """The hash CountSketch of rows whose row i is row row0 + i of the whole
    problem (the oracle's hash of the whole problem's rows)."""
    m = A.shape[0]
    bucket, sign = orc.countsketch_hash(row0 + m, s)
    SA = np.zeros((s, A.shape[1]))
    np.add.at(SA, bucket[row0:], sign[row0:, None] * A)
    return SA


def lsqr(A, b, Rinv, iters, allreduce):
    """Right-preconditioned LSQR in the product's formulation (u kept
    unnormalised, A^T u from the same pass), on this rank's rows; every sum
    over rows goes through allreduce (the identity on one rank)."""
    n = A.shape[1]
    x = np.zeros(n)
    u = b.copy()
    s = allreduce(np.concatenate([A.T @ u, [u @ u]]))
    beta = np.sqrt(s[n])
    v = Rinv.T @ (s[:n] / beta)
    alpha = np.linalg.norm(v)
    v /= alpha
    w = Rinv @ v
    phi_bar, rho_bar = beta, alpha
    for _ in range(iters):
        p = Rinv @ v
        u = A @ p - alpha * (u / beta)  # the next unnormalised u
        s = allreduce(np.concatenate([A.T @ u, [u @ u]]))
        beta = np.sqrt(s[n])
        vh = Rinv.T @ (s[:n] / beta) - beta * v
        alpha = np.linalg.norm(vh)
        v = vh / alpha
        rho = np.hypot(rho_bar, beta)
        c, sn = rho_bar / rho, beta / rho
        theta, rho_bar = sn * alpha, -c * alpha
        phi, phi_bar = c * phi_bar, sn * phi_bar
        x = x + (phi / rho) * w
        w = Rinv @ v - (theta / rho) * w
    return x, abs(phi_bar)


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        idb, r, w = tb.Comm.exchange_id()
        A, b = problem()
        r0, r1 = tb.shard_rows(A.shape[0], rank, world)

        def allreduce(v):
            t = torch.from_numpy(np.ascontiguousarray(v, np.float64))
            dist.all_reduce(t)
            return t.numpy()

        SA = allreduce(sketch(oracle, A[r0:r1], 400, r0))
        Rinv = np.linalg.inv(np.linalg.qr(SA, mode="r"))
        x, res = lsqr(A[r0:r1], b[r0:r1], Rinv, 40, allreduce)
        np.savez(os.path.join(out, f"r{rank}.npz"), idb=np.frombuffer(idb, np.uint8), x=x, res=res, SA=SA)
    finally:
        dist.destroy_process_group()


def test_sharded_lsqr_two_gloo_ranks_matches_one(orc, tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    r = [np.load(tmp_path / f"r{k}.npz") for k in range(world)]
    # one communicator id reached both ranks; the replicated state agrees
    assert np.array_equal(r[0]["idb"], r[1]["idb"]) and r[0]["idb"].any()
    assert np.array_equal(r[0]["x"], r[1]["x"]) and np.array_equal(r[0]["SA"], r[1]["SA"])
    # the single-rank solve of the whole problem
    A, b = problem()
    SA1 = sketch(orc, A, 400, 0)
    np.testing.assert_allclose(r[0]["SA"], SA1, rtol=1e-12, atol=1e-12 * np.abs(SA1).max())
    Rinv = np.linalg.inv(np.linalg.qr(SA1, mode="r"))
    x1, res1 = lsqr(A, b, Rinv, 40, lambda v: v)
    assert np.linalg.norm(r[0]["x"] - x1) <= 1e-6 * np.linalg.norm(x1)
    assert abs(float(r[0]["res"]) - res1) <= 1e-6 * res1 + 1e-12
    # and both reach the least-squares solution
    xo = orc.lstsq_f64(A, b)
    assert np.linalg.norm(x1 - xo) <= 1e-6 * np.linalg.norm(xo)
