"""bench.py with more than one process, on CPU (gloo / no GPU work): the
max-over-ranks timing every rank takes part in, and the reference arm, which
only rank 0 runs and prints while the other ranks exit 0 without work."""
import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        b = _bench()
        got = b.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], "cpu")
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump(got, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_single_process():
    assert _bench().max_over_ranks([3.0, 4.5], "cpu") == [3.0, 4.5]


def test_max_over_ranks_two_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    for r in range(world):
        assert json.load(open(tmp_path / f"r{r}.json")) == [2.0, 10.0, 0.5]


def test_reference_arm_two_ranks():
    """torchrun with 2 processes: one JSON line, from rank 0, with impl
    "reference" (a value, or an `unavailable` reason when the reference's CPU
    build is absent); both ranks exit 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--rows", "4000", "--cols", "40"]
    env = dict(os.environ, OMP_NUM_THREADS="2", OPENBLAS_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" not in d:
        assert d["n_gpus"] == 2 and d["value"] > 0 and d["unit"] == "ms"
        assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
