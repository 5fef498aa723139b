#!/usr/bin/env python
"""LSQR time to relative backward error 1e-6 on one B200: packed 16-bit
(FP32_16) storage against plain FP32 storage, and the GEMV GB/s behind it.

Workload (one step): dense row-major A (1,000,000 x 1000) = G diag(10^u),
G ~ N(0,1), u ~ U(-3,3), b = A x_true + 1e-8 noise -- the matrix already
resident in HBM.  A step is the whole solve: hash CountSketch (s = 4n)
-> FP64 Householder QR -> R^{-1} -> right-preconditioned LSQR with FP32
residual refinement until the normwise backward error
  eta = min(||r|| / (||A||_F ||x|| + ||b||), ||A^T r|| / (||A||_F ||r||))
of the column-scaled problem (A D^{-1}, b, D x), D = the column norms
(recomputed from an exact (wh+wr) FP64-accumulated residual at every
restart), is <= 1e-6.  The plain normwise eta of A itself cannot serve:
with condition 1e6 coming from the column scales it is met by iterates
that are far from the solution (||A||_F ||x|| swamps ||r||).  `value` is the packed run's ms per step; the FP32-storage run of
the same problem is timed beside it (fp32_ms, speedup_vs_fp32).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU runs are replicas (one independent problem per rank, the row
sharding of LSQR is not built); timing is the max over ranks.
"""
import argparse
import json
import math
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LSQR time to rel. backward err 1e-6, packed 16-bit vs FP32 (1 B200); GEMV GB/s"
M_DEF, N_DEF = 1_000_000, 1000
TOL = 1e-6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--m", "--rows", dest="m", type=int, default=M_DEF)
    ap.add_argument("--n", "--cols", dest="n", type=int, default=N_DEF)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-rows", type=int, default=200_000)
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(values, device):
    """Each value's maximum over the ranks of the process group (every rank
    takes part; a single process gets its own values back)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(name):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    v = json.load(open(p)).get(name)
    return v.get("bytes_per_launch") if isinstance(v, dict) else v


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while running."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                fn = getattr(self.nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    self.nv.nvmlDeviceGetCurrentClocksThrottleReasons
                r = fn(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv:
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons)}
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# --------------------------------------------------------------------- GPU

def gpu_solve(tb, torch, A, b, s):
    """One step: sketch (+ column norms) -> QR -> R^{-1} -> LSQR until the
    backward error of the column-scaled problem is <= 1e-6.  Returns (x, report)."""
    packed = A.numeric in (tb.NumericType.FP32_16, tb.NumericType.FP32_BF16)
    m, n = A.size
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if gpu_solve.profile else None
    if ev:
        ev[0].record()
    plane = None
    if A.numeric == tb.NumericType.FP32_16:
        # the sketch pass also writes the fp16 plane the HALF-tier iterations read
        SA, fro2, colsq, plane = tb.apply_count_sketch(A, s, tier=tb.Tier.HALF, with_colsq=True,
                                                       stage=True)
    else:
        SA, fro2, colsq = tb.apply_count_sketch(A, s, tier=tb.Tier.HALF if packed else tb.Tier.AUTO,
                                                with_colsq=True)
    if ev:
        ev[1].record()
    Rinv = tb.generate_sketch_qr_precond(SA, copy=False)
    if ev:
        ev[2].record()
    d, anorm = tb.column_scale(colsq)
    gpu_solve.last_scale = d
    ws = gpu_solve.ws.get((m, n))
    if ws is None:
        ws = tb.create_lsqr_workspace(None, (m, n), tb.NumericType.FP32, tb.NumericType.FP64)
        gpu_solve.ws[(m, n)] = ws
    tb.add_precond(Rinv, ws)
    x = torch.empty(n, device="cuda")  # the solve zeroes x
    rep = tb.lsqr_solve(None, A, b, x, ws, TOL, 200, 0.0, restarts=8,
                        stop_rule=tb.StopRule.BACKWARD, inner_rtol=2e-3 if packed else 0.0,
                        anorm_fro=anorm, col_scale=d, staged_plane=plane,
                        profile=gpu_solve.profile)
    if ev:
        ev[3].record()
        torch.cuda.synchronize()
        rep = dict(rep)
        rep["phase_ms"] = {"sketch": ev[0].elapsed_time(ev[1]), "qr": ev[1].elapsed_time(ev[2]),
                           "solve": ev[2].elapsed_time(ev[3])}
    return x, rep


gpu_solve.ws = {}
gpu_solve.profile = False
gpu_solve.last_scale = None


def count_launches(torch, fn):
    """Kernels of this library (namespace tomos_b200) one call of fn launches."""
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    return sum(1 for e in prof.events()
               if e.device_type.name == "CUDA" and "tomos_b200::" in e.name)


def time_steps(torch, fn, steps, warmup):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    out = None
    for _ in range(steps):
        out = fn()
    ev1.record()
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / steps, out


def run_ours(args):
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import tomos_b200 as tb
    from tomos_b200 import problems

    m, n = args.m, args.n
    s = 4 * n
    A32, xt, b = problems.dense_scaled(m, n, seed=args.seed + rank)
    Af = tb.Dense(tb.NumericType.FP32, tb.Layout.ROW_MAJOR, (m, n), n, A32.view(-1))
    Ap = tb.pack(Af, tb.NumericType.FP32_16)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # timed region: packed 16-bit (the headline), then FP32 storage
    barrier()
    sampler = ClockSampler(local)
    nvtx = torch.cuda.nvtx
    with sampler:
        nvtx.range_push("packed_solve")
        ms_packed, (xp, rep_p) = time_steps(torch, lambda: gpu_solve(tb, torch, Ap, b, s),
                                            args.steps, args.warmup)
        nvtx.range_pop()
        barrier()
        nvtx.range_push("fp32_solve")
        ms_fp32, (xf, rep_f) = time_steps(torch, lambda: gpu_solve(tb, torch, Af, b, s),
                                          args.steps, args.warmup)
        nvtx.range_pop()
    barrier()
    ms_packed, ms_fp32 = max_over_ranks([ms_packed, ms_fp32], "cuda")

    # accurate backward errors of the returned solutions (FP64, exact A):
    # eta_D of the column-scaled problem (the convergence measure) and the
    # plain normwise eta
    ws_be = tb.create_lsqr_workspace(None, (m, n), tb.NumericType.FP32)
    d_exact = gpu_solve.last_scale  # column norms from the last FP32-storage sketch
    be_p = tb.backward_error(Ap, b, xp, ws_be, col_scale=d_exact)["backward_error"]
    be_f = tb.backward_error(Af, b, xf, ws_be, col_scale=d_exact)["backward_error"]
    be_p_plain = tb.backward_error(Ap, b, xp, ws_be)["backward_error"]
    be_f_plain = tb.backward_error(Af, b, xf, ws_be)["backward_error"]
    rel_x = float(torch.linalg.norm((xp - xt).double()) / torch.linalg.norm(xt.double()))

    # roofline of the dominant kernel (the fused pass over the wh plane):
    # one profiled solve times every pass with CUDA events on its stream.
    gpu_solve.profile = True
    for _ in range(2):  # the second of each is kept
        _, prof_p = gpu_solve(tb, torch, Ap, b, s)
        _, prof_f = gpu_solve(tb, torch, Af, b, s)
    gpu_solve.profile = False
    peak, peak_kind = measured_peak()
    pass_ms = prof_p["iter_pass_ms"] / max(1, prof_p["iter_pass_count"])
    alg_bytes = 2.0 * m * n + 8.0 * m  # wh plane + u read/write
    ach = alg_bytes / (pass_ms * 1e-3) / 1e9
    pass_ms_f = prof_f["iter_pass_ms"] / max(1, prof_f["iter_pass_count"])
    ach_f = (4.0 * m * n + 8.0 * m) / (pass_ms_f * 1e-3) / 1e9
    init_ms = prof_p["init_pass_ms"] / max(1, prof_p["init_pass_count"])
    ach_init = (4.0 * m * n + 8.0 * m) / (init_ms * 1e-3) / 1e9

    # end to end through the public API with host buffers: H2D of A (FP32)
    # and b, pack, sketch, QR, solve, D2H of x.
    e2e = None
    if rank == 0 or world > 1:
        hostA = torch.empty((m, n), dtype=torch.float32, pin_memory=True)
        hostA.copy_(A32)
        hostb = torch.empty(m, dtype=torch.float32, pin_memory=True)
        hostb.copy_(b)
        del A32
        Ad = torch.empty((m, n), dtype=torch.float32, device="cuda")
        bd = torch.empty(m, dtype=torch.float32, device="cuda")

        def e2e_step():
            Ad.copy_(hostA, non_blocking=True)
            bd.copy_(hostb, non_blocking=True)
            Dd = tb.Dense(tb.NumericType.FP32, tb.Layout.ROW_MAJOR, (m, n), n, Ad.view(-1))
            P = tb.pack(Dd, tb.NumericType.FP32_16)
            x, _ = gpu_solve(tb, torch, P, bd, s)
            return x.cpu()

        barrier()
        nvtx.range_push("e2e")
        e2e_ms, _ = time_steps(torch, e2e_step, args.e2e_steps, args.warmup)
        nvtx.range_pop()
        barrier()
        e2e_ms = max_over_ranks([e2e_ms], "cuda")[0]
        e2e = {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 4 * m * n + 4 * m,
               "d2h_bytes_per_step": 4 * n}

    # this library's kernels per step, counted from one traced step of each
    # arm (CUPTI through the torch profiler)
    launches = args.steps * (count_launches(torch, lambda: gpu_solve(tb, torch, Ap, b, s)) +
                             count_launches(torch, lambda: gpu_solve(tb, torch, Af, b, s)))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference(args, m, n)
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms_packed, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_packed,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"dense row-major {m}x{n} G diag(10^U(-3,3)), sketch s={s}, "
                                   "FP32_16 packed storage, eta<=1e-6",
                       "m": m, "n": n, "s": s, "storage": "fp32_16 (half tier + exact refinement)",
                       "parallelism": "replicas" if world > 1 else "1 GPU",
                       "l2": "inputs (4 GB) larger than L2 (126 MB)"},
            "fp32_ms": ms_fp32, "speedup_vs_fp32": ms_fp32 / ms_packed,
            "iterations": {"packed": rep_p["iterations"], "fp32": rep_f["iterations"],
                           "packed_restarts": rep_p["restarts_used"],
                           "fp32_restarts": rep_f["restarts_used"]},
            "backward_error": {"measure": "eta_D: backward error of (A D^-1, b, D x), D = column norms",
                               "packed": be_p, "fp32": be_f, "packed_plain_eta": be_p_plain,
                               "fp32_plain_eta": be_f_plain, "x_rel_err_vs_xtrue": rel_x},
            "phase_ms": {"packed": prof_p.get("phase_ms"), "fp32": prof_f.get("phase_ms"),
                         "packed_restart_pass_ms": init_ms,
                         "note": "one profiled solve each (passes timed one by one)"},
            "gemv_gbs": {"fused_pass_fp32_16_half": ach, "fused_pass_fp32": ach_f,
                         "fused_pass_fp32_16_exact_fp64acc": ach_init,
                         "pass_ms_half": pass_ms, "pass_ms_fp32": pass_ms_f},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": peak_kind,
                         "kernel": "fused_rows_mma_kernel (staged fp16 plane, tensor cores; one LSQR "
                                   "iteration's A p and A^T u)",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "traffic": ncu_traffic("fused_pass_mma_f16_1e6x1000")},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": sampler.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------- CPU

def cpu_reference(args, m, n, seed=0):
    """The reference's own CPU path (oracle/_ref: its lsqr_solve, hash
    CountSketch and LAPACK sketch QR) on a row sample of the workload,
    extrapolated linearly in m to the full problem.  Test/baseline
    infrastructure: the product never calls it."""
    import ctypes
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unavailable": "reference CPU build missing"}
    R = oracle.ref()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    ms = min(args.cpu_rows, m)
    rng = np.random.default_rng(seed)
    u = rng.uniform(-3, 3, n)
    A = np.asfortranarray((rng.standard_normal((ms, n)) * 10.0 ** u).astype(np.float32))
    xt = rng.standard_normal(n)
    b = (A.astype(np.float64) @ xt + 1e-8 * rng.standard_normal(ms)).astype(np.float32)
    s = 4 * n
    A64 = np.asfortranarray(A.astype(np.float64))
    SA = np.zeros((s, n), np.float64, order="F")
    t0 = time.perf_counter()
    R.ref_countsketch_apply_f64(ms, n, P(A64), ms, s, P(SA), s)
    t_sketch = time.perf_counter() - t0
    W = SA.copy(order="F")
    t0 = time.perf_counter()
    rc = R.ref_sketch_qr_f64(s, n, P(W))
    t_qr = time.perf_counter() - t0
    Rinv = np.asfortranarray(np.triu(W[:n, :n]).astype(np.float32))
    # its own LSQR to a tight tolerance, timed; the iteration at which the
    # normwise backward error first reaches 1e-6 is read off its residual
    # history (||r_k|| = |phi_bar_k|).
    iters_cap = 60
    x = np.zeros(n, np.float32)
    it = ctypes.c_int(0)
    hist = np.zeros(iters_cap + 2)
    t0 = time.perf_counter()
    R.ref_lsqr_solve_f32(ms, n, P(A), P(b), P(x), P(Rinv), 1e-12, iters_cap, 1e-12, 1,
                         ctypes.byref(it), P(hist))
    t_lsqr = time.perf_counter() - t0
    k = max(1, it.value)
    t_iter = t_lsqr / k
    bn = float(np.linalg.norm(b.astype(np.float64)))
    an = float(np.linalg.norm(A.astype(np.float64)))
    xn = float(np.linalg.norm(x.astype(np.float64)))
    eta_k = hist[:k] * bn / (an * xn + bn)
    hit = np.flatnonzero(eta_k <= TOL)
    k_needed = int(hit[0]) + 1 if hit.size else k
    scale = m / ms
    total_s = t_sketch * scale + t_qr + k_needed * t_iter * scale
    return {"value": total_s * 1e3, "unit": "ms", "cores": os.cpu_count(), "kind": "reference",
            "sample": f"{ms}x{n} row sample of the workload on the reference's CPU lsqr_solve "
                      f"(FP32, OpenBLAS) with its sketch QR; sketch and per-iteration time "
                      f"extrapolated x{scale:g} in m; {k_needed} iterations to eta<=1e-6",
            "extrapolated": True, "sketch_s": t_sketch, "qr_s": t_qr, "iter_s": t_iter,
            "iterations": k_needed, "qr_rc": int(rc)}


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    m, n = args.m, args.n
    vals = []
    last = None
    for _ in range(max(1, args.steps)):
        last = cpu_reference(args, m, n)
        if last.get("value") is None:
            print(json.dumps({"impl": "reference", "unavailable": last.get("unavailable")}))
            return
        vals.append(last["value"])
    v = float(np.mean(vals))
    cpu = dict(last)
    cpu["value"] = v
    line = {"metric": METRIC, "value": v, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"dense {m}x{n} G diag(10^U(-3,3)), sketch s={4 * n}, "
                                   "reference CPU lsqr_solve (FP32 storage), eta<=1e-6",
                       "m": m, "n": n, "s": 4 * n, "parallelism": "host cores"},
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
