"""Named small workloads of the library's hot kernels, for profiling one
kernel at a time (e.g. under ncu) without the whole benchmark around it.

    python -m tomos_b200.cases solve [--m M] [--n N] [--storage fp32_16|fp32] [--reps R] [--profile]
    python -m tomos_b200.cases gemm  [--size S] [--tier half_operands|half|accurate] [--reps R]
    python -m tomos_b200.cases gemv  [--m M] [--n N] [--tier half|accurate|fp32] [--reps R]
    python -m tomos_b200.cases csr   [--m M] [--n N] [--k K] [--reps R] [--profile]

`solve` runs the sketch-preconditioned LSQR pipeline (sketch_lsqr) on the
seeded dense problem A = G diag(10^u) of problems.dense_scaled (--profile: the
solver's profile mode, every iteration launched on its own instead of in the
device-side graph loop, so that a profiler lists each pass); `gemm` runs
mm_apply on S x S column-major operands (A packed FP32_16); `gemv` runs
mv_apply both ways on the packed (or FP32) row-major matrix; `csr` runs
sketch_lsqr (s = 4n) on the FP32_16-packed CSR matrix of problems.csr_scaled
(k nonzeros a row).  Each case
runs `reps` times after one untimed warm-up call and prints one line."""
import argparse
import sys

import torch

import tomos_b200 as tb
from tomos_b200 import problems


def _solve(a):
    A32, _, b = problems.dense_scaled(a.m, a.n, seed=0)
    A = tb.Dense(tb.NumericType.FP32, tb.Layout.ROW_MAJOR, (a.m, a.n), a.n, A32.view(-1))
    if a.storage == "fp32_16":
        A = tb.pack(A, tb.NumericType.FP32_16)
    ws = tb.create_lsqr_workspace(None, (a.m, a.n), tb.NumericType.FP32, tb.NumericType.FP64)
    rep = None
    for _ in range(1 + a.reps):
        _, rep, _ = tb.sketch_lsqr(A, b, 4 * a.n, workspace=ws, profile=a.profile)
    torch.cuda.synchronize()
    return f"solve {a.m}x{a.n} {a.storage}: iterations {rep['iterations']}, eta_D {rep['backward_error']:.3e}"


def _gemm(a):
    T, L = tb.TransposeType, tb.Layout
    n = a.size
    tier = {"half_operands": tb.Tier.HALF_OPERANDS, "half": tb.Tier.HALF, "accurate": tb.Tier.ACCURATE}[a.tier]
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    A = tb.pack(tb.Dense.from_tensor(torch.randn(n, n, device="cuda", generator=g), L.COL_MAJOR),
                tb.NumericType.FP32_16)
    B = tb.Dense.from_tensor(torch.randn(n, n, device="cuda", generator=g), L.COL_MAJOR)
    C = tb.Dense.from_tensor(torch.zeros(n, n, device="cuda"), L.COL_MAJOR)
    for _ in range(1 + a.reps):
        tb.mm_apply(tb.Device.CUDA, T.NO_TRANSPOSE, T.NO_TRANSPOSE, 1.0, A, B, 0.0, C, tier=tier)
    torch.cuda.synchronize()
    return f"gemm {n}^3 {a.tier}"


def _gemv(a):
    A32, _, _ = problems.dense_scaled(a.m, a.n, seed=0)
    A = tb.Dense(tb.NumericType.FP32, tb.Layout.ROW_MAJOR, (a.m, a.n), a.n, A32.view(-1))
    tier = tb.Tier.AUTO
    if a.tier != "fp32":
        A = tb.pack(A, tb.NumericType.FP32_16)
        tier = tb.Tier.HALF if a.tier == "half" else tb.Tier.ACCURATE
    x = torch.randn(a.n, device="cuda")
    u = torch.randn(a.m, device="cuda")
    for _ in range(1 + a.reps):
        tb.mv_apply(tb.Device.CUDA, tb.TransposeType.NO_TRANSPOSE, 1.0, A, x, 0.0, u, tier=tier)
        tb.mv_apply(tb.Device.CUDA, tb.TransposeType.TRANSPOSE, 1.0, A, u, 0.0, x, tier=tier)
    torch.cuda.synchronize()
    return f"gemv {a.m}x{a.n} {a.tier}"


def _csr(a):
    rp, ci, v, _, b = problems.csr_scaled(a.m, a.n, a.k, seed=4)
    t = tb.Dense.from_tensor(v[None, :], tb.Layout.ROW_MAJOR)
    P = tb.pack(t, tb.NumericType.FP32_16)
    A = tb.Csr(tb.NumericType.FP32_16, (a.m, a.n), rp, ci, P.storage)
    ws = tb.create_lsqr_workspace(None, (a.m, a.n), tb.NumericType.FP32, tb.NumericType.FP64)
    rep = None
    for _ in range(1 + a.reps):
        _, rep, _ = tb.sketch_lsqr(A, b, 4 * a.n, workspace=ws, profile=a.profile)
    torch.cuda.synchronize()
    return f"csr {a.m}x{a.n} k={a.k}: iterations {rep['iterations']}, eta_D {rep['backward_error']:.3e}"


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["solve", "gemm", "gemv", "csr"])
    ap.add_argument("--m", type=int, default=200_000)
    ap.add_argument("--n", type=int, default=1000)
    ap.add_argument("--storage", default="fp32_16", choices=["fp32_16", "fp32"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--tier", default="half_operands")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--k", type=int, default=20)
    ap.add_argument("--profile", action="store_true")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    print({"solve": _solve, "gemm": _gemm, "gemv": _gemv, "csr": _csr}[a.case](a))
    return 0


if __name__ == "__main__":
    sys.exit(main())
