"""Regenerates the golden fixtures in this directory from the reference's
own CPU build (oracle/_ref/libtomos_ref.so, compiled from the reference
sources by oracle/Makefile).

    python tests/golden/make_golden.py

Fixtures (small .npz files, committed):
  pack_fp32_16.npz     inputs + wh/wr of fp32_16_split, combine, half_only
                       (edge cases, an exponent sweep and random bit patterns)
  pack_fp32_bf16.npz   truncating and rounding splits and their combines
  countsketch.npz      bucket/sign of rows 0..4095 for s = 64 and 4000, and
                       the reference's countsketch_apply on a 1000 x 3 X
  sketch_qr.npz        the reference's R^{-1} (LAPACK dgeqrf + dtrtri) of a
                       300 x 40 matrix
  lsqr_small.npz       the reference's lsqr_solve (CPU, FP32) on a seeded
                       2000 x 50 Gaussian problem, plain and preconditioned:
                       x, iteration count, residual history
  mv_fp32_16.npz       the reference's CPU FP32_16 GEMV tiers on 37 x 23
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731


def pack_inputs(seed=7):
    rng = np.random.default_rng(seed)
    edge = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0, 65504.0, 65520.0, 6.1035156e-05,
                     6.0e-05, 5.96e-08, 2.0 ** -28, 2.0 ** -29, 2.0 ** 29, 2.0 ** 30, 1e-30, 1e30,
                     3.25, 1.0009765625, 1.00146484375, 0.1, -7.5, 1e-45], dtype=np.float32)
    sweep = []
    for e in range(256):
        mant = rng.integers(0, 1 << 23, 40, dtype=np.uint64).astype(np.uint32)
        sign = rng.integers(0, 2, 40, dtype=np.uint64).astype(np.uint32)
        sweep.append((sign << 31) | (np.uint32(e) << 23) | mant)
    sweep = np.concatenate(sweep).view(np.float32)
    # round-up / carry boundaries: top 9 mantissa bits all ones, ties
    carry = []
    for e in (98, 99, 112, 113, 127, 142, 143, 156, 157):
        for low in (0x1FFF, 0x2000, 0x2001, 0x3FFF):
            carry.append((np.uint32(e) << 23) | np.uint32((0x1FF << 14) | low))
            carry.append((np.uint32(e) << 23) | np.uint32((0x0FE << 14) | low))
    carry = np.array(carry, np.uint32).view(np.float32)
    rnd = rng.integers(0, 1 << 32, 20000, dtype=np.uint64).astype(np.uint32).view(np.float32)
    return np.concatenate([edge, sweep, carry, rnd]).astype(np.float32)


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    R = oracle.ref()
    sz = ctypes.c_size_t

    x = pack_inputs()
    n = x.size
    wh = np.empty(n, np.uint16); wr = np.empty(n, np.uint16)
    R.ref_fp32_16_split(P(x), n, P(wh), P(wr))
    comb = np.empty(n, np.float32)
    R.ref_fp32_16_combine(P(wh), P(wr), n, P(comb))
    allwh = np.arange(65536, dtype=np.uint16)
    ho = np.empty(65536, np.uint16)
    R.ref_fp32_16_half_only(P(allwh), 65536, P(ho))
    np.savez_compressed(os.path.join(HERE, "pack_fp32_16.npz"), x=x, wh=wh, wr=wr, combine=comb,
                        half_only=ho)

    bf = {}
    for rounded, sfn, cfn in ((0, R.ref_fp32_bf16_split, R.ref_fp32_bf16_combine),
                              (1, R.ref_fp32_bf16_split_rounded, R.ref_fp32_bf16_combine_rounded)):
        h = np.empty(n, np.uint16); r = np.empty(n, np.uint16)
        sfn(P(x), n, P(h), P(r))
        c = np.empty(n, np.float32)
        cfn(P(h), P(r), n, P(c))
        bf[f"wh{rounded}"] = h; bf[f"wr{rounded}"] = r; bf[f"combine{rounded}"] = c
    np.savez_compressed(os.path.join(HERE, "pack_fp32_bf16.npz"), x=x, **bf)

    # CountSketch: the hash is pinned through countsketch_apply on unit rows.
    out = {}
    for s in (64, 4000):
        rows = 4096
        X = np.zeros((rows, 1), np.float64)
        bucket = np.empty(rows, np.int32); sign = np.empty(rows, np.int8)
        for i in range(rows):
            X[:] = 0.0
            X[i, 0] = 1.0
            Y = np.zeros((s, 1), np.float64)
            Xf = np.asfortranarray(X)
            R.ref_countsketch_apply_f64(sz(rows), sz(1), P(Xf), sz(rows), sz(s), P(Y), sz(s))
            k = int(np.flatnonzero(Y[:, 0])[0])
            bucket[i] = k
            sign[i] = int(Y[k, 0])
        out[f"bucket_s{s}"] = bucket
        out[f"sign_s{s}"] = sign
    rng = np.random.default_rng(11)
    Xs = np.asfortranarray(rng.standard_normal((1000, 3)).astype(np.float32))
    Ys = np.zeros((64, 3), np.float32, order="F")
    R.ref_countsketch_apply_f32(sz(1000), sz(3), P(Xs), sz(1000), sz(64), P(Ys), sz(64))
    np.savez_compressed(os.path.join(HERE, "countsketch.npz"), X=Xs, Y=Ys, **out)

    rng = np.random.default_rng(5)
    SA = np.asfortranarray(rng.standard_normal((300, 40)) * np.logspace(0, 3, 40))
    W = SA.copy(order="F")
    R.ref_sketch_qr_f64(sz(300), sz(40), P(W))
    np.savez_compressed(os.path.join(HERE, "sketch_qr.npz"), SA=SA, Rinv=np.triu(W[:40, :40]))

    rng = np.random.default_rng(0)
    m, n = 2000, 50
    A = rng.standard_normal((m, n)).astype(np.float32)
    xt = rng.standard_normal(n).astype(np.float32)
    b = (A.astype(np.float64) @ xt + 1e-6 * rng.standard_normal(m)).astype(np.float32)
    x0, it0, h0 = oracle.ref_lsqr_f32(A, b, None, 1e-6, 400, 1e-6, 1)
    # Preconditioned by the reference's own sketch QR (FP64) of the hash sketch.
    Ssk = np.zeros((200, n), np.float64, order="F")
    A64 = np.asfortranarray(A.astype(np.float64))
    R.ref_countsketch_apply_f64(sz(m), sz(n), P(A64), sz(m), sz(200), P(Ssk), sz(200))
    Wq = Ssk.copy(order="F")
    R.ref_sketch_qr_f64(sz(200), sz(n), P(Wq))
    Rinv = np.triu(Wq[:n, :n])
    x1, it1, h1 = oracle.ref_lsqr_f32(A, b, Rinv.astype(np.float32), 1e-6, 400, 1e-6, 1)
    np.savez_compressed(os.path.join(HERE, "lsqr_small.npz"), A=A, b=b, x_plain=x0, it_plain=it0,
                        hist_plain=h0, Rinv=Rinv, x_precond=x1, it_precond=it1, hist_precond=h1)

    rng = np.random.default_rng(101)
    mm, nn = 37, 23
    Am = (rng.uniform(-8, 8, (mm, nn)) * np.where(rng.random((mm, nn)) < 0.1, 1e-4, 1.0)).astype(np.float32)
    Af = np.asfortranarray(Am)
    h = np.empty(mm * nn, np.uint16); r = np.empty(mm * nn, np.uint16)
    Aflat = Af.ravel(order="K")
    R.ref_fp32_16_split(P(Aflat), mm * nn, P(h), P(r))
    xv = rng.uniform(-8, 8, nn).astype(np.float32)
    xt2 = rng.uniform(-8, 8, mm).astype(np.float32)
    res = {}
    for tier in (0, 1, 2):
        y = np.zeros(mm, np.float32)
        R.ref_mv_fp32_16(tier, 0, 1.0, sz(mm), sz(nn), P(h), P(r), sz(mm), P(xv), 0.0, P(y))
        yt = np.zeros(nn, np.float32)
        R.ref_mv_fp32_16(tier, 1, 1.0, sz(mm), sz(nn), P(h), P(r), sz(mm), P(xt2), 0.0, P(yt))
        res[f"y{tier}"] = y
        res[f"yt{tier}"] = yt
    np.savez_compressed(os.path.join(HERE, "mv_fp32_16.npz"), A=Am, x=xv, xt=xt2, **res)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
