"""Seeded synthetic least-squares problems with the benchmark shapes.

The reference ships no test matrices (its MATLAB generator,
scripts/generate_tall_thin_mtx.m, is not runnable here), so the workloads
are generated:

  dense_gaussian   A ~ N(0,1), b = A x_true + noise          (20000 x 200)
  dense_scaled     A = G diag(10^u), G ~ N(0,1), u ~ U(-3,3)  (1e6 x 1000,
                   condition number about 1e6), b = A x_true + noise
  csr_scaled       20 distinct random columns per row, values N(0,1)
                   times a row scale 10^U(-2,2)

Everything is generated on the GPU from a seeded torch generator, in
row blocks, so the 4 GB problems never touch host memory.  b is formed
with FP64 accumulation.
"""
import torch


def _gen(seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed))
    return g


def dense_gaussian(m, n, seed=0, noise=1e-6, layout="row"):
    """A (m x n float32, row-major tensor), x_true, b (float32 CUDA)."""
    g = _gen(seed)
    A = torch.randn(m, n, generator=g, device="cuda", dtype=torch.float32)
    x = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
    e = torch.randn(m, generator=g, device="cuda", dtype=torch.float64)
    b = (A.double() @ x.double() + noise * e).float()
    return A, x, b


def dense_scaled(m, n, seed=0, noise=1e-8, decades=3.0, block_rows=1 << 17, out=None):
    """A = G diag(10^u) (m x n float32 row-major), x_true, b.

    Generated in row blocks of block_rows; `out` may be a preallocated
    (m, n) float32 CUDA tensor to fill."""
    g = _gen(seed)
    u = (torch.rand(n, generator=g, device="cuda", dtype=torch.float64) * 2.0 - 1.0) * decades
    scale = torch.pow(10.0, u)
    x = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
    A = out if out is not None else torch.empty(m, n, device="cuda", dtype=torch.float32)
    b = torch.empty(m, device="cuda", dtype=torch.float32)
    xd = x.double()
    for r0 in range(0, m, block_rows):
        r1 = min(m, r0 + block_rows)
        blk = torch.randn(r1 - r0, n, generator=g, device="cuda", dtype=torch.float64) * scale
        A[r0:r1] = blk.float()
        e = torch.randn(r1 - r0, generator=g, device="cuda", dtype=torch.float64)
        b[r0:r1] = (A[r0:r1].double() @ xd + noise * e).float()
        del blk
    return A, x, b


def csr_scaled(m, n, nnz_per_row=20, seed=0, noise=1e-8, decades=2.0):
    """CSR (row_ptrs int32, col_idxs int32, values float32), x_true, b."""
    g = _gen(seed)
    # distinct columns per row: sample nnz_per_row + slack, keep the first
    # distinct ones in sorted order (rejection on collisions is rare)
    cols = torch.randint(0, n, (m, nnz_per_row * 2), generator=g, device="cuda")
    cols, _ = torch.sort(cols, dim=1)
    dup = torch.zeros_like(cols, dtype=torch.bool)
    dup[:, 1:] = cols[:, 1:] == cols[:, :-1]
    key = cols.masked_fill(dup, n)  # duplicates pushed to the end
    key, _ = torch.sort(key, dim=1)
    cols = key[:, :nnz_per_row]
    if bool((cols >= n).any()):
        raise RuntimeError("csr_scaled: not enough distinct columns sampled")
    rs = torch.pow(10.0, (torch.rand(m, generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * decades)
    vals = (torch.randn(m, nnz_per_row, generator=g, device="cuda", dtype=torch.float64) * rs[:, None])
    x = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
    b = (vals * x.double()[cols]).sum(dim=1)
    b = (b + noise * torch.randn(m, generator=g, device="cuda", dtype=torch.float64)).float()
    row_ptrs = torch.arange(0, (m + 1) * nnz_per_row, nnz_per_row, device="cuda", dtype=torch.int32)
    return row_ptrs, cols.reshape(-1).to(torch.int32).contiguous(), vals.reshape(-1).float().contiguous(), x, b
