"""Seeded synthetic least-squares problems with the benchmark shapes.

The reference ships no test matrices (its MATLAB generator,
scripts/generate_tall_thin_mtx.m, is not runnable here), so the workloads
are generated:

  dense_gaussian   A ~ N(0,1), b = A x_true + noise          (20000 x 200)
  dense_scaled     A = G diag(10^u), G ~ N(0,1), u ~ U(-3,3)  (1e6 x 1000,
                   condition number about 1e6), b = A x_true + noise
  csr_scaled       20 distinct random columns per row, values N(0,1)
                   times a row scale 10^U(-2,2)
  ctr_scaled_rows  dense_scaled's distribution from a counter-based
                   generator: every entry is a function of (seed, row,
                   column), so any row block (a 200,000-row oracle
                   subsample, or the 4e6 x 2000 matrix block by block) is
                   reproducible on its own

Everything is generated on the GPU from a seeded torch generator, in
row blocks, so the 4 GB problems never touch host memory.  b is formed
with FP64 accumulation.
"""
import torch


def _gen(seed, device="cuda"):
    g = torch.Generator(device=device)
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


def dense_scaled(m, n, seed=0, noise=1e-8, decades=3.0, block_rows=1 << 17, out=None, device="cuda"):
    """A = G diag(10^u) (m x n float32 row-major), x_true, b.

    Generated in row blocks of block_rows; `out` may be a preallocated
    (m, n) float32 tensor to fill.  device="cpu" draws from torch's CPU
    generator instead (other values for the same seed)."""
    g = _gen(seed, device)
    u = (torch.rand(n, generator=g, device=device, dtype=torch.float64) * 2.0 - 1.0) * decades
    scale = torch.pow(10.0, u)
    x = torch.randn(n, generator=g, device=device, dtype=torch.float32)
    A = out if out is not None else torch.empty(m, n, device=device, dtype=torch.float32)
    b = torch.empty(m, device=device, dtype=torch.float32)
    xd = x.double()
    for r0 in range(0, m, block_rows):
        r1 = min(m, r0 + block_rows)
        blk = torch.randn(r1 - r0, n, generator=g, device=device, dtype=torch.float64) * scale
        A[r0:r1] = blk.float()
        e = torch.randn(r1 - r0, generator=g, device=device, dtype=torch.float64)
        b[r0:r1] = (A[r0:r1].double() @ xd + noise * e).float()
        del blk
    return A, x, b


def csr_scaled(m, n, nnz_per_row=20, seed=0, noise=1e-8, decades=2.0):
    """CSR (row_ptrs int32, col_idxs int32, values float32), x_true, b."""
    g = _gen(seed)
    # distinct uniform columns per row: sample twice as many, drop repeats,
    # keep a random nnz_per_row of the distinct ones (random priorities, so
    # the choice is not biased toward small indices), then sort them
    cols = torch.randint(0, n, (m, nnz_per_row * 2), generator=g, device="cuda")
    cols, _ = torch.sort(cols, dim=1)
    dup = torch.zeros_like(cols, dtype=torch.bool)
    dup[:, 1:] = cols[:, 1:] == cols[:, :-1]
    pri = torch.rand(cols.shape, generator=g, device="cuda").masked_fill(dup, 2.0)
    pick = torch.topk(pri, nnz_per_row, dim=1, largest=False).indices
    if bool((torch.gather(pri, 1, pick) >= 2.0).any()):
        raise RuntimeError("csr_scaled: not enough distinct columns sampled")
    cols, _ = torch.sort(torch.gather(cols, 1, pick), dim=1)
    rs = torch.pow(10.0, (torch.rand(m, generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * decades)
    vals = (torch.randn(m, nnz_per_row, generator=g, device="cuda", dtype=torch.float64) * rs[:, None])
    x = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
    b = (vals * x.double()[cols]).sum(dim=1)
    b = (b + noise * torch.randn(m, generator=g, device="cuda", dtype=torch.float64)).float()
    row_ptrs = torch.arange(0, (m + 1) * nnz_per_row, nnz_per_row, device="cuda", dtype=torch.int32)
    return row_ptrs, cols.reshape(-1).to(torch.int32).contiguous(), vals.reshape(-1).float().contiguous(), x, b


# ------------------------------------------------------------ counter-based
#
# splitmix64's finaliser on int64 tensors (two's-complement wrapping
# multiplies; >> is arithmetic on int64, so logical shifts are masked).

_M1 = 0xBF58476D1CE4E5B9 - (1 << 64)
_M2 = 0x94D049BB133111EB - (1 << 64)
_G = 0x9E3779B97F4A7C15 - (1 << 64)


def _shr(x, k):
    return (x >> k) & ((1 << (64 - k)) - 1)


def _mix(x):
    x = x + _G
    x = (x ^ _shr(x, 30)) * _M1
    x = (x ^ _shr(x, 27)) * _M2
    return x ^ _shr(x, 31)


def _unif(key):
    """(0, 1) FP64 from an int64 counter tensor."""
    return (_shr(_mix(key), 11).double() + 0.5) * (2.0 ** -53)


def _normal(key):
    """N(0, 1) FP64 (Box-Muller on two counters derived from key)."""
    u1 = _unif(2 * key)
    u2 = _unif(2 * key + 1)
    return torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * torch.pi * u2)


def _stream(seed, tag):
    """Offset of counter stream `tag`: a 26-bit hash of (seed, tag) above
    the 36 bits of an index (rows x columns < 2^36), so keys (and twice
    them) stay within int64."""
    h = int(_mix(torch.tensor([seed * 8 + tag], dtype=torch.int64)).item()) & ((1 << 26) - 1)
    return h << 36


def ctr_scaled_params(n, seed, decades=3.0):
    """(column scales 10^u, x_true) of ctr_scaled_rows (FP64, CUDA)."""
    j = torch.arange(n, device="cuda", dtype=torch.int64)
    u = (_unif(j + _stream(seed, 1)) * 2.0 - 1.0) * decades
    x = _normal(j + _stream(seed, 2)).float()
    return torch.pow(10.0, u), x


def ctr_scaled_rows(r0, r1, n, seed, noise=1e-8, decades=3.0, params=None):
    """Rows [r0, r1) of A = G diag(10^u) (G ~ N(0,1) entrywise from
    (seed, row, column)), and the same rows of b = A x_true + noise
    (FP64 products).  Returns (A block float32, b block float32)."""
    scale, x = params if params is not None else ctr_scaled_params(n, seed, decades)
    i = torch.arange(r0, r1, device="cuda", dtype=torch.int64)
    key = _stream(seed, 0) + i[:, None] * n + torch.arange(n, device="cuda", dtype=torch.int64)[None, :]
    A = (_normal(key) * scale[None, :]).float()
    e = _normal(i + _stream(seed, 3))
    b = (A.double() @ x.double() + noise * e).float()
    return A, b
