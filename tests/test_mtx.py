"""MatrixMarket files (tomos_mtx_*): the reference's read_mtx_host
(benchmarks/solvers/cuda/lsqr_precision_runner.cu:101-125, over
src/io/mmio.c) reads `array real general` files, one value per line
column by column, as scripts/generate_tall_thin_mtx.m writes them
(fprintf '%1.16e').  Checked bit for bit against Python's correctly rounded
parsing and against scipy.io.mmread; the other formats against scipy."""
import os

import numpy as np
import pytest
import scipy.io
import scipy.sparse

import tomos_b200 as tb
from tomos_b200 import _capi as C


def write_text(path, text):
    with open(path, "w") as f:
        f.write(text)
    return str(path)


def matlab_style(path, A):
    """The generator's format: banner, 'M N', '%1.16e' values column-major."""
    m, n = A.shape
    lines = ["%%MatrixMarket matrix array real general", f"{m} {n}"]
    lines += ["%1.16e" % v for v in np.asarray(A, np.float64).ravel(order="F")]
    return write_text(path, "\n".join(lines) + "\n")


def test_generator_format_bit_exact(tmp_path):
    rng = np.random.default_rng(0)
    A = rng.standard_normal((37, 11)) * 10.0 ** rng.uniform(-8, 8, (37, 11))
    A[0, 0], A[1, 0], A[2, 0] = -0.0, 1.0 / 3.0, 5e-324
    p = matlab_style(tmp_path / "a.mtx", A)
    got = tb.read_mtx(p)
    want = np.array([float("%1.16e" % v) for v in A.ravel(order="F")]).reshape(A.shape, order="F")
    assert got.flags["F_CONTIGUOUS"] and got.shape == A.shape
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    assert np.array_equal(got, scipy.io.mmread(p))
    info = tb.mtx_info(p)
    assert info == {"rows": 37, "cols": 11, "entries": 37 * 11, "format": 0, "field": 0, "symmetry": 0}
    rm = tb.read_mtx(p, tb.Layout.ROW_MAJOR)
    assert rm.flags["C_CONTIGUOUS"] and np.array_equal(rm, got)


def test_write_read_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    A = rng.standard_normal((20, 7)) * 10.0 ** rng.uniform(-300, 300, (20, 7))
    p = str(tmp_path / "w.mtx")
    tb.write_mtx(p, A)
    assert np.array_equal(tb.read_mtx(p).view(np.uint64), A.view(np.uint64))
    assert np.array_equal(scipy.io.mmread(p), A)


def test_coordinate_comments_and_repeats(tmp_path):
    p = write_text(tmp_path / "c.mtx", """%%MatrixMarket matrix coordinate real general
% a comment
%another

4 3 6
1 1 1.5
4 3 -2.25e-3
2 2 7
1 1 0.5
3 1 1e10
4 2 -0
""")
    want = scipy.io.mmread(p).toarray()
    assert np.array_equal(tb.read_mtx(p), want)
    r, c, v = tb.read_mtx_coo(p)
    assert list(r) == [0, 3, 1, 0, 2, 3] and list(c) == [0, 2, 1, 0, 0, 1]
    rp, ci, vals, size = tb.read_mtx_csr(p)
    S = scipy.sparse.csr_matrix(scipy.io.mmread(p))
    S.sum_duplicates()
    S.sort_indices()
    assert size == (4, 3)
    assert np.array_equal(rp, S.indptr) and np.array_equal(ci, S.indices)
    assert np.array_equal(vals, S.data)


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate real symmetric\n3 3 4\n1 1 2\n2 1 -1\n3 2 4.5\n3 3 1\n",
    "%%MatrixMarket matrix coordinate real skew-symmetric\n3 3 2\n2 1 -1\n3 2 4.5\n",
    "%%MatrixMarket matrix coordinate integer general\n2 3 3\n1 3 7\n2 1 -4\n2 2 12\n",
    "%%MatrixMarket matrix coordinate pattern general\n3 2 3\n1 1\n3 2\n2 2\n",
    "%%MatrixMarket matrix array real symmetric\n3 3\n1\n2\n3\n4\n5\n6\n",
    "%%MatrixMarket matrix array real skew-symmetric\n3 3\n-1\n2.5\n3\n",
    "%%MatrixMarket matrix array integer general\n2 2\n1\n-2\n3\n4\n",
    "%%MATRIXMARKET MATRIX Array REAL General\n1 2\n3\n4\n",
])
def test_formats_match_scipy(tmp_path, text):
    text = text.replace("%%MATRIXMARKET", "%%MatrixMarket")
    p = write_text(tmp_path / "f.mtx", text)
    want = scipy.io.mmread(p, spmatrix=False)
    want = want.toarray() if scipy.sparse.issparse(want) else np.asarray(want)
    assert np.array_equal(tb.read_mtx(p), want.astype(np.float64))


@pytest.mark.parametrize("text,code,msg", [
    ("not a banner\n2 2\n1\n2\n3\n4\n", C.TOMOS_ERR_INVALID, "not a valid MatrixMarket file"),
    ("%%MatrixMarket matrix array real general\n% only a comment\n", C.TOMOS_ERR_INVALID,
     "could not read array size"),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n", C.TOMOS_ERR_INVALID,
     "truncated/malformed data"),
    ("%%MatrixMarket matrix array real general\n2 1\n1\nabc\n", C.TOMOS_ERR_INVALID,
     "truncated/malformed data"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", C.TOMOS_ERR_INVALID,
     "outside the matrix"),
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", C.TOMOS_ERR_UNSUPPORTED,
     "not supported"),
    ("%%MatrixMarket matrix array real hermitian\n1 1\n1\n", C.TOMOS_ERR_UNSUPPORTED, "not supported"),
])
def test_errors(tmp_path, text, code, msg):
    p = write_text(tmp_path / "e.mtx", text)
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx(p)
    assert e.value.code == code and msg in str(e.value)


def test_missing_file_and_capacity(tmp_path):
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx(str(tmp_path / "nope.mtx"))
    assert "could not open" in str(e.value)
    p = write_text(tmp_path / "c.mtx", "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n2 2 2\n")
    import ctypes
    cnt = ctypes.c_int64(0)
    rc = C.lib().tomos_mtx_read_coo(os.fsencode(p), 0, None, None, None, ctypes.byref(cnt))
    assert rc == C.TOMOS_ERR_INVALID and cnt.value == 2  # cap 0 sizes the call


@pytest.mark.gpu
def test_solve_from_mtx_files(tmp_path, orc):
    """An LSQR solve of a system read from .mtx files (dense and CSR)
    matches the oracle's FP64 least-squares solution."""
    import torch
    rng = np.random.default_rng(3)
    A = rng.standard_normal((3000, 60))
    A[rng.random(A.shape) < 0.7] = 0.0
    b = A @ rng.standard_normal(60) + 1e-8 * rng.standard_normal(3000)
    pa = matlab_style(tmp_path / "A.mtx", A)
    pb = matlab_style(tmp_path / "b.mtx", b[:, None])
    Ah = tb.read_mtx(pa)
    bh = tb.read_mtx(pb)[:, 0].astype(np.float32)
    xo = orc.lstsq_f64(Ah.astype(np.float32).astype(np.float64), bh.astype(np.float64))
    S = scipy.sparse.coo_matrix(Ah)
    pc = str(tmp_path / "S.mtx")
    scipy.io.mmwrite(pc, S, precision=17)
    for M in (tb.dense_from_mtx(pa, tb.NumericType.FP32, tb.Layout.COL_MAJOR),
              tb.dense_from_mtx(pa, tb.NumericType.FP32, tb.Layout.ROW_MAJOR),
              tb.csr_from_mtx(pc, tb.NumericType.FP32)):
        ws = tb.create_lsqr_workspace(None, (3000, 60), tb.NumericType.FP32)
        x = torch.zeros(60, device="cuda")
        rep = tb.lsqr_solve(None, M, torch.from_numpy(bh).cuda(), x, ws, 1e-6, 400, 1e-6)
        assert rep["converged"] == 1
        xx = x.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(xx - xo) / np.linalg.norm(xo) < 1e-4


# ---- the parallel `array` reader: byte ranges parsed by host threads ----

THREADS = [1, 2, 3, 7, 64]


def generator_values(m, n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((m, n)) * 10.0 ** rng.uniform(-12, 12, (m, n))
    A.ravel()[:4] = [-0.0, 5e-324, 1.0 / 3.0, -1e308]
    return A


@pytest.mark.parametrize("threads", THREADS)
def test_array_parallel_bit_exact(tmp_path, monkeypatch, threads):
    """Every thread count gives the sequential parse bit for bit: value t of
    the file lands at (t % m, t / m) whichever range it was parsed in."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    A = generator_values(257, 13, threads)
    p = matlab_style(tmp_path / "p.mtx", A)
    want = np.array([float("%1.16e" % v) for v in A.ravel(order="F")]).reshape(A.shape, order="F")
    for layout in (tb.Layout.COL_MAJOR, tb.Layout.ROW_MAJOR):
        got = tb.read_mtx(p, layout)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (threads, layout)


@pytest.mark.parametrize("threads", THREADS)
def test_array_parallel_layout_of_text(tmp_path, monkeypatch, threads):
    """Several values a line, tabs, blank lines, CRLF endings and trailing
    text past the last value read as the one-value-a-line file does."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    rng = np.random.default_rng(5)
    A = rng.standard_normal((31, 9))
    vals = ["%.17g" % v for v in A.ravel(order="F")]
    out, k = [], 0
    while k < len(vals):
        w = int(rng.integers(1, 5))
        sep = "\t" if rng.random() < 0.3 else "  "
        out.append(sep.join(vals[k:k + w]) + ("\r" if rng.random() < 0.5 else ""))
        if rng.random() < 0.2:
            out.append("")
        k += w
    text = "%%MatrixMarket matrix array real general\n31 9\n" + "\n".join(out) + "\n7 8 9 extra\n"
    p = write_text(tmp_path / "w.mtx", text)
    assert np.array_equal(tb.read_mtx(p), A)


@pytest.mark.parametrize("threads", THREADS)
@pytest.mark.parametrize("sym", ["symmetric", "skew-symmetric"])
def test_array_parallel_symmetric(tmp_path, monkeypatch, threads, sym):
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    rng = np.random.default_rng(7)
    n = 40
    L_ = np.tril(rng.standard_normal((n, n)), 0 if sym == "symmetric" else -1)
    stored = [L_[i, j] for j in range(n) for i in range(j if sym == "symmetric" else j + 1, n)]
    text = f"%%MatrixMarket matrix array real {sym}\n{n} {n}\n" + "\n".join("%.17g" % v for v in stored) + "\n"
    p = write_text(tmp_path / "s.mtx", text)
    want = L_ + (L_.T if sym == "symmetric" else -L_.T)
    if sym == "symmetric":
        want[np.diag_indices(n)] = np.diag(L_)
    got = tb.read_mtx(p)
    assert np.array_equal(got, want)
    assert np.array_equal(got, scipy.io.mmread(p))


@pytest.mark.parametrize("threads", THREADS)
def test_array_parallel_errors(tmp_path, monkeypatch, threads):
    """A value short, or a malformed value in the middle of the file, is
    reported whichever range holds it."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    vals = ["%.17g" % v for v in np.arange(1.0, 601.0)]
    head = "%%MatrixMarket matrix array real general\n20 30\n"
    short = write_text(tmp_path / "short.mtx", head + "\n".join(vals[:-1]) + "\n")
    bad_vals = list(vals)
    bad_vals[377] = "1.5e"
    bad = write_text(tmp_path / "bad.mtx", head + "\n".join(bad_vals) + "\n")
    for p in (short, bad):
        with pytest.raises(tb.TomosError) as e:
            tb.read_mtx(p)
        assert e.value.code == C.TOMOS_ERR_INVALID and "truncated/malformed data" in str(e.value)
    ok = write_text(tmp_path / "ok.mtx", head + "\n".join(vals) + "\nnot-a-number\n")
    assert np.array_equal(tb.read_mtx(ok), np.arange(1.0, 601.0).reshape(20, 30, order="F"))


def test_array_parallel_large_default_threads(tmp_path, monkeypatch):
    """A ~15 MB generator file (several ranges at the default thread count)
    reads bit-exactly."""
    monkeypatch.delenv("TOMOS_MTX_THREADS", raising=False)
    A = generator_values(3000, 200, 11)
    p = matlab_style(tmp_path / "big.mtx", A)
    want = np.array([float("%1.16e" % v) for v in A.ravel(order="F")]).reshape(A.shape, order="F")
    got = tb.read_mtx(p)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def coordinate_text(rng, m, n, nnz, field, split_lines=False):
    r = rng.integers(1, m + 1, nnz)
    c = rng.integers(1, n + 1, nnz)
    if field == "real":
        vals = ["%.17g" % x for x in rng.standard_normal(nnz) * 10.0 ** rng.uniform(-5, 5, nnz)]
    elif field == "integer":
        vals = [str(int(x)) for x in rng.integers(-1000, 1000, nnz)]
    else:
        vals = [None] * nnz
    lines = []
    for a, b, v in zip(r, c, vals):
        toks = [str(a), str(b)] + ([v] if v is not None else [])
        if split_lines and rng.random() < 0.3:
            lines.append(toks[0])
            lines.append("  ".join(toks[1:]))
        else:
            lines.append("\t".join(toks) if rng.random() < 0.2 else " ".join(toks))
    head = f"%%MatrixMarket matrix coordinate {field} general\n% comment\n{m} {n} {nnz}\n"
    return head + "\n".join(lines) + "\n", r - 1, c - 1, vals


@pytest.mark.parametrize("threads", THREADS)
@pytest.mark.parametrize("field", ["real", "integer", "pattern"])
def test_coordinate_parallel_triplets(tmp_path, monkeypatch, threads, field):
    """General coordinate files read by every thread count give the file's
    triplets in file order (entries whose tokens straddle two byte ranges or
    two lines included)."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    rng = np.random.default_rng(threads)
    text, r, c, vals = coordinate_text(rng, 70, 50, 900, field, split_lines=True)
    p = write_text(tmp_path / "c.mtx", text)
    gr, gc, gv = tb.read_mtx_coo(p)
    assert np.array_equal(gr, r) and np.array_equal(gc, c)
    want = np.ones(len(r)) if field == "pattern" else np.array([float(v) for v in vals])
    assert np.array_equal(gv.view(np.uint64), want.view(np.uint64))
    rp, ci, vv, size = tb.read_mtx_csr(p)
    S = scipy.sparse.coo_matrix((want, (r, c)), shape=(70, 50)).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    assert size == (70, 50) and np.array_equal(rp, S.indptr) and np.array_equal(ci, S.indices)
    np.testing.assert_allclose(vv, S.data, rtol=1e-15)


@pytest.mark.parametrize("threads", THREADS)
def test_coordinate_parallel_errors(tmp_path, monkeypatch, threads):
    """The first bad entry in file order is the one reported, whichever
    range holds it: out of the matrix (by its 1-based number), malformed,
    or missing."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    rng = np.random.default_rng(9)
    text, r, c, vals = coordinate_text(rng, 40, 30, 400, "real")
    head, body = text.split("40 30 400\n")
    lines = body.rstrip("\n").split("\n")

    def with_lines(name, ls, nnz=400):
        return write_text(tmp_path / name, head + f"40 30 {nnz}\n" + "\n".join(ls) + "\n")

    out = list(lines)
    out[250] = "41 3 1.0"
    out[300] = "1 2 x"
    p = with_lines("out.mtx", out)
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx_coo(p)
    assert "entry 251 lies outside the matrix" in str(e.value)
    mal = list(lines)
    mal[120] = "3 4 1.0e"
    mal[300] = "0 2 1.0"
    p = with_lines("mal.mtx", mal)
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx_coo(p)
    assert "truncated/malformed data" in str(e.value)
    p = with_lines("short.mtx", lines[:-1])
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx_coo(p)
    assert "truncated/malformed data" in str(e.value)
    p = with_lines("idx.mtx", lines[:7] + ["3.0 4 1.0"] + lines[8:])
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx_coo(p)
    assert "truncated/malformed data" in str(e.value)


@pytest.mark.parametrize("threads", [1, 3, 64])
@pytest.mark.parametrize("layout", ["F", "C"])
def test_write_parallel_bytes(tmp_path, monkeypatch, threads, layout):
    """The writer's blocks, formatted by any number of threads, give the
    bytes of a sequential '%.17g' a line (more values than one block of
    2^18, so several blocks and rounds), and read back bit for bit."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    A = generator_values(1000, 600, threads)
    A.ravel()[5:8] = [np.inf, -np.inf, 0.0]
    A = np.asarray(A, order=layout)
    p = str(tmp_path / "w.mtx")
    tb.write_mtx(p, A)
    want = "%%MatrixMarket matrix array real general\n1000 600\n" + \
        "".join("%.17g\n" % v for v in A.ravel(order="F"))
    assert open(p).read() == want
    assert np.array_equal(tb.read_mtx(p).view(np.uint64), np.asfortranarray(A).view(np.uint64))


@pytest.mark.parametrize("threads", THREADS)
def test_coordinate_dense_parallel_repeats(tmp_path, monkeypatch, threads):
    """A general coordinate file read into a dense matrix: triplets parsed
    by any number of threads, repeated positions summed in file order (the
    sequential sum's bits)."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    rng = np.random.default_rng(21)
    text, r, c, vals = coordinate_text(rng, 12, 9, 700, "real", split_lines=True)
    p = write_text(tmp_path / "d.mtx", text)
    want = np.zeros((12, 9))
    for a, b, v in zip(r, c, vals):
        want[a, b] += float(v)
    got = tb.read_mtx(p)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.timeout(120)
@pytest.mark.parametrize("kind", ["array", "coordinate"])
def test_pipe_reads_sequentially(tmp_path, kind):
    """A file that cannot be mapped (a named pipe) is read by the
    sequential reader, with the same result (one open of the pipe: the C
    entries are called directly)."""
    import ctypes
    import threading
    if kind == "array":
        A = generator_values(50, 7, 3)
        text = "%%MatrixMarket matrix array real general\n50 7\n" + \
            "".join("%1.16e\n" % v for v in A.ravel(order="F"))
    else:
        text, r, c, vals = coordinate_text(np.random.default_rng(4), 30, 20, 200, "real")
    assert len(text) < 60000  # fits the pipe's buffer: the writer never waits on the reader
    fifo = str(tmp_path / "pipe.mtx")
    os.mkfifo(fifo)

    def serve():
        with open(fifo, "w") as f:
            f.write(text)

    th = threading.Thread(target=serve, daemon=True)
    th.start()
    if kind == "array":
        want = np.array([float("%1.16e" % v) for v in A.ravel(order="F")]).reshape(A.shape, order="F")
        out = np.zeros((50, 7), order="F")
        C.check(C.lib().tomos_mtx_read_dense(os.fsencode(fifo), int(tb.Layout.COL_MAJOR), out.ctypes.data, 50))
        assert np.array_equal(out.view(np.uint64), want.view(np.uint64))
    else:
        rr = np.zeros(200, np.int64)
        cc = np.zeros(200, np.int64)
        vv = np.zeros(200)
        cnt = ctypes.c_int64(0)
        C.check(C.lib().tomos_mtx_read_coo(os.fsencode(fifo), 200, rr.ctypes.data, cc.ctypes.data,
                                           vv.ctypes.data, ctypes.byref(cnt)))
        assert cnt.value == 200 and np.array_equal(rr, r) and np.array_equal(cc, c)
        assert np.array_equal(vv, np.array([float(v) for v in vals]))
    th.join(timeout=30)


EMPTY_DATA = [
    ("array", "%%MatrixMarket matrix array real general\n3 2\n"),
    ("array", "%%MatrixMarket matrix array real general\n3 2"),
    ("general", "%%MatrixMarket matrix coordinate real general\n3 3 2\n"),
    ("general", "%%MatrixMarket matrix coordinate real general\n3 3 2"),
    ("general", "%%MatrixMarket matrix coordinate real general\n3 3 2\n\n  \n"),
    ("pattern", "%%MatrixMarket matrix coordinate pattern general\n4 4 3\n"),
]


@pytest.mark.parametrize("threads", [1, 64])
@pytest.mark.parametrize("kind,text", EMPTY_DATA)
def test_empty_data_section(tmp_path, monkeypatch, threads, kind, text):
    """A size line promising values or entries with nothing after it is
    'truncated/malformed data' for every reader (dense, COO, CSR), at any
    thread count -- never a crash."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    p = write_text(tmp_path / "e.mtx", text)
    readers = [tb.read_mtx] if kind == "array" else [tb.read_mtx, tb.read_mtx_coo, tb.read_mtx_csr]
    for rd in readers:
        with pytest.raises(tb.TomosError) as e:
            rd(p)
        assert "truncated/malformed data" in str(e.value)


@pytest.mark.timeout(120)
@pytest.mark.parametrize("kind", ["array", "coordinate"])
def test_long_token_rejected_by_both_readers(tmp_path, kind):
    """A token longer than 127 characters is malformed whether the file is
    mapped (parallel reader) or read from a pipe (sequential reader)."""
    import ctypes
    import threading
    long_num = "1." + "0" * 200
    if kind == "array":
        text = "%%MatrixMarket matrix array real general\n2 1\n" + long_num + "\n2.0\n"
    else:
        text = "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 " + long_num + "\n2 2 1.0\n"
    p = write_text(tmp_path / "long.mtx", text)
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx(p)
    assert "truncated/malformed data" in str(e.value)
    fifo = str(tmp_path / "long_pipe.mtx")
    os.mkfifo(fifo)

    def serve():
        with open(fifo, "w") as f:
            f.write(text)

    th = threading.Thread(target=serve, daemon=True)
    th.start()
    if kind == "array":
        out = np.zeros((2, 1), order="F")
        rc = C.lib().tomos_mtx_read_dense(os.fsencode(fifo), int(tb.Layout.COL_MAJOR), out.ctypes.data, 2)
    else:
        rr = np.zeros(2, np.int64)
        cc = np.zeros(2, np.int64)
        vv = np.zeros(2)
        cnt = ctypes.c_int64(0)
        rc = C.lib().tomos_mtx_read_coo(os.fsencode(fifo), 2, rr.ctypes.data, cc.ctypes.data,
                                        vv.ctypes.data, ctypes.byref(cnt))
    th.join(timeout=30)
    assert rc != 0
    assert "truncated/malformed data" in C.lib().tomos_last_error().decode()


@pytest.mark.parametrize("threads", [1, 64])
def test_long_index_token_rejected(tmp_path, monkeypatch, threads):
    """An index token of 128+ digits is malformed in both readers (the
    sequential reader no longer reads a prefix of it)."""
    monkeypatch.setenv("TOMOS_MTX_THREADS", str(threads))
    text = "%%MatrixMarket matrix coordinate real symmetric\n2 2 1\n" + "0" * 140 + "1 1 1.0\n"
    p = write_text(tmp_path / "li.mtx", text)
    with pytest.raises(tb.TomosError) as e:
        tb.read_mtx(p)
    assert "truncated/malformed data" in str(e.value)
