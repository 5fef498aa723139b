"""The C-ABI library loads, exports every entry point include/tomos_b200.h
declares, and the ctypes mirrors of its structs match the C layout."""
import os
import re
import subprocess
import tempfile

import pytest

from tomos_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tomos_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tomos_[a-z0-9_]+)\s*\(", text)))


def test_library_loads():
    L = C.lib()
    assert b"sm_100a" in L.tomos_version()


def test_every_declared_symbol_is_exported():
    L = C.lib()
    fns = declared_functions()
    assert len(fns) >= 20
    missing = [f for f in fns if not hasattr(L, f)]
    assert not missing, missing
    assert set(fns) == set(C.SIGNATURES), set(fns) ^ set(C.SIGNATURES)


@pytest.mark.parametrize("struct,name", [(C.DenseDesc, "tomos_dense"), (C.CsrDesc, "tomos_csr"),
                                         (C.LsqrOpts, "tomos_lsqr_opts"),
                                         (C.LsqrReport, "tomos_lsqr_report"),
                                         (C.MtxInfo, "tomos_mtx_info")])
def test_struct_layout_matches_header(struct, name):
    fields = [f for f, _ in struct._fields_]
    body = "".join(
        f'printf("%zu %zu\\n", offsetof({name}, {f}), sizeof(((({name}*)0)->{f})));' for f in fields)
    src = ("#include <stdio.h>\n#include <stddef.h>\n#include \"tomos_b200.h\"\n"
           f"int main(void){{ printf(\"%zu\\n\", sizeof({name})); {body} return 0; }}\n")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    import ctypes
    assert int(out[0]) == ctypes.sizeof(struct)
    for i, f in enumerate(fields):
        off, size = map(int, out[1 + i].split())
        assert getattr(struct, f).offset == off, f
        assert getattr(struct, f).size == size, f


def test_errors_are_status_codes_not_exceptions():
    """Invalid arguments come back as TOMOS_ERR_INVALID with a message, on
    any machine (no device work is issued)."""
    import ctypes
    L = C.lib()
    rc = L.tomos_pack_fp32_16(None, 7, 4, 4, 4, None, None, 4, None, None)
    assert rc == C.TOMOS_ERR_INVALID
    assert b"layout" in L.tomos_last_error()
    d = C.DenseDesc()
    d.numeric = 4  # native BF16 storage has no kernel registered
    d.layout = 1
    d.rows = d.cols = d.ld = 4
    rc = L.tomos_gemv(0, 1.0, ctypes.byref(d), 0, None, 0.0, None, None, 0, None)
    assert rc == C.TOMOS_ERR_UNSUPPORTED
    rc = L.tomos_sketch_qr_precond_f64(3, 5, None, 3, None, None, 0, None)
    assert rc == C.TOMOS_ERR_INVALID
    assert b"k >= n" in L.tomos_last_error()
