"""Emit aborting C stubs for every symbol the reference's CPU objects leave
unresolved (its CUDA launchers, which this recipe never compiles).

Test infrastructure for oracle/Makefile.  The link is attempted with
--no-undefined; every mangled name the linker reports as missing gets a
stub that prints the symbol and aborts, so a CPU-Context call that ever
reached the CUDA path would fail loudly instead of silently.
"""
import argparse
import re
import subprocess
import sys


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--cxx", default="g++")
    ap.add_argument("--libs", default="")
    ap.add_argument("objs", nargs="+")
    a = ap.parse_args()
    cmd = [a.cxx, "-shared", "-Wl,--no-undefined", "-Wl,--no-demangle",
           "-o", "/dev/null"] + a.objs + a.libs.split()
    r = subprocess.run(cmd, capture_output=True, text=True)
    missing = sorted(set(re.findall(r"undefined reference to `([^']+)'", r.stderr)))
    lines = ["/* generated by gen_cuda_stubs.py -- do not edit */",
             "#include <stdio.h>", "#include <stdlib.h>",
             "static void oracle_ref_no_cuda(const char* s) {",
             '    fprintf(stderr, "oracle/_ref: CUDA path not built (%s)\\n", s);',
             "    abort();", "}"]
    for i, sym in enumerate(missing):
        lines.append(f'void oracle_stub_{i}(void) __asm__("{sym}");')
        lines.append(f'void oracle_stub_{i}(void) {{ oracle_ref_no_cuda("{sym}"); }}')
    open(a.out, "w").write("\n".join(lines) + "\n")
    print(f"gen_cuda_stubs: {len(missing)} stubs", file=sys.stderr)


if __name__ == "__main__":
    main()
