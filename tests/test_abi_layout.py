"""The Python binding's ctypes structures against include/gpe.h (CPU).

gpe.py mirrors gpe_params, gpe_tuning, gpe_request and gpe_result field by
field; a field added to the header but not to the mirror (or in another order)
would shift every later field of the call.  A small C program compiled here
against the header prints each structure's size and each field's offset, and
the test compares them with the ctypes layout (equal sizes also rule out a
header field after the last mirrored one).
"""
import ctypes as C
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

# C name of the struct, name of the ctypes mirror; Python names that differ
# from the C ones (lambda is a Python keyword)
STRUCTS = [("gpe_params", "Params"), ("gpe_tuning", "Tuning"), ("gpe_request", "Request"), ("gpe_result", "Result")]
RENAME = {"lamda": "lambda"}


def _c_layout(tmp_path, gpe):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "gpe.h"', "int main(void) {"]
    for cname, pyname in STRUCTS:
        lines.append('   printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in getattr(gpe, pyname)._fields_:
            cf = RENAME.get(fname, fname)
            lines.append('   printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, cf))
    lines += ["   return 0;", "}"]
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for ln in out.splitlines():
        cname, key, val = ln.split()
        layout[(cname, key)] = int(val)
    return layout


def test_ctypes_mirrors_match_the_header(gpe_lib, tmp_path):
    gpe = gpe_lib
    layout = _c_layout(tmp_path, gpe)
    for cname, pyname in STRUCTS:
        cls = getattr(gpe, pyname)
        assert C.sizeof(cls) == layout[(cname, "sizeof")], cname
        for fname, _ in cls._fields_:
            assert getattr(cls, fname).offset == layout[(cname, fname)], (cname, fname)

