"""The ctypes mirrors in nopt_b200.rijk of the C-ABI structs in include/rijk.h (rijk_stats_t,
rijk_basis_t, rijk_scf_opts_t, rijk_scf_result_t): every field at the C compiler's offset, and the
same total size, so fields appended to the header are appended to the mirror too.  The C side is
compiled here with gcc from the header alone (no library, no GPU)."""
import ctypes
import os
import shutil
import subprocess
import tempfile

import pytest

from nopt_b200 import rijk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MIRRORS = {"rijk_stats_t": rijk.Stats, "rijk_basis_t": rijk.BasisT, "rijk_scf_opts_t": rijk.ScfOpts,
           "rijk_scf_result_t": rijk.ScfResult}


def _c_layout():
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "rijk.h"', "int main(void) {"]
    for cname, py in MIRRORS.items():
        lines.append('  printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in py._fields_:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines += ["  return 0;", "}"]
    d = tempfile.mkdtemp()
    try:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True,
                       capture_output=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    finally:
        shutil.rmtree(d)
    got = {}
    for ln in out.splitlines():
        cname, field, value = ln.split()
        got[(cname, field)] = int(value)
    return got


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header():
    c = _c_layout()
    for cname, py in MIRRORS.items():
        for f in py._fields_:
            assert getattr(py, f[0]).offset == c[(cname, f[0])], (cname, f[0])
        assert ctypes.sizeof(py) == c[(cname, "sizeof")], cname
