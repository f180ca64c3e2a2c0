"""The C ABI libraries load and export every symbol their headers declare (no GPU needed).

No compute call is made here: only argument validation that precedes any CUDA call.
"""
import ctypes
import os
import re

import pytest

from nopt_b200 import ints, rijk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header, prefix):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(%s\w+)\s*\(" % prefix, src)))


@pytest.mark.parametrize("header,prefix,loader", [("rijk.h", "rijk_", rijk.lib), ("gto_ints.h", "gto_", ints.lib)])
def test_every_declared_symbol_is_exported(header, prefix, loader):
    L = loader()
    names = _declared(header, prefix)
    assert names, header
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_null_arguments_are_rejected_before_any_device_work():
    L = rijk.lib()
    assert L.rijk_create(None, 0) == rijk.ERR_ARG
    assert L.rijk_destroy(None) == rijk.ERR_ARG
    assert L.rijk_set_metric(None, None, 10, 0) == rijk.ERR_ARG
    assert L.rijk_set_3c(None, None, 10, 10, 0) == rijk.ERR_ARG
    assert L.rijk_fock(None, None, None, 1, None, None, 0) == rijk.ERR_ARG
    assert L.rijk_fock_device(None, None, None, 1, None, None, 0) == rijk.ERR_ARG
    buf = ctypes.create_string_buffer(16)
    assert L.rijk_last_error(None, buf, 16) == rijk.ERR_ARG


def test_product_library_is_cuda_only():
    """librijk links the CUDA runtime and holds sm_100a device code: no host fallback."""
    import subprocess
    out = subprocess.run(["readelf", "-d", rijk.lib_path()], capture_output=True, text=True).stdout
    assert "libcudart" in out
    sec = subprocess.run(["readelf", "-S", rijk.lib_path()], capture_output=True, text=True).stdout
    assert ".nv_fatbin" in sec
