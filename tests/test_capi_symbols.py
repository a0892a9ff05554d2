"""The C-ABI library loads and exports every function ``include/oceansar_b200.h`` declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "oceansar_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(ocs_[a-z0-9_]+)\s*\(", hdr)))


@pytest.fixture(scope="module")
def lib():
    from oceansar_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_functions():
    assert "ocs_chan_profile_f64" in declared_functions()


def test_every_declared_symbol_is_exported(lib):
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_python_binding_covers_header():
    from oceansar_b200 import _capi
    assert sorted(_capi.SIGNATURES) == declared_functions()


def test_version_string(lib):
    lib.ocs_version.restype = ctypes.c_char_p
    assert lib.ocs_version().decode().count(".") == 2


def test_argument_errors_need_no_gpu(lib):
    # null pointers are rejected before any CUDA call
    f = lib.ocs_chan_profile_f64
    f.restype = ctypes.c_int
    st = f(None, None, ctypes.c_int64(10), ctypes.c_double(1.0), ctypes.c_double(0.0), None,
           ctypes.c_int(8), ctypes.c_int(20), None, ctypes.c_int64(16), None)
    assert st == -1
