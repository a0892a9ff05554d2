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


STRUCTS = [("ocs_surface_desc", "oceansar_b200.surfaces.ocean", "SurfaceDesc"),
           ("ocs_choppy_desc", "oceansar_b200.surfaces.ocean", "ChoppyDesc"),
           ("ocs_pulse_desc", "oceansar_b200._structs", "PulseDesc"),
           ("ocs_rcs_desc", "oceansar_b200._structs", "RcsDesc"),
           ("ocs_kodis_desc", "oceansar_b200._structs", "KodisDesc"),
           ("ocs_ka_desc", "oceansar_b200._structs", "KaDesc"),
           ("ocs_scene_desc", "oceansar_b200._structs", "SceneDesc")]


def test_python_descriptors_match_the_header(tmp_path):
    """Every ctypes descriptor has the size and field offsets of its C struct (the host C
    compiler lays the header out; no GPU needed)."""
    import importlib
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    expect = {}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "oceansar_b200.h"', 'int main(void) {']
    for cname, mod, pyname in STRUCTS:
        cls = getattr(importlib.import_module(mod), pyname)
        expect[cname] = cls
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split("\n")
    for line in filter(None, out):
        cname, field, value = line.split()
        cls = expect[cname]
        got = ctypes.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert got == int(value), (cname, field, got, int(value))
