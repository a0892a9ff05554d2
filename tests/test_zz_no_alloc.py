"""The allocation-free surface update gives the same fields as the ordinary entry point.

``ocs_surface_update_noalloc`` exists for callers that cannot allocate device memory (a
bare C-ABI host with no allocator of its own, or a loop that must never block on an
allocation): it takes its workspace from a device array compiled into the library instead
of a caller-provided buffer.  This test calls both entry points through the C ABI on the
same inputs, twice in a row with different times, and compares the fields at the
tolerance of the surface tests.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

L2_TOL = 2e-6


def _rel(a, b):
    return float(torch.linalg.norm((a - b).double()) / torch.linalg.norm(b.double()))


def test_noalloc_matches_workspace_entry_point():
    from oceansar_b200 import _capi, build
    from oceansar_b200.surfaces import OceanSurface
    from oceansar_b200.surfaces.ocean import CODES, SurfaceDesc
    build.build()
    np.random.seed(3)
    s = OceanSurface()
    s.init(Lx=512., Ly=512., dx=1., dy=1., cutoff_wl='auto', spec_model='elfouhaily',
           spread_model='elfouhaily', wind_dir=0.4, wind_fetch=500e3, wind_U=9., current_mag=0.1,
           current_dir=0.2, compute=['D', 'Diff', 'Diff2'], opt_res=True, fft_max_prime=2)
    names = ['Dx', 'Dy', 'Dz', 'Diffx', 'Diffy', 'Diffxx', 'Diffyy', 'Diffxy']
    n = len(names)
    shape = (s.Ny, s.Nx)
    ref = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in names]
    got = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in names]
    ws_bytes = _capi.load().ocs_surface_workspace_bytes(s.Nx, s.Ny, n)
    assert 0 < ws_bytes <= (32 << 20)
    ws = torch.empty(int(ws_bytes), dtype=torch.uint8, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_surface_prepare", s.Nx, s.Ny, ctypes.c_void_p(ws.data_ptr()), stream)
    codes = (ctypes.c_int32 * n)(*[CODES[k] for k in names])

    def desc(outs, t, workspace):
        add = (ctypes.c_float * n)(*[float(s.current[0] * np.float32(t)) if k == 'Dx' else
                                     float(s.current[1] * np.float32(t)) if k == 'Dy' else 0.0
                                     for k in names])
        dst = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
        d = SurfaceDesc(s.Nx, s.Ny, s._coefs_d.data_ptr(), s._omega_d.data_ptr(), s._kx_d.data_ptr(),
                        s._ky_d.data_ptr(), float(s.kmin_half), n, codes, dst, add, None, None, 0.0, 0.0,
                        workspace)
        return d, (add, dst)

    for t in (0.3, 1.7):                                   # two calls in a row
        for o in got:
            o.fill_(float('nan'))
        d_ref, keep_ref = desc(ref, t, ws.data_ptr())
        _capi.call("ocs_surface_update", ctypes.addressof(d_ref), ctypes.c_float(t), stream)
        d_new, keep_new = desc(got, t, None)
        _capi.call("ocs_surface_update_noalloc", ctypes.addressof(d_new), ctypes.c_float(t), stream)
        torch.cuda.synchronize()
        for name, a, b in zip(names, got, ref):
            assert torch.isfinite(a).all(), name
            assert _rel(a, b) <= L2_TOL, (name, t, _rel(a, b))


def test_noalloc_rejects_oversized_requests():
    from oceansar_b200 import _capi
    from oceansar_b200.surfaces.ocean import SurfaceDesc
    codes = (ctypes.c_int32 * 8)(*range(8))
    d = SurfaceDesc(4096, 4096, 1, 1, 1, 1, 0.0, 8, codes, None, None, None, None, 0.0, 0.0, None)
    st = _capi.load().ocs_surface_update_noalloc(ctypes.addressof(d), ctypes.c_float(0.0), None)
    assert st == -3                                          # OCS_ERR_SIZE, nothing launched
