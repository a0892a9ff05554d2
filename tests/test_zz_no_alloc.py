"""The allocation-free surface update gives the same fields as the ordinary entry point.

``ocs_surface_update_noalloc`` exists for callers that cannot allocate device memory (a
bare C-ABI host with no allocator of its own, or a loop that must never block on an
allocation): it takes its workspace from a device array compiled into the library instead
of a caller-provided buffer.  These tests call both entry points through the C ABI on the
same inputs, twice in a row with different times, and require bit-identical fields (both
run the same kernels on the same inputs in the same order).  They cover a power-of-two
grid, a non-power-of-two grid (where the staged twiddle tables are not used), the largest
advertised case (1024 x 1024 with 6 fields, close to the 32 MiB limit) and alternating
grid sizes (stale shared state would show up there), and check that the calls allocate no
device memory.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NAMES8 = ['Dx', 'Dy', 'Dz', 'Diffx', 'Diffy', 'Diffxx', 'Diffyy', 'Diffxy']
NAMES6 = ['Dx', 'Dy', 'Dz', 'Diffx', 'Diffy', 'Diffxx']


def _surface(L, seed):
    from oceansar_b200.surfaces import OceanSurface
    np.random.seed(seed)
    pow2 = (L & (L - 1)) == 0
    s = OceanSurface()
    s.init(Lx=float(L), Ly=float(L), dx=1., dy=1., cutoff_wl='auto', spec_model='elfouhaily',
           spread_model='elfouhaily', wind_dir=0.4, wind_fetch=500e3, wind_U=9., current_mag=0.1,
           current_dir=0.2, compute=['D', 'Diff', 'Diff2'], opt_res=pow2, fft_max_prime=2)
    assert (s.Nx, s.Ny) == (L, L)
    return s


class _Case:
    """One surface with both entry points' output buffers and a caller-owned workspace for
    the ordinary entry point."""

    def __init__(self, L, names, seed):
        from oceansar_b200 import _capi
        from oceansar_b200.surfaces.ocean import CODES
        self.s = s = _surface(L, seed)
        self.names = names
        n = len(names)
        shape = (s.Ny, s.Nx)
        self.ref = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in names]
        self.got = [torch.empty(shape, dtype=torch.float32, device="cuda") for _ in names]
        ws_bytes = _capi.load().ocs_surface_workspace_bytes(s.Nx, s.Ny, n)
        assert 0 < ws_bytes <= (32 << 20)
        self.ws = torch.empty(int(ws_bytes), dtype=torch.uint8, device="cuda")
        self.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _capi.call("ocs_surface_prepare", s.Nx, s.Ny, ctypes.c_void_p(self.ws.data_ptr()), self.stream)
        self.codes = (ctypes.c_int32 * n)(*[CODES[k] for k in names])

    def desc(self, outs, t, workspace):
        from oceansar_b200.surfaces.ocean import SurfaceDesc
        s, names, n = self.s, self.names, len(self.names)
        add = (ctypes.c_float * n)(*[float(s.current[0] * np.float32(t)) if k == 'Dx' else
                                     float(s.current[1] * np.float32(t)) if k == 'Dy' else 0.0
                                     for k in names])
        dst = (ctypes.c_void_p * n)(*[o.data_ptr() for o in outs])
        d = SurfaceDesc(s.Nx, s.Ny, s._coefs_d.data_ptr(), s._omega_d.data_ptr(), s._kx_d.data_ptr(),
                        s._ky_d.data_ptr(), float(s.kmin_half), n, self.codes, dst, add, None, None, 0.0, 0.0,
                        workspace)
        return d, (add, dst)

    def run_ref(self, t):
        from oceansar_b200 import _capi
        d, keep = self.desc(self.ref, t, self.ws.data_ptr())
        _capi.call("ocs_surface_update", ctypes.addressof(d), ctypes.c_float(t), self.stream)

    def run_noalloc(self, t):
        from oceansar_b200 import _capi
        for o in self.got:
            o.fill_(float('nan'))
        d, keep = self.desc(self.got, t, None)
        _capi.call("ocs_surface_update_noalloc", ctypes.addressof(d), ctypes.c_float(t), self.stream)

    def check(self, t):
        torch.cuda.synchronize()
        for name, a, b in zip(self.names, self.got, self.ref):
            assert torch.isfinite(a).all(), (name, t)
            assert torch.equal(a, b), (name, t, float((a - b).abs().max()))


@pytest.mark.parametrize("L,names", [(512, NAMES8), (480, NAMES8), (1024, NAMES6)],
                         ids=["512sq_8f", "480sq_8f_non_pow2", "1024sq_6f_near_limit"])
def test_noalloc_matches_workspace_entry_point(L, names):
    from oceansar_b200 import build
    build.build()
    c = _Case(L, names, seed=3)
    for t in (0.3, 1.7):                                   # two calls in a row
        c.run_ref(t)
        c.run_noalloc(t)
        c.check(t)


def test_noalloc_alternating_grids_and_no_allocation():
    """Two grid sizes in turn through the one shared array, each against its own
    workspace entry point; device memory in use is the same before and after."""
    a = _Case(512, NAMES8, seed=4)
    b = _Case(384, NAMES6, seed=5)
    a.run_noalloc(0.1)                                     # warm-up (module load on first use)
    for k, t in enumerate((0.5, 0.9, 1.3, 2.1)):
        c = a if k % 2 == 0 else b
        c.run_ref(t)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        c.run_noalloc(t)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, "the allocation-free call changed free device memory"
        c.check(t)


def test_noalloc_rejects_oversized_requests():
    from oceansar_b200 import _capi
    from oceansar_b200.surfaces.ocean import SurfaceDesc
    codes = (ctypes.c_int32 * 8)(*range(8))
    d = SurfaceDesc(4096, 4096, 1, 1, 1, 1, 0.0, 8, codes, None, None, None, None, 0.0, 0.0, None)
    st = _capi.load().ocs_surface_update_noalloc(ctypes.addressof(d), ctypes.c_float(0.0), None)
    assert st == -3                                          # OCS_ERR_SIZE, nothing launched


def test_noalloc_rejects_bad_descriptor_before_launch():
    """A descriptor with a missing output returns OCS_ERR_ARG and leaves the shared array
    as the previous call left it: the next good call still matches."""
    from oceansar_b200 import _capi
    c = _Case(512, NAMES8, seed=6)
    c.run_ref(0.7)
    c.run_noalloc(0.7)
    c.check(0.7)
    d, keep = c.desc(c.got, 0.7, None)
    keep[1][2] = None                                       # Dz output missing
    st = _capi.load().ocs_surface_update_noalloc(ctypes.addressof(d), ctypes.c_float(0.7), c.stream)
    assert st == -1                                          # OCS_ERR_ARG
    c.run_noalloc(0.7)
    c.check(0.7)
