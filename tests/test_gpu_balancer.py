"""Time-interpolated surface (``OceanSurfaceBalancer``, ``ocs_surface_blend``) on the GPU.

* The blend kernel is float32 w_l a + w_h b with separately rounded products and sum, as
  numpy evaluates it: bit-identical with numpy on any input.
* The balancer's fields against the reference's balancer (golden fixture from one MPI
  process): the end surfaces carry the GPU FFT's float32 rounding, so the surface bar
  applies (relative L2 <= 2e-6, max error <= 2e-5 of the peak); the blend of the GPU's own
  end surfaces is bit-identical.
* A whole interpolated scene against the oracle's interpolated run: relative L2 <= 1e-4
  and phase <= 1e-3 rad, as for the per-pulse surface.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def max_phase(a, b):
    mask = np.abs(b) >= 1e-3 * np.sqrt(np.mean(np.abs(b) ** 2))
    return np.max(np.abs(np.angle(a[mask] * np.conj(b[mask]))))


def test_blend_bit_exact():
    import ctypes
    from oceansar_b200 import _capi, _device
    rng = np.random.default_rng(3)
    for n in (1, 7, 4096, 1000003):
        a = [rng.standard_normal(n).astype(np.float32) for _ in range(3)]
        b = [rng.standard_normal(n).astype(np.float32) for _ in range(3)]
        ad = [torch.from_numpy(x).cuda() for x in a]
        bd = [torch.from_numpy(x).cuda() for x in b]
        dd = [torch.empty(n, dtype=torch.float32, device='cuda') for _ in range(3)]
        arr = lambda ts: (ctypes.c_void_p * 3)(*[t.data_ptr() for t in ts])  # noqa: E731
        w_h = np.float32(np.float32(0.0137) / np.float32(0.05))
        w_l = np.float32(1. - w_h)
        _capi.call("ocs_surface_blend", n, 3, arr(ad), arr(bd), arr(dd), float(w_l), float(w_h),
                   _device.stream_ptr())
        torch.cuda.synchronize()
        for x, y, d in zip(a, b, dd):
            np.testing.assert_array_equal(d.cpu().numpy(), w_l * x + w_h * y)


def test_blend_rejects_bad_arguments():
    import ctypes
    from oceansar_b200 import _capi, _device
    lib = _capi.load()
    t = torch.zeros(64, dtype=torch.float32, device='cuda')
    ok = (ctypes.c_void_p * 1)(t.data_ptr())
    odd = (ctypes.c_void_p * 1)(t.data_ptr() + 4)       # not 16-byte aligned
    sp = _device.stream_ptr()
    assert lib.ocs_surface_blend(-1, 1, ok, ok, ok, ctypes.c_float(1), ctypes.c_float(0), sp) != 0
    assert lib.ocs_surface_blend(16, 99, ok, ok, ok, ctypes.c_float(1), ctypes.c_float(0), sp) != 0
    assert lib.ocs_surface_blend(16, 1, odd, ok, ok, ctypes.c_float(1), ctypes.c_float(0), sp) != 0
    assert lib.ocs_surface_blend(0, 1, ok, ok, ok, ctypes.c_float(1), ctypes.c_float(0), sp) == 0


@pytest.mark.parametrize("choppy", [False, True])
def test_balancer_against_reference(choppy):
    from oceansar_b200.surfaces import OceanSurface, OceanSurfaceBalancer
    from tests.test_oracle_golden import SURF
    d = np.load(os.path.join(G, "balancer_deep_elf.npz"))
    kw, seed = SURF["deep_elf"]
    kw = dict(kw, choppy_enable=choppy) if choppy else dict(kw)
    np.random.seed(seed)
    s = OceanSurface()
    s.init(**kw)
    s.wave_coefs = d["wave_coefs"]
    s._upload()
    ends = OceanSurface()                   # the same surface, for the end fields
    np.random.seed(seed)
    ends.init(**kw)
    ends.wave_coefs = d["wave_coefs"]
    ends._upload()
    b = OceanSurfaceBalancer(s, float(d["dt"]))
    rs = int(d["row_step"])
    for it, t in enumerate(d["times"]):
        b.set_t(t)
        assert b.t_l_last == d["t%d_tl" % it]
        ends.set_t(b.t_l_last)
        lo = {n: getattr(ends, n).copy() for n in b._names}
        ends.set_t(b.t_h_last)
        for n in b._names:
            got = getattr(b, n)
            np.testing.assert_array_equal(got, b.w_l * lo[n] + b.w_h * getattr(ends, n), err_msg=n)
            if not choppy:
                ref = d["t%d_%s" % (it, n)]
                g = got[::rs].astype(np.float64)
                e = (np.linalg.norm(g - ref) / np.linalg.norm(ref), np.max(np.abs(g - ref)) / np.max(np.abs(ref)))
                assert e[0] < 2e-6 and e[1] < 2e-5, (n, t, e)


@pytest.mark.parametrize("name,dt", [("c1small", 0.01), ("c1small", 0.05), ("c3small", 0.003),
                                     ("c1fa", 0.004)])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_interpolated_scene_against_oracle(name, dt, precision):
    from oceansar_b200.radarsim.sar_raw_nompi import RawGenerator
    from oracle.sar_raw import sar_raw as oracle_sar_raw
    cfg = os.path.join(G, "cfg", name + ".cfg")
    ref, nref, osim = oracle_sar_raw(cfg, seed=0, add_noise=False, surface_dt=dt)
    gen = RawGenerator(cfg, precision=precision, seed=0, surface_dt=dt)
    assert gen.balancer is not None and not gen.can_overlap()
    gen.run()
    raw, nrcs_avg = gen.finish(add_noise=False)
    e, ph = rel_l2(raw, ref), max_phase(raw, ref)
    assert e < 1e-4 and ph < 1e-3, (e, ph)
    np.testing.assert_allclose(nrcs_avg, nref, rtol=1e-5)
    # one CUDA graph of the interpolated scene replays the same cube
    gen.capture(overlap=True)
    gen.replay()
    torch.cuda.synchronize()
    raw2, _ = gen.finish(add_noise=False)
    assert rel_l2(raw2, raw) <= (1e-12 if precision == 'f64' else 1e-5)


def test_sarraw_entry(tmp_path):
    """``sarraw`` (the MPI generator's entry) interpolates at the .cfg's ocean dt."""
    from oceansar_b200.ocs_io import RawFile
    from oceansar_b200.radarsim.sar_raw import sarraw
    from oracle.sar_raw import sar_raw as oracle_sar_raw
    cfg = os.path.join(G, "cfg", "c1small.cfg")
    np.random.seed(0)
    out = str(tmp_path / "raw.nc")
    sarraw(cfg, out, None, False, None, False)
    f = RawFile(out, 'r')
    raw = f.get('raw_data*')
    f.close()
    ref = oracle_sar_raw(cfg, seed=0, add_noise=True, surface_dt=0.05)[0]
    assert raw.shape == ref.shape
    assert rel_l2(raw, ref) < 1e-4
