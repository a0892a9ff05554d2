"""GPU parity of the accumulation kernel (ocs_chan_profile_*) against the oracle.

Bar: float64 kernel within 1e-10 relative L2 of the oracle's serial numba-equivalent sum
(only the summation order differs); single-precision kernel within 1e-5.
"""
import os

import numpy as np
import pytest
import torch

from oracle import range_profile as orp

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", autouse=True)
def _built():
    from oceansar_b200 import build
    build.build()


@pytest.mark.parametrize("case", ["smoke", "edges", "ties"])
def test_golden_cases(case):
    from oceansar_b200.radarsim import range_profile as rp
    d = np.load(os.path.join(G, "range_profile.npz"))
    g = {k.split("__", 1)[1]: d[k] for k in d.files if k.startswith(case + "__")}
    out = g["out0"].astype(np.complex128).copy()
    rp.chan_profile_numba(g["srg"], g["scene"], float(g["binsize"]), float(g["min_sr"]), g["sinc"],
                          int(g["n"]), int(g["ovs"]), out)
    assert rel(out, g["out"]) < 1e-12


@pytest.mark.parametrize("name", ["c1small", "c2small", "c3small"])
def test_captured_sar_raw_calls(name):
    from oceansar_b200.radarsim import range_profile as rp
    d = np.load(os.path.join(G, "sar_raw_%s.npz" % name))
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    for i in range(3):
        out = d["call%d_out0" % i].copy()
        rp.chan_profile_numba(d["call%d_srg" % i], d["call%d_scene" % i], float(d["call%d_binsize" % i]),
                              float(d["call%d_min_sr" % i]), sinc, 8, 20, out)
        assert rel(out, d["call%d_out" % i]) < 1e-10


def _synthetic(ny, nx, nbins, seed, binsize=2.725):
    rs = np.random.RandomState(seed)
    col = np.arange(nx) * 0.57 + 5.0
    row = ((np.arange(ny) - ny / 2) ** 2) / 4e5
    srg = col[None, :] + row[:, None] + 0.8 * rs.randn(ny, nx)
    scene = rs.randn(ny, nx) + 1j * rs.randn(ny, nx)
    return srg.ravel(), scene.ravel()


@pytest.mark.parametrize("shape", [(64, 64, 32), (512, 512, 160), (1024, 2048, 512)])
def test_large_against_oracle(shape):
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx, nbins = shape
    srg, scene = _synthetic(ny, nx, nbins, 3)
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref)
    out = np.zeros(nbins, complex)
    rp.chan_profile_numba(srg, scene, 2.725, 0.0, sinc, 8, 20, out)
    assert rel(out, ref) < 1e-10
    # in-place accumulation: a second call doubles the result
    rp.chan_profile_numba(srg, scene, 2.725, 0.0, sinc, 8, 20, out)
    assert rel(out, 2 * ref) < 1e-10


def test_rows_variant():
    from oceansar_b200.radarsim import range_profile as rp
    srg, scene = _synthetic(96, 300, 80, 4)
    srg = srg.reshape(96, 300)
    scene = scene.reshape(96, 300)
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros((96, 80), complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref, rg_only=True)
    out = np.zeros((96, 80), complex)
    rp.chan_profile_numba(srg, scene, 2.725, 0.0, sinc, 8, 20, out, rg_only=True)
    assert rel(out, ref) < 1e-10


def test_empty_and_tensor_inplace():
    from oceansar_b200.radarsim import range_profile as rp
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    out = np.ones(8, complex)
    rp.chan_profile_numba(np.zeros(0), np.zeros(0, complex), 1.0, 0.0, sinc, 8, 20, out)
    assert np.all(out == 1)
    srg, scene = _synthetic(32, 128, 64, 5)
    t = torch.zeros(64, dtype=torch.complex128, device="cuda")
    rp.chan_profile_numba(torch.from_numpy(srg).cuda(), torch.from_numpy(scene).cuda(), 2.725, 0.0,
                          sinc, 8, 20, t)
    ref = np.zeros(64, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref)
    assert rel(t.cpu().numpy(), ref) < 1e-10


def test_nonfinite_scene_touches_only_its_taps():
    from oceansar_b200.radarsim import range_profile as rp
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.0)
    srg = np.array([10.3, 30.7, 31.2])
    scene = np.array([1 + 1j, np.nan + 0j, 2 - 1j])
    ref = np.zeros(48, complex)
    orp.chan_profile(srg, scene, 1.0, 0.0, sinc, 8, 20, ref)
    out = np.zeros(48, complex)
    rp.chan_profile_numba(srg, scene, 1.0, 0.0, sinc, 8, 20, out)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
    fin = ~np.isnan(ref)
    assert rel(out[fin], ref[fin]) < 1e-12


def test_single_precision_kernel():
    from oceansar_b200 import _capi, _device
    from oceansar_b200.radarsim import range_profile as rp
    srg, scene = _synthetic(512, 512, 160, 6)
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros(160, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref)
    srg_d = _device.to_device(srg, np.float64)
    sc_d = _device.to_device(scene.astype(np.complex64), np.complex64)
    out_d = _device.zeros(160, np.complex64)
    sinc_d = _device.to_device(sinc, np.float32)
    _capi.call("ocs_chan_profile_c64", _device.ptr(srg_d), _device.ptr(sc_d), srg.size, 2.725, 0.0,
               _device.ptr(sinc_d), 8, 20, _device.ptr(out_d), 160, _device.stream_ptr())
    assert rel(out_d.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("shape", [(64, 64, 32), (97, 300, 90), (1024, 2048, 512), (5, 7, 16), (97, 301, 90),
                                   (203, 390, 120), (3, 2, 8), (4096, 4096, 2048)])
def test_two_dimensional_layout(shape):
    """The [ny, nx] column-walking kernel gives the flattened sum (edges: ragged tiles,
    bins outside [0, nbins), a non-finite facet; 203 x 390: a ragged last column tile and
    a last row batch of fewer rows); at 4096 x 4096 the persistent CTAs walk several
    tiles each."""
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx, nbins = shape
    srg, scene = _synthetic(ny, nx, nbins, 5)
    srg = srg - 3.0                                     # some facets fall below bin 0
    scene[len(scene) // 3] = np.nan + 0j
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref)
    out = np.zeros(nbins, complex)
    rp.chan_profile_numba(srg.reshape(ny, nx), scene.reshape(ny, nx), 2.725, 0.0, sinc, 8, 20, out)
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(out))
    assert rel(out[fin], ref[fin]) < 1e-10


@pytest.mark.parametrize("misaligned", [False, True], ids=["aligned", "misaligned"])
def test_two_dimensional_c64(misaligned):
    """Single precision in the [ny, nx] layout, also with inputs that start 8 bytes past
    a 16-byte boundary (views into larger buffers)."""
    import ctypes
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx, nbins = 300, 700, 200
    srg, scene = _synthetic(ny, nx, nbins, 6)
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref)
    k = 1 if misaligned else 0
    s_d = torch.tensor(np.concatenate([np.zeros(k), srg]), dtype=torch.float64, device="cuda")[k:]
    c_d = torch.tensor(np.stack([np.concatenate([np.zeros(k), scene.real]), np.concatenate([np.zeros(k), scene.imag])],
                                -1), dtype=torch.float32, device="cuda")[k:]
    assert (s_d.data_ptr() % 16 == 8) == misaligned and (c_d.data_ptr() % 16 == 8) == misaligned
    w_d = torch.tensor(sinc, dtype=torch.float32, device="cuda")
    o_d = torch.zeros(nbins, 2, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_chan_profile_2d_c64", s_d.data_ptr(), c_d.data_ptr(), ny, nx, 2.725, 0.0, w_d.data_ptr(), 8, 20,
               o_d.data_ptr(), nbins, st)
    out = o_d.cpu().numpy().astype(np.float64)
    assert rel(out[:, 0] + 1j * out[:, 1], ref) < 1e-5


@pytest.mark.parametrize("spacing,jitter", [(3.0, 0.8), (10.0, 0.8), (0.57, 40.0), (1.4, 5.0)],
                         ids=["1.1bins_per_col", "3.7bins_per_col", "scattered_40m", "0.5bins_per_col_5m"])
@pytest.mark.parametrize("precision", ["f64", "c64"])
def test_two_dimensional_steep_and_scattered(spacing, jitter, precision):
    """The [ny, nx] kernel on layouts whose columns step more than a bin apart (the strips
    are walked in narrower column groups) and whose ranges scatter far from their column
    (many facets take the per-tap path): same sum as the flattened oracle."""
    import ctypes
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx = 301, 517
    rs = np.random.RandomState(11)
    col = np.arange(nx) * spacing + 40.0
    row = ((np.arange(ny) - ny / 2) ** 2) / 4e4
    srg = col[None, :] + row[:, None] + jitter * rs.randn(ny, nx)
    scene = rs.randn(ny, nx) + 1j * rs.randn(ny, nx)
    nbins = int((srg.max() + 60.0) / 2.725)
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg.ravel(), scene.ravel(), 2.725, 0.0, sinc, 8, 20, ref)
    if precision == "f64":
        out = np.zeros(nbins, complex)
        rp.chan_profile_numba(srg, scene, 2.725, 0.0, sinc, 8, 20, out)
        assert rel(out, ref) < 1e-10
        return
    s_d = torch.tensor(srg, dtype=torch.float64, device="cuda")
    c_d = torch.tensor(np.stack([scene.real, scene.imag], -1), dtype=torch.float32, device="cuda")
    w_d = torch.tensor(sinc, dtype=torch.float32, device="cuda")
    o_d = torch.zeros(nbins, 2, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_chan_profile_2d_c64", s_d.data_ptr(), c_d.data_ptr(), ny, nx, 2.725, 0.0, w_d.data_ptr(), 8, 20,
               o_d.data_ptr(), nbins, st)
    out = o_d.cpu().numpy().astype(np.float64)
    assert rel(out[:, 0] + 1j * out[:, 1], ref) < 1e-5


@pytest.mark.parametrize("precision", ["f64", "c64"])
def test_two_dimensional_scene_off_pair_alignment(precision):
    """The [ny, nx] kernel with a scene that starts one component past its element-pair
    alignment (a view into a larger buffer: 4 bytes for complex64, 8 for complex128), which
    takes the scalar-load path: same sum as the flattened oracle."""
    import ctypes
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx, nbins = 203, 390, 120
    srg, scene = _synthetic(ny, nx, nbins, 8)
    sinc = rp.calc_sinc_vec(8, 20, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 20, ref)
    dt = torch.float64 if precision == "f64" else torch.float32
    inter = np.stack([scene.real, scene.imag], -1).ravel()
    buf = torch.tensor(np.concatenate([[0.0], inter]), dtype=dt, device="cuda")
    c_ptr = buf.data_ptr() + buf.element_size()
    assert c_ptr % (2 * buf.element_size()) == buf.element_size()
    s_d = torch.tensor(srg, dtype=torch.float64, device="cuda")
    w_d = torch.tensor(sinc, dtype=torch.float32, device="cuda")
    o_d = torch.zeros(nbins, 2, dtype=dt, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    fn = "ocs_chan_profile_2d_f64" if precision == "f64" else "ocs_chan_profile_2d_c64"
    _capi.call(fn, s_d.data_ptr(), c_ptr, ny, nx, 2.725, 0.0, w_d.data_ptr(), 8, 20, o_d.data_ptr(), nbins, st)
    out = o_d.cpu().numpy().astype(np.float64)
    assert rel(out[:, 0] + 1j * out[:, 1], ref) < (1e-10 if precision == "f64" else 1e-5)


@pytest.mark.parametrize("precision", ["f64", "c64"])
def test_two_dimensional_fine_oversampling(precision):
    """A pulse oversampled 80 times (the fine-grid histogram would not fit its shared-memory
    budget, so the register-window kernel runs): same sum as the flattened oracle."""
    import ctypes
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx, nbins = 150, 333, 110
    srg, scene = _synthetic(ny, nx, nbins, 9)
    sinc = rp.calc_sinc_vec(8, 80, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, 8, 80, ref)
    if precision == "f64":
        out = np.zeros(nbins, complex)
        rp.chan_profile_numba(srg.reshape(ny, nx), scene.reshape(ny, nx), 2.725, 0.0, sinc, 8, 80, out)
        assert rel(out, ref) < 1e-10
        return
    s_d = torch.tensor(srg, dtype=torch.float64, device="cuda")
    c_d = torch.tensor(np.stack([scene.real, scene.imag], -1), dtype=torch.float32, device="cuda")
    w_d = torch.tensor(sinc, dtype=torch.float32, device="cuda")
    o_d = torch.zeros(nbins, 2, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_chan_profile_2d_c64", s_d.data_ptr(), c_d.data_ptr(), ny, nx, 2.725, 0.0, w_d.data_ptr(), 8, 80,
               o_d.data_ptr(), nbins, st)
    out = o_d.cpu().numpy().astype(np.float64)
    assert rel(out[:, 0] + 1j * out[:, 1], ref) < 1e-5


@pytest.mark.parametrize("taps,ovs", [(5, 10), (7, 3), (16, 4)], ids=["5taps_10x", "7taps_3x", "16taps_4x"])
@pytest.mark.parametrize("precision", ["f64", "c64"])
def test_two_dimensional_other_pulses(taps, ovs, precision):
    """The [ny, nx] kernel with odd and long pulses and other oversampling factors (the
    convolution splits the taps over four lanes unevenly): same sum as the flattened oracle."""
    import ctypes
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim import range_profile as rp
    ny, nx, nbins = 131, 260, 100
    srg, scene = _synthetic(ny, nx, nbins, 10)
    srg = srg - 2.0
    sinc = rp.calc_sinc_vec(taps, ovs, Fs=1.1)
    ref = np.zeros(nbins, complex)
    orp.chan_profile(srg, scene, 2.725, 0.0, sinc, taps, ovs, ref)
    if precision == "f64":
        out = np.zeros(nbins, complex)
        rp.chan_profile_numba(srg.reshape(ny, nx), scene.reshape(ny, nx), 2.725, 0.0, sinc, taps, ovs, out)
        assert rel(out, ref) < 1e-10
        return
    s_d = torch.tensor(srg, dtype=torch.float64, device="cuda")
    c_d = torch.tensor(np.stack([scene.real, scene.imag], -1), dtype=torch.float32, device="cuda")
    w_d = torch.tensor(sinc, dtype=torch.float32, device="cuda")
    o_d = torch.zeros(nbins, 2, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_chan_profile_2d_c64", s_d.data_ptr(), c_d.data_ptr(), ny, nx, 2.725, 0.0, w_d.data_ptr(), taps,
               ovs, o_d.data_ptr(), nbins, st)
    out = o_d.cpu().numpy().astype(np.float64)
    assert rel(out[:, 0] + 1j * out[:, 1], ref) < 1e-5
