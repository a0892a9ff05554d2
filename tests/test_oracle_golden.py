"""Pin the oracle: every CPU restatement against fixtures produced by the reference itself.

The fixtures in ``tests/golden`` were written by ``tests/golden/make_golden.py`` running
the unmodified reference code.  Integer / index work and the serial accumulation must be
bit-identical; float32 surface fields and float64 NRCS values are compared at a few ulp
(numba's transcendental functions and numpy's are not the same code).
"""
import json
import os

import numpy as np
import pytest

from oracle import closure, geometry, nrcs, range_profile, spectra
from oracle.cfg import ConfigFile
from oracle.sar_raw import sar_raw
from oracle.surface import OceanSurface

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(G, name))


def test_sinc_vec_bit_exact():
    d = load("sinc_vec.npz")
    for key in d.files:
        _, n, ovs, fs = key.split("_")
        v = range_profile.calc_sinc_vec(int(n), int(ovs), Fs=float(fs))
        assert v.dtype == np.float32
        np.testing.assert_array_equal(v, d[key])


@pytest.mark.parametrize("case", ["smoke", "edges", "ties"])
def test_chan_profile_bit_exact(case):
    d = load("range_profile.npz")
    g = {k.split("__", 1)[1]: d[k] for k in d.files if k.startswith(case + "__")}
    out = g["out0"].astype(np.complex128).copy()
    range_profile.chan_profile(g["srg"], g["scene"], float(g["binsize"]), float(g["min_sr"]),
                               g["sinc"], int(g["n"]), int(g["ovs"]), out)
    np.testing.assert_array_equal(out, g["out"])


@pytest.mark.parametrize("name", ["c1small", "c2small", "c3small", "c1lut", "c1fa", "c1spa"])
def test_chan_profile_captured_calls_bit_exact(name):
    d = load("sar_raw_%s.npz" % name)
    sinc = range_profile.calc_sinc_vec(8, 20, Fs=1.1)
    for i in range(3):
        out = d["call%d_out0" % i].copy()
        range_profile.chan_profile(d["call%d_srg" % i], d["call%d_scene" % i],
                                   float(d["call%d_binsize" % i]), float(d["call%d_min_sr" % i]),
                                   sinc, 8, 20, out)
        np.testing.assert_array_equal(out, d["call%d_out" % i])


SURF = {
    "deep_elf": (dict(Lx=64., Ly=64., dx=1., dy=1., cutoff_wl='auto', spec_model='elfouhaily',
                      spread_model='elfouhaily', wind_dir=0.0, wind_fetch=500e3, wind_U=10.,
                      current_mag=0., current_dir=0., compute=['D', 'Diff', 'Diff2', 'V', 'A', 'hMTF'],
                      opt_res=True, fft_max_prime=2, depth=None), 0),
    "choppy_swell_cos2s": (dict(Lx=64., Ly=32., dx=1., dy=1., cutoff_wl='auto', spec_model='elfouhaily',
                                spread_model='cos2s', wind_dir=np.deg2rad(45.), wind_fetch=500e3,
                                wind_U=7., current_mag=0.3, current_dir=np.deg2rad(90.),
                                swell_enable=True, swell_ampl=0.5, swell_dir=np.deg2rad(30.),
                                swell_wl=40., compute=['D', 'Diff', 'Diff2', 'V', 'A', 'hMTF'],
                                opt_res=True, fft_max_prime=2, choppy_enable=True, depth=100.), 1),
    "dirswell_p3": (dict(Lx=24., Ly=27., dx=0.5, dy=0.5, cutoff_wl='auto', spec_model='elfouhaily',
                         spread_model='elfouhaily', wind_dir=np.deg2rad(30.), wind_fetch=500e3,
                         wind_U=15., current_mag=0., current_dir=0., dir_swell_dir=120.,
                         freq_r=np.sqrt(9.80665 / (2 * np.pi * 250.)), sigf=0.007, sigs=8., Hs=0.8,
                         swell_dir_enable=True, compute=['D', 'Diff', 'Diff2'],
                         opt_res=True, fft_max_prime=3, depth=1e5,
                         dir_swell_spec=spectra.ardhuin_swell_spec), 2),
}


def ulp_close(a, b, nulp_rel=4):
    a = np.asarray(a)
    b = np.asarray(b)
    eps = np.finfo(b.dtype).eps if b.dtype.kind == 'f' else np.finfo(np.float64).eps
    scale = np.max(np.abs(b)) if b.size else 1.0
    return np.max(np.abs(a - b)) <= nulp_rel * eps * max(scale, 1e-30)


@pytest.mark.parametrize("name", list(SURF))
def test_surface_init_and_fields(name):
    kw, seed = SURF[name]
    d = load("surface_%s.npz" % name)
    np.random.seed(seed)
    s = OceanSurface().init(**kw)
    assert (s.Nx, s.Ny) == tuple(d["Nxy"])
    for k in ("kx", "ky", "omega", "kxn", "kyn", "kinv", "x", "y"):
        np.testing.assert_array_equal(getattr(s, k), d[k], err_msg=k)
    # the spreading function is numba-compiled in the reference: ulp-level differences
    assert ulp_close(s.wave_dirspec, d["wave_dirspec"], 8)
    assert ulp_close(s.wave_coefs, d["wave_coefs"], 8)
    np.testing.assert_allclose([s.rmss_x, s.rmss_y], d["rmss"], rtol=1e-6)
    for it, t in enumerate(d["times"]):
        s.wave_coefs = d["wave_coefs"]          # fields from identical coefficients
        f = s.set_t(t)
        for key in d.files:
            if key.startswith("t%d_" % it):
                fld = key.split("_", 1)[1]
                np.testing.assert_array_equal(f[fld], d[key], err_msg="%s t=%g" % (fld, t))


def test_balancer_interpolation():
    """Time-interpolated surface (balancer.py:126-297) against the reference's balancer on
    one process: bit-identical float32 fields at every time, including a step boundary, a
    step change that reuses the upper end, a backward jump and a jump far ahead."""
    from oracle.balancer import OceanSurfaceBalancer
    kw, seed = SURF["deep_elf"]
    d = load("balancer_deep_elf.npz")
    np.random.seed(seed)
    s = OceanSurface().init(**kw)
    s.wave_coefs = d["wave_coefs"]
    b = OceanSurfaceBalancer(s, float(d["dt"]))
    rs = int(d["row_step"])
    for it, t in enumerate(d["times"]):
        f = b.set_t(t)
        assert b.t_l_last == d["t%d_tl" % it]
        for key in d.files:
            if key.startswith("t%d_" % it) and not key.endswith("_tl"):
                fld = key.split("_", 1)[1]
                np.testing.assert_array_equal(f[fld][::rs], d[key], err_msg="%s t=%g" % (fld, t))


def test_romeiser_rcs():
    d = load("rcs_romeiser.npz")
    k0 = float(d["k0"])
    for spread_name in ("elfouhaily", "cos2s"):
        for pol in ("vv", "hh", "DP"):
            m = nrcs.RCSRomeiser97(k0, d["inc"], pol, 1.0, 1.0, 10.0, np.deg2rad(20.), 500e3,
                                   'elfouhaily', spread_name, 0.125)
            r = m.rcs(d["az_angle"], d["diffx"], d["diffy"])
            key = "%s_%s" % (spread_name, pol)
            if pol == "DP":
                pairs = ((r[0], d[key + "_hh"]), (r[1], d[key + "_vv"]))
            else:
                pairs = ((r, d[key]),)
            for got, ref in pairs:
                assert got.shape == ref.shape
                np.testing.assert_array_equal(np.isfinite(got), np.isfinite(ref))
                fin = np.isfinite(ref)
                np.testing.assert_allclose(got[fin], ref[fin], rtol=1e-12, atol=0)
    np.testing.assert_array_equal(m.interp_k, d["interp_k"])
    np.testing.assert_allclose(m.interp_S, d["interp_S"], rtol=1e-15)


def test_romeiser_lut_mode():
    """LUT mode (romeiser97.py:71-134): the table and the lookups, against the reference."""
    d = load("rcs_romeiser_lut.npz")
    k0 = float(d["k0"])
    for pol in ("vv", "hh", "DP"):
        m = nrcs.RCSRomeiser97(k0, d["inc"], pol, 1.0, 1.0, 10.0, np.deg2rad(20.), 500e3, 'elfouhaily',
                               'elfouhaily', 0.125, rmss_x=0.02, rmss_y=0.015, az_span=np.deg2rad(0.3),
                               use_lut=True)
        np.testing.assert_array_equal(m.lut_az.ravel(), d["lut_az"])
        np.testing.assert_array_equal(m.lut_Diffx.ravel(), d["lut_Diffx"])
        np.testing.assert_array_equal(m.lut_Diffy.ravel(), d["lut_Diffy"])
        r = m.rcs(d["az_angle"], d["diffx"], d["diffy"])
        if pol == "DP":
            pairs = ((m.lut_rcs[0], d["lut_hh"]), (m.lut_rcs[1], d["lut_vv"]), (r[0], d["DP_hh"]), (r[1], d["DP_vv"]))
        else:
            pairs = ((m.lut_rcs, d["lut_%s_single" % pol]), (r, d[pol]))
        for got, ref in pairs:
            assert got.shape == ref.shape
            fin = np.isfinite(ref)
            np.testing.assert_array_equal(np.isfinite(got), fin)
            np.testing.assert_allclose(got[fin], ref[fin], rtol=1e-12, atol=0)


def test_ka_field():
    """Kirchhoff specular field (nrcs/ka.py), facet approach and stationary phase."""
    from oracle.ka import RCSKA
    d = load("ka.npz")
    for mode in ("fa", "spa"):
        m = RCSKA(mode, float(d["k0"]), d["x"], d["y"], 1.0, 1.0)
        for pp in ("hh", "vv", "hv", "vh"):
            E = m.field(1, 1, pp[0], pp[1], d["inc"], d["inc"], d["az"], d["az"] + np.pi, d["Dz"], d["Diffx"],
                        d["Diffy"], d["Diffxx"], d["Diffyy"], d["Diffxy"])
            np.testing.assert_array_equal(E != 0, d["E_%s_%s" % (mode, pp)] != 0)
            np.testing.assert_allclose(E, d["E_%s_%s" % (mode, pp)], rtol=1e-13, atol=0)
        r = m.rcs('v', 'v', d["inc"], d["inc"], d["az"], d["az"] + np.pi, d["Dz"], d["Diffx"], d["Diffy"],
                  d["Diffxx"], d["Diffyy"], d["Diffxy"])
        np.testing.assert_allclose(r, d["rcs_%s_vv" % mode], rtol=1e-12, atol=0)


def test_sar_focus():
    """Range-Doppler focusing (radarsim/sar_processor.py) against the reference's SLC."""
    from oracle.sar_processor import focus_cube
    d = load("sar_focus.npz")
    sar = dict(f0=5.405e9, prf=1000., num_ch=2, v_ground=7600., rg_bw=50e6, over_fs=1.1, ant_L_tx=2.742,
               ant_L_rx=2.742)
    slc = focus_cube(d["raw"], sar, dict(doppler_bw=100., az_weighting=0.54), d["sr0"])
    assert slc.shape == d["slc"].shape
    np.testing.assert_allclose(slc, d["slc"], rtol=1e-12, atol=1e-12 * np.abs(d["slc"]).max())


def test_kodis_field():
    d = load("kodis.npz")
    m = nrcs.RCSKodis(d["inc"], float(d["k0"]), 1.0, 1.0)
    E = m.field(d["az_angle"], d["sr"], d["diffx"], d["diffy"], d["diffxx"], d["diffyy"], d["diffxy"])
    np.testing.assert_array_equal(E != 0, d["E"] != 0)
    np.testing.assert_allclose(E, d["E"], rtol=1e-13, atol=0)


def test_closure():
    d = load("closure.npz")
    np.testing.assert_allclose([closure.grid_coherence(u, 1.0, 5.405e9) for u in d["tau_U"]],
                               d["tau_c"], rtol=1e-15)
    np.testing.assert_allclose([closure.grid_coherence(u, 0.5, 5.405e9) for u in d["tau_U"]],
                               d["tau_c_res05"], rtol=1e-15)
    np.random.seed(21)
    r = closure.RandomScatTS(float(d["r_tau"]), (24, 20), 1000.0)
    assert r.N == int(d["r_N"])
    np.testing.assert_array_equal(r.s, d["r_s"])
    np.testing.assert_array_equal(r.ind0, d["r_ind0"])
    for t, sc in zip(d["r_ts"], d["r_scats"]):
        np.testing.assert_array_equal(r.scats(t), sc)


def test_geometry():
    d = load("geometry.npz")
    for ia, a in enumerate(d["alts"]):
        for ii, i in enumerate(d["incs"]):
            assert geometry.inc_to_sr(i, a) == d["sr0"][ia, ii]
            assert geometry.inc_to_gr(i, a) == d["gr0"][ia, ii]
    sr, inc, look = geometry.gr_to_geo(d["gr"], 514e3)
    np.testing.assert_array_equal(sr, d["gr_sr"])
    np.testing.assert_array_equal(inc, d["gr_inc"])
    np.testing.assert_array_equal(look, d["gr_look"])
    assert geometry.orbit_to_vel(514e3, ground=True) == d["v_ground_auto"]
    for p in (2, 3, 5):
        got = [int(geometry.optimize_fftsize(int(v), p)) for v in d["fft_vals"]]
        assert got == list(d["fft_opt_%d" % p])


def _cfg_json(cfg):
    out = {}
    for sec in cfg.sections[1:]:
        s = vars(cfg)[sec]
        out[sec] = {}
        for el in s.elements:
            v = vars(s)[el]
            if isinstance(v, np.ndarray):
                out[sec][el] = {"ndarray": v.tolist(), "dtype": str(v.dtype)}
            elif isinstance(v, bool):
                out[sec][el] = {"bool": v}
            elif isinstance(v, int):
                out[sec][el] = {"int": v}
            elif isinstance(v, float):
                out[sec][el] = {"float": v}
            elif isinstance(v, list):
                out[sec][el] = {"list": v}
            else:
                out[sec][el] = {"str": v}
    return out


def test_cfg_parser():
    with open(os.path.join(G, "cfg_parsed.json")) as f:
        ref = json.load(f)
    for name in ("quirks", "c1small", "c2small", "c3small", "c1lut", "c1fa", "c1spa"):
        cfg = ConfigFile(os.path.join(G, "cfg", name + ".cfg"))
        assert cfg.sections[1:] == ref[name]["sections"]
        assert _cfg_json(cfg) == ref[name]["values"]


@pytest.mark.parametrize("name", ["c1small", "c2small", "c3small", "c1lut", "c1fa", "c1spa"])
def test_sar_raw_end_to_end(name):
    d = load("sar_raw_%s.npz" % name)
    raw, nrcs_avg, sim = sar_raw(os.path.join(G, "cfg", name + ".cfg"), seed=0)
    assert raw.shape == d["raw"].shape
    np.testing.assert_allclose(sim.surface.wave_coefs, d["wave_coefs"], rtol=0, atol=1e-3)
    err = np.linalg.norm(raw - d["raw"]) / np.linalg.norm(d["raw"])
    assert err < 1e-9, err
    np.testing.assert_allclose(nrcs_avg, d["NRCS_avg"], rtol=1e-9)
    assert float(d["sr0"]) == pytest.approx(sim.sr_near, rel=1e-15)


def test_sar_raw_interpolated_surface_one_step():
    """With the interpolation step equal to the pulse interval, the time-interpolated run
    reproduces the per-pulse surface of the reference's sar_raw (the blend weights are 0/1
    up to float32 rounding of the pulse times)."""
    d = load("sar_raw_c1small.npz")
    cfg = os.path.join(G, "cfg", "c1small.cfg")
    raw, _, sim = sar_raw(cfg, seed=0, surface_dt=0.001)
    assert sim.balancer is not None and sim.t_step == 0.001
    err = np.linalg.norm(raw - d["raw"]) / np.linalg.norm(d["raw"])
    assert err < 1e-5, err


@pytest.mark.parametrize("name", ["dsc1", "dsc2"])
def test_dopsca_end_to_end(name):
    """DopSCA scatterometer generator (dopscasim/dopsca_raw.py) against the reference's run:
    range blocks, rolled surface rows, sub-pulses, two-way range scaling."""
    from oracle.dopsca_raw import dopsca_raw
    d = load("dopsca_%s.npz" % name)
    raw, nrcs_avg, sim = dopsca_raw(os.path.join(G, "cfg", name + ".cfg"), seed=0)
    assert raw.shape == d["raw"].shape
    np.testing.assert_array_equal(sim.surface.wave_coefs, d["wave_coefs"])
    err = np.linalg.norm(raw - d["raw"]) / np.linalg.norm(d["raw"])
    assert err < 1e-12, err
    np.testing.assert_allclose(nrcs_avg, d["NRCS_avg"], rtol=1e-12)
    assert float(d["sr0"]) == pytest.approx(sim.sr_near, rel=1e-15)


@pytest.mark.parametrize("name", ["skim1", "skim2", "skim3"])
def test_skim_end_to_end(name):
    """SKIM generator (radarsim/skim_raw.py) against the reference's run on one process:
    time-interpolated surface, per-facet beam, two-scale Doppler (row groups, up-sampling,
    geometric Doppler) and the single-scale form."""
    from oracle.skim_raw import skimraw
    d = load("skim_%s.npz" % name)
    raw, nrcs_avg, sim = skimraw(os.path.join(G, "cfg", name + ".cfg"), seed=0)
    assert raw.shape == d["raw"].shape
    np.testing.assert_array_equal(sim.surface_full.wave_coefs, d["wave_coefs"])
    err = np.linalg.norm(raw - d["raw"]) / np.linalg.norm(d["raw"])
    assert err < 1e-12, err
    np.testing.assert_allclose(nrcs_avg, d["NRCS_avg"], rtol=1e-12)
    np.testing.assert_array_equal(sim.dop_ref.ravel(), d["dop_ref"].ravel())
