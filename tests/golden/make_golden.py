"""Generate the golden fixtures in this folder by running the OCEANSAR reference itself.

Run from the repository root, in a container where the reference tree is mounted:

    python tests/golden/make_golden.py

It imports the unmodified reference (``ref_shims.install()`` documents the
import-time shims it needs) and records, for small seeded inputs, the outputs of the
reference functions on the raw-data-generation path:

* ``radarsim/range_profile.py``  ``calc_sinc_vec`` / ``chan_profile_numba``
* ``surfaces/ocean.py``          ``OceanSurface.init`` and the ``t`` setter
* ``surfaces/balancer.py``       ``OceanSurfaceBalancer`` time interpolation (one process)
* ``nrcs/romeiser97.py``         ``RCSRomeiser97.rcs`` (numba path and LUT mode)
* ``nrcs/kodis.py``              ``RCSKodis.field``
* ``nrcs/ka.py``                 ``RCSKA.field`` / ``rcs`` (facet approach, stationary phase)
* ``closure/*.py``               ``grid_coherence`` / ``randomscat_ts``
* ``utils/geometry.py``, ``utils/misc.py``  geometry helpers and ``optimize_fftsize``
* ``ocs_io/cfg.py``              ``ConfigFile`` parsing of the ``.cfg`` files in ``cfg/``
* ``radarsim/sar_processor.py``  ``sar_focus`` on a seeded raw cube
* ``radarsim/sar_raw_nompi.py``  ``sar_raw`` end to end (noise at -300 dB), plus the
  arguments and results of its first ``chan_profile_numba`` calls.
* ``dopscasim/dopsca_raw.py``    ``dopsca_raw`` end to end (range blocks, sub-pulses).
* ``radarsim/skim_raw.py``       ``skimraw`` end to end on one process (two-scale Doppler).

The fixtures are committed; tests never import the reference.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_shims  # noqa: E402

ref_shims.install()

from oceansar import closure, spec, spread  # noqa: E402
from oceansar import constants as const  # noqa: E402
from oceansar import nrcs  # noqa: E402
from oceansar import ocs_io  # noqa: E402
from oceansar import utils  # noqa: E402
from oceansar.radarsim import range_profile as rp  # noqa: E402
from oceansar.radarsim import sar_raw_nompi  # noqa: E402
from oceansar.surfaces import OceanSurface  # noqa: E402
from oceansar.swell_spec import dir_swell_spec  # noqa: E402
from oceansar.utils import geometry as geo  # noqa: E402

OUT = HERE


def save(name, **arrays):
    path = os.path.join(OUT, name)
    np.savez_compressed(path, **arrays)
    print("wrote", path, sum(np.asarray(a).nbytes for a in arrays.values()), "bytes raw")


# --------------------------------------------------------------------------------------
def gen_sinc():
    out = {}
    for n, ovs, fs in ((8, 20, 1.1), (8, 20, 1.0), (6, 10, 1.0), (3, 10, 1.0), (8, 20, 1.25)):
        out["sinc_%d_%d_%g" % (n, ovs, fs)] = rp.calc_sinc_vec(n, ovs, Fs=fs)
    save("sinc_vec.npz", **out)


def gen_range_profile():
    cases = {}
    # (a) the reference's own smoke layout: unit point target at srg=50.5 in a
    #     random field, 3-sample sinc oversampled 10x, 110 output bins.
    np.random.seed(11)
    N = 1024
    srg = np.random.rand(N) * 100
    scat = np.random.randn(N) + 1j * np.random.randn(N)
    scat[100] = 1.0
    srg[100] = 50.5
    sincv = rp.calc_sinc_vec(3, 10)
    out = np.zeros(110, dtype=complex)
    rp.chan_profile_numba(srg, scat, 1.0, 0.0, sincv, 3, 10, out)
    cases["smoke"] = dict(srg=srg, scene=scat, binsize=1.0, min_sr=0.0, sinc=sincv,
                          n=3, ovs=10, out0=np.zeros(110, dtype=complex), out=out)
    # (b) ranges spilling over both edges, 8x20 sinc at over_fs 1.1, accumulation
    #     into a non-zero output (the call is an in-place +=).
    np.random.seed(12)
    N = 5000
    binsize = 2.998e8 / 2 / 50e6 / 1.1
    srg = np.random.uniform(-20.0, 64 * binsize + 20.0, N)
    scat = (np.random.randn(N) + 1j * np.random.randn(N))
    sincv = rp.calc_sinc_vec(8, 20, Fs=1.1)
    out0 = (np.random.randn(64) + 1j * np.random.randn(64))
    out = out0.copy()
    rp.chan_profile_numba(srg, scat, binsize, 3.5, sincv, 8, 20, out)
    cases["edges"] = dict(srg=srg, scene=scat, binsize=binsize, min_sr=3.5, sinc=sincv,
                          n=8, ovs=20, out0=out0, out=out)
    # (c) exact rounding ties of the LUT index (20*(1-frac) = k + 0.5 for dyadic frac):
    #     numpy rounds half to even.
    fr = np.array([1 / 8, 3 / 8, 5 / 8, 7 / 8, 0.0, 0.5, 0.25, 0.999999999])
    srg = (np.arange(fr.size)[:, None] * 3 + 10 + fr[None, :]).ravel()
    scat = np.exp(1j * np.arange(srg.size) * 0.7) * (1 + np.arange(srg.size))
    sincv = rp.calc_sinc_vec(8, 20, Fs=1.0)
    out = np.zeros(48, dtype=complex)
    rp.chan_profile_numba(srg, scat, 1.0, 0.0, sincv, 8, 20, out)
    cases["ties"] = dict(srg=srg, scene=scat, binsize=1.0, min_sr=0.0, sinc=sincv,
                         n=8, ovs=20, out0=np.zeros(48, dtype=complex), out=out)
    flat = {}
    for cname, d in cases.items():
        for k, v in d.items():
            flat["%s__%s" % (cname, k)] = np.asarray(v)
    save("range_profile.npz", **flat)


# --------------------------------------------------------------------------------------
SURFACE_CASES = {
    # name: (init kwargs, seed, times)
    "deep_elf": (dict(Lx=64., Ly=64., dx=1., dy=1., cutoff_wl='auto', spec_model='elfouhaily',
                      spread_model='elfouhaily', wind_dir=0.0, wind_fetch=500e3, wind_U=10.,
                      current_mag=0., current_dir=0., compute=['D', 'Diff', 'Diff2', 'V', 'A', 'hMTF'],
                      opt_res=True, fft_max_prime=2, depth=None), 0, (0.0, 0.37, 1.5)),
    "choppy_swell_cos2s": (dict(Lx=64., Ly=32., dx=1., dy=1., cutoff_wl='auto', spec_model='elfouhaily',
                                spread_model='cos2s', wind_dir=np.deg2rad(45.), wind_fetch=500e3,
                                wind_U=7., current_mag=0.3, current_dir=np.deg2rad(90.),
                                swell_enable=True, swell_ampl=0.5, swell_dir=np.deg2rad(30.),
                                swell_wl=40., compute=['D', 'Diff', 'Diff2', 'V', 'A', 'hMTF'],
                                opt_res=True, fft_max_prime=2, choppy_enable=True, depth=100.),
                           1, (0.0, 0.25, 2.0)),
    "dirswell_p3": (dict(Lx=24., Ly=27., dx=0.5, dy=0.5, cutoff_wl='auto', spec_model='elfouhaily',
                         spread_model='elfouhaily', wind_dir=np.deg2rad(30.), wind_fetch=500e3,
                         wind_U=15., current_mag=0., current_dir=0., dir_swell_dir=120.,
                         freq_r=np.sqrt(const.g / (2 * np.pi * 250.)), sigf=0.007, sigs=8., Hs=0.8,
                         swell_dir_enable=True, compute=['D', 'Diff', 'Diff2'],
                         opt_res=True, fft_max_prime=3, depth=1e5,
                         dir_swell_spec=dir_swell_spec.ardhuin_swell_spec), 2, (0.0, 0.5)),
}

FIELDS = ['Dx', 'Dy', 'Dz', 'Diffx', 'Diffy', 'Diffxx', 'Diffyy', 'Diffxy',
          'Vx', 'Vy', 'Vz', 'Ax', 'Ay', 'Az', 'hMTF']


def gen_surfaces():
    for name, (kw, seed, times) in SURFACE_CASES.items():
        np.random.seed(seed)
        s = OceanSurface()
        s.init(**kw)
        out = dict(wave_coefs=s.wave_coefs, kx=s.kx, ky=s.ky, omega=s.omega,
                   kxn=s.kxn, kyn=s.kyn, kinv=s.kinv, wave_dirspec=s.wave_dirspec,
                   rmss=np.array([s.rmss_x, s.rmss_y]), dxdy=np.array([s.dx, s.dy], dtype=np.float64),
                   Nxy=np.array([s.Nx, s.Ny]), x=s.x, y=s.y, times=np.array(times))
        if kw.get('swell_enable'):
            out['swell_ph0'] = np.array(s.swell_ph0)
        for it, t in enumerate(times):
            s.t = t
            for f in FIELDS:
                if hasattr(s, f):
                    out['t%d_%s' % (it, f)] = getattr(s, f).copy()
        save("surface_%s.npz" % name, **out)


# --------------------------------------------------------------------------------------
BALANCER_DT = 0.05
BALANCER_TIMES = (0.0, 0.013, 0.05, 0.071, 0.12, 0.02, 0.5, 0.5371)
BALANCER_ROW_STEP = 4                    # every 4th surface row is stored


def gen_balancer():
    """``OceanSurfaceBalancer`` over the deep_elf surface: pulse times inside one step, on a
    step boundary, into the next step (upper end reused), backwards and far ahead."""
    from oceansar.surfaces import OceanSurfaceBalancer
    kw, seed, _ = SURFACE_CASES["deep_elf"]
    np.random.seed(seed)
    s = OceanSurface()
    s.init(**kw)
    b = OceanSurfaceBalancer(s, BALANCER_DT)
    out = dict(wave_coefs=s.wave_coefs, dt=np.array(BALANCER_DT), times=np.array(BALANCER_TIMES),
               row_step=np.array(BALANCER_ROW_STEP))
    for it, t in enumerate(BALANCER_TIMES):
        b.t = t
        out['t%d_tl' % it] = np.array(b.t_l_last)
        for f in FIELDS:
            if hasattr(b, f):
                out['t%d_%s' % (it, f)] = getattr(b, f)[::BALANCER_ROW_STEP].copy()
    save("balancer_deep_elf.npz", **out)


# --------------------------------------------------------------------------------------
def gen_rcs():
    f0 = 5.405e9
    k0 = 2 * np.pi * f0 / const.c
    Ny, Nx = 48, 40
    rs = np.random.RandomState(5)
    diffx = (0.05 * rs.randn(Ny, Nx)).astype(np.float32)
    diffy = (0.05 * rs.randn(Ny, Nx)).astype(np.float32)
    diffx[0, :4] = [0.0, 0.7, -0.7, 0.45]          # around the near-specular / bad_ones region
    diffy[0, :4] = [0.0, 0.0, 0.3, -0.2]
    inc = np.deg2rad(np.linspace(30., 40., Nx)).reshape(1, Nx)
    # float64 azimuth angles, as sar_raw_nompi.py:363 produces them
    y = np.linspace(-300, 300, Ny).astype(np.float32).astype(np.float64)
    az_angle = np.arcsin((y / 5e5)).reshape(Ny, 1)
    out = dict(diffx=diffx, diffy=diffy, inc=inc, az_angle=az_angle, k0=np.array(k0))
    for spread_name in ('elfouhaily', 'cos2s'):
        for pol in ('vv', 'hh', 'DP'):
            m = nrcs.RCSRomeiser97(k0, inc, pol, 1.0, 1.0, 10.0, np.deg2rad(20.), 500e3,
                                   'elfouhaily', spread_name, 0.125, use_lut=False)
            r = m.rcs(az_angle, diffx, diffy)
            key = "%s_%s" % (spread_name, pol)
            if pol == 'DP':
                out[key + "_hh"], out[key + "_vv"] = r
            else:
                out[key] = r
    # the interpolation table the model uses (k grid + omni-directional spectrum)
    kk = np.arange(1, 2 * k0, 0.1)
    out['interp_k'] = kk
    out['interp_S'] = spec.models['elfouhaily'](kk, 10.0, 500e3)
    save("rcs_romeiser.npz", **out)


def gen_rcs_lut():
    """RCSRomeiser97 in LUT mode (romeiser97.py:71-92, 109-134): a small LUT (rmss 0.02 /
    0.015, 0.3 deg azimuth span) and its lookups on slopes that partly fall outside it."""
    f0 = 5.405e9
    k0 = 2 * np.pi * f0 / const.c
    Ny, Nx = 48, 40
    rs = np.random.RandomState(9)
    diffx = (0.04 * rs.randn(Ny, Nx)).astype(np.float32)
    diffy = (0.03 * rs.randn(Ny, Nx)).astype(np.float32)
    inc = np.deg2rad(np.linspace(30., 40., Nx)).reshape(1, Nx)
    y = np.linspace(-1200, 1200, Ny).astype(np.float32).astype(np.float64)
    az_angle = np.arcsin((y / 5e5)).reshape(Ny, 1)
    out = dict(diffx=diffx, diffy=diffy, inc=inc, az_angle=az_angle, k0=np.array(k0))
    for pol in ('vv', 'hh', 'DP'):
        m = nrcs.RCSRomeiser97(k0, inc, pol, 1.0, 1.0, 10.0, np.deg2rad(20.), 500e3, 'elfouhaily', 'elfouhaily',
                               0.125, rmss_x=0.02, rmss_y=0.015, az_span=np.deg2rad(0.3), use_lut=True)
        r = m.rcs(az_angle, diffx, diffy)
        if pol == 'DP':
            out["lut_hh"], out["lut_vv"] = np.asarray(m.lut_rcs[0]), np.asarray(m.lut_rcs[1])
            out["DP_hh"], out["DP_vv"] = r
        else:
            out["lut_" + pol + "_single"] = np.asarray(m.lut_rcs)
            out[pol] = r
    out["lut_az"] = m.lut_az.ravel()
    out["lut_Diffx"] = m.lut_Diffx.ravel()
    out["lut_Diffy"] = m.lut_Diffy.ravel()
    save("rcs_romeiser_lut.npz", **out)


def gen_ka():
    """RCSKA (nrcs/ka.py:41-310) field and rcs, facet approach and stationary phase, all four
    polarisation pairs, monostatic, on seeded float32 surface derivatives."""
    f0 = 5.405e9
    k0 = 2 * np.pi * f0 / const.c
    Ny, Nx = 40, 36
    rs = np.random.RandomState(11)
    x = np.arange(Nx) * 1.0 - Nx / 2
    y = np.arange(Ny) * 1.0 - Ny / 2
    Dz = (0.4 * rs.randn(Ny, Nx)).astype(np.float32)
    Diffx = (0.08 * rs.randn(Ny, Nx)).astype(np.float32)
    Diffy = (0.08 * rs.randn(Ny, Nx)).astype(np.float32)
    Diffxx = (0.05 * rs.randn(Ny, Nx)).astype(np.float32)
    Diffyy = (0.05 * rs.randn(Ny, Nx)).astype(np.float32)
    Diffxy = (0.03 * rs.randn(Ny, Nx)).astype(np.float32)
    Diffxx[0, 0] = Diffyy[0, 0] = Diffxy[0, 0] = 0.0          # J = 0
    # slopes near tan(inc) so that some stationary points fall inside their facet
    inc = np.deg2rad(np.linspace(30., 40., Nx)).reshape(1, Nx)
    # rows 2-9: slopes facing the radar and strong curvature, so that stationary points fall
    # inside their facets (both signs of J)
    for r in range(2, 10):
        Diffx[r, :] = (np.tan(inc[0]) + 0.3 * rs.randn(Nx)).astype(np.float32)
        Diffy[r, :] = (0.3 * rs.randn(Nx)).astype(np.float32)
        Diffxx[r, :] = 1.0
        Diffyy[r, :] = 1.0 if r < 6 else -1.0
        Diffxy[r, :] = 0.2
    az = np.arcsin(np.linspace(-300, 300, Ny) / 5e5).reshape(Ny, 1)
    out = dict(x=x, y=y, Dz=Dz, Diffx=Diffx, Diffy=Diffy, Diffxx=Diffxx, Diffyy=Diffyy, Diffxy=Diffxy,
               inc=inc, az=az, k0=np.array(k0))
    for mode in ('fa', 'spa'):
        m = nrcs.RCSKA(mode, k0, x, y, 1.0, 1.0)
        for pi_, ps in (('h', 'h'), ('v', 'v'), ('h', 'v'), ('v', 'h')):
            E = m.field(1, 1, pi_, ps, inc, inc, az, az + np.pi, Dz, Diffx, Diffy, Diffxx, Diffyy, Diffxy)
            out['E_%s_%s%s' % (mode, pi_, ps)] = E
        out['rcs_%s_vv' % mode] = m.rcs('v', 'v', inc, inc, az, az + np.pi, Dz, Diffx, Diffy, Diffxx, Diffyy,
                                        Diffxy)
    save("ka.npz", **out)


PROC_CFG = """\
[sar]
f0=5.405e9
prf=1000.
num_ch=2
alt=514e3
v_ground=7600.
rg_bw=50e6
over_fs=1.1
ant_L_tx=2.742
ant_L_rx=2.742
inc_angle=35.
pol=vv

[processing]
az_weighting=0.54
doppler_bw=100.
plot_format=png
plot_tex=False
plot_save=False
plot_path=plots
plot_raw=False
plot_rcmc_dopp=False
plot_rcmc_time=False
plot_image_valid=False
"""


def gen_focus():
    """sar_focus (radarsim/sar_processor.py:30-274) on a seeded raw cube (1 pol, 2 channels,
    500 azimuth x 40 range samples, padded by the processor to 512 x 64)."""
    from oceansar.radarsim import sar_processor
    path = os.path.join(OUT, "cfg", "proc.cfg")
    with open(path, "w") as f:
        f.write(PROC_CFG)
    rs = np.random.RandomState(21)
    raw = (rs.randn(1, 2, 500, 40) + 1j * rs.randn(1, 2, 500, 40)).astype(np.complex64)
    raw_file = "/tmp/golden_focus_raw.nc"
    rf = ocs_io.RawFile(raw_file, 'w', raw.shape)
    rf.set('raw_data*', raw)
    for k, v in dict(sr0=627e3, inc_angle=35., b_ati=np.array([0., 10.]), b_xti=np.zeros(2)).items():
        rf.set(k, v)
    rf.close()
    out_file = "/tmp/golden_focus_slc.nc"
    sar_processor.sar_focus(path, raw_file, out_file)
    v = ref_shims.NC_STORE[out_file].variables
    save("sar_focus.npz", raw=raw, slc=v['slc_r'].data + 1j * v['slc_i'].data, sr0=np.array(627e3))


def gen_kodis():
    f0 = 5.405e9
    k0 = 2 * np.pi * f0 / const.c
    Ny, Nx = 64, 48
    rs = np.random.RandomState(6)
    inc = np.deg2rad(np.linspace(2., 12., Nx)).reshape(1, Nx)
    # curvatures of either sign so that J > 0 and J < 0 both occur, and slopes near
    # tan(inc) so that stationary points fall inside some facets
    diffxx = (0.5 * rs.randn(Ny, Nx)).astype(np.float32)
    diffyy = (0.5 * rs.randn(Ny, Nx)).astype(np.float32)
    diffxy = (0.2 * rs.randn(Ny, Nx)).astype(np.float32)
    diffx = (np.tan(inc) + 0.1 * rs.randn(Ny, Nx)).astype(np.float32)
    diffy = (0.1 * rs.randn(Ny, Nx)).astype(np.float32)
    diffxx[0, 0] = 1.0; diffyy[0, 0] = 1.0; diffxy[0, 0] = 1.0       # J == 0 exactly
    sr = 1000.0 + rs.uniform(0, 50, (Ny, Nx))
    # float64 azimuth angles, as sar_raw_nompi.py:363 produces them
    y = np.linspace(-100, 100, Ny).astype(np.float32).astype(np.float64)
    # a full [Ny, Nx] azimuth-angle array: with the [Ny, 1] vector that sar_raw passes,
    # kodis.py:61 raises IndexError as soon as a stationary point lies outside column 0
    az = np.repeat(np.arcsin(y / 3e4).reshape(Ny, 1), Nx, axis=1)
    m = nrcs.RCSKodis(inc, k0, 1.0, 1.0)
    E = m.field(az, sr, diffx, diffy, diffxx, diffyy, diffxy)
    save("kodis.npz", inc=inc, k0=np.array(k0), diffx=diffx, diffy=diffy, diffxx=diffxx,
         diffyy=diffyy, diffxy=diffxy, sr=sr, az_angle=az, E=E)


def gen_closure():
    out = {}
    us = np.array([3.0, 7.0, 10.0, 15.0, 20.0])
    out['tau_U'] = us
    out['tau_c'] = np.array([closure.grid_coherence(u, 1.0, 5.405e9) for u in us])
    out['tau_c_res05'] = np.array([closure.grid_coherence(u, 0.5, 5.405e9) for u in us])
    np.random.seed(21)
    tau = closure.grid_coherence(10.0, 1.0, 5.405e9)
    r = closure.randomscat_ts(tau, (24, 20), 1000.0)
    out['r_tau'] = np.array(tau)
    out['r_N'] = np.array(r.N)
    out['r_s'] = r.s
    out['r_ind0'] = r.ind0
    ts = np.array([0.0, 0.001, 0.0123, 0.2, 3.0, 21.7])
    out['r_ts'] = ts
    out['r_scats'] = np.stack([r.scats(t) for t in ts])
    save("closure.npz", **out)


def gen_geometry():
    out = {}
    incs = np.deg2rad(np.array([20., 30., 35., 45.]))
    alts = np.array([514e3, 693e3])
    out['incs'] = incs
    out['alts'] = alts
    out['sr0'] = np.array([[geo.inc_to_sr(i, a) for i in incs] for a in alts])
    out['gr0'] = np.array([[geo.inc_to_gr(i, a) for i in incs] for a in alts])
    gr = geo.inc_to_gr(np.deg2rad(35.), 514e3) + np.linspace(-256, 256, 512).astype(np.float32)
    sr, inc, look = geo.gr_to_geo(gr, 514e3)
    out['gr'] = gr
    out['gr_sr'] = sr
    out['gr_inc'] = inc
    out['gr_look'] = look
    out['v_ground_auto'] = np.array(geo.orbit_to_vel(514e3, ground=True))
    vals = np.array([5, 17, 100, 127, 129, 500, 1000, 1023, 2049, 4095, 21000, 21600, 5159])
    out['fft_vals'] = vals
    for p in (2, 3, 5):
        out['fft_opt_%d' % p] = np.array([utils.optimize_fftsize(int(v), p) for v in vals])
    save("geometry.npz", **out)


# --------------------------------------------------------------------------------------
CFG_TEMPLATE = """\
# OCEANSAR raw-generation test configuration ({name})
[sar]
f0=5.405e9
inc_angle={inc}
pol={pol}
squint=0
prf={prf}
rg_bw=50e6
over_fs=1.1
alt=514e3
v_ground={v_ground}
heading=0.
ant_L_tx={ant_l}
ant_L_rx={ant_l}
num_ch={num_ch}
b_ati={b_ati}
b_xti={b_xti}
sigma_n_tx=0.
phase_n_tx=0.
sigma_beta_tx=0.
phase_beta_tx=0.
sigma_n_rx=0.
phase_n_rx=0.
sigma_beta_rx=0.
phase_beta_rx=0.

[ocean]
Lx={Lx}
Ly={Ly}
dx={dx}
dy={dy}
opt_res=True
fft_max_prime={fmp}
dt=0.05
depth={depth}
wind_dir={wind_dir}
wind_U={wind_U}
wind_fetch=500e3
swell_dir_enable={dswell}
sigf=0.007
freq_r={freq_r}
dir_swell_dir=120
sigs=8
Hs=0.8
swell_enable={swell}
swell_wl=60
swell_dir=20
swell_ampl=0.3
spec_model=elfouhaily
spread_model={spread}
cutoff_wl=auto
current_mag={cur}
current_dir=60.
choppy_enable={choppy}
frozen_ocean=False

[srg]
use_hmtf={hmtf}
nesz=-300.
wh_tol=2.73    ; wave-height tolerance added to the range window
scat_spec_enable={spec_on}
scat_spec_mode={spec_mode}
scat_bragg_enable=True
scat_bragg_model=romeiser97
scat_bragg_spec=elfouhaily
scat_bragg_spread={bspread}
scat_bragg_d=0.125
use_lut={lut}
"""

SAR_CASES = {
    # single channel vv, cos^2 spreading, Kodis specular on (the first benchmark family)
    "c1small": dict(inc=35., pol='vv', prf=1000., v_ground=7600., ant_l=120., num_ch=1, b_ati=0,
                    b_xti=0, Lx=64, Ly=64, dx=1., dy=1., fmp=2, depth=1e5, wind_dir=0., wind_U=10.,
                    dswell=False, freq_r=0.079, swell=False, spread='cos2s', cur=0., choppy=False,
                    hmtf=False, spec_on=True, bspread='cos2s', lut=False, spec_mode='kodis'),
    # two along-track channels, dual pol, hMTF, choppy waves, monochromatic swell, current
    "c2small": dict(inc=35., pol='DP', prf=1500., v_ground=7600., ant_l=100., num_ch=2, b_ati=10.,
                    b_xti=0, Lx=64, Ly=32, dx=1., dy=1., fmp=2, depth=1e5, wind_dir=45., wind_U=7.,
                    dswell=False, freq_r=0.079, swell=True, spread='elfouhaily', cur=0.2,
                    choppy=True, hmtf=True, spec_on=True, bspread='elfouhaily', lut=False, spec_mode='kodis'),
    # four channels (ATI 0/5/10/0 m, one 2 m XTI), directional swell, 0.5 m grid, hh
    "c3small": dict(inc=30., pol='hh', prf=2000., v_ground=7600., ant_l=130., num_ch=4,
                    b_ati='[0., 5., 10., 0.]', b_xti='[0., 0., 0., 2.]', Lx=24, Ly=27, dx=0.5, dy=0.5,
                    fmp=3, depth=1e5, wind_dir=30., wind_U=15., dswell=True,
                    freq_r=float(np.sqrt(const.g / (2 * np.pi * 250.))), swell=False,
                    spread='elfouhaily', cur=0., choppy=False, hmtf=False, spec_on=True,
                    bspread='elfouhaily', lut=False, spec_mode='kodis'),
    # the single-channel case with the Romeiser LUT mode (romeiser97.py:71-134)
    # Kirchhoff specular scattering (nrcs/ka.py): facet approach and stationary phase, dual pol
    "c1fa": dict(inc=35., pol='DP', prf=1000., v_ground=7600., ant_l=120., num_ch=1, b_ati=0,
                 b_xti=0, Lx=64, Ly=64, dx=1., dy=1., fmp=2, depth=1e5, wind_dir=0., wind_U=10.,
                 dswell=False, freq_r=0.079, swell=False, spread='cos2s', cur=0., choppy=False,
                 hmtf=False, spec_on=True, bspread='cos2s', lut=False, spec_mode='fa'),
    "c1spa": dict(inc=35., pol='vv', prf=1000., v_ground=7600., ant_l=120., num_ch=1, b_ati=0,
                  b_xti=0, Lx=64, Ly=64, dx=1., dy=1., fmp=2, depth=1e5, wind_dir=0., wind_U=10.,
                  dswell=False, freq_r=0.079, swell=False, spread='cos2s', cur=0., choppy=False,
                  hmtf=False, spec_on=True, bspread='cos2s', lut=False, spec_mode='spa'),
    "c1lut": dict(inc=35., pol='vv', prf=1000., v_ground=7600., ant_l=120., num_ch=1, b_ati=0,
                  b_xti=0, Lx=64, Ly=64, dx=1., dy=1., fmp=2, depth=1e5, wind_dir=0., wind_U=10.,
                  dswell=False, freq_r=0.079, swell=False, spread='cos2s', cur=0., choppy=False,
                  hmtf=False, spec_on=True, bspread='cos2s', lut=True, spec_mode='kodis'),
}


def write_cfg(name, kw):
    path = os.path.join(OUT, "cfg", name + ".cfg")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write(CFG_TEMPLATE.format(name=name, **kw))
    return path


def cfg_to_json(cfg):
    d = {}
    for sec in cfg.sections[1:]:
        s = vars(cfg)[sec]
        d[sec] = {}
        for el in s.elements:
            v = vars(s)[el]
            if isinstance(v, np.ndarray):
                d[sec][el] = {"ndarray": v.tolist(), "dtype": str(v.dtype)}
            elif isinstance(v, bool):
                d[sec][el] = {"bool": v}
            elif isinstance(v, int):
                d[sec][el] = {"int": v}
            elif isinstance(v, float):
                d[sec][el] = {"float": v}
            elif isinstance(v, list):
                d[sec][el] = {"list": v}
            else:
                d[sec][el] = {"str": v}
    top = {}
    for el in cfg.elements:
        top[el] = repr(vars(cfg)[el])
    return {"sections": cfg.sections[1:], "values": d, "top": top}


QUIRKS_CFG = """\
top_level=3
# comment line
; another comment
[alpha]
an_int=42
neg_int=-3
a_float=2.5e3
a_bool=True
b_bool=False
a_str=elfouhaily
a_path=/some/dir/file.nc
with_comment=7.5   ; trailing comment
f_array=[1.5, 2, -3e2]
s_array=['hh', 'vv']
b_array=[True, False, True]
none_value=None
auto_value=auto
spaced = 12
[beta]
one_elem=[0]
after_trap=1.0
"""


def gen_cfg_and_sar(only=None):
    res = {}
    qpath = os.path.join(OUT, "cfg", "quirks.cfg")
    os.makedirs(os.path.dirname(qpath), exist_ok=True)
    with open(qpath, "w") as f:
        f.write(QUIRKS_CFG)
    res["quirks"] = cfg_to_json(ocs_io.ConfigFile(qpath))
    for name, kw in SAR_CASES.items():
        path = write_cfg(name, kw)
        res[name] = cfg_to_json(ocs_io.ConfigFile(path))
    with open(os.path.join(OUT, "cfg_parsed.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    print("wrote cfg_parsed.json")

    for name in SAR_CASES:
        if only and name not in only:
            continue
        path = os.path.join(OUT, "cfg", name + ".cfg")
        calls = []
        orig = sar_raw_nompi.raw.chan_profile_numba

        def recorder(srg, scene, binsize, min_sr, sinc_vec, n, ovs, output, rg_only=False):
            before = output.copy()
            orig(srg, scene, binsize, min_sr, sinc_vec, n, ovs, output, rg_only)
            if len(calls) < 3:
                calls.append(dict(srg=srg.copy(), scene=scene.copy(), binsize=binsize,
                                  min_sr=min_sr, out0=before, out=output.copy()))

        sar_raw_nompi.raw.chan_profile_numba = recorder
        try:
            np.random.seed(0)
            out_file = "/tmp/golden_%s_raw.nc" % name
            ocean_file = "/tmp/golden_%s_ocean.nc" % name
            sar_raw_nompi.sar_raw(path, out_file, ocean_file, False, None, False, plot_save=False)
        finally:
            sar_raw_nompi.raw.chan_profile_numba = orig
        ds = ref_shims.NC_STORE[out_file]
        v = ds.variables
        raw = v['raw_data_r'].data + 1j * v['raw_data_i'].data
        oc = ref_shims.NC_STORE[ocean_file].variables
        arrs = dict(raw=raw, NRCS_avg=v['NRCS_avg'].data,
                    sr0=v['sr0'].data, b_ati=v['b_ati'].data, b_xti=v['b_xti'].data,
                    v_ground=v['v_ground'].data, rg_sampling=v['rg_sampling'].data,
                    wave_coefs=(oc['wave_coefs_r'].data + 1j * oc['wave_coefs_i'].data))
        for i, c in enumerate(calls):
            for k, val in c.items():
                arrs["call%d_%s" % (i, k)] = np.asarray(val)
        save("sar_raw_%s.npz" % name, **arrs)


# --------------------------------------------------------------------------------------
DOPSCA_TEMPLATE = """\
# OCEANSAR DopSCA test configuration ({name})
[sca]
f0=5.4e9
inc_angle={inc}
pol={pol}
prf={prf}
rg_bw={rg_bw}
over_fs=2.0
squint=0
alt=817e3
v_ground={v_ground}
heading=-11.2
ant_L_tx=3
ant_L_rx=3
num_ch=1
n_subpulses={n_sub}
sub_pulse_length={sub_len}
sub_pulse_bw=1e6
nesz=-26
use_errors=False
sigma_n_tx=0.12
phase_n_tx=2.3
sigma_beta_tx=0.2
phase_beta_tx=0.2
sigma_n_rx=0.04
phase_n_rx=0.2
sigma_beta_rx=0.04
phase_beta_rx=0.2

[acquisition]
length={length}

[ocean]
N_repeat_x={n_rep}
Lx={Lx}
Ly={Ly}
dx={dx}
dy={dy}
opt_res=True
dt=0.05
depth=500
wind_dir={wind_dir}
wind_U=10
wind_fetch=500e3
swell_dir_enable=False
sigf=0.007
freq_r= .068
dir_swell_dir = 70
sigs=8
Hs=1
swell_enable=False
swell_wl=80
swell_dir=45
swell_ampl=0.5
spec_model=elfouhaily
spread_model={spread}
cutoff_wl=auto
current_mag=0
current_dir=0.
frozen_ocean=False
fft_max_prime=3
choppy_enable={choppy}
use_buoy_data=False

[srg]
use_hmtf=False
nesz=-30.
wh_tol=2.73
scat_spec_enable={spec}
scat_spec_mode=kodis
scat_bragg_enable=True
scat_bragg_model=romeiser97
scat_bragg_spec=elfouhaily
scat_bragg_spread={spread}
scat_bragg_d=0.125
use_lut = False
"""

# The sub-pulse lengths keep the scatterer series short (N ~ 200 tau / sub_pulse_length):
# the reference factorises N by trial division in optimize_fftsize, which takes many
# minutes for the ~1e6-sample series of microsecond sub-pulses.
DOPSCA_CASES = {
    # vv, Kodis + Bragg, three range blocks, two sub-pulses
    "dsc1": dict(inc=35., pol='vv', prf=20., rg_bw=5e6, v_ground=7000., n_sub=2, sub_len=1e-3, length=2500.,
                 n_rep=3, Lx=512, Ly=256, dx=4, dy=4, wind_dir=30., spread='cos2s', choppy=False, spec=True),
    # dual pol, Bragg only, choppy surface, two blocks, three sub-pulses, orbital velocity
    "dsc2": dict(inc=30., pol='DP', prf=10., rg_bw=2e6, v_ground='auto', n_sub=3, sub_len=5e-4, length=4000.,
                 n_rep=2, Lx=256, Ly=128, dx=4, dy=4, wind_dir=0., spread='elfouhaily', choppy=True, spec=False),
}


def gen_dopsca():
    from oceansar.dopscasim import dopsca_raw as ref_dopsca
    for name, kw in DOPSCA_CASES.items():
        path = os.path.join(OUT, "cfg", name + ".cfg")
        with open(path, "w") as f:
            f.write(DOPSCA_TEMPLATE.format(name=name, **kw))
        np.random.seed(0)
        out_file = "/tmp/golden_%s/raw.nc" % name
        ocean_file = "/tmp/golden_%s/ocean.nc" % name
        os.makedirs(os.path.dirname(out_file), exist_ok=True)
        ref_dopsca.dopsca_raw(path, out_file, ocean_file, False, None, False, plot_save=False)
        v = ref_shims.NC_STORE[out_file].variables
        oc = ref_shims.NC_STORE[ocean_file].variables
        save("dopsca_%s.npz" % name, raw=v['raw_data_r'].data + 1j * v['raw_data_i'].data,
             NRCS_avg=v['NRCS_avg'].data, sr0=v['sr0'].data, v_ground=v['v_ground'].data,
             wave_coefs=(oc['wave_coefs_r'].data + 1j * oc['wave_coefs_i'].data))


# --------------------------------------------------------------------------------------
SKIM_TEMPLATE = """\
# OCEANSAR SKIM test configuration ({name})
[sim]
verbosity=0

[radar]
f0=35e9
inc_angle={inc}
pol={pol}
prf=32e3
rg_bw=200e6
Fs = 250e6
n_pulses = {n_pulses}
n_rg = 128
over_fs=1.1
azimuth = {azimuth}
alt=690e3
v_ground=auto
heading=-11.2
ant_L={ant_L}
L_total={L_total}
Spacing=50
num_ch={num_ch}
use_errors=False
sigma_n_tx=0.12
phase_n_tx=2.3
sigma_beta_tx=0.2
phase_beta_tx=0.2
sigma_n_rx=0.04
phase_n_rx=0.2
sigma_beta_rx=0.04
phase_beta_rx=0.2

[ocean]
Lx=64.
Ly=64.
dx=1
dy=1
opt_res=True
depth=100
wind_dir=45.
wind_U={wind_U}
wind_fetch=500e3
swell_enable=False
swell_wl=12.5
swell_dir=90
swell_ampl=1
swell_dir_enable={dir_swell}
sigf=0.007
freq_r= .068
dir_swell_dir=90
sigs=8
Hs=1.45
spec_model=elfouhaily
spread_model=elfouhaily
cutoff_wl=auto
current_mag=0.2
current_dir=90.
dt=0.002
fft_max_prime=3
choppy_enable={choppy}
use_buoy_data=False

[srg]
use_hmtf=False
nesz=-300.
wh_tol=5.
scat_spec_enable={spec}
scat_spec_mode={spec_mode}
scat_bragg_enable=True
scat_bragg_model=romeiser97
scat_bragg_spec=elfouhaily
scat_bragg_spread=elfouhaily
scat_bragg_d=0.125
two_scale_Doppler={two_scale}
surface_coh_time=2e-3
phase_err_tol=0.5
rcm = {rcm}
"""

# The antenna lengths keep at least two samples in the calibration's azimuth axis (step
# sr0 c / (pi f0 L 10)) over these short acquisitions; with one sample the reference's
# calibration factor is 1/sqrt(0).
SKIM_CASES = {
    # the shipped SKIM set-up, scaled down: vv, stationary-phase specular + Bragg, choppy,
    # directional swell, two-scale Doppler (8 simulated steps, groups of 16 rows)
    "skim1": dict(inc=12., pol='vv', n_pulses=256, azimuth=90, ant_L=10, L_total=False, num_ch=1, wind_U=3.,
                  dir_swell=True, choppy=True, spec=True, spec_mode='spa', two_scale=True, rcm=False),
    # dual pol, facet-approach specular + Bragg, squinted beam, L_total with two channels,
    # rcm in the bins (the reference's Kodis field fails on [Ny, 1] azimuth angles as soon
    # as a stationary point lies outside column 0, kodis.py:61)
    "skim2": dict(inc=10., pol='DP', n_pulses=256, azimuth=60, ant_L=10, L_total=True, num_ch=2, wind_U=7.,
                  dir_swell=False, choppy=False, spec=True, spec_mode='fa', two_scale=True, rcm=True),
    # single-scale form: every pulse simulated, all rows in one profile
    "skim3": dict(inc=12., pol='vv', n_pulses=64, azimuth=90, ant_L=30, L_total=False, num_ch=1, wind_U=5.,
                  dir_swell=False, choppy=False, spec=False, spec_mode='kodis', two_scale=False, rcm=False),
}


def gen_skim():
    from oceansar.radarsim import skim_raw as ref_skim
    for name, kw in SKIM_CASES.items():
        path = os.path.join(OUT, "cfg", name + ".cfg")
        with open(path, "w") as f:
            f.write(SKIM_TEMPLATE.format(name=name, **kw))
        np.random.seed(0)
        out_file = "/tmp/golden_%s/raw.nc" % name
        ocean_file = "/tmp/golden_%s/ocean.nc" % name
        os.makedirs(os.path.dirname(out_file), exist_ok=True)
        ref_skim.skimraw(path, out_file, ocean_file, False, None, False, plot_save=False)
        v = ref_shims.NC_STORE[out_file].variables
        oc = ref_shims.NC_STORE[ocean_file].variables
        save("skim_%s.npz" % name, raw=v['raw_data_r'].data + 1j * v['raw_data_i'].data,
             NRCS_avg=v['NRCS_avg'].data, dop_ref=v['dop_ref'].data, sr0=v['sr0'].data,
             wave_coefs=(oc['wave_coefs_r'].data + 1j * oc['wave_coefs_i'].data))


if __name__ == "__main__":
    which = sys.argv[1:] or ["sinc", "range_profile", "surfaces", "rcs", "kodis", "closure",
                             "geometry", "sar"]
    if "sinc" in which:
        gen_sinc()
    if "range_profile" in which:
        gen_range_profile()
    if "surfaces" in which:
        gen_surfaces()
    if "balancer" in which:
        gen_balancer()
    if "rcs" in which:
        gen_rcs()
    if "rcs_lut" in which:
        gen_rcs_lut()
    if "kodis" in which:
        gen_kodis()
    if "ka" in which:
        gen_ka()
    if "focus" in which:
        gen_focus()
    if "closure" in which:
        gen_closure()
    if "geometry" in which:
        gen_geometry()
    if "sar" in which:
        gen_cfg_and_sar()
    if "sar_lut" in which:
        gen_cfg_and_sar(only=["c1lut"])
    if "dopsca" in which:
        gen_dopsca()
    if "skim" in which:
        gen_skim()
    if "sar_ka" in which:
        gen_cfg_and_sar(only=["c1fa", "c1spa"])
