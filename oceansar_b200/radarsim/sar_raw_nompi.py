"""The raw-data generator ``sar_raw`` (``oceansar/radarsim/sar_raw_nompi.py:32-641``) on the GPU.

``RawGenerator`` does the reference's set-up on the host -- in the same order, so that the
global numpy RNG produces the same surface, the same random scatterer series and the same
noise for the same seed -- and then keeps everything per pulse on the device:

* ``OceanSurface.set_t`` -> ``ocs_surface_update`` (surface fields of the pulse),
* ``ocs_pulse`` -> slant range, Kodis specular field, Romeiser Bragg RCS (refreshed when
  ``t_now - t_last > ocean_dt``, ``:432``), Bragg phases and sub-grid scatterers, antenna
  pattern, ATI / XTI phases and the accumulation into the raw cube.

``precision='f64'`` is the drop-in (float64 throughout, slant range and bin indices
bit-identical with numpy); ``precision='mixed'`` keeps the slant range, the bin / LUT indices
and the 2 k0 r phase reduction in float64 and runs the rest in float32, with a complex64
raw cube.  ``sar_raw`` wraps it with the reference's signature and writes the raw file.
"""
import ctypes
import math

import numpy as np
import torch
from scipy import linalg

from .. import _capi, _device, nrcs, swell_spec
from .._structs import PulseDesc
from ..closure import grid_coherence, randomscat_ts
from ..ocs_io.cfg import ConfigFile
from ..ocs_io.raw import RawFile
from ..surfaces import OceanSurface
from ..utils import geometry as geo
from ..utils.misc import db2lin, optimize_fftsize
from .range_profile import calc_sinc_vec

C_LIGHT = 2.99792458e8
G = 9.80665
PRECISIONS = {'f64': 0, 'mixed': 1}


def sinc_bp(sin_angle, L, f0, field=False):
    """Uniform-aperture pattern (``oceansar/radarsim/antenna.py:5-25``, no squint)."""
    pattern = np.sinc(L / (C_LIGHT / f0) * sin_angle)
    return pattern if field else pattern ** 2


def scene_device_bytes(nx, ny, nfields, npol, nch, az_steps, rg_samp, precision, bragg=True):
    """Device memory a scene holds while it runs (bytes): spectrum, omega, surface fields and
    FFT scratch, sqrt(RCS), scatterer index maps, raw cube and small tables.  Used to admit
    scenes under a memory budget before they are allocated."""
    nf = float(nx) * ny
    npair = (nfields + 1) // 2
    cb = 16 if precision == 'f64' else 8
    b = nf * (8 + 4)                         # wave coefficients, omega
    b += nf * 4 * nfields                    # fields
    b += nf * 8 * npair                      # FFT scratch planes
    if bragg:
        b += nf * (8 if precision == 'f64' else 4) * 2 * npol + nf * 4 * 2
    b += float(npol) * nch * az_steps * rg_samp * cb
    b += az_steps * (8 + 8 * npol + 64) + ny * (5 + 2 * nch) * 8 + (nx + ny) * 64 + (1 << 20)
    return int(b)


class RawGenerator(object):
    """Device-resident state of one ``sar_raw`` scene; see the module docstring.

    ``overrides`` may fix ``az_steps`` / ``rg_samp`` / ``rg_samp_orig`` (the reference
    derives them from the geometry, ``sar_raw_nompi.py:264-278``).  ``device=False`` does
    only the host set-up (no GPU touched; the object pickles), and ``to_device()`` then
    uploads and allocates -- scene preparation in worker processes.  ``surface_dt`` (e.g. the
    .cfg's ocean dt) selects the time-interpolated surface of the reference's MPI generator
    (``OceanSurfaceBalancer``, ``sar_raw.py:233-353``): surfaces synthesised every
    ``surface_dt`` seconds, fields interpolated linearly in between.
    """

    def __init__(self, cfg, precision='f64', overrides=None, seed=None, stream=None, device=True,
                 surface_dt=None):
        if precision not in PRECISIONS:
            raise ValueError('precision must be f64 or mixed')
        self.precision = precision
        self.stream = stream
        if isinstance(cfg, str):
            cfg = ConfigFile(cfg)
        self.cfg = cfg
        ov = dict(overrides or {})
        if seed is not None:
            np.random.seed(seed)
        srg, sar, oc = cfg.srg, cfg.sar, cfg.ocean
        self.nesz = srg.nesz
        self.wh_tol = srg.wh_tol
        self.use_hmtf = bool(srg.use_hmtf)
        self.scat_spec_enable = bool(srg.scat_spec_enable)
        self.scat_bragg_enable = bool(srg.scat_bragg_enable)
        self.scat_spec_mode = srg.scat_spec_mode if self.scat_spec_enable else 'kodis'
        if self.scat_spec_enable and self.scat_spec_mode not in ('kodis', 'fa', 'spa'):
            raise NotImplementedError('RCS mode %s for specular scattering not implemented' % srg.scat_spec_mode)
        if self.scat_bragg_enable and srg.scat_bragg_model != 'romeiser97':
            raise NotImplementedError('RCS model %s for Bragg scattering not implemented' % srg.scat_bragg_model)
        self.inc_angle = np.deg2rad(sar.inc_angle)
        self.f0 = f0 = sar.f0
        self.pol = pol = sar.pol
        self.do_hh = pol in ('DP', 'hh')
        self.do_vv = pol not in ('hh',)
        self.npol = 2 if pol == 'DP' else 1
        self.prf = sar.prf
        self.num_ch = int(sar.num_ch)
        if self.num_ch > 8:
            raise ValueError('at most 8 channels')
        alt = sar.alt
        v_ground = sar.v_ground
        self.rg_bw = sar.rg_bw
        self.over_fs = sar.over_fs
        self.ocean_dt = oc.dt
        self.chan_sinc_vec = calc_sinc_vec(8, 20, Fs=self.over_fs)

        # ---- surface (global RNG draw 1: random_cg, then swell) -------------------------
        compute = ['D', 'Diff']
        if self.scat_spec_enable:
            compute.append('Diff2')
        if self.use_hmtf:
            compute.append('hMTF')
        if hasattr(oc, 'use_buoy_data') and oc.use_buoy_data:
            raise NotImplementedError('buoy-spectrum input is not built')
        dir_swell = swell_spec.ardhuin_swell_spec if oc.swell_dir_enable else None
        s = self.surface = OceanSurface()
        s.init(oc.Lx, oc.Ly, oc.dx, oc.dy, oc.cutoff_wl, oc.spec_model, oc.spread_model,
               np.deg2rad(oc.wind_dir), oc.wind_fetch, oc.wind_U, oc.current_mag,
               np.deg2rad(oc.current_dir), oc.dir_swell_dir, oc.freq_r, oc.sigf, oc.sigs, oc.Hs,
               oc.swell_dir_enable, oc.swell_enable, oc.swell_ampl, np.deg2rad(oc.swell_dir),
               oc.swell_wl, compute, oc.opt_res, oc.fft_max_prime, choppy_enable=oc.choppy_enable,
               depth=oc.depth, dirspectrum_func=None, dir_swell_spec=dir_swell, device=device)
        self.frozen = bool(getattr(oc, 'frozen_ocean', False))
        self.surface_dt = surface_dt if (surface_dt and not self.frozen) else None
        self.balancer = None

        # ---- geometry (:231-278) ----------------------------------------------------------
        self.sr0 = sr0 = geo.inc_to_sr(self.inc_angle, alt)
        self.gr0 = gr0 = geo.inc_to_gr(self.inc_angle, alt)
        sr, inc, _ = geo.gr_to_geo(s.x + gr0, alt)
        self.sr_near = sr[0] - self.wh_tol + C_LIGHT / 2 / (self.rg_bw * self.over_fs)
        sr -= np.min(sr)
        self.inc = inc.reshape(1, inc.size)
        self.sr = sr.reshape(1, sr.size)
        self.sin_inc = np.sin(self.inc)
        self.cos_inc = np.cos(self.inc)
        self.k0 = k0 = 2. * np.pi * f0 / C_LIGHT
        self.sr_res = C_LIGHT / (2. * self.rg_bw)
        self.ant_l_tx = sar.ant_L_tx
        self.ant_l_rx = sar.ant_L_rx
        b_ati = sar.b_ati
        if not type(b_ati) == np.ndarray:
            b_ati = np.arange(self.num_ch) * b_ati
        b_xti = sar.b_xti
        if not type(b_xti) == np.ndarray:
            b_xti = np.arange(self.num_ch) * b_xti
        self.b_ati, self.b_xti = np.asarray(b_ati, float), np.asarray(b_xti, float)
        if v_ground == 'auto':
            v_ground = geo.orbit_to_vel(alt, ground=True)
        self.v_ground = v_ground
        self.t_step = 1. / self.prf
        self.t_span = (1.5 * (sr0 * (C_LIGHT / f0) / self.ant_l_tx) + s.Ly) / v_ground
        self.az_steps = int(ov.get('az_steps', int(np.floor(self.t_span / self.t_step))))
        max_sr = (np.max(sr) + self.wh_tol + (np.max(s.y) + (self.t_span / 2.) * v_ground) ** 2. / (2. * sr0))
        self.min_sr = np.min(sr) - self.wh_tol
        self.rg_samp_orig = int(ov.get('rg_samp_orig',
                                       int(np.ceil(((max_sr - self.min_sr) / self.sr_res) * self.over_fs))))
        self.rg_samp = int(ov.get('rg_samp', int(optimize_fftsize(self.rg_samp_orig))))
        self.surface_area = s.dx * s.dy * s.Nx * s.Ny

        # ---- scattering models (:293-340; global RNG draw 2: rndscat_p then rndscat_m) ---
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                self.rcs_spec = nrcs.RCSKodis(self.inc, k0, s.dx, s.dy)
            else:
                # sar_raw_nompi.py:296-299: the reference draws a phase screen here (unused)
                self.spec_ph0 = np.random.uniform(0., 2. * np.pi, size=[s.Ny, s.Nx])
                self.rcs_spec = nrcs.RCSKA(self.scat_spec_mode, k0, s.x, s.y, s.dx, s.dy)
        if self.scat_bragg_enable:
            tau_c = grid_coherence(oc.wind_U, s.dx, f0)
            self.rndscat_p = randomscat_ts(tau_c, (s.Ny, s.Nx), self.prf)
            self.rndscat_m = randomscat_ts(tau_c, (s.Ny, s.Nx), self.prf)
            k_b = 2. * k0 * self.sin_inc
            self.c_b = self.sin_inc * np.sqrt(G / k_b + 0.072e-3 * k_b)
            cdir = np.deg2rad(oc.current_dir)
            cur = oc.current_mag * np.array([np.cos(cdir), np.sin(cdir)])
            udir = np.deg2rad(oc.wind_dir)
            u_eff = oc.wind_U * np.array([np.cos(udir), np.sin(udir)]) - cur
            self.rcs_bragg = nrcs.RCSRomeiser97(k0, self.inc, pol, s.dx, s.dy, linalg.norm(u_eff),
                                                np.arctan2(u_eff[1], u_eff[0]), s.wind_fetch,
                                                srg.scat_bragg_spec, srg.scat_bragg_spread,
                                                srg.scat_bragg_d, rmss_x=s.rmss_x, rmss_y=s.rmss_y,
                                                az_span=(self.t_span * v_ground + s.Ly) / gr0,
                                                use_lut=bool(srg.use_lut))
        self._on_device = False
        if device:
            self.to_device()
        self.t_last_rcs_bragg = -1.

    def to_device(self):
        """Upload the host set-up and allocate the device buffers (once)."""
        if not self._on_device:
            self.surface.to_device()
            self._alloc()
            self._on_device = True
        return self

    def device_bytes(self):
        """Device memory of the scene's buffers (bytes), known before ``to_device``."""
        nfields = 5 + (3 if self.scat_spec_enable else 0) + (1 if self.use_hmtf else 0)
        return scene_device_bytes(self.surface.Nx, self.surface.Ny, nfields, self.npol, self.num_ch,
                                  self.az_steps, self.rg_samp, self.precision, self.scat_bragg_enable)

    # ------------------------------------------------------------------------------------
    def _alloc(self):
        s = self.surface
        cdt = np.complex128 if self.precision == 'f64' else np.complex64
        sdt = np.float64 if self.precision == 'f64' else np.float32
        nout = self.npol * self.num_ch
        self.raw_d = _device.zeros((nout, self.az_steps, self.rg_samp), cdt)
        self.nrcs_spec_d = _device.zeros((self.az_steps,), np.float64)
        self.nrcs_bragg_d = _device.zeros((self.npol, self.az_steps), np.float64)
        col = lambda a: _device.to_device(np.ravel(a), np.float64)  # noqa: E731
        self._cols = dict(sr=col(self.sr), sin=col(self.sin_inc), cos=col(self.cos_inc),
                          tan=col(np.tan(self.inc)), inc=col(self.inc))
        self._y_d = _device.to_device(s.y, np.float32)
        self._sinc_d = _device.to_device(self.chan_sinc_vec, np.float32)
        self._b_ati = (ctypes.c_double * self.num_ch)(*[float(v) for v in self.b_ati])
        self._b_xti = (ctypes.c_double * self.num_ch)(*[float(v) for v in self.b_xti])
        d = self.desc = PulseDesc()
        d.nx, d.ny, d.npol, d.nch = s.Nx, s.Ny, self.npol, self.num_ch
        d.pol = nrcs.POL_CODES[self.pol]
        f = s.field
        if self.surface_dt:
            from ..surfaces import OceanSurfaceBalancer
            self.balancer = OceanSurfaceBalancer(s, self.surface_dt)
            f = self.balancer.field
        d.dx_d, d.dy_d, d.dz_d = f('Dx').data_ptr(), f('Dy').data_ptr(), f('Dz').data_ptr()
        d.diffx_d, d.diffy_d = f('Diffx').data_ptr(), f('Diffy').data_ptr()
        if self.scat_spec_enable:
            d.diffxx_d, d.diffyy_d, d.diffxy_d = (f('Diffxx').data_ptr(), f('Diffyy').data_ptr(),
                                                  f('Diffxy').data_ptr())
        if self.use_hmtf:
            d.hmtf_d = f('hMTF').data_ptr()
        d.y_d = self._y_d.data_ptr()
        c = self._cols
        d.sr_col_d, d.sin_inc_d, d.cos_inc_d = c['sr'].data_ptr(), c['sin'].data_ptr(), c['cos'].data_ptr()
        d.tan_inc_d, d.inc_d = c['tan'].data_ptr(), c['inc'].data_ptr()
        d.inc_angle, d.sr0, d.gr0, d.k0, d.f0 = (float(self.inc_angle), float(self.sr0), float(self.gr0),
                                                 float(self.k0), float(self.f0))
        d.min_sr, d.binsize, d.t_step = float(self.min_sr), float(self.sr_res / self.over_fs), float(self.t_step)
        d.az_steps = self.az_steps
        d.ant_l_tx, d.ant_l_rx = float(self.ant_l_tx), float(self.ant_l_rx)
        d.b_ati, d.b_xti = self._b_ati, self._b_xti
        d.do_kodis, d.do_bragg, d.use_hmtf = int(self.scat_spec_enable), int(self.scat_bragg_enable), \
            int(self.use_hmtf)
        d.facet_dx, d.facet_dy = float(s.dx), float(s.dy)
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                d.kodis_R_re, d.kodis_R_im = float(self.rcs_spec.R.real), float(self.rcs_spec.R.imag)
            else:
                d.spec_mode = 1 if self.scat_spec_mode == 'fa' else 2
                self._x_d = _device.to_device(s.x, np.float32)
                d.x_d = self._x_d.data_ptr()
                d.ka_dx, d.ka_dy = float(s.dx), float(s.dy)
                K = self.rcs_spec.constant(1, 1)
                d.ka_K_re, d.ka_K_im = K.real, K.imag
        if self.scat_bragg_enable:
            self.rcs_bragg.fill(d)
            d.bragg_d = float(self.rcs_bragg.d)
            self._c_b_d = col(self.c_b)
            d.c_b_d = self._c_b_d.data_ptr()
            self._scat_d = torch.empty((self.npol, 2, s.Ny, s.Nx), dtype=torch.float64 if sdt == np.float64
                                       else torch.float32, device=_device.device())
            d.scat_d = self._scat_d.data_ptr()
            sm, im = self.rndscat_m.device()
            sp, ip = self.rndscat_p.device()
            d.s_m_d, d.s_p_d, d.n_m, d.n_p = sm.data_ptr(), sp.data_ptr(), int(self.rndscat_m.N), \
                int(self.rndscat_p.N)
            if self.precision == 'mixed':
                d.s_m32_d, d.s_p32_d = self.rndscat_m.device32().data_ptr(), self.rndscat_p.device32().data_ptr()
            d.ind0_m_d, d.ind0_p_d = im.data_ptr(), ip.data_ptr()
            if self.rcs_bragg.use_lut:
                self._lut_d = self.rcs_bragg.lut_device(self.precision)
                d.lut_d = self._lut_d.data_ptr()
                (d.lut_naz, d.lut_ndy, d.lut_ndx, d.lut_az0, d.lut_daz, d.lut_dy0, d.lut_ddy, d.lut_dx0,
                 d.lut_ddx) = self.rcs_bragg.lut_params()
        d.sinc_d = self._sinc_d.data_ptr()
        d.raw_d = self.raw_d.data_ptr()
        d.nbins = self.rg_samp
        d.nrcs_spec_d = self.nrcs_spec_d.data_ptr()
        d.nrcs_bragg_d = self.nrcs_bragg_d.data_ptr()
        nb = _capi.load().ocs_pulse_workspace_bytes(s.Ny, self.num_ch)
        self._rowtab = torch.empty(int(nb), dtype=torch.uint8, device=_device.device())
        d.rowtab_d = self._rowtab.data_ptr()
        if self.precision == 'mixed':
            # compensation row of the raw cube's compensated float32 accumulation
            self._raw_lo = _device.zeros((nout, self.rg_samp), cdt)
            d.raw_lo_d = self._raw_lo.data_ptr()
        _capi.call("ocs_pulse_reset", ctypes.addressof(d), _device.stream_ptr(self.stream))
        self._refreshes = []

    # ------------------------------------------------------------------------------------
    def pulse(self, az_step, update_surface=True, buffer=0, surface_stream=None):
        """One iteration of the azimuth loop (``sar_raw_nompi.py:349-535``).

        ``update_surface=False`` keeps whatever the surface field buffers hold (used to
        feed externally computed fields, stage by stage).  ``buffer`` selects the field set
        (1: the second set of ``run_overlapped``); ``surface_stream`` the stream of the
        surface update (default: the pulse's)."""
        t_now = az_step * self.t_step
        az_now = (t_now - self.t_span / 2.) * self.v_ground
        if update_surface and self.balancer is not None:
            self.balancer.set_t(t_now, stream=self.stream)
        elif update_surface and ((not self.frozen) or az_step == 0):
            # a frozen ocean keeps the t = 0 surface (the reference leaves it unset)
            self.surface.set_t(t_now, stream=surface_stream if surface_stream is not None else self.stream,
                               buffer=buffer)
        d = self.desc if buffer == 0 else self._desc_b
        d.az_step = int(az_step)
        d.az_now = float(az_now)
        d.refresh = 0
        if self.scat_bragg_enable:
            d.tind = self.rndscat_m.tind(t_now)
            if (t_now - self.t_last_rcs_bragg) > self.ocean_dt:
                self._lut_check(az_now)
                d.refresh = 1
                self.t_last_rcs_bragg = t_now
                self._refreshes.append(az_step)
        _capi.call("ocs_pulse", ctypes.addressof(d), PRECISIONS[self.precision],
                   _device.stream_ptr(self.stream))

    def pulse_schedule(self):
        """Per-pulse inputs of the whole scene, computed as ``pulse`` computes them pulse
        by pulse (same float32 time, additive terms, swell rotation, azimuth position,
        surface-update and Bragg-refresh decisions and scatterer offsets), for the scene
        batch.  Returns (tables, refresh pulses, time of the last refresh)."""
        s = self.surface
        n = self.az_steps
        nf = max(1, len(s._raw))
        t32 = np.zeros(n, np.float32)
        add = np.zeros((n, nf), np.float32)
        rot = np.zeros((n, 2), np.float32)
        az_now = np.zeros(n, np.float64)
        flags = np.zeros(n, np.int32)
        tmod = np.zeros((n, 2), np.int32)
        t_last = -1.
        refreshes = []
        for a in range(n):
            t_now = a * self.t_step
            az_now[a] = (t_now - self.t_span / 2.) * self.v_ground
            if (not self.frozen) or a == 0:
                flags[a] |= 1
            tt, ad, ro = s.time_terms(t_now)
            t32[a] = tt
            add[a, :len(ad)] = ad
            rot[a] = (np.real(ro), np.imag(ro))
            if self.scat_bragg_enable:
                tind = self.rndscat_m.tind(t_now)
                tmod[a] = (tind % int(self.rndscat_m.N), tind % int(self.rndscat_p.N))
                if (t_now - t_last) > self.ocean_dt:
                    self._lut_check(az_now[a])
                    flags[a] |= 2
                    t_last = t_now
                    refreshes.append(a)
        tables = dict(t=t32, add=add, swell_rot=rot if s.swell_enable else None, az_now=az_now,
                      flags=flags, tmod=tmod)
        return tables, refreshes, t_last

    def _lut_check(self, az_now):
        """LUT mode: the rows' azimuth indices must exist in the table, as numpy indexing
        requires (negative ones count from the end); raise IndexError as the reference's
        lookup would (romeiser97.py:117, 134)."""
        if not (self.scat_bragg_enable and self.rcs_bragg.use_lut):
            return
        m = self.rcs_bragg
        az = (self.surface.y - az_now).reshape((self.surface.Ny, 1))
        ind = np.round((np.arcsin(az / self.gr0) - m.lut_az.min()) /
                       (m.lut_az[1, 0, 0] - m.lut_az[0, 0, 0])).astype(int)
        n = m.lut_az.shape[0]
        if ind.max() >= n or ind.min() < -n:
            bad = int(ind.max() if ind.max() >= n else ind.min())
            raise IndexError('index %d is out of bounds for axis 0 with size %d' % (bad, n))

    def run(self, steps=None):
        for a in (range(self.az_steps) if steps is None else steps):
            self.pulse(a)
        self.flush()

    def flush(self, stream=None):
        """Fold the last pulse's compensation row into the raw cube (mixed form; a no-op
        otherwise).  ``run``, ``run_overlapped`` and ``raw`` call it."""
        _capi.call("ocs_pulse_flush", ctypes.addressof(self.desc),
                   _device.stream_ptr(stream if stream is not None else self.stream))

    def check(self):
        """Raise if a bounded device-side wait of the pulse kernel gave up (synchronises)."""
        st = _capi.load().ocs_pulse_error(ctypes.addressof(self.desc))
        if st != 0:
            raise RuntimeError('ocs_pulse: a device-side wait gave up (status %d)' % st)

    def can_overlap(self):
        """Whether ``run_overlapped`` applies (not for choppy, frozen or time-interpolated
        surfaces)."""
        return not self.surface._aux and not self.frozen and self.balancer is None

    def _second_desc(self):
        """The pulse descriptor reading the second field set."""
        if getattr(self, '_desc_b', None) is None:
            fb = self.surface.second_buffer()
            d = PulseDesc.from_buffer_copy(self.desc)
            d.b_ati, d.b_xti = self._b_ati, self._b_xti
            d.dx_d, d.dy_d, d.dz_d = fb['Dx'].data_ptr(), fb['Dy'].data_ptr(), fb['Dz'].data_ptr()
            d.diffx_d, d.diffy_d = fb['Diffx'].data_ptr(), fb['Diffy'].data_ptr()
            if 'Diffxx' in fb:
                d.diffxx_d, d.diffyy_d, d.diffxy_d = (fb['Diffxx'].data_ptr(), fb['Diffyy'].data_ptr(),
                                                      fb['Diffxy'].data_ptr())
            if 'hMTF' in fb:
                d.hmtf_d = fb['hMTF'].data_ptr()
            self._desc_b = d
        return self._desc_b

    def run_overlapped(self, steps=None):
        """The azimuth loop with the surface of pulse a + 1 synthesised on a second stream,
        into the other of two field sets, while pulse a's kernels read theirs.  Same result
        as ``run`` (only the kernels' overlap on the GPU differs).  Enqueued on the current
        stream (forked and joined), so it can be recorded into a CUDA graph."""
        if not self.can_overlap():
            return self.run(steps)
        self._second_desc()
        steps = list(range(self.az_steps) if steps is None else steps)
        main = torch.cuda.current_stream()
        if getattr(self, '_surf_stream', None) is None:
            self._surf_stream = torch.cuda.Stream()
        side = self._surf_stream
        side.wait_stream(main)
        done_surf, done_pulse = {}, {}
        saved = self.stream
        self.stream = main
        try:
            for i, a in enumerate(steps):
                buf = i % 2
                if i >= 2:
                    side.wait_event(done_pulse[i - 2])          # its fields were read by pulse i-2
                t_now = a * self.t_step
                self.surface.set_t(t_now, stream=side, buffer=buf)
                ev = torch.cuda.Event()
                ev.record(side)
                done_surf[i] = ev
                main.wait_event(ev)
                self.pulse(a, update_surface=False, buffer=buf)
                evp = torch.cuda.Event()
                evp.record(main)
                done_pulse[i] = evp
            self.flush(stream=main)
        finally:
            self.stream = saved
        main.wait_stream(side)

    def reset(self):
        """Clear the raw cube and NRCS accumulators and restart the Bragg refresh clock."""
        self.raw_d.zero_()
        self.nrcs_spec_d.zero_()
        self.nrcs_bragg_d.zero_()
        _capi.call("ocs_pulse_reset", ctypes.addressof(self.desc), _device.stream_ptr(self.stream))
        self.t_last_rcs_bragg = -1.
        self._refreshes = []
        if self.balancer is not None:
            self.balancer.restart()

    # ------------------------------------------------------------------------------------
    def capture(self, overlap=True):
        """Record reset + every pulse of the scene into one CUDA graph (with ``overlap``,
        the surface of the next pulse on a second stream, as ``run_overlapped``).

        The per-pulse host work (time, azimuth, refresh decision, launch arguments) is
        done once, at capture; ``replay()`` then re-issues the whole scene with a single
        graph launch.  One ordinary pass runs first (warm-up and lazy set-up)."""
        self.reset()
        self.run()
        if overlap and self.can_overlap():
            self._second_desc()                 # second field set, allocated outside the capture
            self._surf_stream = getattr(self, '_surf_stream', None) or torch.cuda.Stream()
        torch.cuda.synchronize()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        saved, self.stream = self.stream, None
        with torch.cuda.graph(g, stream=side):
            self.reset()
            if overlap and self.can_overlap():
                self.run_overlapped()
            else:
                self.run()
        self.stream = saved
        torch.cuda.current_stream().wait_stream(side)
        self._graph = g
        return g

    def replay(self):
        """Re-run the captured scene (raw cube and NRCS start from zero)."""
        self._graph.replay()

    def kernel_launches_per_scene(self):
        """Kernels of this library launched by one pass over the scene."""
        surf = 2 + (1 if self.surface._aux else 0)
        nout = self.npol * self.num_ch
        group = 2 if self.precision == 'f64' else 4
        pulse = 1 + (nout + group - 1) // group          # row table + pulse kernel(s)
        if self.balancer is not None:                    # syntheses at the ends + one blend per pulse
            times = [a * self.t_step for a in range(self.az_steps)]
            return self.balancer.syntheses(times) * surf + self.az_steps * (1 + pulse)
        return self.az_steps * (surf + pulse)

    def time_stages(self, steps):
        """Average device time [ms] of the surface update and of the pulse kernel(s) over
        ``steps`` pulses, from CUDA events on the launching stream."""
        t = self.time_kernels(steps)
        return t['surface_rows'] + t['surface_cols'], t['pulse'], None, None

    def time_kernels(self, steps, repeats=1):
        """Average device time [ms] per pulse of each kernel of the scene loop over ``steps``
        pulses: 'surface_rows' (row pass), 'surface_cols' (column pass) and 'pulse' (the
        per-pulse row table and the fused NRCS / scene / accumulation kernel(s)), each from
        CUDA events recorded on the launching stream around that launch alone.  The window
        runs ``repeats`` times (same pulses, same Bragg refresh decisions); the result is the
        median of the windows' averages, and 'windows' holds every window's average."""
        st = torch.cuda.current_stream()
        mk = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
        steps = list(steps)
        names = ('surface_rows', 'surface_cols', 'pulse')
        saved_last = self.t_last_rcs_bragg
        wins = {n: [] for n in names}
        for _ in range(max(1, int(repeats))):
            self.t_last_rcs_bragg = saved_last
            ev = [[mk() for _ in range(4)] for _ in steps]
            for e, a in zip(ev, steps):
                t_now = a * self.t_step
                e[0].record(st)
                self.surface.set_t(t_now, passes=1)
                e[1].record(st)
                self.surface.set_t(t_now, passes=2)
                e[2].record(st)
                self.pulse(a, update_surface=False)
                e[3].record(st)
            torch.cuda.synchronize()
            for i, n in enumerate(names):
                wins[n].append(float(np.mean([e[i].elapsed_time(e[i + 1]) for e in ev])))
        self.t_last_rcs_bragg = saved_last
        out = {n: float(np.median(wins[n])) for n in names}
        out['windows'] = wins
        return out

    # ------------------------------------------------------------------------------------
    def nrcs_avg(self):
        """NRCS_avg[pol, az] (``:427-467``): specular plus Bragg, per unit surface area."""
        spec = self.nrcs_spec_d.cpu().numpy()
        bragg = self.nrcs_bragg_d.cpu().numpy()
        out = np.zeros((self.npol, self.az_steps))
        last = None
        filled = np.zeros_like(bragg)
        for a in range(self.az_steps):
            if a in self._refreshes:
                last = a
            if last is not None:
                filled[:, a] = bragg[:, last]
        for p in range(self.npol):
            if self.scat_spec_enable:
                out[p] += spec / self.surface_area
            if self.scat_bragg_enable:
                out[p] += filled[p] / self.surface_area
        return out

    def raw(self):
        """Accumulated raw cube [pol, ch, az, rg_samp] before calibration (host copy)."""
        self.flush()
        self.check()
        r = self.raw_d.cpu().numpy()
        return r.reshape(self.npol, self.num_ch, self.az_steps, self.rg_samp)

    def finish(self, add_noise=True):
        """Truncation, calibration factor and noise (``:552-574``) -> (raw, NRCS_avg)."""
        t_span, v = self.t_span, self.v_ground
        az_axis = np.arange(-t_span / 2. * v, t_span / 2. * v,
                            self.sr0 * C_LIGHT / (np.pi * self.f0 * self.ant_l_tx * 10.))
        pattern = (sinc_bp(az_axis / self.sr0, self.ant_l_tx, self.f0, field=True) *
                   sinc_bp(az_axis / self.sr0, self.ant_l_rx, self.f0, field=True))
        self.cal_factor = (1. / np.sqrt(np.trapezoid(np.abs(pattern) ** 2., az_axis) *
                                        self.sr_res / np.sin(self.inc_angle)))
        raw = self.raw()[:, :, :, :self.rg_samp_orig].astype(np.complex128)
        out = []
        for p in range(self.npol):
            r = raw[p]
            noise = 0.
            if add_noise:
                noise = (db2lin(self.nesz, amplitude=True) / np.sqrt(2.) *
                         (np.random.normal(size=r.shape) + 1j * np.random.normal(size=r.shape)))
            out.append(r * self.cal_factor + noise)
        return np.stack(out), self.nrcs_avg()


def sar_raw(cfg_file, output_file, ocean_file, reuse_ocean_file, errors_file, reuse_errors_file,
            plot_save=True, precision='f64', surface_dt=None):
    """Drop-in for ``sar_raw_nompi.sar_raw``: simulate and write the raw file.

    The raw file (``RawFile``: ``raw_data_r``/``raw_data_i`` [pol, ch, az, rg], ``NRCS_avg``,
    geometry scalars, baselines) and the ocean state file (``OceanStateFile``) are netCDF
    classic files with the reference's dimensions, variables and units; a file name ending
    in ``.npz`` gets the same variables in a numpy container instead.  ``errors_file`` /
    ``plot_save`` are accepted and unused, as in the reference.  ``surface_dt`` selects the
    time-interpolated surface (``RawGenerator``).
    """
    cfg = cfg_file if isinstance(cfg_file, ConfigFile) else ConfigFile(cfg_file)
    gen = RawGenerator(cfg, precision=precision, surface_dt=surface_dt)
    if ocean_file and not reuse_ocean_file:
        gen.surface.save(ocean_file)
    gen.run()
    total_raw, nrcs_avg = gen.finish(add_noise=True)
    if output_file:
        values = dict(NRCS_avg=nrcs_avg, inc_angle=np.rad2deg(gen.inc_angle), f0=gen.f0, num_ch=gen.num_ch,
                      ant_L=gen.ant_l_tx, prf=gen.prf, v_ground=gen.v_ground, orbit_alt=cfg.sar.alt,
                      sr0=gen.sr_near, rg_sampling=gen.rg_bw * gen.over_fs, rg_bw=gen.rg_bw, b_ati=gen.b_ati,
                      b_xti=gen.b_xti)
        if str(output_file).endswith('.npz'):
            np.savez(output_file, raw_data_r=total_raw.real, raw_data_i=total_raw.imag, **values)
        else:
            # sar_raw_nompi.py:580-600
            f = RawFile(output_file, 'w', raw_dim=total_raw.shape)
            f.set('raw_data*', total_raw)
            for k, v in values.items():
                f.set(k, v)
            f.close()
    return total_raw, nrcs_avg
