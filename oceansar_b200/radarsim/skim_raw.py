"""The SKIM raw-data generator (``oceansar/radarsim/skim_raw.py:84-689``) on the GPU.

SKIM is a near-nadir Doppler radar with a rotating beam; the reference simulates one beam
azimuth.  Compared with ``sar_raw`` its loop differs in these ways, all reproduced here:

* the surface is time-interpolated every ocean ``dt`` (``OceanSurfaceBalancer``) and set
  at every step;
* the slant range of a column is absolute, sin_az = az / sr per facet, and the antenna
  pattern (``sinc_1tx_nrx``, power units) is evaluated per facet;
* range profiles use a 10-tap pulse on the ``Fs`` sampling grid centred on the mean slant
  range (``sr_prof``);
* with ``two_scale_Doppler`` (the shipped configurations) the pulses are simulated at
  a reduced rate (one every ``n_pulses_b``), range-only profiles are summed over
  ``ny_integ`` surface rows, the phase range leaves out the az^2/(2 sr) term (it goes to
  the range bins only with ``rcm``), and ``upsample_and_dopplerize`` restores the PRF and
  applies the geometric Doppler of each row group.

The device does the surface, the row table and one pulse-kernel launch per simulated step
(the SKIM mode of ``ocs_pulse``, which writes the row-group profiles directly); the host
does the set-up in the reference's order (same RNG stream), calibration and noise; the
up-sampling and Doppler of the two-scale form run on the device (``ocs_skim_upsample``).  The
calibration target (``sim.cal_targets``) is the pulse kernel's centre-facet substitution.
Not built: buoy-spectrum input, which raises ``NotImplementedError``.
"""
import ctypes

import numpy as np
import torch
from scipy import linalg

from .. import _capi, _device, nrcs, swell_spec
from .._structs import PulseDesc
from ..closure import grid_coherence, randomscat_ts
from ..ocs_io.cfg import ConfigFile
from ..ocs_io.raw import SkimRawFile
from ..surfaces import OceanSurface, OceanSurfaceBalancer
from ..utils import geometry as geo
from ..utils.misc import db2lin, optimize_fftsize
from .range_profile import calc_sinc_vec
from .sar_processor import sinc_1tx_nrx
from .sar_raw_nompi import C_LIGHT, G, PRECISIONS

N_SINC, SINC_OVS = 10, 20


def upsample_and_dopplerize(ssraw, dop, n_up, prf, stream=None):
    """Up-sample the step profiles ``ssraw`` [steps, groups, rg] by ``n_up`` and apply the
    geometric Doppler ``dop`` [groups, rg] of each row group, summed over the groups
    (``skim_raw.py:51-81``); returns complex128 [steps * n_up, rg].

    On the device (``ocs_skim_upsample``): the reference's zero-padded azimuth spectrum
    transformed back is the band-limited (Dirichlet-kernel) interpolation of the step
    samples, which the kernel evaluates directly for every output sample and range bin, with
    the Doppler ramp applied in the same pass.  ``ssraw`` may be a numpy array or a device
    tensor (the generator passes its device profiles)."""
    dev = _device.device()
    x = torch.as_tensor(ssraw).to(device=dev, dtype=torch.complex128).contiguous()
    if x.dim() != 3:
        raise ValueError('ssraw must be [steps, groups, rg]')
    N, G, R = (int(v) for v in x.shape)
    n_up = int(n_up)
    d = torch.as_tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(dop, dtype=np.float64), (G, R))),
                        device=dev)
    y = torch.empty((N * n_up, R), dtype=torch.complex128, device=dev)
    D = torch.empty((N * n_up,), dtype=torch.complex128, device=dev)
    _capi.call("ocs_skim_upsample", x.data_ptr(), d.data_ptr(), y.data_ptr(), D.data_ptr(), N, G, R, n_up,
               float(prf), _device.stream_ptr(stream))
    return y.cpu().numpy()


class SkimGenerator(object):
    """Device-resident state of one SKIM acquisition; see the module docstring."""

    def __init__(self, cfg, precision='f64', seed=None, stream=None, ocean_file=None, reuse_ocean_file=False):
        if precision not in PRECISIONS:
            raise ValueError('precision must be f64 or mixed')
        self.precision = precision
        self.stream = stream
        if isinstance(cfg, str):
            cfg = ConfigFile(cfg)
        self.cfg = cfg
        if seed is not None:
            np.random.seed(seed)
        srg, radar, oc = cfg.srg, cfg.radar, cfg.ocean
        # calibration target at the scene centre (skim_raw.py:151-164): absent or False:
        # none; 'floating' (any case): moves with the surface; any other string: fixed
        cal = getattr(cfg.sim, 'cal_targets', False) if hasattr(cfg, 'sim') else False
        self.pt_mode = 0 if cal is False else (1 if str(cal).lower() == 'floating' else 2)
        self.wh_tol, self.nesz = srg.wh_tol, srg.nesz
        self.use_hmtf = bool(srg.use_hmtf)
        self.scat_spec_enable = bool(srg.scat_spec_enable)
        self.scat_spec_mode = srg.scat_spec_mode if self.scat_spec_enable else 'kodis'
        self.scat_bragg_enable = bool(srg.scat_bragg_enable)
        if self.scat_spec_enable and self.scat_spec_mode not in ('kodis', 'fa', 'spa'):
            raise NotImplementedError('RCS mode %s for specular scattering not implemented' % self.scat_spec_mode)
        if self.scat_bragg_enable and srg.scat_bragg_model != 'romeiser97':
            raise NotImplementedError('RCS model %s for Bragg scattering not implemented' % srg.scat_bragg_model)
        self.inc_angle = np.deg2rad(radar.inc_angle)
        self.f0 = f0 = radar.f0
        self.pol = pol = radar.pol
        self.squint_r = np.radians(90 - radar.azimuth)
        self.do_hh = pol in ('DP', 'hh')
        self.do_vv = pol not in ('hh',)
        self.npol = 2 if pol == 'DP' else 1
        self.prf = prf = radar.prf
        self.num_ch = num_ch = int(radar.num_ch)
        ant_L = radar.ant_L
        alt = radar.alt
        v_ground = radar.v_ground
        self.rg_bw = radar.rg_bw
        self.over_fs = radar.Fs / radar.rg_bw
        self.ocean_dt = oc.dt
        self.chan_sinc_vec = calc_sinc_vec(N_SINC, SINC_OVS, Fs=self.over_fs)
        wind_dir = radar.azimuth - oc.wind_dir          # wind relative to the beam (:171)

        # ---- surface (:173-305; global RNG draw 1) ---------------------------------------
        compute = ['D', 'Diff', 'Diff2']
        if self.use_hmtf:
            compute.append('hMTF')
        s = self.surface = OceanSurface()
        if reuse_ocean_file:
            try:
                s.load(ocean_file, compute)
            except RuntimeError:
                pass
        if (not reuse_ocean_file) or (not s.initialized):
            if getattr(oc, 'use_buoy_data', False):
                raise NotImplementedError('buoy-spectrum input is not built')
            dir_swell = swell_spec.ardhuin_swell_spec if oc.swell_dir_enable else None
            s.init(oc.Lx, oc.Ly, oc.dx, oc.dy, oc.cutoff_wl, oc.spec_model, oc.spread_model,
                   np.deg2rad(wind_dir), oc.wind_fetch, oc.wind_U, oc.current_mag,
                   np.deg2rad(radar.azimuth - oc.current_dir), radar.azimuth - oc.dir_swell_dir,
                   oc.freq_r, oc.sigf, oc.sigs, oc.Hs, oc.swell_dir_enable, oc.swell_enable, oc.swell_ampl,
                   np.deg2rad(radar.azimuth - oc.swell_dir), oc.swell_wl, compute, oc.opt_res,
                   oc.fft_max_prime, choppy_enable=oc.choppy_enable, depth=oc.depth,
                   dirspectrum_func=None, dir_swell_spec=dir_swell)
            if ocean_file:
                s.save(ocean_file)
        self.balancer = OceanSurfaceBalancer(s, self.ocean_dt)

        # ---- geometry (:311-394) ----------------------------------------------------------
        self.sr0 = geo.inc_to_sr(self.inc_angle, alt)
        self.gr0 = gr0 = geo.inc_to_gr(self.inc_angle, alt)
        sr, inc, _ = geo.gr_to_geo(s.x + gr0, alt)
        self.min_sr = np.min(sr)
        self.inc = inc.reshape(1, inc.size)
        self.sr = sr.reshape(1, sr.size)
        self.sin_inc, self.cos_inc = np.sin(self.inc), np.cos(self.inc)
        self.l0 = l0 = C_LIGHT / f0
        self.k0 = k0 = 2. * np.pi * f0 / C_LIGHT
        self.sr_res = C_LIGHT / (2. * self.rg_bw)
        self.sr_smp = C_LIGHT / (2 * radar.Fs)
        self.L_total = bool(radar.L_total)
        if self.L_total:
            ant_L = ant_L / float(num_ch)
        self.ant_L = ant_L
        if v_ground == 'auto':
            v_ground = geo.orbit_to_vel(alt, ground=True)
            v_orb = geo.orbit_to_vel(alt, ground=False)
        else:
            v_orb = v_ground
        self.v_ground, self.v_orb = v_ground, v_orb
        self.t_step = 1. / prf
        self.az_steps = int(radar.n_pulses)
        self.t_span = self.az_steps / prf
        self.n_rg = int(radar.n_rg)
        self.rg_samp = rg_samp = int(optimize_fftsize(radar.n_rg))
        sr_prof = (np.arange(rg_samp) - rg_samp / 2) * self.sr_smp + np.mean(sr)
        gr_prof, inc_prof, look_prof, b_prof = geo.sr_to_geo(sr_prof, alt)
        look_prof = look_prof.reshape((1, look_prof.size))
        self.sr_prof = sr_prof.reshape((1, look_prof.size))
        self.dop_ref = 2 * v_orb * np.sin(look_prof) * np.sin(self.squint_r) / l0
        self.two_scale = bool(srg.two_scale_Doppler)
        self.rcm = bool(getattr(srg, 'rcm', False)) if self.two_scale else False
        if self.two_scale:
            self.n_pulses_b = optimize_fftsize(int(srg.surface_coh_time * prf)) / 2
            self.steps = int(np.ceil(self.az_steps / self.n_pulses_b))
            self.t_step = self.t_step * self.n_pulses_b
            dy_integ = srg.phase_err_tol / (2 * k0 * v_ground / self.min_sr * srg.surface_coh_time)
            ny_integ = dy_integ / s.dy
            ny_integ = 1 if ny_integ < 1 else int(2 ** np.floor(np.log2(ny_integ)))
            if s.Ny % ny_integ:
                raise ValueError('the row-group size %d does not divide Ny = %d' % (ny_integ, s.Ny))
            self.ny_integ = ny_integ
            az = s.y.reshape((s.Ny, 1))
            da = az / gr_prof
            sin_az = np.sin(self.squint_r) + np.cos(self.squint_r) * da - 0.5 * np.sin(self.squint_r) * da ** 2
            dop0 = 2 * v_orb * np.sin(look_prof) * sin_az / l0
            s_int = int(s.Ny / ny_integ)
            self.dop0 = np.mean(np.reshape(dop0, (s_int, int(ny_integ), rg_samp)), axis=1)
        else:
            self.n_pulses_b = 1
            self.steps = self.az_steps
            self.ny_integ = s.Ny
        self.s_int = s.Ny // self.ny_integ
        self.surface_area = s.dx * s.dy * s.Nx * s.Ny

        # ---- scattering models (:402-461; global RNG draw 2) --------------------------------
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                self.rcs_spec = nrcs.RCSKodis(self.inc, k0, s.dx, s.dy)
            else:
                self.spec_ph0 = np.random.uniform(0., 2. * np.pi, size=[s.Ny, s.Nx])
                self.rcs_spec = nrcs.RCSKA(self.scat_spec_mode, k0, s.x, s.y, s.dx, s.dy)
        if self.scat_bragg_enable:
            tau_c = grid_coherence(oc.wind_U, s.dx, f0)
            self.rndscat_p = randomscat_ts(tau_c, (s.Ny, s.Nx), prf)
            self.rndscat_m = randomscat_ts(tau_c, (s.Ny, s.Nx), prf)
            k_b = 2. * k0 * self.sin_inc
            self.c_b = self.sin_inc * np.sqrt(G / k_b + 0.072e-3 * k_b)
            cdir = np.deg2rad(oc.current_dir)
            cur = oc.current_mag * np.array([np.cos(cdir), np.sin(cdir)])
            udir = np.deg2rad(oc.wind_dir)          # the .cfg's wind direction, as the reference
            u_eff = oc.wind_U * np.array([np.cos(udir), np.sin(udir)]) - cur
            # the reference builds the model with the constructor's defaults (LUT mode)
            self.rcs_bragg = nrcs.RCSRomeiser97(k0, self.inc, pol, s.dx, s.dy, linalg.norm(u_eff),
                                                np.arctan2(u_eff[1], u_eff[0]), s.wind_fetch,
                                                srg.scat_bragg_spec, srg.scat_bragg_spread, srg.scat_bragg_d)
        self._alloc()
        self.t_last_rcs_bragg = -1.
        self._refreshes = []

    # ------------------------------------------------------------------------------------
    def _alloc(self):
        s = self.surface
        cdt = np.complex128 if self.precision == 'f64' else np.complex64
        sdt = torch.float64 if self.precision == 'f64' else torch.float32
        self.raw_d = _device.zeros((self.npol, self.steps, self.s_int, self.rg_samp), cdt)
        self.nrcs_spec_d = _device.zeros((self.steps,), np.float64)
        self.nrcs_bragg_d = _device.zeros((self.npol, self.steps), np.float64)
        col = lambda a: _device.to_device(np.ravel(a), np.float64)  # noqa: E731
        self._cols = dict(sr=col(self.sr), sin=col(self.sin_inc), cos=col(self.cos_inc),
                          tan=col(np.tan(self.inc)), inc=col(self.inc))
        self._y_d = _device.to_device(s.y, np.float32)
        self._sinc_d = _device.to_device(self.chan_sinc_vec, np.float32)
        self._b0 = (ctypes.c_double * 1)(0.0)
        d = self.desc = PulseDesc()
        d.nx, d.ny, d.npol, d.nch = s.Nx, s.Ny, self.npol, 1
        d.pol = nrcs.POL_CODES[self.pol]
        f = self.balancer.field
        d.dx_d, d.dy_d, d.dz_d = f('Dx').data_ptr(), f('Dy').data_ptr(), f('Dz').data_ptr()
        d.diffx_d, d.diffy_d = f('Diffx').data_ptr(), f('Diffy').data_ptr()
        d.diffxx_d, d.diffyy_d, d.diffxy_d = f('Diffxx').data_ptr(), f('Diffyy').data_ptr(), f('Diffxy').data_ptr()
        if self.use_hmtf:
            d.hmtf_d = f('hMTF').data_ptr()
        d.y_d = self._y_d.data_ptr()
        c = self._cols
        d.sr_col_d, d.sin_inc_d, d.cos_inc_d = c['sr'].data_ptr(), c['sin'].data_ptr(), c['cos'].data_ptr()
        d.tan_inc_d, d.inc_d = c['tan'].data_ptr(), c['inc'].data_ptr()
        d.inc_angle, d.sr0, d.gr0, d.k0, d.f0 = (float(self.inc_angle), float(self.sr0), float(self.gr0),
                                                 float(self.k0), float(self.f0))
        d.min_sr, d.binsize, d.t_step = float(self.sr_prof.min()), float(self.sr_smp), float(self.t_step)
        d.az_steps = self.steps
        # sinc_1tx_nrx(sin_az, L, f0, n): transmit length L, receive length L / n
        if self.L_total:
            L = self.ant_L * self.num_ch
            d.ant_l_tx, d.ant_l_rx = float(L), float(L / self.num_ch)
        else:
            d.ant_l_tx, d.ant_l_rx = float(self.ant_L), float(self.ant_L / 1)
        d.b_ati, d.b_xti = self._b0, self._b0
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
            self._scat_d = torch.empty((self.npol, 2, s.Ny, s.Nx), dtype=sdt, device=_device.device())
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
        d.skim, d.skim_ny_integ = 1, self.ny_integ
        d.skim_az2 = int(not self.two_scale)
        d.skim_rcm = int(self.rcm)
        d.pt_mode = self.pt_mode
        d.pt_x, d.pt_y, d.pt_amp = int(s.Nx / 2), int(s.Ny / 2), 1000.0
        nb = _capi.load().ocs_pulse_workspace_bytes(s.Ny, 1)
        self._rowtab = torch.empty(int(nb), dtype=torch.uint8, device=_device.device())
        d.rowtab_d = self._rowtab.data_ptr()

    def _lut_check(self, az_now):
        """LUT mode: every row's azimuth index must exist in the table, as numpy indexing
        requires; raise IndexError as the reference's lookup would."""
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

    # ------------------------------------------------------------------------------------
    def step(self, az_step, update_surface=True):
        """One simulated step of the loop (``skim_raw.py:465-689``).  ``update_surface=False``
        keeps whatever the interpolated field buffers hold."""
        t_now = az_step * self.t_step
        az_now = (t_now - self.t_span / 2.) * self.v_ground * np.cos(self.squint_r)
        if update_surface:
            self.balancer.set_t(t_now, stream=self.stream)
        d = self.desc
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
        _capi.call("ocs_pulse", ctypes.addressof(d), PRECISIONS[self.precision], _device.stream_ptr(self.stream))

    def run(self):
        for a in range(self.steps):
            self.step(a)

    # ------------------------------------------------------------------------------------
    def profiles(self):
        """Step profiles [pol, steps, row groups, rg_samp] (complex128 host copy)."""
        torch.cuda.synchronize()
        return self.raw_d.cpu().numpy().astype(np.complex128)

    def nrcs_avg(self):
        """NRCS_avg [pol, n_pulses] (:526-577): specular plus the Bragg sum of the last
        refresh, per unit area, at the simulated steps (zero after them)."""
        torch.cuda.synchronize()
        spec = self.nrcs_spec_d.cpu().numpy()
        bragg = self.nrcs_bragg_d.cpu().numpy()
        out = np.zeros((self.npol, self.az_steps))
        last = None
        for a in range(self.steps):
            if a in self._refreshes:
                last = a
            for p in range(self.npol):
                if self.scat_spec_enable:
                    out[p, a] += spec[a] / self.surface_area
                if self.scat_bragg_enable and last is not None:
                    out[p, a] += bragg[p, last] / self.surface_area
        return out

    def cal_factor(self):
        """Calibration by the azimuth-integrated antenna pattern (:632-640)."""
        az_axis = np.arange(-self.t_span / 2. * self.v_ground, self.t_span / 2. * self.v_ground,
                            self.sr0 * C_LIGHT / (np.pi * self.f0 * self.ant_L * 10.))
        if self.L_total:
            pattern = sinc_1tx_nrx(az_axis / self.sr0, self.ant_L * self.num_ch, self.f0, self.num_ch, field=True)
        else:
            pattern = sinc_1tx_nrx(az_axis / self.sr0, self.ant_L, self.f0, 1, field=True)
        trapz = getattr(np, 'trapezoid', None) or np.trapz
        return 1. / np.sqrt(trapz(np.abs(pattern) ** 2., az_axis) * self.sr_res / np.sin(self.inc_angle))

    def finish(self, add_noise=True):
        """(raw [pol, az, n_rg], NRCS_avg [pol, n_pulses]): up-sampling and Doppler of the
        two-scale form, truncation, calibration and noise (:661-677)."""
        prof = None if self.two_scale else self.profiles()
        out = []
        cal = self.cal_factor()
        for p in range(self.npol):
            if self.two_scale:
                r = upsample_and_dopplerize(self.raw_d[p], self.dop0, self.n_pulses_b, self.prf, stream=self.stream)
            else:
                r = prof[p][:, 0, :]
            r = r[:, :self.n_rg]
            if add_noise:
                noise = (db2lin(self.nesz, amplitude=True) / np.sqrt(2.) *
                         (np.random.normal(size=r.shape) + 1j * np.random.normal(size=r.shape)))
                r = r * cal + noise
            else:
                r = r * cal
            out.append(r)
        return np.array(out), self.nrcs_avg()


def skimraw(cfg_file, output_file, ocean_file, reuse_ocean_file, errors_file, reuse_errors_file,
            plot_save=True, precision='f64'):
    """Drop-in for ``skim_raw.skimraw``: simulate one beam azimuth and write the SKIM raw
    file (``SkimRawFile``: ``raw_data_r``/``raw_data_i`` [pol, az, rg], ``NRCS_avg``,
    ``dop_ref``, geometry).  No MPI: one GPU holds the whole surface."""
    cfg = cfg_file if isinstance(cfg_file, ConfigFile) else ConfigFile(cfg_file)
    gen = SkimGenerator(cfg, precision=precision, ocean_file=ocean_file, reuse_ocean_file=reuse_ocean_file)
    gen.run()
    total_raw, nrcs_avg = gen.finish(add_noise=True)
    if output_file:
        f = SkimRawFile(output_file, 'w', raw_dim=total_raw.shape)
        f.set('inc_angle', np.rad2deg(gen.inc_angle))
        f.set('f0', gen.f0)
        f.set('ant_L', gen.ant_L)
        f.set('prf', gen.prf)
        f.set('v_ground', gen.v_ground)
        f.set('orbit_alt', cfg.radar.alt)
        f.set('sr0', gen.sr0)
        f.set('rg_sampling', gen.rg_bw * gen.over_fs)
        f.set('rg_bw', gen.rg_bw)
        f.set('raw_data*', total_raw)
        f.set('NRCS_avg', nrcs_avg)
        f.set('azimuth', cfg.radar.azimuth)
        f.set('dop_ref', gen.dop_ref)
        f.close()
    return total_raw, nrcs_avg
