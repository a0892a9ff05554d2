"""The DopSCA scatterometer raw-data generator (``oceansar/dopscasim/dopsca_raw.py:34-632``)
on the GPU.

The reference simulates a Doppler scatterometer over a long acquisition: the surface tile
is repeated ``N_repeat_x`` times in ground range (each repetition a range block with its
own incidence, slant range and scattering models), the platform motion is applied by
rolling the surface rows by whole azimuth samples, every pulse is made of ``n_subpulses``
sub-pulses (the surface, the Bragg phases and the range delay advance with the sub-pulse
time), the scene is scaled by the two-way spreading (sr0 / (sr0 + r))^2, and the Bragg RCS
is evaluated on every sub-pulse.  Everything per sub-pulse runs on the device: the surface
update, the row table and one pulse-kernel launch over all range blocks (the
scatterometer mode of ``ocs_pulse``: columns of the blocks side by side, fields read at
column mod Nx and at the rolled row).

The host set-up follows the reference's order so that the global numpy RNG gives the same
surface and scatterer series for the same seed: surface (random phases, swell), then the
Bragg scatterer series ``rndscat_p`` and ``rndscat_m`` of shape (N_repeat_x, Ny, Nx) at the
sub-pulse rate.

Scope: Kodis or Kirchhoff specular, the Romeiser Bragg model (direct or LUT) and the hMTF
modulation.  The
reference's hMTF branch weights the Bragg RCS by 1 + hMTF of the rolled rows without
clipping and writes its clipping mask (computed on the rolled rows) into the unrolled
surface, where it persists while the ocean is frozen; both are reproduced.  The
reference's Kirchhoff branch (marked FIXME there) is reproduced as written: the
tangent-plane field of every facet at the block's incidence, times exp(-2 i k0 r) and
(4 pi)^1.5, scaled by the two-way spreading, after one unused phase screen per block from
the global RNG.  Buoy-spectrum input raises ``NotImplementedError``.  The Romeiser LUT mode keeps
one table per range block (the reference builds one model per block), stacked on the
device and selected by the column's block in the kernel.
The reference adds no noise in this generator; neither does this one.
"""
import ctypes

import numpy as np
import torch
from scipy import linalg

from .. import _capi, _device, nrcs, swell_spec
from .._structs import PulseDesc
from ..closure import grid_coherence, randomscat_ts
from ..ocs_io.cfg import ConfigFile
from ..ocs_io.raw import DopscaRawFile
from ..radarsim.range_profile import calc_sinc_vec
from ..radarsim.sar_raw_nompi import C_LIGHT, G, PRECISIONS, sinc_bp
from ..surfaces import OceanSurface
from ..utils import geometry as geo
from ..utils.misc import optimize_fftsize


class DopscaGenerator(object):
    """Device-resident state of one DopSCA acquisition; see the module docstring.

    ``overrides`` may fix ``az_steps`` / ``rg_samp`` / ``rg_samp_orig`` (derived from the
    geometry by the reference, ``dopsca_raw.py:276-289``)."""

    def __init__(self, cfg, precision='f64', overrides=None, seed=None, stream=None,
                 ocean_file=None, reuse_ocean_file=False):
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
        srg, sca, oc = cfg.srg, cfg.sca, cfg.ocean
        self.wh_tol = srg.wh_tol
        self.use_hmtf = bool(srg.use_hmtf)
        self.scat_spec_enable = bool(srg.scat_spec_enable)
        self.scat_bragg_enable = bool(srg.scat_bragg_enable)
        self.scat_spec_mode = srg.scat_spec_mode if self.scat_spec_enable else 'kodis'
        if self.scat_spec_enable and self.scat_spec_mode not in ('kodis', 'fa', 'spa'):
            raise NotImplementedError('RCS mode %s for specular scattering not implemented' % self.scat_spec_mode)
        if self.scat_bragg_enable and srg.scat_bragg_model != 'romeiser97':
            raise NotImplementedError('RCS model %s for Bragg scattering not implemented' % srg.scat_bragg_model)
        self.use_lut = bool(getattr(srg, 'use_lut', False))
        self.inc_angle = np.deg2rad(sca.inc_angle)
        self.f0 = f0 = sca.f0
        self.pol = pol = sca.pol
        self.do_hh = pol in ('DP', 'hh')
        self.do_vv = pol not in ('hh',)
        self.npol = 2 if pol == 'DP' else 1
        self.prf = sca.prf
        alt = sca.alt
        v_ground = sca.v_ground
        self.rg_bw = sca.rg_bw
        self.over_fs = sca.over_fs
        self.n_sub = int(sca.n_subpulses)
        self.sub_len = float(sca.sub_pulse_length)
        self.sub_bw = float(getattr(sca, 'sub_pulse_bw', 0.0))
        self.ocean_dt = oc.dt
        self.frozen = oc.frozen_ocean is not False           # dopsca_raw.py:375 tests `is False`
        self.chan_sinc_vec = calc_sinc_vec(8, 20, Fs=self.over_fs)

        # ---- surface (dopsca_raw.py:134-198; global RNG draw 1) -------------------------
        compute = ['D', 'Diff']
        if self.scat_spec_enable:
            compute.append('Diff2')
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
                   np.deg2rad(oc.wind_dir), oc.wind_fetch, oc.wind_U, oc.current_mag,
                   np.deg2rad(oc.current_dir), oc.dir_swell_dir, oc.freq_r, oc.sigf, oc.sigs, oc.Hs,
                   oc.swell_dir_enable, oc.swell_enable, oc.swell_ampl, np.deg2rad(oc.swell_dir),
                   oc.swell_wl, compute, oc.opt_res, oc.fft_max_prime, choppy_enable=oc.choppy_enable,
                   depth=oc.depth, dirspectrum_func=None, dir_swell_spec=dir_swell)
            if ocean_file:
                s.save(ocean_file)

        # ---- geometry of the range blocks (:245-289) ------------------------------------
        self.n_rep = n_rep = int(oc.N_repeat_x)
        self.sr0 = sr0 = geo.inc_to_sr(self.inc_angle, alt)
        self.gr0 = gr0 = geo.inc_to_gr(self.inc_angle, alt)
        gr_s = np.zeros((n_rep, s.Nx))
        sr_s = np.zeros((n_rep, s.Nx))
        inc_s = np.zeros((n_rep, s.Nx))
        for ind in range(n_rep):
            gr_s[ind, :] = s.x + ind * s.Lx + gr0
            sr, inc, _ = geo.gr_to_geo(gr_s[ind, :], alt)
            sr_s[ind, :] = sr
            inc_s[ind, :] = inc
        rg_sampling = self.rg_bw * self.over_fs
        self.sr_near = sr_s[0, 0] - self.wh_tol + C_LIGHT / 2 / rg_sampling
        sr_s -= np.min(sr_s)
        self.sr_s, self.inc_s = sr_s, inc_s
        self.sin_inc_s, self.cos_inc_s = np.sin(inc_s), np.cos(inc_s)
        self.l0 = C_LIGHT / f0
        self.k0 = k0 = 2. * np.pi * f0 / C_LIGHT
        self.sr_res = C_LIGHT / (2. * self.rg_bw)
        self.ant_l_tx = sca.ant_L_tx
        self.ant_l_rx = sca.ant_L_rx
        if v_ground == 'auto':
            v_ground = geo.orbit_to_vel(alt, ground=True)
        self.v_ground = v_ground
        self.t_step = 1. / self.prf
        self.t_span = cfg.acquisition.length / v_ground
        self.az_steps = int(ov.get('az_steps', int(np.ceil(self.t_span * self.prf))))
        az_span = (self.t_span * v_ground + s.Ly) / gr0
        max_sr = (np.max(sr_s) + self.wh_tol + (np.max(s.y) + (self.t_span / 2.) * v_ground) ** 2. / (2. * sr0)
                  + self.sub_len * C_LIGHT / 2 * (self.n_sub - 1))
        self.min_sr = np.min(sr_s) - self.wh_tol
        self.rg_samp_orig = int(ov.get('rg_samp_orig',
                                       int(np.ceil(((max_sr - self.min_sr) / self.sr_res) * self.over_fs))))
        self.rg_samp = int(ov.get('rg_samp', int(optimize_fftsize(self.rg_samp_orig))))
        self.surface_area = s.dx * s.dy * s.Nx * s.Ny

        # ---- scattering models (:297-360; global RNG draw 2: rndscat_p then rndscat_m) ---
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                self.rcs_spec = nrcs.RCSKodis(inc_s, k0, s.dx, s.dy)
            else:
                # Kirchhoff (the reference's FIXME branch, dopsca_raw.py:302-308): one model
                # per block after an unused phase screen per block, drawn to keep the RNG
                # stream; the models differ in nothing the kernel reads
                for _ in range(n_rep):
                    np.random.uniform(0., 2. * np.pi, size=[s.Ny, s.Nx])
                self.rcs_spec = nrcs.RCSKA(self.scat_spec_mode, k0, s.x, s.y, s.dx, s.dy)
        if self.scat_bragg_enable:
            tau_c = grid_coherence(oc.wind_U, s.dx, f0)
            self.rndscat_p = randomscat_ts(tau_c, (n_rep, s.Ny, s.Nx), 1 / self.sub_len)
            self.rndscat_m = randomscat_ts(tau_c, (n_rep, s.Ny, s.Nx), 1 / self.sub_len)
            k_b_s = 2. * k0 * self.sin_inc_s
            self.c_b_s = self.sin_inc_s * np.sqrt(G / k_b_s + 0.072e-3 * k_b_s)
            cdir = np.deg2rad(oc.current_dir)
            cur = oc.current_mag * np.array([np.cos(cdir), np.sin(cdir)])
            udir = np.deg2rad(oc.wind_dir)
            u_eff = oc.wind_U * np.array([np.cos(udir), np.sin(udir)]) - cur
            # one model for all blocks: its constants do not depend on the incidence, which
            # the kernel reads per column
            self.rcs_bragg = nrcs.RCSRomeiser97(k0, inc_s, pol, s.dx, s.dy, linalg.norm(u_eff),
                                                np.arctan2(u_eff[1], u_eff[0]), s.wind_fetch,
                                                srg.scat_bragg_spec, srg.scat_bragg_spread,
                                                srg.scat_bragg_d, rmss_x=s.rmss_x, rmss_y=s.rmss_y,
                                                az_span=az_span, use_lut=False)
            if self.use_lut:
                # LUT mode: one table per range block at the block's mean incidence
                # (dopsca_raw.py:329-356 builds one model per block); the lookup grids are
                # the same for every block
                self.rcs_lut_s = [nrcs.RCSRomeiser97(k0, inc_s[b], pol, s.dx, s.dy, linalg.norm(u_eff),
                                                     np.arctan2(u_eff[1], u_eff[0]), s.wind_fetch,
                                                     srg.scat_bragg_spec, srg.scat_bragg_spread,
                                                     srg.scat_bragg_d, rmss_x=s.rmss_x, rmss_y=s.rmss_y,
                                                     az_span=az_span, use_lut=True)
                                  for b in range(n_rep)]
                params = {m.lut_params() for m in self.rcs_lut_s}
                if len(params) != 1:
                    raise ValueError('the range blocks\' LUT grids differ')
        self._alloc()

    # ------------------------------------------------------------------------------------
    def _alloc(self):
        s = self.surface
        s.to_device()
        cdt = np.complex128 if self.precision == 'f64' else np.complex64
        nblk, nx = self.n_rep, self.n_rep * s.Nx
        self.raw_d = _device.zeros((self.npol, self.az_steps, self.rg_samp), cdt)
        nrows = self.az_steps * self.n_sub
        self.nrcs_spec_d = _device.zeros((nrows, nblk), np.float64)
        self.nrcs_bragg_d = _device.zeros((self.npol, nrows, nblk), np.float64)
        col = lambda a: _device.to_device(np.ravel(a), np.float64)  # noqa: E731
        self._cols = dict(sr=col(self.sr_s), sin=col(self.sin_inc_s), cos=col(self.cos_inc_s),
                          tan=col(np.tan(self.inc_s)), inc=col(self.inc_s))
        self._y_d = _device.to_device(s.y, np.float32)
        self._sinc_d = _device.to_device(self.chan_sinc_vec, np.float32)
        self._b0 = (ctypes.c_double * 1)(0.0)
        d = self.desc = PulseDesc()
        d.nx, d.ny, d.npol, d.nch = nx, s.Ny, self.npol, 1
        d.pol = nrcs.POL_CODES[self.pol]
        f = s.field
        d.dx_d, d.dy_d, d.dz_d = f('Dx').data_ptr(), f('Dy').data_ptr(), f('Dz').data_ptr()
        d.diffx_d, d.diffy_d = f('Diffx').data_ptr(), f('Diffy').data_ptr()
        if self.scat_spec_enable:
            d.diffxx_d, d.diffyy_d, d.diffxy_d = (f('Diffxx').data_ptr(), f('Diffyy').data_ptr(),
                                                  f('Diffxy').data_ptr())
            if self.scat_spec_mode == 'kodis':
                d.kodis_R_re, d.kodis_R_im = float(self.rcs_spec.R.real), float(self.rcs_spec.R.imag)
            else:
                d.spec_mode = 1 if self.scat_spec_mode == 'fa' else 2
                self._x_d = _device.to_device(s.x, np.float32)
                d.x_d = self._x_d.data_ptr()
                d.ka_dx, d.ka_dy = float(s.dx), float(s.dy)
                K = self.rcs_spec.constant(1, 1)
                d.ka_K_re, d.ka_K_im = K.real, K.imag
        d.y_d = self._y_d.data_ptr()
        c = self._cols
        d.sr_col_d, d.sin_inc_d, d.cos_inc_d = c['sr'].data_ptr(), c['sin'].data_ptr(), c['cos'].data_ptr()
        d.tan_inc_d, d.inc_d = c['tan'].data_ptr(), c['inc'].data_ptr()
        d.inc_angle, d.sr0, d.gr0, d.k0, d.f0 = (float(self.inc_angle), float(self.sr0), float(self.gr0),
                                                 float(self.k0), float(self.f0))
        d.min_sr, d.binsize, d.t_step = float(self.min_sr), float(self.sr_res / self.over_fs), float(self.t_step)
        d.az_steps = self.az_steps
        d.ant_l_tx, d.ant_l_rx = float(self.ant_l_tx), float(self.ant_l_rx)
        d.b_ati, d.b_xti = self._b0, self._b0
        d.do_kodis, d.do_bragg = int(self.scat_spec_enable), int(self.scat_bragg_enable)
        d.use_hmtf = int(self.use_hmtf and self.scat_bragg_enable)
        if d.use_hmtf:
            d.hmtf_d = f('hMTF').data_ptr()
        d.facet_dx, d.facet_dy = float(s.dx), float(s.dy)
        if self.scat_bragg_enable:
            self.rcs_bragg.fill(d)
            d.bragg_d = float(self.rcs_bragg.d)
            self._c_b_d = col(self.c_b_s)
            d.c_b_d = self._c_b_d.data_ptr()
            # per-facet start indices as [Ny][N_repeat_x * Nx] (block-major columns)
            if max(self.rndscat_m.ind0.max(initial=0), self.rndscat_p.ind0.max(initial=0)) >= 2 ** 31:
                raise ValueError('scatterer start index exceeds int32')
            ind = lambda r: _device.to_device(  # noqa: E731
                np.ascontiguousarray(r.ind0.transpose(1, 0, 2).reshape(s.Ny, nx)).astype(np.int32), np.int32)
            self._ind_m, self._ind_p = ind(self.rndscat_m), ind(self.rndscat_p)
            sm, _ = self.rndscat_m.device()
            sp, _ = self.rndscat_p.device()
            d.s_m_d, d.s_p_d, d.n_m, d.n_p = sm.data_ptr(), sp.data_ptr(), int(self.rndscat_m.N), \
                int(self.rndscat_p.N)
            if self.precision == 'mixed':
                d.s_m32_d, d.s_p32_d = self.rndscat_m.device32().data_ptr(), self.rndscat_p.device32().data_ptr()
            d.ind0_m_d, d.ind0_p_d = self._ind_m.data_ptr(), self._ind_p.data_ptr()
            if self.use_lut:
                tabs = [m.lut_device(self.precision) for m in self.rcs_lut_s]
                self._lut_d = torch.stack(tabs).contiguous()     # [block][npol][2][naz][ndy][ndx]
                d.lut_d = self._lut_d.data_ptr()
                d.lut_block = int(tabs[0].numel())
                (d.lut_naz, d.lut_ndy, d.lut_ndx, d.lut_az0, d.lut_daz, d.lut_dy0, d.lut_ddy, d.lut_dx0,
                 d.lut_ddx) = self.rcs_lut_s[0].lut_params()
        d.sinc_d = self._sinc_d.data_ptr()
        d.raw_d = self.raw_d.data_ptr()
        d.nbins = self.rg_samp
        d.nrcs_spec_d = self.nrcs_spec_d.data_ptr()
        d.nrcs_bragg_d = self.nrcs_bragg_d.data_ptr()
        d.sca, d.field_nx, d.refresh = 1, s.Nx, 1
        d.nrcs_rows = nrows
        nb = _capi.load().ocs_pulse_workspace_bytes(s.Ny, 1)
        self._rowtab = torch.empty(int(nb), dtype=torch.uint8, device=_device.device())
        d.rowtab_d = self._rowtab.data_ptr()

    # ------------------------------------------------------------------------------------
    def sub_pulse(self, az_step, sub, update_surface=True):
        """One sub-pulse of the azimuth loop (``dopsca_raw.py:367-519``), all range blocks.
        ``update_surface=False`` keeps whatever the surface field buffers hold."""
        s = self.surface
        t_now = az_step * self.t_step + sub * self.sub_len
        az_now = (t_now - self.t_span / 2.) * self.v_ground
        shift = int(np.floor(az_now / s.dy))
        az_res = az_now - shift * s.dy
        if update_surface and ((not self.frozen) or az_step == 0):
            s.set_t(t_now, stream=self.stream)
        d = self.desc
        d.az_step = az_step
        d.az_now = float(az_res)
        # numpy gives a float32 residual (and float32 y - residual) when az_now is not a
        # float64 scalar; mirror it
        d.az_f32 = int(np.asarray(az_res).dtype == np.float32)
        d.roll = int(shift % s.Ny)                  # np.roll(field, -shift, axis=0)
        d.sr_bin_offset = sub * self.sub_len * C_LIGHT / 2
        d.cap_t = self.t_step * (az_step + 1) + sub * self.sub_len
        d.nrcs_row = az_step * self.n_sub + sub
        if self.scat_bragg_enable:
            d.tind = self.rndscat_m.tind(t_now)
        _capi.call("ocs_pulse", ctypes.byref(d), PRECISIONS[self.precision], _device.stream_ptr(self.stream))
        if d.use_hmtf and self.frozen:
            # the reference's clipping of the rolled hMTF writes -1 into the unrolled
            # surface where the rolled value is below -1 (dopsca_raw.py:463-466); a frozen
            # surface keeps those writes for the following sub-pulses
            with torch.cuda.stream(self.stream):          # None: the current stream
                h = s.field('hMTF')
                h.masked_fill_(torch.roll(h, -shift, dims=0) < -1, -1.0)

    def run(self, steps=None):
        for a in (range(self.az_steps) if steps is None else steps):
            for sub in range(self.n_sub):
                self.sub_pulse(a, sub)

    # ------------------------------------------------------------------------------------
    def nrcs_avg(self):
        """NRCS_avg [pol, az] with the reference's running sums (``dopsca_raw.py:447-475``):
        per sub-pulse and range block, hh += specular; vv += hh; then each polarisation adds
        its Bragg sum."""
        torch.cuda.synchronize()
        area = self.surface_area
        spec = self.nrcs_spec_d.cpu().numpy()
        bragg = self.nrcs_bragg_d.cpu().numpy()
        hh = np.zeros(self.az_steps)
        vv = np.zeros(self.az_steps)
        p_hh, p_vv = 0, (1 if self.pol == 'DP' else 0)
        for a in range(self.az_steps):
            for sub in range(self.n_sub):
                row = a * self.n_sub + sub
                for blk in range(self.n_rep):
                    if self.scat_spec_enable:
                        hh[a] += spec[row, blk] / area
                        vv[a] += hh[a]
                    if self.scat_bragg_enable:
                        if self.do_hh:
                            hh[a] += bragg[p_hh, row, blk] / area
                        if self.do_vv:
                            vv[a] += bragg[p_vv, row, blk] / area
        out = []
        if self.do_hh:
            out.append(hh)
        if self.do_vv:
            out.append(vv)
        return np.array(out)

    def cal_factor(self):
        """Calibration by the azimuth-integrated antenna pattern (``dopsca_raw.py:555-561``)."""
        az_axis = np.arange(-self.t_span / 2. * self.v_ground, self.t_span / 2. * self.v_ground,
                            self.sr0 * C_LIGHT / (np.pi * self.f0 * self.ant_l_tx * 10.))
        pattern = (sinc_bp(az_axis / self.sr0, self.ant_l_tx, self.f0, field=True) *
                   sinc_bp(az_axis / self.sr0, self.ant_l_rx, self.f0, field=True))
        trapz = getattr(np, 'trapezoid', None) or np.trapz
        return 1. / np.sqrt(trapz(np.abs(pattern) ** 2., az_axis) * self.sr_res / np.sin(self.inc_angle))

    def raw(self):
        """Raw cube [pol, az, rg_samp] on the host, uncalibrated."""
        torch.cuda.synchronize()
        return self.raw_d.cpu().numpy()

    def finish(self):
        """(raw [pol, az, rg_samp_orig] calibrated, NRCS_avg [pol, az])."""
        raw = self.raw().astype(np.complex128)[:, :, :self.rg_samp_orig]
        return raw * self.cal_factor(), self.nrcs_avg()


def dopsca_raw(cfg_file, output_file, ocean_file, reuse_ocean_file, errors_file, reuse_errors_file,
               plot_save=True, precision='f64'):
    """Drop-in for ``dopscasim.dopsca_raw.dopsca_raw``: simulate and write the DopSCA raw file
    (``DopscaRawFile``: ``raw_data_r``/``raw_data_i`` [pol, az, rg], ``NRCS_avg``, geometry,
    sub-pulse length and bandwidth).  ``errors_file`` / ``plot_save`` are unused, as in the
    reference (no plots here)."""
    cfg = cfg_file if isinstance(cfg_file, ConfigFile) else ConfigFile(cfg_file)
    gen = DopscaGenerator(cfg, precision=precision, ocean_file=ocean_file, reuse_ocean_file=reuse_ocean_file)
    gen.run()
    total_raw, nrcs_avg = gen.finish()
    if output_file:
        f = DopscaRawFile(output_file, 'w', raw_dim=total_raw.shape)
        f.set('inc_angle', np.rad2deg(gen.inc_angle))
        f.set('f0', gen.f0)
        f.set('ant_L', gen.ant_l_tx)
        f.set('prf', gen.prf)
        f.set('v_ground', gen.v_ground)
        f.set('orbit_alt', cfg.sca.alt)
        f.set('sr0', gen.sr_near)
        f.set('rg_sampling', gen.rg_bw * gen.over_fs)
        f.set('rg_bw', gen.rg_bw)
        f.set('raw_data*', total_raw)
        f.set('subpulse_length', gen.sub_len)
        f.set('subpulse_bandwidth', gen.sub_bw)
        f.set('NRCS_avg', nrcs_avg)
        f.close()
    return total_raw, nrcs_avg
