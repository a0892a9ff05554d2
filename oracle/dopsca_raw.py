"""Oracle (test infrastructure only): the DopSCA scatterometer generator ``dopsca_raw``.

Restates ``oceansar/dopscasim/dopsca_raw.py:34-632`` for the Kodis or Kirchhoff specular
and the Romeiser Bragg models (with the hMTF weighting of ``:461-472``) with the oracle's own surface, NRCS, closure, geometry and
accumulation restatements:

* set-up ``:66-360``: configuration (``[sca]``, ``[acquisition]``, ``ocean.N_repeat_x``),
  surface init with the global numpy RNG, geometry of the range blocks, sizes, one
  Kodis / Romeiser model per block, random scatterer series ``rndscat_p`` then
  ``rndscat_m`` of shape (N_repeat_x, Ny, Nx) at the sub-pulse rate;
* the loop ``:367-519``: per azimuth step and sub-pulse, surface time, whole-sample roll of
  the fields, per block slant range, two-way range scaling, specular field, Bragg RCS and
  phases, antenna pattern and the accumulation at the sub-pulse's range delay;
* post-processing ``:538-562``: truncation and calibration (no noise in this generator).
"""
import numpy as np
from scipy import linalg

from . import closure, geometry as geo, ka, nrcs, range_profile as rp, spectra
from .cfg import ConfigFile
from .sar_raw import C_LIGHT, sinc_bp
from .surface import OceanSurface

G = 9.80665


class DopscaSim:
    def __init__(self, cfg, overrides=None, seed=None):
        if isinstance(cfg, str):
            cfg = ConfigFile(cfg)
        self.cfg = cfg
        ov = dict(overrides or {})
        if seed is not None:
            np.random.seed(seed)
        srg, sca, oc = cfg.srg, cfg.sca, cfg.ocean
        self.wh_tol = srg.wh_tol
        self.scat_spec_enable = srg.scat_spec_enable
        self.scat_bragg_enable = srg.scat_bragg_enable
        self.use_hmtf = bool(srg.use_hmtf)
        self.scat_spec_mode = srg.scat_spec_mode
        self.inc_angle = np.deg2rad(sca.inc_angle)
        self.f0 = f0 = sca.f0
        pol = self.pol = sca.pol
        self.do_hh = pol in ('DP', 'hh')
        self.do_vv = pol != 'hh'
        self.prf = sca.prf
        alt = sca.alt
        v_ground = sca.v_ground
        self.rg_bw = sca.rg_bw
        self.over_fs = sca.over_fs
        self.n_sub = int(sca.n_subpulses)
        self.sub_len = sca.sub_pulse_length
        self.frozen = oc.frozen_ocean
        self.n_sinc_samples, self.sinc_ovs = 8, 20
        self.chan_sinc_vec = rp.calc_sinc_vec(8, 20, Fs=self.over_fs)
        s = self.surface = OceanSurface()
        s.init(oc.Lx, oc.Ly, oc.dx, oc.dy, oc.cutoff_wl, oc.spec_model, oc.spread_model,
               np.deg2rad(oc.wind_dir), oc.wind_fetch, oc.wind_U, oc.current_mag,
               np.deg2rad(oc.current_dir), oc.dir_swell_dir, oc.freq_r, oc.sigf, oc.sigs, oc.Hs,
               oc.swell_dir_enable, oc.swell_enable, oc.swell_ampl, np.deg2rad(oc.swell_dir),
               oc.swell_wl, ['D', 'Diff', 'Diff2'] + (['hMTF'] if self.use_hmtf else []), oc.opt_res,
               oc.fft_max_prime,
               choppy_enable=oc.choppy_enable, depth=oc.depth, dirspectrum_func=None,
               dir_swell_spec=spectra.ardhuin_swell_spec if oc.swell_dir_enable else None)
        n_rep = self.n_rep = int(oc.N_repeat_x)
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
        self.inc_s = inc_s.reshape(n_rep, 1, s.Nx)
        self.sr_s = sr_s.reshape(n_rep, 1, s.Nx)
        self.sin_inc_s = np.sin(self.inc_s)
        self.cos_inc_s = np.cos(self.inc_s)
        self.k0 = k0 = 2. * np.pi * f0 / C_LIGHT
        self.sr_res = C_LIGHT / (2. * self.rg_bw)
        self.ant_l_tx, self.ant_l_rx = sca.ant_L_tx, sca.ant_L_rx
        if v_ground == 'auto':
            v_ground = geo.orbit_to_vel(alt, ground=True)
        self.v_ground = v_ground
        self.t_step = 1. / self.prf
        self.t_span = cfg.acquisition.length / v_ground
        self.az_steps = int(ov.get('az_steps', int(np.ceil(self.t_span * self.prf))))
        az_span = (self.t_span * v_ground + s.Ly) / gr0
        max_sr = (np.max(self.sr_s) + self.wh_tol + (np.max(s.y) + (self.t_span / 2.) * v_ground) ** 2. / (2. * sr0)
                  + self.sub_len * C_LIGHT / 2 * (self.n_sub - 1))
        self.min_sr = np.min(self.sr_s) - self.wh_tol
        self.rg_samp_orig = int(ov.get('rg_samp_orig',
                                       int(np.ceil(((max_sr - self.min_sr) / self.sr_res) * self.over_fs))))
        self.rg_samp = int(ov.get('rg_samp', int(geo.optimize_fftsize(self.rg_samp_orig))))
        if self.do_hh:
            self.proc_raw_hh = np.zeros([self.az_steps, self.rg_samp], dtype=complex)
        if self.do_vv:
            self.proc_raw_vv = np.zeros([self.az_steps, self.rg_samp], dtype=complex)
        self.NRCS_avg_vv = np.zeros(self.az_steps, dtype=float)
        self.NRCS_avg_hh = np.zeros(self.az_steps, dtype=float)
        if self.scat_spec_enable:                          # dopsca_raw.py:297-309
            self.rcs_spec_s = []
            for b in range(n_rep):
                if self.scat_spec_mode == 'kodis':
                    self.rcs_spec_s.append(nrcs.RCSKodis(self.inc_s[b], k0, s.dx, s.dy))
                else:
                    np.random.uniform(0., 2. * np.pi, size=[s.Ny, s.Nx])     # spec_ph0, unused
                    self.rcs_spec_s.append(ka.RCSKA(self.scat_spec_mode, k0, s.x, s.y, s.dx, s.dy))
        if self.scat_bragg_enable:
            tau_c = closure.grid_coherence(oc.wind_U, s.dx, f0)
            self.rndscat_p = closure.RandomScatTS(tau_c, (n_rep, s.Ny, s.Nx), 1 / self.sub_len)
            self.rndscat_m = closure.RandomScatTS(tau_c, (n_rep, s.Ny, s.Nx), 1 / self.sub_len)
            k_b_s = 2. * k0 * self.sin_inc_s
            self.c_b_s = self.sin_inc_s * np.sqrt(G / k_b_s + 0.072e-3 * k_b_s)
            cdir = np.deg2rad(oc.current_dir)
            cur = oc.current_mag * np.array([np.cos(cdir), np.sin(cdir)])
            udir = np.deg2rad(oc.wind_dir)
            u_eff = oc.wind_U * np.array([np.cos(udir), np.sin(udir)]) - cur
            self.rcs_bragg_s = [nrcs.RCSRomeiser97(k0, self.inc_s[b], pol, s.dx, s.dy, linalg.norm(u_eff),
                                                   np.arctan2(u_eff[1], u_eff[0]), s.wind_fetch,
                                                   srg.scat_bragg_spec, srg.scat_bragg_spread, srg.scat_bragg_d,
                                                   rmss_x=s.rmss_x, rmss_y=s.rmss_y, az_span=az_span,
                                                   use_lut=bool(getattr(srg, 'use_lut', False)))
                                for b in range(n_rep)]
            self.phase_bragg = np.zeros([2, s.Ny, s.Nx])
            self.bragg_scats = np.zeros([2, s.Ny, s.Nx], dtype=complex)
        self.surface_area = s.dx * s.dy * s.Nx * s.Ny

    def step(self, az_step):
        """All sub-pulses and range blocks of one azimuth step (``dopsca_raw.py:367-519``)."""
        for sub_pulse in range(self.n_sub):
            self.sub_pulse(az_step, sub_pulse)

    def sub_pulse(self, az_step, sub_pulse):
        """One sub-pulse, all range blocks (``dopsca_raw.py:369-519``)."""
        s = self.surface
        t_now = az_step * self.t_step + sub_pulse * self.sub_len
        az_now = (t_now - self.t_span / 2.) * self.v_ground
        az_now_int_smp = int(np.floor(az_now / s.dy))
        az_now_res = az_now - az_now_int_smp * s.dy
        az = (s.y - az_now_res).reshape((s.Ny, 1))
        if self.frozen is False or az_step == 0:
            s.set_t(t_now)
        roll = lambda f: np.roll(f.copy(), -az_now_int_smp, axis=0)  # noqa: E731
        Dz, Dx, Dy = roll(s.Dz), roll(s.Dx), roll(s.Dy)
        Diffx, Diffy = roll(s.Diffx), roll(s.Diffy)
        Diffxx, Diffyy, Diffxy = roll(s.Diffxx), roll(s.Diffyy), roll(s.Diffxy)
        for blk in range(self.n_rep):
            sin_az = az / self.sr0
            az_proj_angle = np.arcsin(az / self.gr0)
            sr_surface = (self.sr_s[blk] - self.cos_inc_s[blk] * Dz + az / 2 * sin_az
                          + Dx * self.sin_inc_s[blk] + Dy * sin_az)
            range_scaling = (self.sr0 / (self.sr0 + sr_surface)) ** 2
            scene_hh = np.zeros([s.Ny, s.Nx], dtype=complex)
            scene_vv = np.zeros([s.Ny, s.Nx], dtype=complex)
            if self.scat_spec_enable:
                if self.scat_spec_mode == 'kodis':
                    Esn_sp = np.sqrt(4. * np.pi) * self.rcs_spec_s[blk].field(az_proj_angle, sr_surface, Diffx,
                                                                              Diffy, Diffxx, Diffyy, Diffxy)
                    if self.do_hh:
                        scene_hh += Esn_sp * range_scaling
                    if self.do_vv:
                        scene_vv += Esn_sp * range_scaling
                else:                                      # dopsca_raw.py:426-445
                    for do, pol_tmp in ((self.do_hh, 'hh'), (self.do_vv, 'vv')):
                        if not do:
                            continue
                        Esn_sp = (np.exp(-1j * (2. * self.k0 * sr_surface)) * (4. * np.pi) ** 1.5 *
                                  self.rcs_spec_s[blk].field(1, 1, pol_tmp[0], pol_tmp[1], self.inc_s[blk],
                                                             self.inc_s[blk], az_proj_angle, az_proj_angle + np.pi,
                                                             Dz, Diffx, Diffy, Diffxx, Diffyy, Diffxy))
                        if pol_tmp == 'hh':
                            scene_hh += Esn_sp * range_scaling
                        else:
                            scene_vv += Esn_sp * range_scaling
                self.NRCS_avg_hh[az_step] += (np.sum(np.abs(Esn_sp) ** 2) / self.surface_area)
                self.NRCS_avg_vv[az_step] += self.NRCS_avg_hh[az_step]
            if self.scat_bragg_enable:
                r = self.rcs_bragg_s[blk].rcs(az_proj_angle, Diffx, Diffy)
                if self.pol == 'DP':
                    RCS_bragg_hh, RCS_bragg_vv = r
                elif self.pol == 'hh':
                    RCS_bragg_hh = r
                else:
                    RCS_bragg_vv = r
                if self.use_hmtf:                      # dopsca_raw.py:461-472
                    if blk == 0:
                        self.hmtf_in = s.hMTF.copy()       # the field this sub-pulse reads
                        hmtf = np.roll(s.hMTF.copy(), -az_now_int_smp, axis=0)
                        s.hMTF[np.where(hmtf < -1)] = -1
                    if self.do_hh:
                        RCS_bragg_hh[0] *= (1 + hmtf)
                        RCS_bragg_hh[1] *= (1 + hmtf)
                    if self.do_vv:
                        RCS_bragg_vv[0] *= (1 + hmtf)
                        RCS_bragg_vv[1] *= (1 + hmtf)
                if self.do_hh:
                    scat_bragg_hh = np.sqrt(RCS_bragg_hh)
                    self.NRCS_avg_hh[az_step] += np.sum(RCS_bragg_hh) / self.surface_area
                if self.do_vv:
                    scat_bragg_vv = np.sqrt(RCS_bragg_vv)
                    self.NRCS_avg_vv[az_step] += np.sum(RCS_bragg_vv) / self.surface_area
                surf_phase = - (2 * self.k0) * sr_surface
                cap_phase = (2 * self.k0) * self.c_b_s[blk] * (self.t_step * (az_step + 1) + sub_pulse * self.sub_len)
                self.phase_bragg[0] = surf_phase - cap_phase
                self.phase_bragg[1] = surf_phase + cap_phase
                self.bragg_scats[0] = np.roll(self.rndscat_m.scats(t_now)[blk], -az_now_int_smp, axis=0)
                self.bragg_scats[1] = np.roll(self.rndscat_p.scats(t_now)[blk], -az_now_int_smp, axis=0)
                if self.do_hh:
                    scene_hh += np.sum(scat_bragg_hh * np.exp(1j * self.phase_bragg) * self.bragg_scats,
                                       axis=0) * range_scaling
                if self.do_vv:
                    scene_vv += np.sum(scat_bragg_vv * np.exp(1j * self.phase_bragg) * self.bragg_scats,
                                       axis=0) * range_scaling
            beam_pattern = (sinc_bp(sin_az, self.ant_l_tx, self.f0, field=True) *
                            sinc_bp(sin_az, self.ant_l_rx, self.f0, field=True))
            sr_surface_mod = sr_surface.flatten() + sub_pulse * self.sub_len * C_LIGHT / 2
            for do, scene, raw in ((self.do_hh, scene_hh, getattr(self, 'proc_raw_hh', None)),
                                   (self.do_vv, scene_vv, getattr(self, 'proc_raw_vv', None))):
                if not do:
                    continue
                this = np.zeros(self.rg_samp, dtype=complex)
                scene_bp = scene * beam_pattern
                rp.chan_profile(sr_surface_mod, scene_bp.flatten(), self.sr_res / self.over_fs, self.min_sr,
                                self.chan_sinc_vec, self.n_sinc_samples, self.sinc_ovs, this)
                raw[az_step] = raw[az_step] + this

    def run(self, steps=None):
        for a in (range(self.az_steps) if steps is None else steps):
            self.step(a)

    def finish(self):
        """Truncation and calibration (``dopsca_raw.py:538-562``)."""
        t_span, v = self.t_span, self.v_ground
        az_axis = np.arange(-t_span / 2. * v, t_span / 2. * v,
                            self.sr0 * C_LIGHT / (np.pi * self.f0 * self.ant_l_tx * 10.))
        pattern = (sinc_bp(az_axis / self.sr0, self.ant_l_tx, self.f0, field=True) *
                   sinc_bp(az_axis / self.sr0, self.ant_l_rx, self.f0, field=True))
        cal_factor = (1. / np.sqrt(np.trapezoid(np.abs(pattern) ** 2., az_axis) *
                                   self.sr_res / np.sin(self.inc_angle)))
        out, nrcs_avg = [], []
        if self.do_hh:
            out.append(self.proc_raw_hh[:, :self.rg_samp_orig] * cal_factor)
            nrcs_avg.append(self.NRCS_avg_hh)
        if self.do_vv:
            out.append(self.proc_raw_vv[:, :self.rg_samp_orig] * cal_factor)
            nrcs_avg.append(self.NRCS_avg_vv)
        return np.stack(out), np.stack(nrcs_avg)


def dopsca_raw(cfg_file, seed=0, overrides=None):
    """Whole run: (raw [pol, az, rg], NRCS_avg [pol, az], sim)."""
    sim = DopscaSim(cfg_file, overrides=overrides, seed=seed)
    sim.run()
    raw, nrcs_avg = sim.finish()
    return raw, nrcs_avg, sim
