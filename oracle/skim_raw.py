"""Oracle (test infrastructure only): the SKIM raw-data generator ``skimraw``.

Restates ``oceansar/radarsim/skim_raw.py:51-689`` on one process (the MPI row scattering
is the identity there) with the oracle's surface, balancer, NRCS, Kirchhoff, closure,
geometry and accumulation restatements:

* ``upsample_and_dopplerize`` ``:51-81``;
* set-up ``:102-461``: the ``[radar]`` section, beam-relative wind / current / swell
  directions, the surface and its time-interpolating balancer, absolute slant range,
  ``sr_prof`` and the reference Doppler, the two-scale Doppler decimation (``n_pulses_b``,
  ``ny_integ``, ``dop0``), Kodis or Kirchhoff specular, scatterer series at the PRF and
  the Romeiser model with its constructor defaults (LUT mode);
* the loop ``:465-684`` (with the calibration target of ``:151-164``, ``:490-493`` and
  ``:608-615``) and the post-processing ``:686-773`` (up-sampling, truncation,
  calibration, noise).
"""
import numpy as np
from scipy import linalg

from . import closure, geometry as geo, ka, nrcs, range_profile as rp, spectra
from .balancer import OceanSurfaceBalancer
from .cfg import ConfigFile
from .sar_raw import C_LIGHT, sinc_bp
from .surface import OceanSurface

G = 9.80665


def sinc_1tx_nrx(sin_angle, L, f0, num_chan, field=False, sin_squint=0):
    """``antenna.py:28-42``: the field flag reaches sinc_bp's positional catch-all, so both
    patterns are in power units."""
    return sinc_bp(sin_angle - sin_squint, L, f0) * sinc_bp(sin_angle - sin_squint, L / num_chan, f0)


def upsample_and_dopplerize(ssraw, dop, n_up, prf):
    dims = ssraw.shape
    out = np.zeros((dims[0] * int(n_up), dims[2]), dtype=np.complex64)
    t = (np.arange(dims[0] * int(n_up)) / prf).reshape((dims[0] * int(n_up), 1))
    t2pi = t * (np.pi * 2)
    for ind in range(dims[1]):
        raw_zp = np.zeros((dims[0] * int(n_up), dims[2]), dtype=np.complex64)
        raw_zp[0:dims[0]] = np.fft.fftshift(np.fft.fft(ssraw[:, ind, :], axis=0), axes=(0,))
        raw_zp = np.roll(raw_zp, int(-dims[0] / 2), axis=0)
        raw_zp = np.conj(np.fft.fft(np.conj(raw_zp), axis=0)) / dims[0]
        dop_phase = t2pi * (dop[ind]).reshape((1, dims[2]))
        out = out + raw_zp * np.exp(1j * dop_phase)
    return out


class SkimSim:
    def __init__(self, cfg, seed=None):
        if isinstance(cfg, str):
            cfg = ConfigFile(cfg)
        self.cfg = cfg
        if seed is not None:
            np.random.seed(seed)
        srg, radar, oc = cfg.srg, cfg.radar, cfg.ocean
        # calibration target (skim_raw.py:151-164)
        self.add_point_target, self.point_target_floats = False, True
        if hasattr(cfg, 'sim') and hasattr(cfg.sim, 'cal_targets') and cfg.sim.cal_targets is not False:
            self.add_point_target = True
            self.point_target_floats = cfg.sim.cal_targets.lower() == 'floating'
        self.wh_tol, self.nesz = srg.wh_tol, srg.nesz
        self.use_hmtf = srg.use_hmtf
        self.scat_spec_enable, self.scat_spec_mode = srg.scat_spec_enable, srg.scat_spec_mode
        self.scat_bragg_enable = srg.scat_bragg_enable
        self.inc_angle = np.deg2rad(radar.inc_angle)
        self.f0 = f0 = radar.f0
        pol = self.pol = radar.pol
        self.squint_r = np.radians(90 - radar.azimuth)
        self.do_hh = pol in ('DP', 'hh')
        self.do_vv = pol != 'hh'
        self.prf = prf = radar.prf
        num_ch = int(radar.num_ch)
        ant_L = radar.ant_L
        alt = radar.alt
        v_ground = radar.v_ground
        self.rg_bw = radar.rg_bw
        self.over_fs = radar.Fs / radar.rg_bw
        self.ocean_dt = oc.dt
        self.n_sinc_samples, self.sinc_ovs = 10, 20
        self.chan_sinc_vec = rp.calc_sinc_vec(10, 20, Fs=self.over_fs)
        wind_dir = radar.azimuth - oc.wind_dir
        compute = ['D', 'Diff', 'Diff2']
        if self.use_hmtf:
            compute.append('hMTF')
        s = self.surface_full = OceanSurface()
        s.init(oc.Lx, oc.Ly, oc.dx, oc.dy, oc.cutoff_wl, oc.spec_model, oc.spread_model,
               np.deg2rad(wind_dir), oc.wind_fetch, oc.wind_U, oc.current_mag,
               np.deg2rad(radar.azimuth - oc.current_dir), radar.azimuth - oc.dir_swell_dir,
               oc.freq_r, oc.sigf, oc.sigs, oc.Hs, oc.swell_dir_enable, oc.swell_enable, oc.swell_ampl,
               np.deg2rad(radar.azimuth - oc.swell_dir), oc.swell_wl, compute, oc.opt_res, oc.fft_max_prime,
               choppy_enable=oc.choppy_enable, depth=oc.depth, dirspectrum_func=None,
               dir_swell_spec=spectra.ardhuin_swell_spec if oc.swell_dir_enable else None)
        b = self.surface = OceanSurfaceBalancer(s, self.ocean_dt)
        self.sr0 = geo.inc_to_sr(self.inc_angle, alt)
        self.gr0 = gr0 = geo.inc_to_gr(self.inc_angle, alt)
        sr, inc, _ = geo.gr_to_geo(b.x + gr0, alt)
        self.min_sr = np.min(sr)
        self.inc = inc.reshape(1, inc.size)
        self.sr = sr.reshape(1, sr.size)
        self.sin_inc, self.cos_inc = np.sin(self.inc), np.cos(self.inc)
        self.l0 = l0 = C_LIGHT / f0
        self.k0 = k0 = 2. * np.pi * f0 / C_LIGHT
        self.sr_res = C_LIGHT / (2. * self.rg_bw)
        self.sr_smp = C_LIGHT / (2 * radar.Fs)
        self.L_total = radar.L_total
        if radar.L_total:
            ant_L = ant_L / float(num_ch)
        self.ant_L, self.num_ch = ant_L, num_ch
        if v_ground == 'auto':
            v_ground = geo.orbit_to_vel(alt, ground=True)
            v_orb = geo.orbit_to_vel(alt, ground=False)
        else:
            v_orb = v_ground
        self.v_ground = v_ground
        self.t_step = 1. / prf
        self.az_steps = int(radar.n_pulses)
        self.t_span = self.az_steps / prf
        self.n_rg = radar.n_rg
        self.rg_samp = rg_samp = int(geo.optimize_fftsize(radar.n_rg))
        sr_prof = (np.arange(rg_samp) - rg_samp / 2) * self.sr_smp + np.mean(sr)
        gr_prof, inc_prof, look_prof, b_prof = geo.sr_to_geo(sr_prof, alt)
        look_prof = look_prof.reshape((1, look_prof.size))
        self.sr_prof = sr_prof.reshape((1, look_prof.size))
        self.dop_ref = 2 * v_orb * np.sin(look_prof) * np.sin(self.squint_r) / l0
        self.two_scale = srg.two_scale_Doppler
        self.rcm = srg.rcm if self.two_scale else False
        if self.two_scale:
            self.n_pulses_b = geo.optimize_fftsize(int(srg.surface_coh_time * prf)) / 2
            self.az_steps_ = int(np.ceil(self.az_steps / self.n_pulses_b))
            self.t_step = self.t_step * self.n_pulses_b
            dy_integ = srg.phase_err_tol / (2 * k0 * v_ground / self.min_sr * srg.surface_coh_time)
            ny_integ = dy_integ / b.dy
            ny_integ = 1 if ny_integ < 1 else int(2 ** np.floor(np.log2(ny_integ)))
            self.ny_integ = ny_integ
            s_int = int(b.Ny / ny_integ)
            shape = [self.az_steps_, s_int, rg_samp]
            az = b.y.reshape((b.Ny, 1))
            da = az / gr_prof
            sin_az = np.sin(self.squint_r) + np.cos(self.squint_r) * da - 0.5 * np.sin(self.squint_r) * da ** 2
            dop0 = 2 * v_orb * np.sin(look_prof) * sin_az / l0
            self.dop0 = np.mean(np.reshape(dop0, (s_int, int(ny_integ), rg_samp)), axis=1)
        else:
            self.az_steps_ = self.az_steps
            shape = [self.az_steps, rg_samp]
        if self.do_hh:
            self.proc_raw_hh = np.zeros(shape, dtype=complex)
        if self.do_vv:
            self.proc_raw_vv = np.zeros(shape, dtype=complex)
        self.t_last_rcs_bragg = -1.
        self.NRCS_avg_vv = np.zeros(self.az_steps, dtype=float)
        self.NRCS_avg_hh = np.zeros(self.az_steps, dtype=float)
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                self.rcs_spec = nrcs.RCSKodis(self.inc, k0, b.dx, b.dy)
            else:
                self.spec_ph0 = np.random.uniform(0., 2. * np.pi, size=[b.Ny, b.Nx])
                self.rcs_spec = ka.RCSKA(self.scat_spec_mode, k0, b.x, b.y, b.dx, b.dy)
        if self.scat_bragg_enable:
            self.phase_bragg = np.zeros([2, b.Ny, b.Nx])
            self.bragg_scats = np.zeros([2, b.Ny, b.Nx], dtype=complex)
            tau_c = closure.grid_coherence(oc.wind_U, b.dx, f0)
            self.rndscat_p = closure.RandomScatTS(tau_c, (b.Ny, b.Nx), prf)
            self.rndscat_m = closure.RandomScatTS(tau_c, (b.Ny, b.Nx), prf)
            k_b = 2. * k0 * self.sin_inc
            self.c_b = self.sin_inc * np.sqrt(G / k_b + 0.072e-3 * k_b)
            cdir = np.deg2rad(oc.current_dir)
            cur = oc.current_mag * np.array([np.cos(cdir), np.sin(cdir)])
            udir = np.deg2rad(oc.wind_dir)
            u_eff = oc.wind_U * np.array([np.cos(udir), np.sin(udir)]) - cur
            # the reference relies on the constructor's defaults: LUT mode
            self.rcs_bragg = nrcs.RCSRomeiser97(k0, self.inc, pol, b.dx, b.dy, linalg.norm(u_eff),
                                                np.arctan2(u_eff[1], u_eff[0]), s.wind_fetch,
                                                srg.scat_bragg_spec, srg.scat_bragg_spread, srg.scat_bragg_d,
                                                use_lut=True)
        self.surface_area = b.dx * b.dy * b.Nx * b.Ny

    def step(self, az_step):
        """One iteration of ``skim_raw.py:465-684``."""
        s = self.surface
        t_now = az_step * self.t_step
        az_now = (t_now - self.t_span / 2.) * self.v_ground * np.cos(self.squint_r)
        az = (s.y - az_now).reshape((s.Ny, 1))
        s.set_t(t_now)
        sin_az = az / self.sr
        az_proj_angle = np.arcsin(az / self.gr0)
        pt_y, pt_x = int(s.Ny / 2), int(s.Nx / 2)
        if not self.point_target_floats:                      # skim_raw.py:490-493
            s.Dx[pt_y, pt_x] = 0
            s.Dy[pt_y, pt_x] = 0
            s.Dz[pt_y, pt_x] = 0
        if self.two_scale:
            sr_surface = self.sr - self.cos_inc * s.Dz + s.Dx * self.sin_inc + s.Dy * sin_az
            sr_surface4rcm = sr_surface + az / 2 * sin_az if self.rcm else sr_surface
        else:
            sr_surface = (self.sr - self.cos_inc * s.Dz + az / 2 * sin_az + s.Dx * self.sin_inc + s.Dy * sin_az)
            sr_surface4rcm = sr_surface
        scene_hh = np.zeros([s.Ny, s.Nx], dtype=complex)
        scene_vv = np.zeros([s.Ny, s.Nx], dtype=complex)
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                Esn_sp = np.sqrt(4. * np.pi) * self.rcs_spec.field(az_proj_angle, sr_surface, s.Diffx, s.Diffy,
                                                                   s.Diffxx, s.Diffyy, s.Diffxy)
                scene_hh += Esn_sp
                scene_vv += Esn_sp
            else:
                for do, pol_tmp in ((self.do_hh, 'hh'), (self.do_vv, 'vv')):
                    if not do:
                        continue
                    Esn_sp = (np.exp(-1j * (2. * self.k0 * sr_surface)) * (4. * np.pi) ** 1.5 *
                              self.rcs_spec.field(1, 1, pol_tmp[0], pol_tmp[1], self.inc, self.inc, az_proj_angle,
                                                  az_proj_angle + np.pi, s.Dz, s.Diffx, s.Diffy, s.Diffxx,
                                                  s.Diffyy, s.Diffxy))
                    if pol_tmp == 'hh':
                        scene_hh += Esn_sp
                    else:
                        scene_vv += Esn_sp
            self.NRCS_avg_hh[az_step] += (np.sum(np.abs(Esn_sp) ** 2) / self.surface_area)
            self.NRCS_avg_vv[az_step] += self.NRCS_avg_hh[az_step]
        if self.scat_bragg_enable:
            if (t_now - self.t_last_rcs_bragg) > self.ocean_dt:
                r = self.rcs_bragg.rcs(az_proj_angle, s.Diffx, s.Diffy)
                if self.pol == 'DP':
                    self.RCS_bragg_hh, self.RCS_bragg_vv = r
                elif self.pol == 'hh':
                    self.RCS_bragg_hh = r
                else:
                    self.RCS_bragg_vv = r
                if self.use_hmtf:
                    s.hMTF[np.where(s.hMTF < -1)] = -1
                    for attr in ('RCS_bragg_hh', 'RCS_bragg_vv'):
                        if hasattr(self, attr):
                            getattr(self, attr)[0] *= (1 + s.hMTF)
                            getattr(self, attr)[1] *= (1 + s.hMTF)
                self.t_last_rcs_bragg = t_now
            if self.do_hh:
                scat_bragg_hh = np.sqrt(self.RCS_bragg_hh)
                self.NRCS_avg_hh[az_step] += np.sum(self.RCS_bragg_hh) / self.surface_area
            if self.do_vv:
                scat_bragg_vv = np.sqrt(self.RCS_bragg_vv)
                self.NRCS_avg_vv[az_step] += np.sum(self.RCS_bragg_vv) / self.surface_area
            surf_phase = - (2 * self.k0) * sr_surface
            cap_phase = (2 * self.k0) * self.t_step * self.c_b * (az_step + 1)
            self.phase_bragg[0] = surf_phase - cap_phase
            self.phase_bragg[1] = surf_phase + cap_phase
            self.bragg_scats[0] = self.rndscat_m.scats(t_now)
            self.bragg_scats[1] = self.rndscat_p.scats(t_now)
            if self.do_hh:
                scene_hh += np.sum(scat_bragg_hh * np.exp(1j * self.phase_bragg) * self.bragg_scats, axis=0)
            if self.do_vv:
                scene_vv += np.sum(scat_bragg_vv * np.exp(1j * self.phase_bragg) * self.bragg_scats, axis=0)
        if self.add_point_target:                             # skim_raw.py:608-615
            pt = 1000 * np.exp(-1j * 2 * self.k0 * sr_surface[pt_y, pt_x])
            scene_hh[pt_y, pt_x] = pt
            scene_vv[pt_y, pt_x] = pt
        if self.L_total:
            beam_pattern = sinc_1tx_nrx(sin_az, self.ant_L * self.num_ch, self.f0, self.num_ch, field=True)
        else:
            beam_pattern = sinc_1tx_nrx(sin_az, self.ant_L, self.f0, 1, field=True)
        for do, scene, raw in ((self.do_hh, scene_hh, getattr(self, 'proc_raw_hh', None)),
                               (self.do_vv, scene_vv, getattr(self, 'proc_raw_vv', None))):
            if not do:
                continue
            if self.two_scale:
                step = np.zeros([s.Ny, self.rg_samp], dtype=complex)
                rp.chan_profile(sr_surface4rcm, scene * beam_pattern, self.sr_smp, self.sr_prof.min(),
                                self.chan_sinc_vec, self.n_sinc_samples, self.sinc_ovs, step, rg_only=True)
                s_int = int(s.Ny / self.ny_integ)
                raw[az_step] = np.sum(np.reshape(step, (s_int, self.ny_integ, self.rg_samp)), axis=1)
            else:
                rp.chan_profile(sr_surface4rcm.flatten(), (scene * beam_pattern).flatten(), self.sr_smp,
                                self.sr_prof.min(), self.chan_sinc_vec, self.n_sinc_samples, self.sinc_ovs,
                                raw[az_step])

    def run(self):
        for a in range(self.az_steps_):
            self.step(a)

    def finish(self, add_noise=True):
        """Up-sampling, truncation, calibration and noise (``skim_raw.py:686-739``)."""
        out = []
        raws = [r for do, r in ((self.do_hh, getattr(self, 'proc_raw_hh', None)),
                                (self.do_vv, getattr(self, 'proc_raw_vv', None))) if do]
        if self.two_scale:
            raws = [upsample_and_dopplerize(r, self.dop0, self.n_pulses_b, self.prf) for r in raws]
        raws = [r[:, :self.n_rg] for r in raws]
        az_axis = np.arange(-self.t_span / 2. * self.v_ground, self.t_span / 2. * self.v_ground,
                            self.sr0 * C_LIGHT / (np.pi * self.f0 * self.ant_L * 10.))
        if self.L_total:
            pattern = sinc_1tx_nrx(az_axis / self.sr0, self.ant_L * self.num_ch, self.f0, self.num_ch, field=True)
        else:
            pattern = sinc_1tx_nrx(az_axis / self.sr0, self.ant_L, self.f0, 1, field=True)
        cal_factor = (1. / np.sqrt(np.trapezoid(np.abs(pattern) ** 2., az_axis) * self.sr_res / np.sin(self.inc_angle)))
        for r in raws:
            if add_noise:
                noise = (geo.db2lin(self.nesz, amplitude=True) / np.sqrt(2.) *
                         (np.random.normal(size=r.shape) + 1j * np.random.normal(size=r.shape)))
                out.append(r * cal_factor + noise)
            else:
                out.append(r * cal_factor)
        nrcs_avg = [n for do, n in ((self.do_hh, self.NRCS_avg_hh), (self.do_vv, self.NRCS_avg_vv)) if do]
        return np.stack(out), np.stack(nrcs_avg)


def skimraw(cfg_file, seed=0, add_noise=True):
    """Whole run: (raw [pol, az, n_rg], NRCS_avg [pol, n_pulses], sim)."""
    sim = SkimSim(cfg_file, seed=seed)
    sim.run()
    raw, nrcs_avg = sim.finish(add_noise=add_noise)
    return raw, nrcs_avg, sim
