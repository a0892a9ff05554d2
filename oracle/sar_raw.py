"""Oracle (test infrastructure only): the raw-data generator ``sar_raw``.

Restates ``oceansar/radarsim/sar_raw_nompi.py:32-574`` with the oracle's own surface,
NRCS, closure, geometry and accumulation restatements:

* set-up ``:66-341`` (configuration, surface init with the global numpy RNG, geometry,
  sizes, Kodis / Romeiser models, random scatterer series ``rndscat_p`` then ``rndscat_m``)
* the per-pulse loop ``:349-535`` (surface update, slant range, specular field, Bragg RCS
  refreshed only when ``t_now - t_last > ocean_dt``, Bragg phases, scene, antenna pattern,
  per-channel ATI / XTI phases, accumulation)
* post-processing ``:552-574`` (truncation, calibration factor, complex noise)

``SarRawSim`` keeps the state between pulses so that a test or the CPU baseline can run
any window of pulses; ``overrides`` may force ``az_steps`` / ``rg_samp`` (the reference
derives them from the geometry, ``:264-278``).
"""
import numpy as np
from scipy import linalg

from . import closure, geometry as geo, ka, nrcs, range_profile as rp, spectra
from .cfg import ConfigFile
from .surface import OceanSurface

C_LIGHT = 2.99792458e8


def sinc_bp(sin_angle, L, f0, field=False):
    """``oceansar/radarsim/antenna.py:5-25`` (no squint, no beamwidth override)."""
    l = C_LIGHT / f0
    pattern = np.sinc(L / l * sin_angle)
    return pattern if field else pattern ** 2


class SarRawSim:
    def __init__(self, cfg, overrides=None, seed=None, surface_dt=None):
        if isinstance(cfg, str):
            cfg = ConfigFile(cfg)
        self.cfg = cfg
        ov = dict(overrides or {})
        if seed is not None:
            np.random.seed(seed)
        srg, sar, oc = cfg.srg, cfg.sar, cfg.ocean
        self.wh_tol = srg.wh_tol
        self.nesz = srg.nesz
        self.use_hmtf = srg.use_hmtf
        self.scat_spec_enable = srg.scat_spec_enable
        self.scat_spec_mode = srg.scat_spec_mode
        self.scat_bragg_enable = srg.scat_bragg_enable
        self.inc_angle = np.deg2rad(sar.inc_angle)
        self.f0 = f0 = sar.f0
        pol = self.pol = sar.pol
        self.do_hh = pol in ('DP', 'hh')
        self.do_vv = pol != 'hh'
        self.prf = sar.prf
        self.num_ch = int(sar.num_ch)
        alt = sar.alt
        v_ground = sar.v_ground
        self.rg_bw = sar.rg_bw
        self.over_fs = sar.over_fs
        self.ocean_dt = oc.dt
        self.n_sinc_samples = 8
        self.sinc_ovs = 20
        self.chan_sinc_vec = rp.calc_sinc_vec(8, 20, Fs=self.over_fs)
        compute = ['D', 'Diff', 'Diff2']
        if self.use_hmtf:
            compute.append('hMTF')
        dir_swell = spectra.ardhuin_swell_spec if oc.swell_dir_enable else None
        s = self.surface = OceanSurface()
        s.init(oc.Lx, oc.Ly, oc.dx, oc.dy, oc.cutoff_wl, oc.spec_model, oc.spread_model,
               np.deg2rad(oc.wind_dir), oc.wind_fetch, oc.wind_U, oc.current_mag,
               np.deg2rad(oc.current_dir), oc.dir_swell_dir, oc.freq_r, oc.sigf, oc.sigs, oc.Hs,
               oc.swell_dir_enable, oc.swell_enable, oc.swell_ampl, np.deg2rad(oc.swell_dir),
               oc.swell_wl, compute, oc.opt_res, oc.fft_max_prime, choppy_enable=oc.choppy_enable,
               depth=oc.depth, dirspectrum_func=None, dir_swell_spec=dir_swell)
        self.frozen = bool(getattr(oc, 'frozen_ocean', False))
        self.sr0 = sr0 = geo.inc_to_sr(self.inc_angle, alt)
        self.gr0 = gr0 = geo.inc_to_gr(self.inc_angle, alt)
        gr = s.x + gr0
        sr, inc, _ = geo.gr_to_geo(gr, alt)
        rg_sampling = self.rg_bw * self.over_fs
        self.sr_near = sr[0] - self.wh_tol + C_LIGHT / 2 / rg_sampling
        sr -= np.min(sr)
        self.inc = inc.reshape(1, inc.size)
        self.sr = sr.reshape(1, sr.size)
        self.sin_inc = np.sin(self.inc)
        self.cos_inc = np.cos(self.inc)
        self.l0 = C_LIGHT / f0
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
        self.b_ati, self.b_xti = b_ati, b_xti
        if v_ground == 'auto':
            v_ground = geo.orbit_to_vel(alt, ground=True)
        self.v_ground = v_ground
        self.t_step = t_step = 1. / self.prf
        self.t_span = t_span = (1.5 * (sr0 * self.l0 / self.ant_l_tx) + s.Ly) / v_ground
        self.az_steps = int(ov.get('az_steps', int(np.floor(t_span / t_step))))
        az_span = (t_span * v_ground + s.Ly) / gr0
        max_sr = (np.max(sr) + self.wh_tol +
                  (np.max(s.y) + (t_span / 2.) * v_ground) ** 2. / (2. * sr0))
        self.min_sr = np.min(sr) - self.wh_tol
        self.rg_samp_orig = int(ov.get('rg_samp_orig',
                                       int(np.ceil(((max_sr - self.min_sr) / self.sr_res) * self.over_fs))))
        self.rg_samp = int(ov.get('rg_samp', int(geo.optimize_fftsize(self.rg_samp_orig))))
        if self.do_hh:
            self.proc_raw_hh = np.zeros([self.num_ch, self.az_steps, self.rg_samp], dtype=complex)
        if self.do_vv:
            self.proc_raw_vv = np.zeros([self.num_ch, self.az_steps, self.rg_samp], dtype=complex)
        self.t_last_rcs_bragg = -1.
        self.NRCS_avg_vv = np.zeros(self.az_steps, dtype=float)
        self.NRCS_avg_hh = np.zeros(self.az_steps, dtype=float)
        if self.scat_spec_enable:
            if self.scat_spec_mode == 'kodis':
                self.rcs_spec = nrcs.RCSKodis(self.inc, k0, s.dx, s.dy)
            elif self.scat_spec_mode in ('fa', 'spa'):
                # sar_raw_nompi.py:296-299: a phase screen is drawn (and not used afterwards)
                self.spec_ph0 = np.random.uniform(0., 2. * np.pi, size=[s.Ny, s.Nx])
                self.rcs_spec = ka.RCSKA(self.scat_spec_mode, k0, s.x, s.y, s.dx, s.dy)
            else:
                raise NotImplementedError('specular mode %s' % self.scat_spec_mode)
        if self.scat_bragg_enable:
            if srg.scat_bragg_model != 'romeiser97':
                raise NotImplementedError('Bragg model %s' % srg.scat_bragg_model)
            self.phase_bragg = np.zeros([2, s.Ny, s.Nx])
            self.bragg_scats = np.zeros([2, s.Ny, s.Nx], dtype=complex)
            tau_c = closure.grid_coherence(oc.wind_U, s.dx, f0)
            self.rndscat_p = closure.RandomScatTS(tau_c, (s.Ny, s.Nx), self.prf)
            self.rndscat_m = closure.RandomScatTS(tau_c, (s.Ny, s.Nx), self.prf)
            k_b = 2. * k0 * self.sin_inc
            self.c_b = self.sin_inc * np.sqrt(9.80665 / k_b + 0.072e-3 * k_b)
            current_dir = np.deg2rad(oc.current_dir)
            current_vec = oc.current_mag * np.array([np.cos(current_dir), np.sin(current_dir)])
            U_dir = np.deg2rad(oc.wind_dir)
            U_vec = oc.wind_U * np.array([np.cos(U_dir), np.sin(U_dir)])
            U_eff_vec = U_vec - current_vec
            self.rcs_bragg = nrcs.RCSRomeiser97(k0, self.inc, pol, s.dx, s.dy, linalg.norm(U_eff_vec),
                                                np.arctan2(U_eff_vec[1], U_eff_vec[0]), s.wind_fetch,
                                                srg.scat_bragg_spec, srg.scat_bragg_spread,
                                                srg.scat_bragg_d, rmss_x=s.rmss_x, rmss_y=s.rmss_y,
                                                az_span=az_span, use_lut=srg.use_lut)
        self.surface_area = s.dx * s.dy * s.Nx * s.Ny
        self.next_step = 0
        # time-interpolated surface of the MPI generator (sar_raw.py:233-353)
        self.balancer = None
        if surface_dt and not self.frozen:
            from .balancer import OceanSurfaceBalancer
            self.balancer = OceanSurfaceBalancer(s, surface_dt)

    # ------------------------------------------------------------------------------
    def set_threads(self, threads):
        """Run the per-facet work of each pulse on ``threads`` host threads (row blocks in a
        thread pool; numpy and the C accumulator release the GIL) and the surface FFTs with
        ``threads`` workers.  Only the CPU baseline uses more than one thread: with one
        thread (the default) every operation is the whole-array operation of the reference,
        bit for bit; with several, the NRCS sums and the range profiles are summed block by
        block (rounding order differs)."""
        import concurrent.futures
        import functools
        self.threads = max(1, int(threads))
        self._pool = (concurrent.futures.ThreadPoolExecutor(self.threads) if self.threads > 1 else None)
        if self.threads > 1:
            import scipy.fft
            self.surface.fft_ifft2 = functools.partial(scipy.fft.ifft2, workers=self.threads)
        else:
            self.surface.fft_ifft2 = None

    def pulse(self, az_step, record=None):
        """One iteration of ``sar_raw_nompi.py:349-535``."""
        s = self.surface
        t_now = az_step * self.t_step
        az_now = (t_now - self.t_span / 2.) * self.v_ground
        az = (s.y - az_now).reshape((s.Ny, 1))
        if self.balancer is not None:
            s = self.balancer
            s.set_t(t_now)
        elif (not self.frozen) or az_step == 0:
            s.set_t(t_now)
        sin_az = az / self.sr0
        az_proj_angle = np.arcsin(az / self.gr0)
        refresh = self.scat_bragg_enable and (t_now - self.t_last_rcs_bragg) > self.ocean_dt
        if refresh:
            self.t_last_rcs_bragg = t_now
            if record is not None:
                record['rcs_refresh'] = True
        if self.scat_bragg_enable:
            scats = (self.rndscat_m.scats(t_now), self.rndscat_p.scats(t_now))
        else:
            scats = None
        threads = getattr(self, 'threads', 1)
        ny = s.Ny
        kirchhoff = self.scat_spec_enable and self.scat_spec_mode != 'kodis'   # needs whole rows of x, y
        if threads == 1 or record is not None or kirchhoff:
            blocks = [(0, ny)]
        else:
            nb = 4 * threads
            edges = [ny * i // nb for i in range(nb + 1)]
            blocks = [(edges[i], edges[i + 1]) for i in range(nb) if edges[i + 1] > edges[i]]
        if refresh and len(blocks) > 1:
            shape = (2, s.Ny, s.Nx)
            if self.do_hh:
                self.RCS_bragg_hh = np.empty(shape)
            if self.do_vv:
                self.RCS_bragg_vv = np.empty(shape)
        args = (s, az_step, t_now, az, sin_az, az_proj_angle, refresh, scats, record, len(blocks) == 1)
        if len(blocks) == 1:
            parts = [self._pulse_rows(0, ny, *args)]
        else:
            parts = list(self._pool.map(lambda blk: self._pulse_rows(blk[0], blk[1], *args), blocks))
        spec = [p[0] for p in parts]
        if self.scat_spec_enable:
            self.NRCS_avg_hh[az_step] += (spec[0] if len(spec) == 1 else sum(spec)) / self.surface_area
            self.NRCS_avg_vv[az_step] += self.NRCS_avg_hh[az_step]
        if self.scat_bragg_enable:
            for k, (do, attr) in enumerate(((self.do_hh, 'NRCS_avg_hh'), (self.do_vv, 'NRCS_avg_vv'))):
                if do:
                    rs = [p[1][k] for p in parts]
                    getattr(self, attr)[az_step] += (rs[0] if len(rs) == 1 else sum(rs)) / self.surface_area
        if len(parts) > 1:
            for key in parts[0][2]:
                pol, ch = key
                raw = self.proc_raw_hh if pol == 'hh' else self.proc_raw_vv
                for p in parts:
                    raw[ch][az_step] += p[2][key]

    def _pulse_rows(self, r0, r1, s, az_step, t_now, az, sin_az, az_proj_angle, refresh, scats, record, whole):
        """The per-facet part of a pulse for facet rows r0:r1.  ``whole``: the block is the
        whole surface (whole-array operations, profiles accumulated in place)."""
        rows = slice(r0, r1)
        az, sin_az, az_proj_angle = az[rows], sin_az[rows], az_proj_angle[rows]
        Dx, Dy, Dz = s.Dx[rows], s.Dy[rows], s.Dz[rows]
        Diffx, Diffy = s.Diffx[rows], s.Diffy[rows]
        ny = r1 - r0
        sr_surface = (self.sr - self.cos_inc * Dz + az / 2 * sin_az
                      + Dx * self.sin_inc + Dy * sin_az)
        wave_dinc = (Dz * self.sin_inc + Dx * self.sin_inc) / self.sr0
        if self.do_hh:
            scene_hh = np.zeros([ny, s.Nx], dtype=complex)
        if self.do_vv:
            scene_vv = np.zeros([ny, s.Nx], dtype=complex)
        spec_sum = 0.
        if self.scat_spec_enable and self.scat_spec_mode == 'kodis':
            Esn_sp = np.sqrt(4. * np.pi) * self.rcs_spec.field(az_proj_angle, sr_surface, Diffx,
                                                                Diffy, s.Diffxx[rows], s.Diffyy[rows],
                                                                s.Diffxy[rows])
            if self.do_hh:
                scene_hh += Esn_sp
            if self.do_vv:
                scene_vv += Esn_sp
        elif self.scat_spec_enable:
            # Kirchhoff modes (sar_raw_nompi.py:402-426): per polarisation, two-way phase of the
            # facet's slant range times the monostatic field
            for do, pol_tmp in ((self.do_hh, 'hh'), (self.do_vv, 'vv')):
                if not do:
                    continue
                Esn_sp = (np.exp(-1j * (2. * self.k0 * sr_surface)) * (4. * np.pi) ** 1.5 *
                          self.rcs_spec.field(1, 1, pol_tmp[0], pol_tmp[1], self.inc, self.inc, az_proj_angle,
                                              az_proj_angle + np.pi, Dz, Diffx, Diffy, s.Diffxx[rows],
                                              s.Diffyy[rows], s.Diffxy[rows]))
                if pol_tmp == 'hh':
                    scene_hh += Esn_sp
                else:
                    scene_vv += Esn_sp
        if self.scat_spec_enable:
            spec_sum = np.sum(np.abs(Esn_sp) ** 2)
        bragg_sums = [0., 0.]
        if self.scat_bragg_enable:
            if refresh:
                r = self.rcs_bragg.rcs(az_proj_angle, Diffx, Diffy)
                if self.pol == 'DP':
                    r_hh, r_vv = r
                elif self.pol == 'hh':
                    r_hh, r_vv = r, None
                else:
                    r_hh, r_vv = None, r
                if self.use_hmtf:
                    hm = s.hMTF[rows]
                    hm[np.where(hm < -1)] = -1
                    if self.do_hh:
                        r_hh[0] *= (1 + hm)
                        r_hh[1] *= (1 + hm)
                    if self.do_vv:
                        r_vv[0] *= (1 + hm)
                        r_vv[1] *= (1 + hm)
                if whole:
                    if self.do_hh:
                        self.RCS_bragg_hh = r_hh
                    if self.do_vv:
                        self.RCS_bragg_vv = r_vv
                else:
                    if self.do_hh:
                        self.RCS_bragg_hh[:, rows] = r_hh
                    if self.do_vv:
                        self.RCS_bragg_vv[:, rows] = r_vv
            if self.do_hh:
                rcs = self.RCS_bragg_hh if whole else self.RCS_bragg_hh[:, rows]
                scat_bragg_hh = np.sqrt(rcs)
                bragg_sums[0] = np.sum(rcs)
            if self.do_vv:
                rcs = self.RCS_bragg_vv if whole else self.RCS_bragg_vv[:, rows]
                scat_bragg_vv = np.sqrt(rcs)
                bragg_sums[1] = np.sum(rcs)
            surf_phase = - (2 * self.k0) * sr_surface
            cap_phase = (2 * self.k0) * self.t_step * self.c_b * (az_step + 1)
            if whole:
                phase_bragg, bragg_scats = self.phase_bragg, self.bragg_scats
            else:
                phase_bragg = np.zeros([2, ny, s.Nx])
                bragg_scats = np.zeros([2, ny, s.Nx], dtype=complex)
            phase_bragg[0] = surf_phase - cap_phase
            phase_bragg[1] = surf_phase + cap_phase
            bragg_scats[0] = scats[0][rows]
            bragg_scats[1] = scats[1][rows]
            if self.do_hh:
                scene_hh += np.sum(scat_bragg_hh * np.exp(1j * phase_bragg) * bragg_scats, axis=0)
            if self.do_vv:
                scene_vv += np.sum(scat_bragg_vv * np.exp(1j * phase_bragg) * bragg_scats, axis=0)
        beam_pattern = (sinc_bp(sin_az, self.ant_l_tx, self.f0, field=True) *
                        sinc_bp(sin_az, self.ant_l_rx, self.f0, field=True))
        if record is not None:
            record.update(sr_surface=sr_surface, sin_az=sin_az, az=az, beam_pattern=beam_pattern)
            if self.do_vv:
                record['scene_vv'] = scene_vv.copy()
            if self.do_hh:
                record['scene_hh'] = scene_hh.copy()
        profiles = {}
        for ch in np.arange(self.num_ch, dtype=int):
            tot_dinc = (self.inc - self.inc_angle) + wave_dinc
            for do, pol, scene, raw in ((self.do_hh, 'hh', scene_hh if self.do_hh else None,
                                         self.proc_raw_hh if self.do_hh else None),
                                        (self.do_vv, 'vv', scene_vv if self.do_vv else None,
                                         self.proc_raw_vv if self.do_vv else None)):
                if not do:
                    continue
                scene_bp = scene * beam_pattern
                scene_bp *= np.exp(-1j * self.k0 * self.b_ati[ch] * sin_az)
                scene_bp *= np.exp(-1j * self.k0 * self.b_xti[ch] * tot_dinc)
                out = raw[ch][az_step] if whole else np.zeros(self.rg_samp, dtype=complex)
                rp.chan_profile(sr_surface.flatten(), scene_bp.flatten(), self.sr_res / self.over_fs,
                                self.min_sr, self.chan_sinc_vec, self.n_sinc_samples, self.sinc_ovs, out)
                if not whole:
                    profiles[(pol, int(ch))] = out
        return spec_sum, bragg_sums, profiles

    def run(self, steps=None, record_steps=()):
        recs = {}
        steps = range(self.az_steps) if steps is None else steps
        for a in steps:
            rec = {} if a in record_steps else None
            self.pulse(a, rec)
            if rec is not None:
                recs[a] = rec
        return recs

    def finish(self, add_noise=True):
        """Truncation, calibration and noise (``sar_raw_nompi.py:552-600``)."""
        t_span, v = self.t_span, self.v_ground
        az_axis = np.arange(-t_span / 2. * v, t_span / 2. * v,
                            self.sr0 * C_LIGHT / (np.pi * self.f0 * self.ant_l_tx * 10.))
        pattern = (sinc_bp(az_axis / self.sr0, self.ant_l_tx, self.f0, field=True) *
                   sinc_bp(az_axis / self.sr0, self.ant_l_rx, self.f0, field=True))
        cal_factor = (1. / np.sqrt(np.trapezoid(np.abs(pattern) ** 2., az_axis) *
                                   self.sr_res / np.sin(self.inc_angle)))
        out = []
        for do, raw in ((self.do_hh, getattr(self, 'proc_raw_hh', None)),
                        (self.do_vv, getattr(self, 'proc_raw_vv', None))):
            if not do:
                continue
            raw = raw[:, :, :self.rg_samp_orig]
            if add_noise:
                noise = (geo.db2lin(self.nesz, amplitude=True) / np.sqrt(2.) *
                         (np.random.normal(size=raw.shape) + 1j * np.random.normal(size=raw.shape)))
            else:
                noise = 0.
            out.append(raw * cal_factor + noise)
        nrcs_avg = []
        if self.do_hh:
            nrcs_avg.append(self.NRCS_avg_hh)
        if self.do_vv:
            nrcs_avg.append(self.NRCS_avg_vv)
        self.cal_factor = cal_factor
        return np.stack(out), np.stack(nrcs_avg)


def sar_raw(cfg_file, seed=0, overrides=None, add_noise=True, surface_dt=None):
    """Whole run: returns (raw[pol, ch, az, rg], NRCS_avg[pol, az], sim)."""
    sim = SarRawSim(cfg_file, overrides=overrides, seed=seed, surface_dt=surface_dt)
    sim.run()
    raw, nrcs_avg = sim.finish(add_noise=add_noise)
    return raw, nrcs_avg, sim
