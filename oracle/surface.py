"""Oracle (test infrastructure only): linear-wave ocean surface.

Restates ``oceansar/surfaces/ocean.py``:

* ``OceanSurface.init``  -- ``:29-242`` (grid, k-space polar quantities, dispersion,
  directional spectrum, rms slopes, global-RNG complex Gaussian coefficients, optional
  directional and monochromatic swell; the numpy dtype flow is kept so that the float32
  results match the reference bit for bit)
* ``OceanSurface.set_t``  -- the ``t`` setter ``:418-526`` (propagation and one numpy
  ``ifft2`` per field, complex64 throughout)

``precision='f64'`` evaluates the same fields from complex128 coefficients with complex128
FFTs (the FP64 restatement the FP64 surface kernel is checked against).
"""
import numpy as np
from scipy import linalg

from . import spectra
from .geometry import optimize_fftsize

G = 9.80665


class OceanSurface:
    def __init__(self):
        self.initialized = False

    def init(self, Lx, Ly, dx, dy, cutoff_wl, spec_model, spread_model, wind_dir, wind_fetch,
             wind_U, current_mag, current_dir, dir_swell_dir=0, freq_r=100, sigf=1, sigs=1, Hs=2,
             swell_dir_enable=False, swell_enable=False, swell_ampl=0., swell_dir=0.,
             swell_wl=0., compute=[], opt_res=True, fft_max_prime=2, choppy_enable=False,
             dirspectrum_func=None, depth=None, dir_swell_spec=None):
        self.Lx, self.Ly, self.dx, self.dy = Lx, Ly, dx, dy
        self.wind_dir, self.wind_fetch, self.wind_U = wind_dir, wind_fetch, wind_U
        self.current_mag, self.current_dir = current_mag, current_dir
        self.swell_enable, self.swell_ampl, self.swell_dir, self.swell_wl = (
            swell_enable, swell_ampl, swell_dir, swell_wl)
        self.compute = list(compute)
        self.choppy_enable = choppy_enable
        self.Nx = int(self.Lx / self.dx)
        self.Ny = int(self.Ly / self.dy)
        if opt_res:
            self.Nx = int(optimize_fftsize(self.Nx, fft_max_prime))
            self.Ny = int(optimize_fftsize(self.Ny, fft_max_prime))
            self.dx = np.float32(self.Lx / float(self.Nx))
            self.dy = np.float32(self.Ly / float(self.Ny))
        self.x = np.linspace(-self.Lx / 2., self.Lx / 2., self.Nx, dtype=np.float32)
        self.y = np.linspace(-self.Ly / 2., self.Ly / 2., self.Ny, dtype=np.float32)
        self.current = (self.current_mag * np.array([np.cos(self.current_dir),
                                                     np.sin(self.current_dir)])).astype(np.float32)
        U_eff_vec = (self.wind_U * np.array([np.cos(self.wind_dir), np.sin(self.wind_dir)]) -
                     self.current).astype(np.float32)
        self.wind_U_eff = linalg.norm(U_eff_vec)
        self.wind_dir_eff = np.arctan2(U_eff_vec[1], U_eff_vec[0])
        kmax_x = np.float32(np.pi / self.dx)
        kmax_y = np.float32(np.pi / self.dy)
        kx_s = (2 * np.pi * np.fft.fftfreq(self.Nx, self.dx)).astype(np.float32)
        ky_s = (2 * np.pi * np.fft.fftfreq(self.Ny, self.dy)).astype(np.float32)
        self.kx, self.ky = np.meshgrid(kx_s, ky_s)
        self.kx_res = kx_res = self.kx[0, 1] - self.kx[0, 0]
        self.ky_res = ky_res = self.ky[1, 0] - self.ky[0, 0]
        self.k = np.sqrt(self.kx ** 2 + self.ky ** 2)
        good_k = np.where(self.k > np.min(np.array([kx_res, ky_res])) / 2.0)
        self.kxn = np.zeros_like(self.kx, dtype=np.float32)
        self.kyn = np.zeros_like(self.kx, dtype=np.float32)
        self.kxn[good_k] = self.kx[good_k] / self.k[good_k]
        self.kyn[good_k] = self.ky[good_k] / self.k[good_k]
        self.kinv = np.zeros(self.k.shape, dtype=np.float32)
        self.kinv[good_k] = 1. / self.k[good_k]
        self.theta = np.angle(np.exp(1j * (np.arctan2(self.ky, self.kx) -
                                           self.wind_dir_eff))).astype(np.float32)
        self.theta_swell = np.angle(np.exp(1j * (np.arctan2(self.ky, self.kx)))).astype(np.float32)
        if depth is None:
            self.omega = np.sqrt(np.float32(G) * self.k)
        else:
            self.omega = np.sqrt(np.float32(G) * self.k * np.tanh(self.k * np.float32(depth)))
        if callable(dirspectrum_func):
            self.wave_dirspec = np.zeros(self.k.shape, dtype=np.float32)
            self.wave_dirspec[good_k] = dirspectrum_func(self.kx[good_k], self.ky[good_k])
        else:
            if spec_model not in spectra.SPEC_MODELS:
                raise NotImplementedError('%s spectrum function not implemented' % spec_model)
            if spread_model not in spectra.SPREAD_MODELS:
                raise NotImplementedError('%s spreading function not implemented' % spread_model)
            wave_spec = np.zeros(self.k.shape, dtype=np.float32)
            wave_spec[good_k] = spectra.SPEC_MODELS[spec_model](self.k[good_k], self.wind_U_eff,
                                                                self.wind_fetch)
            wave_spread = np.zeros(self.k.shape, dtype=np.float32)
            sfun = spectra.SPREAD_MODELS[spread_model]
            if spread_model == 'elfouhaily':
                # numba-compiled in the reference: every operand promoted to float64
                wave_spread[good_k] = sfun(self.k[good_k].astype(np.float64),
                                           self.theta[good_k].astype(np.float64),
                                           float(self.wind_U_eff), float(self.wind_fetch))
            else:
                wave_spread[good_k] = sfun(self.k[good_k], self.theta[good_k], self.wind_U_eff,
                                           self.wind_fetch)
            self.wave_dirspec = self.kinv * wave_spec * wave_spread
        self.rmss_x = np.sqrt(np.sum(self.wave_dirspec * self.kx ** 2 * self.kx_res * ky_res))
        self.rmss_y = np.sqrt(np.sum(self.wave_dirspec * self.ky ** 2 * self.kx_res * ky_res))
        if cutoff_wl and (cutoff_wl != 'auto'):
            raise NotImplementedError('numeric cutoff_wl (float slice indices in the reference)')
        random_cg = (1. / np.sqrt(2) * (np.random.normal(0., 1., size=[self.Ny, self.Nx]) +
                                        1j * np.random.normal(0., 1., size=[self.Ny, self.Nx]))
                     ).astype(np.complex64)
        if swell_dir_enable:
            swell_dirspec = np.zeros(self.k.shape, dtype=np.float32)
            swell_dirspec[good_k] = dir_swell_spec(self.k[good_k], self.theta_swell[good_k],
                                                   dir_swell_dir, freq_r, sigf, sigs, Hs)
            self.swell_dirspec = self.kinv * swell_dirspec
            random_swell = (1. / np.sqrt(2) * (np.random.normal(0., 1., size=[self.Ny, self.Nx]) +
                                               1j * np.random.normal(0., 1., size=[self.Ny, self.Nx]))
                            ).astype(np.complex64)
        if self.swell_enable:
            x, y = np.meshgrid(self.x, self.y)
            self.swell_k = np.float32(2. * np.pi / self.swell_wl)
            self.swell_kx = np.float32(self.swell_k * np.cos(self.swell_dir))
            self.swell_ky = np.float32(self.swell_k * np.sin(self.swell_dir))
            if depth is None:
                self.swell_omega = np.float32(np.sqrt(self.swell_k * G))
            else:
                self.swell_omega = np.float32(np.sqrt(self.swell_k * G * np.tanh(self.swell_k * depth)))
            self.swell_ph0 = np.float32(np.random.uniform(0., 2. * np.pi))
            self.swell_exp = (self.swell_ampl *
                              np.exp(1j * (self.swell_k * (np.cos(self.swell_dir) * x +
                                                           np.sin(self.swell_dir) * y) + self.swell_ph0))
                              ).astype(np.complex64)
        self.wave_coefs = (self.Nx * self.Ny * np.sqrt(2. * self.wave_dirspec * kx_res * ky_res) *
                           random_cg).astype(np.complex64)
        if swell_dir_enable:
            self.swell_coefs = (self.Nx * self.Ny * np.sqrt(2. * self.swell_dirspec * kx_res * ky_res) *
                                random_swell).astype(np.complex64)
            self.wave_coefs = self.wave_coefs + self.swell_coefs
        self.initialized = True
        return self

    # ------------------------------------------------------------------------------
    def set_t(self, value, precision='f32'):
        """Fields at time ``value`` as a dict (``ocean.py:418-526``)."""
        if not self.initialized:
            raise Exception('Surface not initialized')
        cdt = np.complex64 if precision == 'f32' else np.complex128
        rdt = np.float32 if precision == 'f32' else np.float64
        t = np.float32(value)
        self._t = t
        if precision == 'f32':
            wcp = (self.wave_coefs * np.exp(-1j * self.omega * t)).astype(np.complex64)
        else:
            om = self.omega.astype(np.float64)
            wcp = self.wave_coefs.astype(np.complex128) * np.exp(-1j * om * np.float64(t))
        kx, ky, kxn, kyn, kinv, om = self.kx, self.ky, self.kxn, self.kyn, self.kinv, self.omega
        if precision != 'f32':
            kx, ky, kxn, kyn, kinv, om = (a.astype(np.float64) for a in (kx, ky, kxn, kyn, kinv, om))
        # numpy's transform (as the reference); a threaded one only for the CPU baseline
        ifft2 = getattr(self, 'fft_ifft2', None) or np.fft.ifft2
        cur = self.current if precision == 'f32' else self.current.astype(np.float64)
        tt = t if precision == 'f32' else np.float64(t)
        if self.swell_enable:
            sw_ph = (self.swell_exp * np.exp(-1j * self.swell_omega * t)).astype(np.complex64)
            if precision != 'f32':
                sw_ph = sw_ph.astype(np.complex128)
            skx, sky, sk, som = self.swell_kx, self.swell_ky, self.swell_k, self.swell_omega
        out = {}
        comp = self.compute
        if 'D' in comp:
            out['Dx'] = (-np.imag(ifft2(kxn * wcp)) + cur[0] * tt).astype(rdt)
            out['Dy'] = (-np.imag(ifft2(kyn * wcp)) + cur[1] * tt).astype(rdt)
            out['Dz'] = np.real(ifft2(wcp)).astype(rdt)
            if self.swell_enable:
                out['Dx'] = (out['Dx'] + np.real(1j * skx / sk * sw_ph).astype(np.float32)).astype(rdt)
                out['Dy'] = (out['Dy'] + np.real(1j * sky / sk * sw_ph).astype(np.float32)).astype(rdt)
                out['Dz'] = (out['Dz'] + np.real(sw_ph).astype(np.float32)).astype(rdt)
        if 'Diff' in comp:
            if not self.choppy_enable:
                out['Diffx'] = np.real(ifft2(1j * kx * wcp)).astype(rdt)
                out['Diffy'] = np.real(ifft2(1j * ky * wcp)).astype(rdt)
            else:
                out['Diffx'] = (np.real(ifft2(1j * kx * wcp)) /
                                (1. + np.real(ifft2(-kx ** 2. * kinv * wcp)))).astype(rdt)
                out['Diffy'] = (np.real(ifft2(1j * ky * wcp)) /
                                (1. + np.real(ifft2(-ky ** 2. * kinv * wcp)))).astype(rdt)
            if self.swell_enable:
                out['Diffx'] = (out['Diffx'] + np.real(1j * skx * sw_ph)).astype(rdt)
                out['Diffy'] = (out['Diffy'] + np.real(1j * sky * sw_ph)).astype(rdt)
        if 'Diff2' in comp:
            if not self.choppy_enable:
                out['Diffxx'] = np.real(ifft2(-kx ** 2. * wcp)).astype(rdt)
                out['Diffyy'] = np.real(ifft2(-ky ** 2. * wcp)).astype(rdt)
                out['Diffxy'] = np.real(ifft2(-kx * ky * wcp)).astype(rdt)
            else:
                aux_x = np.real(ifft2(1j * kx * wcp))
                aux_y = np.real(ifft2(1j * ky * wcp))
                aux_xx = np.real(ifft2(-kx ** 2. * kinv * wcp))
                aux_yy = np.real(ifft2(-ky ** 2. * kinv * wcp))
                aux_xxx = np.real(ifft2(-1j * kx ** 3. * kinv * wcp))
                aux_yyy = np.real(ifft2(-1j * ky ** 3. * kinv * wcp))
                aux_xxy = np.real(ifft2(-1j * kx ** 2. * ky * kinv * wcp))
                out['Diffxx'] = (((1. + aux_xx) * np.real(ifft2(-kx ** 2. * wcp)) - aux_xxx * aux_x) /
                                 ((1 + aux_xx) ** 3.)).astype(rdt)
                out['Diffyy'] = (((1. + aux_yy) * np.real(ifft2(-ky ** 2. * wcp)) - aux_yyy * aux_y) /
                                 ((1 + aux_yy) ** 3.)).astype(rdt)
                out['Diffxy'] = (((1. + aux_xx) * np.real(ifft2(-kx * ky * wcp)) - aux_xxy * aux_x) /
                                 ((1 + aux_xx) ** 2. * (1 + aux_yy))).astype(rdt)
            if self.swell_enable:
                out['Diffxx'] = (out['Diffxx'] + np.real(-skx ** 2. * sw_ph)).astype(rdt)
                out['Diffyy'] = (out['Diffyy'] + np.real(-sky ** 2. * sw_ph)).astype(rdt)
                out['Diffxy'] = (out['Diffxy'] + np.real(-skx * sky * sw_ph)).astype(rdt)
        if 'V' in comp:
            wdt = -1j * om * wcp
            out['Vx'] = (-np.imag(ifft2(kxn * wdt)) + cur[0]).astype(rdt)
            out['Vy'] = (-np.imag(ifft2(kyn * wdt)) + cur[1]).astype(rdt)
            out['Vz'] = np.real(ifft2(wdt)).astype(rdt)
            if self.swell_enable:
                sdt = -1j * som * sw_ph
                out['Vx'] = (out['Vx'] + np.real(1j * skx / sk * sdt)).astype(rdt)
                out['Vy'] = (out['Vy'] + np.real(1j * sky / sk * sdt)).astype(rdt)
                out['Vz'] = (out['Vz'] + np.real(sdt)).astype(rdt)
        if 'A' in comp:
            wdt2 = -om ** 2. * wcp
            out['Ax'] = np.real(ifft2(1j * kx * kinv * wdt2)).astype(rdt)
            out['Ay'] = np.real(ifft2(1j * ky * kinv * wdt2)).astype(rdt)
            out['Az'] = np.real(ifft2(wdt2)).astype(rdt)
            if self.swell_enable:
                sdt2 = -som ** 2. * sw_ph
                out['Ax'] = (out['Ax'] + np.real(1j * skx / sk * sdt2)).astype(rdt)
                out['Ay'] = (out['Ay'] + np.real(1j * sky / sk * sdt2)).astype(rdt)
                out['Az'] = (out['Az'] + np.real(sdt2)).astype(rdt)
        if 'hMTF' in comp:
            k = self.k if precision == 'f32' else self.k.astype(np.float64)
            k_max = 2. * np.pi / 20.
            mu = 0.04 / 16.
            dlnS_dlnk = -3.
            Vg_c = 0.5
            M_h = 1j * k * om * (om + 1j * mu) / (om ** 2. + mu ** 2.) * (dlnS_dlnk - Vg_c)
            wh = M_h * wcp
            wh[np.where(k > k_max)] = 0.
            out['hMTF'] = np.real(ifft2(wh)).astype(rdt)
        for name, arr in out.items():
            setattr(self, name, arr)
        return out
