"""Oracle (test infrastructure only): NRCS models.

* ``RCSRomeiser97`` -- ``oceansar/nrcs/romeiser97.py:38-393``: constructor (``:38-92``,
  interpolation table of the omni-directional spectrum on k = 1, 1.1, ... < 2 k0), the
  numba kernel ``_rcs_numba`` (``:252-322``) evaluated in float64 numpy, and ``rcs_numba``
  (``:324-393``: folded spectrum, spreading, ``bad_ones`` mask; in DP mode line 0 of the
  hh RCS is deliberately *not* masked, ``:391-392``).  The LUT mode is not restated.
* ``RCSKodis`` -- ``oceansar/nrcs/kodis.py:27-73``.  ``field`` accepts an azimuth-angle
  array of any shape that broadcasts to the facet grid (the reference indexes it with
  the facet coordinates and so needs a full [Ny, Nx] array, ``:61-62``).
"""
import numpy as np
from scipy import interpolate

from . import spectra

EPS_SW = 73 + 18j


class RCSRomeiser97:
    def __init__(self, k0, inc_angle, pol, dx, dy, wind_U, wind_dir, wind_fetch,
                 sw_spec_func, sw_spread_func, d, numba=True, rmss_x=0.1, rmss_y=0.1,
                 az_span=np.radians(1), use_lut=False):
        self.wind_U, self.wind_dir, self.wind_fetch = wind_U, wind_dir, wind_fetch
        self.dx, self.dy, self.pol, self.k0 = dx, dy, pol, k0
        self.inc_angle, self.d = inc_angle, d
        self.sw_spec_func, self.sw_dir_func = sw_spec_func, sw_spread_func
        k = np.arange(1, 2 * k0, 0.1)
        spectrum = spectra.SPEC_MODELS[sw_spec_func](k, self.wind_U, self.wind_fetch)
        self.interp_k = k
        self.interp_S = spectrum
        self.spec_interpolator = interpolate.interp1d(k, spectrum, bounds_error=False, fill_value=1)
        self.use_lut = False
        if use_lut:
            self._build_lut(rmss_x, rmss_y, az_span)

    def _build_lut(self, rmss_x, rmss_y, az_span):
        """LUT over (azimuth, slope_y, slope_x) at the mean incidence (romeiser97.py:71-92):
        slope steps 0.0025 over +-5 rms slopes (rms floored at 0.01), azimuth steps 0.05 deg
        over az_span plus one step either side; every entry is the direct model."""
        step = 0.0025
        nsig = 5
        # np.max over a list: float32 rms slopes are promoted to float64 (as the reference's)
        sx, sy = np.max([rmss_x, 0.01]), np.max([rmss_y, 0.01])
        nx = int(sx * nsig * 2 / step)
        ny = int(sy * nsig * 2 / step)
        self.lut_Diffx = (-nsig * sx + np.arange(nx) * step)[np.newaxis, np.newaxis, :]
        self.lut_Diffy = (-nsig * sy + np.arange(ny) * step)[np.newaxis, :, np.newaxis]
        az_step = np.radians(0.05)
        naz_in = int(az_span / az_step)
        self.lut_az = (-az_span / 2 + np.arange(-1, naz_in + 2) * az_step)[:, np.newaxis, np.newaxis]
        shape = (naz_in + 3, ny, nx)
        inc_keep = self.inc_angle
        self.inc_angle = inc_keep.mean() + np.zeros_like(self.lut_Diffx)
        self.lut_rcs = self.rcs(self.lut_az + np.zeros(shape), self.lut_Diffx + np.zeros(shape),
                                self.lut_Diffy + np.zeros(shape))
        self.inc_angle = inc_keep
        self.use_lut = True

    def lut_indices(self, az_angle, diffx, diffy):
        """LUT indices of facets (romeiser97.py:109-123): round half to even, slopes clamped
        to the table, azimuth indices as numpy indexing takes them."""
        az_ind = np.round((az_angle - self.lut_az.min()) /
                          (self.lut_az[1, 0, 0] - self.lut_az[0, 0, 0])).astype(int)
        dy = np.round((diffy - self.lut_Diffy[0, 0, 0]) /
                      (self.lut_Diffy[0, 1, 0] - self.lut_Diffy[0, 0, 0])).astype(int)
        dx = np.round((diffx - self.lut_Diffx[0, 0, 0]) /
                      (self.lut_Diffx[0, 0, 1] - self.lut_Diffx[0, 0, 0])).astype(int)
        dy = np.clip(dy, 0, self.lut_Diffy.shape[1] - 1)
        dx = np.clip(dx, 0, self.lut_Diffx.shape[2] - 1)
        return az_ind, dy, dx

    def rcs_lut(self, az_angle, diffx, diffy):
        a, dy, dx = self.lut_indices(az_angle, diffx, diffy)
        if self.pol == 'DP':
            return (np.stack([self.lut_rcs[0][0][a, dy, dx], self.lut_rcs[0][1][a, dy, dx]]),
                    np.stack([self.lut_rcs[1][0][a, dy, dx], self.lut_rcs[1][1][a, dy, dx]]))
        return self.lut_rcs[:, a, dy, dx]

    @staticmethod
    def _kernel(inc_angle, az_angle, diffx, diffy, k0, pol, wind_dir, d):
        cos_az = np.cos(az_angle)
        sin_az = np.sin(az_angle)
        s_p = np.arctan(cos_az * diffx + sin_az * diffy)
        s_t = np.arctan(-sin_az * diffx + cos_az * diffy)
        cos_s_t = np.cos(s_t)
        cos_s_t_2 = cos_s_t ** 2
        sin_s_t_2 = 1 - cos_s_t_2
        sin_inc_anglep = np.sin(inc_angle - s_p)
        cos_inc_anglep = np.cos(inc_angle - s_p)
        cos_inc_anglep_2 = cos_inc_anglep ** 2
        sin_inc_anglep_2 = sin_inc_anglep ** 2
        cos_theta_i = cos_inc_anglep * cos_s_t
        sin_theta_i_2 = 1 - cos_theta_i ** 2
        b_hh = EPS_SW / (cos_theta_i + np.sqrt(EPS_SW)) ** 2.
        b_vv = ((EPS_SW ** 2.) * (1. + sin_theta_i_2)) / ((EPS_SW * cos_theta_i + np.sqrt(EPS_SW)) ** 2.)
        w = cos_inc_anglep / (np.cos(inc_angle) * np.cos(s_p))
        a = sin_s_t_2 / sin_theta_i_2
        b = sin_inc_anglep_2 * cos_s_t_2 / sin_theta_i_2
        F0 = 8 * np.pi * (k0 * cos_theta_i) ** 4
        T_vv = w * (F0 * np.abs(b * b_vv + a * b_hh) ** 2.)
        T_hh = w * (F0 * np.abs(b * b_hh + a * b_vv) ** 2.)
        k_b = 2 * k0 * np.sqrt(sin_inc_anglep_2 + (cos_inc_anglep_2 * sin_s_t_2))
        k_b = np.where(k_b > (2 * k0), 0, k_b)
        phi_b = az_angle + np.arctan((cos_inc_anglep * np.sin(-s_t)) / np.sin(inc_angle - s_p))
        theta_inp = np.empty((2,) + phi_b.shape)
        theta_inp[0] = phi_b - wind_dir
        theta_inp[1] = phi_b + np.pi - wind_dir
        theta_inp = np.angle(np.exp(1j * theta_inp))
        bad = 4 * sin_inc_anglep_2 < (d ** 2)
        return k_b, theta_inp, T_hh, T_vv, bad

    def rcs(self, az_angle, diffx, diffy):
        if self.use_lut:
            return self.rcs_lut(az_angle, diffx, diffy)
        diffx = np.asarray(diffx, dtype=np.float64)
        diffy = np.asarray(diffy, dtype=np.float64)
        az = np.broadcast_to(np.asarray(az_angle, dtype=np.float64), diffx.shape)
        inc = np.broadcast_to(np.asarray(self.inc_angle, dtype=np.float64), diffx.shape)
        with np.errstate(divide='ignore', invalid='ignore'):
            k_b, theta_inp, T_hh, T_vv, bad = self._kernel(inc, az, diffx, diffy, self.k0, self.pol,
                                                           self.wind_dir, self.d)
            k_inp = np.array([k_b, k_b])
            spectrum_1D = self.spec_interpolator(k_b.flatten()).reshape((1,) + k_b.shape)
            spectrum = (spectrum_1D / k_inp *
                        spectra.SPREAD_MODELS[self.sw_dir_func](k_inp, theta_inp, self.wind_U,
                                                                self.wind_fetch))
            rcs_vv = T_vv * spectrum * self.dx * self.dy
            rcs_hh = T_hh * spectrum * self.dx * self.dy
        if self.pol == 'vv':
            rcs_vv[:, bad] = 0
            return rcs_vv
        if self.pol == 'hh':
            rcs_hh[:, bad] = 0
            return rcs_hh
        rcs_vv[:, bad] = 0
        rcs_hh[1][bad] = 0
        return rcs_hh, rcs_vv


class RCSKodis:
    def __init__(self, inc, k0, dx, dy):
        self.dx, self.dy, self.k0 = dx, dy, k0
        self.sin_inc = np.sin(inc)
        self.cos_inc = np.cos(inc)
        self.tan_inc = np.tan(inc)
        self.R = (EPS_SW - np.sqrt(EPS_SW)) / (EPS_SW + np.sqrt(EPS_SW))

    def field(self, az_angle, sr, diffx, diffy, diffxx, diffyy, diffxy):
        shape = np.broadcast(sr, diffx).shape
        az = np.broadcast_to(np.asarray(az_angle), shape)
        cos_az = np.cos(az)
        sin_az = np.sin(az)
        with np.errstate(divide='ignore', invalid='ignore'):
            J = diffxx * diffyy - diffxy ** 2
            J = np.where(J == 0., np.nan, J)
            J_abs = np.abs(J)
            delta_x = (1. / J_abs) * (diffxy * (diffy - self.tan_inc * sin_az) -
                                      diffyy * (diffx - self.tan_inc * cos_az))
            delta_y = (1. / J_abs) * (diffxy * (diffx - self.tan_inc * cos_az) -
                                      diffxx * (diffy - self.tan_inc * sin_az))
            epsilon = np.where(J > 0., np.sign(diffxx), 1j)
        hdx = self.dx / 2
        hdy = self.dy / 2
        E = np.zeros(delta_x.shape, dtype=complex)
        sps = np.where(((-hdx < delta_x) & (delta_x < hdx)) & ((-hdy < delta_y) & (delta_y < hdy)))
        if sps[0].size > 0:
            delta_z = delta_x[sps] * diffx[sps] + delta_y[sps] * diffy[sps]
            sin_inc = np.broadcast_to(self.sin_inc, shape)
            cos_inc = np.broadcast_to(self.cos_inc, shape)
            sr_p2 = (sr[sps] + (sin_inc[sps] * cos_az[sps] * delta_x[sps] +
                                sin_inc[sps] * sin_az[sps] * delta_y[sps] -
                                cos_inc[sps] * delta_z))
            E[sps] = ((0.5 * self.R * epsilon[sps]) * ((diffx[sps] ** 2. + diffy[sps] ** 2. + 1.)) *
                      np.exp(-1j * 2. * self.k0 * sr_p2) / np.sqrt(J_abs[sps]))
        return E
