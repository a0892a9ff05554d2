"""NRCS models (``oceansar/nrcs``) evaluated on the GPU.

* ``RCSRomeiser97`` -- Bragg scattering (``nrcs/romeiser97.py:38-393``).  The constructor
  builds the reference's interpolation table of the omni-directional spectrum on the host
  (k = 1, 1.1, ... < 2 k0); ``rcs`` runs the float64 sm_100a kernel behind
  ``ocs_rcs_romeiser``.  Inside ``sar_raw`` the same device function runs fused in the
  per-pulse kernel.  The LUT mode (``use_lut=True``, ``:71-92, 109-134``) tabulates the
  model over (azimuth, slope_y, slope_x) at the mean incidence with the same device
  function, on first use; lookups round half to even and clamp the slopes as the reference
  does (on the host for ``rcs``, inside the pulse kernel for ``sar_raw``).
* ``RCSKodis`` -- stationary-phase specular field (``nrcs/kodis.py:27-73``) behind
  ``ocs_field_kodis``.
* ``RCSKA`` -- Kirchhoff-approximation specular field (``nrcs/ka.py:41-310``), facet
  approach ('fa') or stationary phase ('spa'), monostatic, behind ``ocs_field_ka``.
"""
import ctypes

import numpy as np

from .. import _capi, _device, spec, spread
from .._structs import KaDesc, KodisDesc, RcsDesc

EPS_SW = 73 + 18j
POL_CODES = {'vv': 0, 'hh': 1, 'DP': 2}


def _broadcast_strides(arr, ny, nx):
    """Device float64 copy of ``arr`` and its (row, col) strides over a [ny, nx] grid."""
    a = np.asarray(arr, dtype=np.float64)
    if a.ndim == 0:
        return _device.to_device(a.reshape(1), np.float64), 0, 0
    if a.ndim == 1:
        a = a.reshape(1, -1)
    if a.shape == (ny, nx):
        return _device.to_device(a, np.float64), nx, 1
    if a.shape == (ny, 1):
        return _device.to_device(a.ravel(), np.float64), 1, 0
    if a.shape == (1, nx):
        return _device.to_device(a.ravel(), np.float64), 0, 1
    raise ValueError('angle array of shape %s does not broadcast to (%d, %d)' % (a.shape, ny, nx))


class RCSRomeiser97(object):
    def __init__(self, k0, inc_angle, pol, dx, dy, wind_U, wind_dir, wind_fetch, sw_spec_func,
                 sw_spread_func, d, numba=True, rmss_x=0.1, rmss_y=0.1, az_span=np.radians(1),
                 use_lut=True):
        if pol not in POL_CODES:
            raise ValueError('pol must be vv, hh or DP')
        if (sw_spread_func == 'none') and (sw_spec_func == 'elfouhaily'):
            raise Exception('Elfouhaily spectrum requires a direction function')
        if sw_spec_func not in spec.models:
            raise NotImplementedError('%s spectrum function not implemented' % sw_spec_func)
        if sw_spread_func not in spread.DEVICE_CODES:
            raise NotImplementedError('%s spreading function not implemented on the GPU' % sw_spread_func)
        self.wind_U, self.wind_dir, self.wind_fetch = wind_U, wind_dir, wind_fetch
        self.dx, self.dy, self.pol, self.k0 = dx, dy, pol, k0
        self.inc_angle, self.d = inc_angle, d
        self.sw_spec_func, self.sw_dir_func = sw_spec_func, sw_spread_func
        self.numba = numba
        self.use_lut = False
        k = np.arange(1, 2 * k0, 0.1)
        self.interp_k = k
        self.interp_S = np.asarray(spec.models[sw_spec_func](k, self.wind_U, self.wind_fetch), dtype=np.float64)
        self.spread_code = spread.DEVICE_CODES[sw_spread_func]
        self.spread_consts = spread.elfouhaily_delta_coeffs(self.wind_U, self.wind_fetch)
        self._tab = None
        self._lut_dev = {}
        self._lut_rcs = None
        if use_lut:
            self._lut_grid(rmss_x, rmss_y, az_span)
            self.use_lut = True

    # ---- LUT mode (romeiser97.py:71-92) --------------------------------------------------
    def _lut_grid(self, rmss_x, rmss_y, az_span):
        """Table axes: slopes in steps of 0.0025 over +-5 rms slopes (rms floored at 0.01),
        azimuth in steps of 0.05 deg over az_span plus one step either side."""
        step, nsig = 0.0025, 5
        # np.max over a list: float32 rms slopes are promoted to float64 (as the reference's)
        sx, sy = np.max([rmss_x, 0.01]), np.max([rmss_y, 0.01])
        nx = int(sx * nsig * 2 / step)
        ny = int(sy * nsig * 2 / step)
        self.lut_Diffx = (-nsig * sx + np.arange(nx) * step)[np.newaxis, np.newaxis, :]
        self.lut_Diffy = (-nsig * sy + np.arange(ny) * step)[np.newaxis, :, np.newaxis]
        az_step = np.radians(0.05)
        naz_in = int(az_span / az_step)
        self.lut_az = (-az_span / 2 + np.arange(-1, naz_in + 2) * az_step)[:, np.newaxis, np.newaxis]
        self._lut_shape = (naz_in + 3, ny, nx)

    def lut_params(self):
        """(naz, ndy, ndx, az0, daz, dy0, ddy, dx0, ddx) of the table, float64 as numpy forms them."""
        naz, ndy, ndx = self._lut_shape
        return (naz, ndy, ndx, float(self.lut_az.min()), float(self.lut_az[1, 0, 0] - self.lut_az[0, 0, 0]),
                float(self.lut_Diffy[0, 0, 0]), float(self.lut_Diffy[0, 1, 0] - self.lut_Diffy[0, 0, 0]),
                float(self.lut_Diffx[0, 0, 0]), float(self.lut_Diffx[0, 0, 1] - self.lut_Diffx[0, 0, 0]))

    def _lut_device64(self):
        """The table on the device, float64 [npol][2][naz][ndy][ndx] (pol order: the
        model's outputs, hh then vv for 'DP'), evaluated by the direct model at the mean
        incidence (romeiser97.py:83-91)."""
        if 'f64' not in self._lut_dev:
            naz, ndy, ndx = self._lut_shape
            az = np.repeat(self.lut_az.ravel(), ndy).reshape(naz * ndy, 1)
            dx = np.broadcast_to(self.lut_Diffx.reshape(1, ndx), (naz * ndy, ndx))
            dy = np.broadcast_to(np.tile(self.lut_Diffy.ravel(), naz).reshape(naz * ndy, 1), (naz * ndy, ndx))
            inc_keep = self.inc_angle
            self.inc_angle = np.float64(np.mean(inc_keep))
            try:
                outs = self._rcs_direct_device(az, dx, dy)
            finally:
                self.inc_angle = inc_keep
            import torch
            self._lut_dev['f64'] = torch.stack([o.reshape(2, naz, ndy, ndx) for o in outs]).contiguous()
        return self._lut_dev['f64']

    def lut_device(self, precision):
        """Device table in the pulse kernel's real type (float64 'f64', float32 'mixed')."""
        t = self._lut_device64()
        if precision == 'f64':
            return t
        if 'f32' not in self._lut_dev:
            import torch
            self._lut_dev['f32'] = t.to(torch.float32).contiguous()
        return self._lut_dev['f32']

    @property
    def lut_rcs(self):
        """The table as the reference holds it: [2][naz][ndy][ndx] or an (hh, vv) pair."""
        if self._lut_rcs is None:
            t = self._lut_device64().cpu().numpy()
            self._lut_rcs = (t[0], t[1]) if self.pol == 'DP' else t[0]
        return self._lut_rcs

    def rcs_lut(self, az_angle, diffx, diffy):
        """Table lookup (romeiser97.py:109-134)."""
        az_ind = (np.round((az_angle - self.lut_az.min()) /
                           (self.lut_az[1, 0, 0] - self.lut_az[0, 0, 0]))).astype(int)
        dy = (np.round((diffy - self.lut_Diffy[0, 0, 0]) /
                       (self.lut_Diffy[0, 1, 0] - self.lut_Diffy[0, 0, 0]))).astype(int)
        dx = (np.round((diffx - self.lut_Diffx[0, 0, 0]) /
                       (self.lut_Diffx[0, 0, 1] - self.lut_Diffx[0, 0, 0]))).astype(int)
        dy = np.where(dy > 0, dy, 0)
        dx = np.where(dx > 0, dx, 0)
        dy = np.where(dy < self.lut_Diffy.shape[1], dy, self.lut_Diffy.shape[1] - 1)
        dx = np.where(dx < self.lut_Diffx.shape[2], dx, self.lut_Diffx.shape[2] - 1)
        lut = self.lut_rcs
        if self.pol == 'DP':
            return (np.stack([lut[0][0][az_ind, dy, dx], lut[0][1][az_ind, dy, dx]]),
                    np.stack([lut[1][0][az_ind, dy, dx], lut[1][1][az_ind, dy, dx]]))
        return lut[:, az_ind, dy, dx]

    def device_tables(self):
        if self._tab is None:
            self._tab = (_device.to_device(self.interp_k, np.float64),
                         _device.to_device(self.interp_S, np.float64))
        return self._tab

    def fill(self, desc):
        """Write the model constants into a pulse / RCS descriptor."""
        tk, ts = self.device_tables()
        desc.k0 = float(self.k0)
        desc.wind_dir = float(self.wind_dir)
        desc.wind_U = float(self.wind_U)
        desc.spread = int(self.spread_code)
        (desc.spread_ck_p, desc.spread_ck_m, desc.spread_a0, desc.spread_ap,
         desc.spread_am) = [float(v) for v in self.spread_consts]
        desc.spec_k_d, desc.spec_s_d, desc.spec_n = tk.data_ptr(), ts.data_ptr(), int(tk.numel())
        se = np.sqrt(EPS_SW)
        desc.sqrt_eps_re, desc.sqrt_eps_im = float(se.real), float(se.imag)

    def rcs(self, az_angle, diffx, diffy):
        """RCS of both Bragg lines, float64 [2, Ny, Nx]; a (hh, vv) pair for 'DP'."""
        if self.use_lut:
            return self.rcs_lut(az_angle, diffx, diffy)
        outs = self._rcs_direct_device(az_angle, diffx, diffy)
        if self.pol == 'DP':
            return outs[0].cpu().numpy(), outs[1].cpu().numpy()
        return outs[0].cpu().numpy()

    def _rcs_direct_device(self, az_angle, diffx, diffy):
        """Direct model on the device: list of float64 [2, Ny, Nx] tensors (hh, vv for 'DP')."""
        diffx = np.asarray(diffx)
        ny, nx = diffx.shape
        dxd = _device.to_device(diffx, np.float64)
        dyd = _device.to_device(diffy, np.float64)
        azd, ars, acs = _broadcast_strides(az_angle, ny, nx)
        incd, irs, ics = _broadcast_strides(self.inc_angle, ny, nx)
        want_hh = self.pol in ('hh', 'DP')
        want_vv = self.pol in ('vv', 'DP')
        out_hh = _device.empty((2, ny, nx), np.float64) if want_hh else None
        out_vv = _device.empty((2, ny, nx), np.float64) if want_vv else None
        desc = RcsDesc()
        desc.nx, desc.ny = nx, ny
        desc.az_d, desc.az_row_stride, desc.az_col_stride = azd.data_ptr(), ars, acs
        desc.inc_d, desc.inc_row_stride, desc.inc_col_stride = incd.data_ptr(), irs, ics
        desc.diffx_d, desc.diffy_d = dxd.data_ptr(), dyd.data_ptr()
        self.fill(desc)
        desc.d, desc.dx, desc.dy = float(self.d), float(self.dx), float(self.dy)
        desc.pol = POL_CODES[self.pol]
        desc.out_hh_d = out_hh.data_ptr() if want_hh else None
        desc.out_vv_d = out_vv.data_ptr() if want_vv else None
        _capi.call("ocs_rcs_romeiser", ctypes.addressof(desc), _device.stream_ptr())
        if self.pol == 'DP':
            return [out_hh, out_vv]
        return [out_hh if want_hh else out_vv]

    def rcs_numba(self, az_angle, diffx, diffy):
        """The direct model (romeiser97.py:252-393), whatever the LUT setting."""
        outs = self._rcs_direct_device(az_angle, diffx, diffy)
        if self.pol == 'DP':
            return outs[0].cpu().numpy(), outs[1].cpu().numpy()
        return outs[0].cpu().numpy()


class RCSKodis(object):
    def __init__(self, inc, k0, dx, dy):
        self.dx, self.dy, self.k0 = dx, dy, k0
        self.inc = np.asarray(inc, dtype=np.float64)
        self.sin_inc = np.sin(self.inc)
        self.cos_inc = np.cos(self.inc)
        self.tan_inc = np.tan(self.inc)
        self.R = (EPS_SW - np.sqrt(EPS_SW)) / (EPS_SW + np.sqrt(EPS_SW))
        self._dev = None

    def device_columns(self):
        """float64 [nx] sin / cos / tan of the incidence angle on the device."""
        if self._dev is None:
            self._dev = tuple(_device.to_device(np.ravel(a), np.float64)
                              for a in (self.sin_inc, self.cos_inc, self.tan_inc))
        return self._dev

    def field(self, az_angle, sr, diffx, diffy, diffxx, diffyy, diffxy):
        sr = np.asarray(sr, dtype=np.float64)
        ny, nx = sr.shape
        if np.size(self.inc) not in (1, nx):
            raise ValueError('incidence must be a scalar or a [1, Nx] row')
        si, ci, ti = self.device_columns()
        if si.numel() == 1:
            si, ci, ti = (t.expand(nx).contiguous() for t in (si, ci, ti))
        azd, ars, acs = _broadcast_strides(az_angle, ny, nx)
        out = _device.empty((ny, nx), np.complex128)
        f = [_device.to_device(a, np.float32) for a in (diffx, diffy, diffxx, diffyy, diffxy)]
        srd = _device.to_device(sr, np.float64)
        desc = KodisDesc(nx, ny, azd.data_ptr(), ars, acs, si.data_ptr(), ci.data_ptr(), ti.data_ptr(),
                         srd.data_ptr(), *[t.data_ptr() for t in f], float(self.k0), float(self.R.real),
                         float(self.R.imag), float(self.dx), float(self.dy),
                         out.data_ptr())
        _capi.call("ocs_field_kodis", ctypes.addressof(desc), _device.stream_ptr())
        return out.cpu().numpy()




class RCSKA(object):
    """Kirchhoff approximation (``nrcs/ka.py:41-310``), mode 'fa' or 'spa'."""

    def __init__(self, mode, k0, x, y, dx, dy):
        if mode not in ('fa', 'spa'):
            raise ValueError('mode must be fa or spa')
        self.mode, self.k0, self.dx, self.dy = mode, k0, dx, dy
        self.x = np.asarray(x, dtype=np.float64)
        self.y = np.asarray(y, dtype=np.float64)
        self.shape = [self.y.shape[0], self.x.shape[0], 3]
        self._xy = None

    def constant(self, R_i=1, R_s=1):
        """K = -1j k0 exp(-1j k0 (R_i + R_s)) / ((4 pi)^2 R_i R_s), as numpy evaluates it."""
        return complex(-1j * self.k0 * np.exp(-1j * self.k0 * (R_i + R_s)) / ((4. * np.pi) ** 2. * R_i * R_s))

    def device_positions(self):
        if self._xy is None:
            self._xy = (_device.to_device(self.x, np.float64), _device.to_device(self.y, np.float64))
        return self._xy

    def field(self, R_i, R_s, pol_i, pol_s, theta_i, theta_s, phi_i, phi_s, Dz, Diffx, Diffy, Diffxx, Diffyy,
              Diffxy, monostatic=True):
        if not monostatic:
            raise NotImplementedError('bistatic Kirchhoff geometry is not built')
        ny, nx = np.shape(Dz)
        xd, yd = self.device_positions()
        th = np.asarray(theta_i, dtype=np.float64).reshape(1, -1)
        thd, trs, tcs = _broadcast_strides(th if th.size > 1 else th.reshape(()), ny, nx)
        phd, prs, pcs = _broadcast_strides(phi_i, ny, nx)
        f = [_device.to_device(a, np.float32) for a in (Dz, Diffx, Diffy, Diffxx, Diffyy, Diffxy)]
        out = _device.empty((ny, nx), np.complex128)
        K = self.constant(R_i, R_s)
        desc = KaDesc(nx, ny, xd.data_ptr(), yd.data_ptr(), thd.data_ptr(), trs, tcs, phd.data_ptr(), prs, pcs,
                      *[t.data_ptr() for t in f], float(self.k0), float(self.dx), float(self.dy), K.real, K.imag,
                      0 if self.mode == 'fa' else 1, 0 if pol_i == 'h' else 1, 0 if pol_s == 'h' else 1,
                      out.data_ptr())
        _capi.call("ocs_field_ka", ctypes.addressof(desc), _device.stream_ptr())
        return out.cpu().numpy()

    def rcs(self, pol_i, pol_s, theta_i, theta_s, phi_i, phi_s, Dz, Diffx, Diffy, Diffxx, Diffyy, Diffxy):
        return (4. * np.pi) ** 2. * np.abs(self.field(1, 1, pol_i, pol_s, theta_i, theta_s, phi_i, phi_s, Dz, Diffx,
                                                     Diffy, Diffxx, Diffyy, Diffxy)) ** 2.


models = {'ka': RCSKA, 'kodis': RCSKodis, 'romeiser97': RCSRomeiser97}
