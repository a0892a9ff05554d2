"""NRCS models (``oceansar/nrcs``) evaluated on the GPU.

* ``RCSRomeiser97`` -- Bragg scattering (``nrcs/romeiser97.py:38-393``).  The constructor
  builds the reference's interpolation table of the omni-directional spectrum on the host
  (k = 1, 1.1, ... < 2 k0); ``rcs`` runs the float64 sm_100a kernel behind
  ``ocs_rcs_romeiser``.  Inside ``sar_raw`` the same device function runs fused in the
  per-pulse kernel.  The LUT mode (``use_lut=True``, ``:71-92, 109-134``) is not built.
* ``RCSKodis`` -- stationary-phase specular field (``nrcs/kodis.py:27-73``) behind
  ``ocs_field_kodis``.
"""
import ctypes

import numpy as np

from .. import _capi, _device, spec, spread
from .._structs import KodisDesc, RcsDesc

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
        if use_lut:
            raise NotImplementedError('RCSRomeiser97 LUT mode (use_lut=True) is not built; '
                                      'use use_lut=False (direct evaluation)')
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
            return out_hh.cpu().numpy(), out_vv.cpu().numpy()
        return (out_hh if want_hh else out_vv).cpu().numpy()

    rcs_numba = rcs


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


models = {'kodis': RCSKodis, 'romeiser97': RCSRomeiser97}
