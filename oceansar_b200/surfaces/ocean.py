"""``OceanSurface`` with the reference's API (``oceansar/surfaces/ocean.py``), fields on the GPU.

* ``init`` (``ocean.py:29-242``) runs on the host once per scene, exactly as in the
  reference: wavenumber grid, dispersion relation, directional spectrum, global-numpy-RNG
  complex Gaussian coefficients, optional swell.  The numpy dtype flow is the reference's,
  so ``wave_coefs`` is bit-identical for the same seed.  The coefficients, the dispersion
  relation and the 1-D wavenumber axes are then uploaded once.
* Setting ``t`` (``ocean.py:418-526``) launches the sm_100a surface kernels
  (``ocs_surface_update``): phase evolution fused into a packed 2-D inverse FFT that
  writes the requested float32 fields into device buffers.  Reading an attribute such
  as ``surface.Dz`` returns a host numpy copy (the reference's type); ``field(name)``
  returns the device tensor without copying.
* ``save`` / ``load`` (``ocean.py:244-373``) write / read the state-file variables as a
  netCDF classic ``OceanStateFile`` (or a ``.npz`` container for names ending in ``.npz``).
"""
import ctypes

import numpy as np
import torch
from scipy import linalg

from .. import _capi, _device, spec, spread
from ..ocs_io import netcdf3
from ..ocs_io.state import OceanStateFile

G = 9.80665

# field name -> C ABI code (include/oceansar_b200.h)
CODES = {'Dz': 0, 'Dx': 1, 'Dy': 2, 'Diffx': 3, 'Diffy': 4, 'Diffxx': 5, 'Diffyy': 6, 'Diffxy': 7,
         'Vx': 8, 'Vy': 9, 'Vz': 10, 'Ax': 11, 'Ay': 12, 'Az': 13, 'hMTF': 14,
         'aux_xx': 15, 'aux_yy': 16, 'aux_xxx': 17, 'aux_yyy': 18, 'aux_xxy': 19}
GROUPS = {'D': ['Dx', 'Dy', 'Dz'], 'Diff': ['Diffx', 'Diffy'], 'Diff2': ['Diffxx', 'Diffyy', 'Diffxy'],
          'V': ['Vx', 'Vy', 'Vz'], 'A': ['Ax', 'Ay', 'Az'], 'hMTF': ['hMTF']}
FIELD_NAMES = [f for g in ('D', 'Diff', 'Diff2', 'V', 'A', 'hMTF') for f in GROUPS[g]]


class _Vars(dict):
    """Variables of a state file, with the ``files`` listing of an ``.npz`` archive."""
    @property
    def files(self):
        return list(self.keys())


class SurfaceDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("coefs_d", ctypes.c_void_p), ("omega_d", ctypes.c_void_p),
                ("kx_d", ctypes.c_void_p), ("ky_d", ctypes.c_void_p),
                ("kmin_half", ctypes.c_float), ("nfields", ctypes.c_int32),
                ("codes", ctypes.POINTER(ctypes.c_int32)), ("dst_d", ctypes.POINTER(ctypes.c_void_p)),
                ("add", ctypes.POINTER(ctypes.c_float)), ("swell_mult", ctypes.POINTER(ctypes.c_float)),
                ("swell_exp_d", ctypes.c_void_p), ("swell_rot_re", ctypes.c_float),
                ("swell_rot_im", ctypes.c_float), ("workspace_d", ctypes.c_void_p)]


class ChoppyDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64)] + \
        [(n, ctypes.c_void_p) for n in ("ax_d", "ay_d", "axx_d", "ayy_d", "axxx_d", "ayyy_d", "axxy_d",
                                       "fxx_d", "fyy_d", "fxy_d", "diffx_d", "diffy_d", "diffxx_d",
                                       "diffyy_d", "diffxy_d", "swell_exp_d")] + \
        [("swell_rot_re", ctypes.c_float), ("swell_rot_im", ctypes.c_float),
         ("swell_mult", ctypes.POINTER(ctypes.c_float))]


def optimize_fftsize(value, max_prime=2):
    """``oceansar/utils/misc.py:60-83`` for a scalar: next power of two, or the next
    integer whose largest prime factor is <= max_prime."""
    value = int(value)
    if max_prime == 2:
        return int(2 ** np.ceil(np.log2(value)))
    b = value
    while _largest_prime(b) > max_prime:
        b += 1
    return b


def _largest_prime(n):
    best, p = 1, 2
    while p * p <= n:
        while n % p == 0:
            best, n = p, n // p
        p += 1 if p == 2 else 2
    return max(best, n) if n > 1 else best


class OceanSurface(object):
    """Ocean surface simulator; see the module docstring."""

    def __init__(self):
        self.initialized = False
        self._fields = {}
        self._host_cache = {}

    # ------------------------------------------------------------------------------
    def init(self, Lx, Ly, dx, dy, cutoff_wl, spec_model, spread_model, wind_dir, wind_fetch,
             wind_U, current_mag, current_dir, dir_swell_dir=0, freq_r=100, sigf=1, sigs=1, Hs=2,
             swell_dir_enable=False, swell_enable=False, swell_ampl=0., swell_dir=0., swell_wl=0.,
             compute=[], opt_res=True, fft_max_prime=2, choppy_enable=False, dirspectrum_func=None,
             depth=None, dir_swell_spec=None, device=True):
        """``device=False`` stops after the host-side spectrum (no GPU touched); ``to_device()``
        uploads it later (a scene prepared in another process)."""
        self.Lx, self.Ly, self.dx, self.dy = Lx, Ly, dx, dy
        self.wind_dir, self.wind_fetch, self.wind_U = wind_dir, wind_fetch, wind_U
        self.current_mag, self.current_dir = current_mag, current_dir
        self.swell_enable, self.swell_ampl, self.swell_dir, self.swell_wl = (
            swell_enable, swell_ampl, swell_dir, swell_wl)
        self.compute = list(compute)
        self.choppy_enable = choppy_enable
        self.dir_swell_dir, self.freq_r, self.sigf, self.sigs, self.Hs = dir_swell_dir, freq_r, sigf, sigs, Hs
        self.depth = depth

        self.Nx = int(self.Lx / self.dx)
        self.Ny = int(self.Ly / self.dy)
        if opt_res:
            self.Nx = optimize_fftsize(self.Nx, fft_max_prime)
            self.Ny = optimize_fftsize(self.Ny, fft_max_prime)
            self.dx = np.float32(self.Lx / float(self.Nx))
            self.dy = np.float32(self.Ly / float(self.Ny))
        self.x = np.linspace(-self.Lx / 2., self.Lx / 2., self.Nx, dtype=np.float32)
        self.y = np.linspace(-self.Ly / 2., self.Ly / 2., self.Ny, dtype=np.float32)

        self.current = (self.current_mag * np.array([np.cos(self.current_dir),
                                                     np.sin(self.current_dir)])).astype(np.float32)
        u_eff = (self.wind_U * np.array([np.cos(self.wind_dir), np.sin(self.wind_dir)]) -
                 self.current).astype(np.float32)
        self.wind_U_eff = linalg.norm(u_eff)
        self.wind_dir_eff = np.arctan2(u_eff[1], u_eff[0])

        kx_s = (2 * np.pi * np.fft.fftfreq(self.Nx, self.dx)).astype(np.float32)
        ky_s = (2 * np.pi * np.fft.fftfreq(self.Ny, self.dy)).astype(np.float32)
        self.kx_s, self.ky_s = kx_s, ky_s
        self.kx, self.ky = np.meshgrid(kx_s, ky_s)
        self.kx_res = kx_res = self.kx[0, 1] - self.kx[0, 0]
        self.ky_res = ky_res = self.ky[1, 0] - self.ky[0, 0]
        self.k = np.sqrt(self.kx ** 2 + self.ky ** 2)
        self.kmin_half = np.min(np.array([kx_res, ky_res])) / 2.0
        good_k = np.where(self.k > self.kmin_half)
        self.kxn = np.zeros_like(self.kx, dtype=np.float32)
        self.kyn = np.zeros_like(self.kx, dtype=np.float32)
        self.kxn[good_k] = self.kx[good_k] / self.k[good_k]
        self.kyn[good_k] = self.ky[good_k] / self.k[good_k]
        self.kinv = np.zeros(self.k.shape, dtype=np.float32)
        self.kinv[good_k] = 1. / self.k[good_k]
        self.theta = np.angle(np.exp(1j * (np.arctan2(self.ky, self.kx) -
                                           self.wind_dir_eff))).astype(np.float32)
        self.theta_swell = np.angle(np.exp(1j * np.arctan2(self.ky, self.kx))).astype(np.float32)
        if depth is None:
            self.omega = np.sqrt(np.float32(G) * self.k)
        else:
            self.omega = np.sqrt(np.float32(G) * self.k * np.tanh(self.k * np.float32(depth)))

        if callable(dirspectrum_func):
            self.wave_dirspec = np.zeros(self.k.shape, dtype=np.float32)
            self.wave_dirspec[good_k] = dirspectrum_func(self.kx[good_k], self.ky[good_k])
        else:
            if spec_model not in spec.models:
                raise NotImplementedError('%s spectrum function not implemented' % spec_model)
            if spread_model not in spread.models or spread.models[spread_model] is None:
                raise NotImplementedError('%s spreading function not implemented' % spread_model)
            wave_spec = np.zeros(self.k.shape, dtype=np.float32)
            wave_spec[good_k] = spec.models[spec_model](self.k[good_k], self.wind_U_eff, self.wind_fetch)
            wave_spread = np.zeros(self.k.shape, dtype=np.float32)
            wave_spread[good_k] = spread.models[spread_model](self.k[good_k], self.theta[good_k],
                                                              self.wind_U_eff, self.wind_fetch)
            self.wave_dirspec = self.kinv * wave_spec * wave_spread
        self.rmss_x = np.sqrt(np.sum(self.wave_dirspec * self.kx ** 2 * self.kx_res * ky_res))
        self.rmss_y = np.sqrt(np.sum(self.wave_dirspec * self.ky ** 2 * self.kx_res * ky_res))
        if cutoff_wl and (cutoff_wl != 'auto'):
            kco = 2. * np.pi / cutoff_wl
            if (kco > np.pi / self.dx) or (kco > np.pi / self.dy):
                raise ValueError('Cutoff wavelength is too small for the specified grid resolution')
            # the reference builds this box filter with float slice bounds (ocean.py:192-196),
            # which numpy rejects; the box it describes is applied here
            kmax_x = np.float32(np.pi / self.dx)
            kmax_y = np.float32(np.pi / self.dy)
            k_f = np.zeros([self.Ny, self.Nx], dtype=np.float32)
            ys = int(np.ceil((self.Ny / 2) * kco / kmax_y))
            xs = int(np.ceil((self.Nx / 2) * kco / kmax_x))
            k_f[self.Ny // 2 - ys:self.Ny // 2 + ys, self.Nx // 2 - xs:self.Nx // 2 + xs] = 1.
            self.wave_dirspec *= np.fft.fftshift(k_f)

        random_cg = (1. / np.sqrt(2) * (np.random.normal(0., 1., size=[self.Ny, self.Nx]) +
                                        1j * np.random.normal(0., 1., size=[self.Ny, self.Nx]))
                     ).astype(np.complex64)
        if swell_dir_enable:
            swell_dirspec = np.zeros(self.k.shape, dtype=np.float32)
            swell_dirspec[good_k] = dir_swell_spec(self.k[good_k], self.theta_swell[good_k],
                                                   self.dir_swell_dir, self.freq_r, self.sigf,
                                                   self.sigs, self.Hs)
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
        self._on_device = False
        if device:
            self._upload()
        self.initialized = True
        return self

    def to_device(self):
        """Upload a surface initialised with ``device=False`` (no-op once on the device)."""
        if not getattr(self, '_on_device', True):
            self._upload()
        return self

    # ------------------------------------------------------------------------------
    def _upload(self):
        """Copy the spectral state to the device and lay out the field program."""
        self._coefs_d = _device.to_device(self.wave_coefs, np.complex64)
        self._omega_d = _device.to_device(self.omega, np.float32)
        self._kx_d = _device.to_device(self.kx_s, np.float32)
        self._ky_d = _device.to_device(self.ky_s, np.float32)
        self._swell_d = (_device.to_device(self.swell_exp, np.complex64)
                         if self.swell_enable else None)
        self._plan_fields()
        self._on_device = True

    def _plan_fields(self):
        names = []
        for g in ('D', 'Diff', 'Diff2', 'V', 'A', 'hMTF'):
            if g in self.compute:
                names += GROUPS[g]
        self._out_names = names
        shape = (self.Ny, self.Nx)
        # one contiguous block, fields in FIELD_NAMES order: the pulse kernel fetches a row
        # of every field with a single tensor copy
        block = _device.empty((max(1, len(names)),) + shape, np.float32)
        self._fields = {n: block[i] for i, n in enumerate(names)}
        raw = []                      # (code, destination tensor, additive key, swell key)
        self._aux = {}
        chop = self.choppy_enable
        for n in names:
            if chop and n in ('Diffx', 'Diffy', 'Diffxx', 'Diffyy', 'Diffxy'):
                continue
            raw.append((CODES[n], self._fields[n], n, n))
        if chop and ('Diff' in self.compute or 'Diff2' in self.compute):
            aux = ['Diffx', 'Diffy', 'aux_xx', 'aux_yy']
            if 'Diff2' in self.compute:
                aux += ['aux_xxx', 'aux_yyy', 'aux_xxy', 'Diffxx', 'Diffyy', 'Diffxy']
            for a in aux:
                t = _device.empty(shape, np.float32)
                self._aux[a] = t
                raw.append((CODES[a], t, None, None))
        self._raw = raw
        n = len(raw)
        if n == 0:
            return
        ws = _capi.load().ocs_surface_workspace_bytes(self.Nx, self.Ny, n)
        if ws < 0:
            raise ValueError('unsupported surface size %dx%d' % (self.Nx, self.Ny))
        self._ws = torch.empty(int(ws), dtype=torch.uint8, device=_device.device())
        _capi.call("ocs_surface_prepare", self.Nx, self.Ny, _device.ptr(self._ws), _device.stream_ptr())
        self._codes = (ctypes.c_int32 * n)(*[c for c, _, _, _ in raw])
        self._dsts = (ctypes.c_void_p * n)(*[t.data_ptr() for _, t, _, _ in raw])
        self._swm = (ctypes.c_float * (2 * n))()
        if self.swell_enable:
            for i, (_, _, _, key) in enumerate(raw):
                m = self._swell_mult(key)
                self._swm[2 * i], self._swm[2 * i + 1] = float(m.real), float(m.imag)

    def _swell_mult(self, name):
        """Complex factor m with field += Re(m * swell_phased) (ocean.py:438-506)."""
        if name is None or not self.swell_enable:
            return np.complex64(0)
        skx, sky, sk, som = self.swell_kx, self.swell_ky, self.swell_k, self.swell_omega
        dt = -1j * som
        table = {
            'Dx': 1j * skx / sk, 'Dy': 1j * sky / sk, 'Dz': np.complex64(1),
            'Diffx': 1j * skx, 'Diffy': 1j * sky,
            'Diffxx': -skx ** 2., 'Diffyy': -sky ** 2., 'Diffxy': -skx * sky,
            'Vx': 1j * skx / sk * dt, 'Vy': 1j * sky / sk * dt, 'Vz': dt,
            'Ax': 1j * skx / sk * (-som ** 2.), 'Ay': 1j * sky / sk * (-som ** 2.), 'Az': -som ** 2.,
        }
        return np.complex64(table.get(name, 0))

    # ------------------------------------------------------------------------------
    def load(self, state_file, compute=[]):
        """Restore a surface written by ``save`` (``ocean.py:244-332``)."""
        try:
            if netcdf3.is_netcdf3(state_file):
                ds = netcdf3.Dataset(state_file, 'r')
                st = {k: v[:] for k, v in ds.variables.items()}
                st = _Vars(st)
            else:
                st = np.load(state_file, allow_pickle=False)
        except (OSError, ValueError):
            raise RuntimeError('Error loading OTGI File')
        g = lambda k: st[k][()]  # noqa: E731
        self.Nx, self.Ny = int(g('Nx')), int(g('Ny'))
        self.Lx, self.Ly = g('Lx'), g('Ly')
        self.dx, self.dy = g('dx'), g('dy')
        self.wind_dir = np.deg2rad(g('wind_dir'))
        self.wind_dir_eff = np.deg2rad(g('wind_dir_eff'))
        self.wind_fetch, self.wind_U, self.wind_U_eff = g('wind_fetch'), g('wind_U'), g('wind_U_eff')
        self.current_mag = g('current_mag')
        self.current_dir = np.deg2rad(g('current_dir'))
        self.swell_enable = bool(g('swell_enable') == 1)
        self.swell_ampl, self.swell_wl = g('swell_ampl'), g('swell_wl')
        self.swell_dir = np.deg2rad(g('swell_dir'))
        self.swell_ph0 = g('swell_ph0') if 'swell_ph0' in st.files else np.float32(0)
        self.kx, self.ky = st['kx'], st['ky']
        self.kx_s, self.ky_s = self.kx[0].copy(), self.ky[:, 0].copy()
        self.wave_coefs = (st['wave_coefs_r'] + 1j * st['wave_coefs_i']).astype(np.complex64)
        self.choppy_enable = bool(g('choppy_enable') == 1)
        self.k = np.sqrt(self.kx ** 2 + self.ky ** 2)
        kx_res = self.kx[0, 1] - self.kx[0, 0]
        ky_res = self.ky[1, 0] - self.ky[0, 0]
        self.kmin_half = np.min(np.array([kx_res, ky_res])) / 2.0
        self.current = self.current_mag * np.array([np.cos(self.current_dir), np.sin(self.current_dir)])
        self.current = self.current.astype(np.float32)
        self.x = np.linspace(-self.Lx / 2, self.Lx / 2., self.Nx).astype(np.float32)
        self.y = np.linspace(-self.Ly / 2., self.Ly / 2., self.Ny).astype(np.float32)
        # the reference's load() uses the deep-water dispersion relation (ocean.py:317)
        self.omega = np.sqrt(np.float32(G) * self.k).astype(np.float32)
        if self.swell_enable:
            x, y = np.meshgrid(self.x, self.y)
            self.swell_k = np.float32(2. * np.pi / self.swell_wl)
            self.swell_kx = np.float32(self.swell_k * np.cos(self.swell_dir))
            self.swell_ky = np.float32(self.swell_k * np.sin(self.swell_dir))
            self.swell_omega = np.float32(np.sqrt(self.swell_k * G))
            self.swell_exp = (self.swell_ampl * np.exp(1j * (self.swell_k * (np.cos(self.swell_dir) * x +
                                                                             np.sin(self.swell_dir) * y) +
                                                             self.swell_ph0))).astype(np.complex64)
        self.compute = list(compute)
        self._upload()
        self.initialized = True

    def save(self, state_file):
        """Write the state-file variables (``ocean.py:334-373``) to ``state_file``: a netCDF
        classic ``OceanStateFile``, or a numpy container for names ending in ``.npz``."""
        if not self.initialized:
            raise Exception('Surface not initialized')
        d = dict(Nx=np.uint32(self.Nx), Ny=np.uint32(self.Ny), Lx=np.float32(self.Lx),
                 Ly=np.float32(self.Ly), dx=np.float32(self.dx), dy=np.float32(self.dy),
                 wind_dir=np.float32(np.rad2deg(self.wind_dir)),
                 wind_dir_eff=np.float32(np.rad2deg(self.wind_dir_eff)),
                 wind_fetch=np.float32(self.wind_fetch), wind_U=np.float32(self.wind_U),
                 wind_U_eff=np.float32(self.wind_U_eff), current_mag=np.float32(self.current_mag),
                 current_dir=np.float32(np.rad2deg(self.current_dir)),
                 swell_enable=np.float32(1 if self.swell_enable else 0),
                 swell_ampl=np.float32(self.swell_ampl), swell_dir=np.float32(np.rad2deg(self.swell_dir)),
                 swell_wl=np.float32(self.swell_wl), kx=self.kx.astype(np.float32),
                 ky=self.ky.astype(np.float32), wave_coefs_r=self.wave_coefs.real.astype(np.float64),
                 wave_coefs_i=self.wave_coefs.imag.astype(np.float64),
                 choppy_enable=np.float32(1 if self.choppy_enable else 0))
        if self.swell_enable:
            d['swell_ph0'] = np.float32(self.swell_ph0)
        if str(state_file).endswith('.npz'):
            with open(state_file, 'wb') as f:
                np.savez(f, **d)
            return
        # netCDF classic OceanStateFile (ocean.py:334-373)
        f = OceanStateFile(state_file, 'w', ocean_dim=(self.Ny, self.Nx))
        for k, v in d.items():
            f.set(k, v)
        f.close()

    # ------------------------------------------------------------------------------
    @property
    def t(self):
        if not self.initialized:
            raise Exception('Surface not initialized')
        return self._t

    @t.setter
    def t(self, value):
        self.set_t(value)

    def set_t(self, value, stream=None, passes=3, buffer=0):
        """Propagate to time ``value`` and synthesise every requested field on the GPU.

        ``passes`` selects the row pass (1), the column pass (2) or both (3, the default);
        the column pass consumes what the row pass of the same time left in the workspace.
        ``buffer`` 1 writes the second field set (``second_buffer``)."""
        if not self.initialized:
            raise Exception('Surface not initialized')
        self._t = np.float32(value)
        self._host_cache = {}
        if not self._raw:
            return
        _, add, rot = self.time_terms(value)
        desc = self.update_desc(add, rot, buffer)
        sp = _device.stream_ptr(stream)
        if passes == 3:
            _capi.call("ocs_surface_update", ctypes.addressof(desc), ctypes.c_float(float(self._t)), sp)
        else:
            _capi.call("ocs_surface_update_passes", ctypes.addressof(desc), ctypes.c_float(float(self._t)),
                       int(passes), sp)
        if self._aux and passes & 2:
            self._choppy(rot, sp)

    def time_terms(self, value):
        """(float32 t, additive term of every synthesised field, swell rotation) at time
        ``value``: the per-call inputs of the surface update besides the spectrum."""
        t = np.float32(value)
        add = []
        for _, _, key, _ in self._raw:
            if key == 'Dx':
                add.append(float(self.current[0] * t))
            elif key == 'Dy':
                add.append(float(self.current[1] * t))
            elif key == 'Vx':
                add.append(float(self.current[0]))
            elif key == 'Vy':
                add.append(float(self.current[1]))
            else:
                add.append(0.0)
        rot = np.complex64(0)
        if self.swell_enable:
            rot = np.exp(-1j * self.swell_omega * t)
        return t, add, rot

    def second_buffer(self):
        """Allocate a second set of field buffers (once) so that the fields of the next time
        can be synthesised while the current ones are still being read; returns the
        field-name -> tensor dict of that set.  Not for choppy surfaces."""
        if self._aux:
            raise NotImplementedError('choppy surfaces keep a single field buffer')
        if getattr(self, '_fields_b', None) is None:
            shape = (self.Ny, self.Nx)
            block = _device.empty((max(1, len(self._fields)),) + shape, np.float32)
            self._fields_b = {n: block[i] for i, n in enumerate(self._fields)}
            self._dsts_b = (ctypes.c_void_p * len(self._raw))(*[self._fields_b[key].data_ptr()
                                                                  for _, _, key, _ in self._raw])
        return self._fields_b

    def update_desc(self, add=None, rot=np.complex64(0), buffer=0):
        """``ocs_surface_desc`` of this surface (the caller keeps it alive while in use);
        ``buffer`` 1 writes the second field set (``second_buffer``)."""
        n = len(self._raw)
        add_c = (ctypes.c_float * n)(*(add if add is not None else [0.0] * n))
        dsts = self._dsts if buffer == 0 else self._dsts_b
        desc = SurfaceDesc(self.Nx, self.Ny, self._coefs_d.data_ptr(), self._omega_d.data_ptr(),
                           self._kx_d.data_ptr(), self._ky_d.data_ptr(), float(self.kmin_half), n,
                           self._codes, dsts, add_c, self._swm,
                           self._swell_d.data_ptr() if self._swell_d is not None else None,
                           float(np.real(rot)), float(np.imag(rot)), self._ws.data_ptr())
        desc._keep = add_c
        return desc

    def choppy_desc(self, rot=np.complex64(0)):
        """``ocs_choppy_desc`` of a choppy surface (the caller keeps it alive while in use):
        the slopes / curvatures from this surface's auxiliary fields, swell rotation ``rot``."""
        a, f = self._aux, self._fields
        p = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        m = (ctypes.c_float * 10)()
        for i, name in enumerate(('Diffx', 'Diffy', 'Diffxx', 'Diffyy', 'Diffxy')):
            v = self._swell_mult(name)
            m[2 * i], m[2 * i + 1] = float(v.real), float(v.imag)
        d2 = 'aux_xxx' in a
        desc = ChoppyDesc(self.Nx * self.Ny, p(a['Diffx']), p(a['Diffy']), p(a['aux_xx']), p(a['aux_yy']),
                          p(a.get('aux_xxx')), p(a.get('aux_yyy')), p(a.get('aux_xxy')),
                          p(a.get('Diffxx')), p(a.get('Diffyy')), p(a.get('Diffxy')),
                          p(f.get('Diffx')), p(f.get('Diffy')),
                          p(f.get('Diffxx')) if d2 else None, p(f.get('Diffyy')) if d2 else None,
                          p(f.get('Diffxy')) if d2 else None,
                          self._swell_d.data_ptr() if self._swell_d is not None else None,
                          float(np.real(rot)), float(np.imag(rot)), m)
        desc._keep = m
        return desc

    def _choppy(self, rot, sp):
        desc = self.choppy_desc(rot)
        _capi.call("ocs_surface_choppy", ctypes.addressof(desc), sp)

    # ------------------------------------------------------------------------------
    def field(self, name):
        """Device tensor (float32 [Ny, Nx]) of a computed field, no copy."""
        return self._fields[name]

    def __getattr__(self, name):
        fields = self.__dict__.get('_fields', {})
        if name in fields:
            cache = self.__dict__['_host_cache']
            if name not in cache:
                cache[name] = fields[name].cpu().numpy()
            return cache[name]
        raise AttributeError(name)
