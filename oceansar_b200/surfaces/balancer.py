"""``OceanSurfaceBalancer`` (oceansar/surfaces/balancer.py:8-297) on one GPU.

The reference's MPI generator (``sar_raw.py:233-353``) does not synthesise the surface at
every pulse: it synthesises it at the multiples t_l, t_h = t_l + dt of the ocean time step
around the pulse time and interpolates every field linearly in float32,
w_l F(t_l) + w_h F(t_h), w_h = (t - t_l) / dt.  Here the two end surfaces live in the
wrapped surface's two field sets (``OceanSurface.second_buffer``); when t moves into the
next step only the new end is synthesised (the old upper end becomes the lower one), and
``ocs_surface_blend`` writes the interpolated fields into a third set.  The time
arithmetic is float32, as in the reference.  MPI scattering is replaced by nothing: the
whole surface is on the device.  A choppy surface keeps a single field set (its
synthesis needs auxiliary fields in place), so for it the two ends are separate buffers
that each new end is copied into on the device.
"""
import ctypes

import numpy as np
import torch

from .. import _capi, _device

PROPS = ('Lx', 'Ly', 'dx', 'dy', 'Nx', 'Ny', 'x', 'y', 'wind_dir', 'wind_dir_eff', 'wind_fetch', 'wind_U',
         'wind_U_eff', 'current_mag', 'current_dir', 'compute')


class OceanSurfaceBalancer(object):
    def __init__(self, surface, dt, t0=0., root=0):
        if not surface:
            raise ValueError('Surface is needed by root process')
        self.surface = surface
        for p in PROPS:
            if hasattr(surface, p):
                setattr(self, p, getattr(surface, p))
        shape = (surface.Ny, surface.Nx)
        self._copy_ends = bool(surface._aux)
        if self._copy_ends:
            self._sets = tuple({n: _device.empty(shape, np.float32) for n in surface._fields} for _ in range(2))
        else:
            surface.second_buffer()
            self._sets = (surface._fields, surface._fields_b)
        self._lo = 0                            # which field set holds F(t_l)
        self._names = list(surface._fields)
        block = _device.empty((max(1, len(self._names)),) + shape, np.float32)      # contiguous, in order
        self._fields = {n: block[i] for i, n in enumerate(self._names)}
        self._dst = (ctypes.c_void_p * len(self._names))(*[self._fields[n].data_ptr() for n in self._names])
        self._host_cache = {}
        self.dt = dt
        self.t_l_last = -1.
        self.t_h_last = -1.
        self.stream = None
        self.t = t0

    @property
    def t(self):
        return self._t

    @t.setter
    def t(self, value):
        self.set_t(value, self.stream)

    def restart(self):
        """Forget both ends: the next ``set_t`` synthesises the two of them."""
        self.t_l_last = -1.
        self.t_h_last = -1.

    def _plan(self, value, t_l_last, t_h_last, lo):
        """Host side of the ``t`` setter (balancer.py:133-166): (t, t_l, t_h, syntheses as
        (field set, time), field set of the lower end)."""
        t = np.float32(value)
        t_l = np.float32(np.floor(t / self.dt) * self.dt)
        t_h = t_l + self.dt
        updates = ()
        if (t_l != t_l_last) or (t_h != t_h_last):
            if t_l == t_h_last:
                lo = 1 - lo                     # the old upper end is the new lower end
                updates = ((1 - lo, t_h),)
            else:
                updates = ((lo, t_l), (1 - lo, t_h))
        return t, t_l, t_h, updates, lo

    def syntheses(self, times):
        """Surface syntheses that ``set_t`` over ``times`` makes after ``restart``."""
        tl, th, lo, n = -1., -1., 0, 0
        for v in times:
            _, tl, th, upd, lo = self._plan(v, tl, th, lo)
            n += len(upd)
        return n

    def set_t(self, value, stream=None):
        """Interpolated fields at ``value`` (balancer.py:130-297)."""
        self._host_cache = {}
        self._t, t_l, t_h, updates, self._lo = self._plan(value, self.t_l_last, self.t_h_last, self._lo)
        s = self.surface
        for buf, tt in updates:
            if self._copy_ends:
                s.set_t(float(tt), stream=stream)
                with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
                    for n in self._names:
                        self._sets[buf][n].copy_(s._fields[n])
            else:
                s.set_t(float(tt), stream=stream, buffer=buf)
        self.t_l_last = t_l
        self.t_h_last = t_h
        w_h = np.float32((self._t - t_l) / self.dt)
        w_l = np.float32(1. - w_h)
        lo, hi = self._sets[self._lo], self._sets[1 - self._lo]
        a = (ctypes.c_void_p * len(self._names))(*[lo[n].data_ptr() for n in self._names])
        b = (ctypes.c_void_p * len(self._names))(*[hi[n].data_ptr() for n in self._names])
        n = s.Nx * s.Ny
        _capi.call("ocs_surface_blend", n, len(self._names), a, b, self._dst, float(w_l), float(w_h),
                   _device.stream_ptr(stream))
        self.w_l, self.w_h = w_l, w_h

    def field(self, name):
        """Device tensor of an interpolated field."""
        return self._fields[name]

    def __getattr__(self, name):
        fields = self.__dict__.get('_fields', {})
        if name in fields:
            cache = self.__dict__['_host_cache']
            if name not in cache:
                cache[name] = fields[name].cpu().numpy()
            return cache[name]
        raise AttributeError(name)
