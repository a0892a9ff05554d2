"""Time-interpolated surface (CPU restatement for the tests).

Test infrastructure only (see ``oracle/__init__.py``).  Restates
``OceanSurfaceBalancer.t`` (oceansar/surfaces/balancer.py:126-297) without MPI: fields of
the surface at t_l = floor(t / dt) dt and t_h = t_l + dt (float32 time arithmetic, the
upper end reused as the lower one when t enters the next step), blended as
w_l F(t_l) + w_h F(t_h) in float32 with w_h = (t - t_l) / dt.
"""
import numpy as np


class OceanSurfaceBalancer:
    def __init__(self, surface, dt, t0=0.):
        self.surface = surface
        for p in ('Nx', 'Ny', 'x', 'y', 'dx', 'dy', 'Lx', 'Ly', 'compute'):
            setattr(self, p, getattr(surface, p))
        self.dt = dt
        self.t_l_last = -1.
        self.t_h_last = -1.
        self._ends = [None, None]
        self.set_t(t0)

    def set_t(self, value):
        t = np.float32(value)
        self._t = t
        t_l = np.float32(np.floor(t / self.dt) * self.dt)
        t_h = t_l + self.dt
        if (t_l != self.t_l_last) or (t_h != self.t_h_last):
            if t_l == self.t_h_last:
                self._ends[0] = self._ends[1]
                self._ends[1] = dict(self.surface.set_t(np.array([[1, t_h]])[0, 1]))
            else:
                self._ends[0] = dict(self.surface.set_t(np.array([[0, t_l], [1, t_h]])[0, 1]))
                self._ends[1] = dict(self.surface.set_t(np.array([[0, t_l], [1, t_h]])[1, 1]))
        self.t_l_last = t_l
        self.t_h_last = t_h
        w_h = np.float32((t - t_l) / self.dt)
        w_l = np.float32(1. - w_h)
        out = {}
        for k in self._ends[0]:
            out[k] = w_l * self._ends[0][k] + w_h * self._ends[1][k]
            setattr(self, k, out[k])
        return out
