"""Kirchhoff-approximation specular field (CPU restatement for the tests).

Test infrastructure only (see ``oracle/__init__.py``).  Restates ``RCSKA``
(oceansar/nrcs/ka.py:41-310): the monostatic tangent-plane field of every facet, either
by the facet approach (``fa``: the Stratton-Chu integral over the facet, ka.py:277-284) or
by the stationary-phase approximation (``spa``: only facets whose stationary point lies
inside them contribute, ka.py:243-274).  The float32 surface derivatives enter exactly
as numpy combines them in the reference: the normal's norm and components, the
curvature determinant and its inverse are float32 quantities.
"""
import numpy as np

EPS_SW = 73 + 18j


def _cross(a, b):
    return np.stack([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


class RCSKA:
    def __init__(self, mode, k0, x, y, dx, dy):
        self.mode, self.k0, self.dx, self.dy = mode, k0, dx, dy
        self.x = np.asarray(x, dtype=np.float64)
        self.y = np.asarray(y, dtype=np.float64)

    def field(self, R_i, R_s, pol_i, pol_s, theta_i, theta_s, phi_i, phi_s, Dz, Diffx, Diffy, Diffxx,
              Diffyy, Diffxy, monostatic=True):
        if not monostatic:
            raise NotImplementedError('bistatic geometry')
        ny, nx = Dz.shape
        st = np.sin(theta_i).reshape(1, -1)
        ct = np.cos(theta_i).reshape(1, -1)
        tt = np.tan(theta_i)
        sp = np.sin(phi_i)
        cp = np.cos(phi_i)
        full = lambda v: np.broadcast_to(v, (ny, nx)).astype(np.float64)  # noqa: E731
        h = np.stack([full(-sp), full(cp), np.zeros((ny, nx))])
        v = np.stack([full(-ct * cp), full(-ct * sp), full(-st)])
        a_i = h if pol_i == 'h' else v
        a_s = h if pol_s == 'h' else v
        # surface normal from the float32 slopes (float32 arithmetic, as in the reference)
        n_norm = np.sqrt(Diffx ** 2. + Diffy ** 2. + 1.)
        n = np.stack([(-Diffx / n_norm).astype(np.float64), (-Diffy / n_norm).astype(np.float64),
                      (1. / n_norm).astype(np.float64)])
        n_i = np.stack([full(st * cp), full(st * sp), full(-ct)])
        n_s = np.stack([full(-st * cp), full(-st * sp), full(ct)])
        q = self.k0 * (n_s - n_i)
        t = _cross(n_i, n)
        t = t / np.sqrt(np.sum(t ** 2, axis=0))
        d = _cross(n_i, t)
        cos_l = -np.sum(n * n_i, axis=0)
        root = np.sqrt(EPS_SW + cos_l ** 2. - 1.)
        r_v = (EPS_SW * cos_l - root) / (EPS_SW * cos_l + root)
        r_h = (cos_l - root) / (cos_l + root)
        a_t = np.sum(a_i * t, axis=0)
        a_d = np.sum(a_i * d, axis=0)
        n_ni = -cos_l
        n_x_t = _cross(n, t)
        e_s = ((1. + r_h) * a_t) * n_x_t - ((1. - r_v) * n_ni * a_d) * t
        h_s = -(((1. - r_h) * n_ni * a_t) * t + ((1. + r_v) * a_d) * n_x_t)
        p = np.sum(a_s * _cross(n_s, e_s - _cross(n_s, h_s)), axis=0)
        K = -1j * self.k0 * np.exp(-1j * self.k0 * (R_i + R_s)) / ((4. * np.pi) ** 2. * R_i * R_s)
        if self.mode == 'spa':
            with np.errstate(divide='ignore', invalid='ignore'):
                J = Diffxx * Diffyy - Diffxy ** 2
                J = np.where(J == 0., np.nan, J)
                J_abs = np.abs(J)
                dxv = (1. / J_abs) * (Diffxy * (Diffy - tt * sp) - Diffyy * (Diffx - tt * cp))
                dyv = (1. / J_abs) * (Diffxy * (Diffx - tt * cp) - Diffxx * (Diffy - tt * sp))
                dzv = dxv * Diffx + dyv * Diffy
                eps = np.where(J > 0., np.sign(Diffxx), 1j)
            E = np.zeros((ny, nx), dtype=complex)
            hit = np.where(((-0.5 * self.dx < dxv) & (dxv < 0.5 * self.dx)) &
                           ((-0.5 * self.dy < dyv) & (dyv < 0.5 * self.dy)))
            if hit[0].size:
                E[hit] = (eps[hit] * p[hit] * K *
                          np.exp(1j * (q[0][hit] * dxv[hit] + q[1][hit] * dyv[hit] + q[2][hit] * dzv[hit])) *
                          2. * np.pi / q[2][hit] * n_norm[hit] / np.sqrt(J_abs[hit]))
            return E
        X, Y = np.meshgrid(self.x, self.y)
        r = np.stack([X, Y, Dz.astype(np.float64)])
        I = (np.exp(-1j * np.sum(q * r, axis=0)) * n_norm * self.dx * self.dy *
             np.sinc((q[0] + q[2] * Diffx) * self.dx / 2.) * np.sinc((q[1] + q[2] * Diffy) * self.dy / 2.))
        return K * I * p

    def rcs(self, pol_i, pol_s, theta_i, theta_s, phi_i, phi_s, Dz, Diffx, Diffy, Diffxx, Diffyy, Diffxy):
        return (4. * np.pi) ** 2. * np.abs(self.field(1, 1, pol_i, pol_s, theta_i, theta_s, phi_i, phi_s, Dz, Diffx,
                                                     Diffy, Diffxx, Diffyy, Diffxy)) ** 2.
