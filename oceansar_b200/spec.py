"""Omni-directional wave-number spectra (registry ``models``), evaluated on the host at set-up.

``elfouhaily`` follows ``oceansar/spec/elfouhaily.py:43-99`` (Elfouhaily, Chapron and Katsaros
1997, with the L_pm factor on both the long- and short-wave curvature spectra).  Called
once per scene by ``OceanSurface.init`` and ``RCSRomeiser97``; numpy's dtype flow is kept
(float32 wavenumbers stay float32) so that the wave coefficients match the reference's.
"""
import warnings

import numpy as np

G = 9.80665          # scipy.constants.g
RHO_W = 1000.        # water density [kg/m^3]
SIGMA_W = 0.072      # surface tension [N/m]
X0 = 22e3            # dimensionless fetch of fully developed seas


def _peak_enhancement(omega_c):
    if 0.84 < omega_c < 1.0:
        return 1.7
    if 1.0 < omega_c < 5.0:
        return 1.7 + 6. * np.log10(omega_c)
    warnings.warn('Omega_c is out of range. Returning  value for 5.0', RuntimeWarning)
    return 1.7 + 6. * np.log10(5.0)


def _alpha_m(ustar, c_m):
    if ustar < c_m:
        return 1e-2 * (1. + np.log(ustar / c_m))
    return 1e-2 * (1. + 3. * np.log(ustar / c_m))


def elfouhaily(k, U_10, fetch):
    k_m = 2 * np.pi / 0.017
    k_0 = G / U_10 ** 2
    omega_c = 0.84 * np.tanh((k_0 * fetch / X0) ** 0.4) ** (-0.75)
    c = np.sqrt(G / k + SIGMA_W / RHO_W * k)
    k_p = k_0 * omega_c ** 2
    c_p = np.sqrt(G / k_p + SIGMA_W / RHO_W * k_p)
    omega = U_10 / c_p
    alpha_p = 6e-3 * np.sqrt(omega)
    sigma = 0.08 * (1. + 4. * omega_c ** (-3.))
    gam = np.exp(-(np.sqrt(k / k_p) - 1.) ** 2 / (2. * sigma ** 2))
    j_p = _peak_enhancement(omega_c) ** gam
    l_pm = np.exp(-5. / 4. * (k_p / k) ** 2)
    f_p = l_pm * j_p * np.exp(-omega / np.sqrt(10.) * (np.sqrt(k / k_p) - 1.))
    b_l = 0.5 * alpha_p * c_p / c * f_p
    ustar = np.sqrt((0.8 + 0.065 * U_10) * 1e-3) * U_10
    c_m = np.sqrt(G / k_m + SIGMA_W / RHO_W * k_m)
    f_m = l_pm * np.exp(-0.25 * (k / k_m - 1.) ** 2)
    b_h = 0.5 * _alpha_m(ustar, c_m) * c_m / c * f_m
    return (b_l + b_h) / k ** 3


models = {'elfouhaily': elfouhaily}
