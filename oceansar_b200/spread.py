"""Directional spreading functions (registry ``models``), evaluated on the host at set-up.

* ``elfouhaily`` -- ``oceansar/spread/elfouhaily.py:23-56``: G = (1 + Delta cos 2 theta)/pi
  inside |theta| < pi/2, 0 outside.  The reference compiles it with numba, which evaluates
  every operand in float64; this host version promotes its inputs to float64 likewise.
* ``cos2s`` -- the cos^2 spreading that ``oceansar/spread/cos2s.py:13-19`` intends
  (G = cos^2(theta)/pi inside |theta| <= pi/2, 0 outside; the reference body raises on
  arrays).
The Bragg kernel evaluates the same two functions on the device.
"""
import numpy as np

from .spec import G, RHO_W, SIGMA_W, X0


def elfouhaily_delta_coeffs(U_10, fetch):
    """Constants of the Elfouhaily Delta(k): (cK_p, cK_m, a_0, a_p, a_m) in float64."""
    U_10 = float(U_10)
    k_0 = G / U_10 ** 2
    omega_c = 0.84 * np.tanh((k_0 * fetch / X0) ** 0.4) ** (-0.75)
    k_p = k_0 * omega_c ** 2
    ck_p = np.sqrt(G / k_p + SIGMA_W / RHO_W * k_p)
    k_m = np.sqrt(RHO_W * G / SIGMA_W)
    ck_m = np.sqrt(G / k_m + SIGMA_W / RHO_W * k_m)
    ustar = np.sqrt((0.8 + 0.065 * U_10) * 1e-3) * U_10
    return ck_p, ck_m, np.log(2.) / 4., 4., 0.13 * ustar / ck_m


def elfouhaily(k, theta, U_10, fetch):
    k = np.asarray(k, dtype=np.float64)
    theta = np.asarray(theta, dtype=np.float64)
    ck_p, ck_m, a_0, a_p, a_m = elfouhaily_delta_coeffs(U_10, fetch)
    ck = np.sqrt(G / k + SIGMA_W / RHO_W * k)
    delta = np.tanh(a_0 + a_p * (ck / ck_p) ** 2.5 + a_m * (ck_m / ck) ** 2.5)
    return np.where((theta > -np.pi / 2.) & (theta < np.pi / 2.),
                    (1. + delta * np.cos(2. * theta)) / np.pi, 0)


def cos2s(k, theta, U_10, fetch):
    theta = np.asarray(theta)
    g = np.cos(theta) ** 2 / np.pi
    return np.where((theta < -np.pi / 2.0) | (theta > np.pi / 2.0), 0.0, g)


models = {'elfouhaily': elfouhaily, 'cos2s': cos2s, 'none': None}
# device-side codes of the spreading functions the Bragg kernel implements
DEVICE_CODES = {'elfouhaily': 0, 'cos2s': 1}
