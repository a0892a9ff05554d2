"""Oracle (test infrastructure only): wave spectra and spreading functions.

* ``elfouhaily_spec``  -- ``oceansar/spec/elfouhaily.py:43-99`` (with the gamma / alpha_m
  helpers of ``:20-40``)
* ``elfouhaily_spread`` -- ``oceansar/spread/elfouhaily.py:23-56``
* ``cos2s``            -- the intent of ``oceansar/spread/cos2s.py:13-19`` (the reference
  body raises on arrays; G = cos^2(theta)/pi inside |theta| <= pi/2, else 0)
* ``ardhuin_swell_spec`` -- ``oceansar/swell_spec/dir_swell_spec.py:24-39``
"""
import warnings

import numpy as np

G = 9.80665           # scipy.constants.g
RHO = 1000.
S_TENSION = 0.072
X_0 = 22e3


def _gamma(omega_c):
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


def elfouhaily_spec(k, U_10, fetch):
    k_m = 2 * np.pi / 0.017
    k_0 = G / U_10 ** 2
    X = k_0 * fetch
    Omega_c = 0.84 * np.tanh((X / X_0) ** 0.4) ** (-0.75)
    c = np.sqrt(G / k + S_TENSION / RHO * k)
    k_p = k_0 * Omega_c ** 2
    c_p = np.sqrt(G / k_p + S_TENSION / RHO * k_p)
    Omega = U_10 / c_p
    alpha_p = 6e-3 * np.sqrt(Omega)
    sigma = 0.08 * (1. + 4. * Omega_c ** (-3.))
    Gamma = np.exp(-(np.sqrt(k / k_p) - 1.) ** 2 / (2. * sigma ** 2))
    J_p = _gamma(Omega_c) ** Gamma
    L_pm = np.exp(-5. / 4. * (k_p / k) ** 2)
    F_p = L_pm * J_p * np.exp(-Omega / np.sqrt(10.) * (np.sqrt(k / k_p) - 1.))
    B_l = 0.5 * alpha_p * c_p / c * F_p
    C_10 = (0.8 + 0.065 * U_10) * 1e-3
    ustar = np.sqrt(C_10) * U_10
    c_m = np.sqrt(G / k_m + S_TENSION / RHO * k_m)
    alpha_m = _alpha_m(ustar, c_m)
    F_m = L_pm * np.exp(-0.25 * (k / k_m - 1.) ** 2)
    B_h = 0.5 * alpha_m * c_m / c * F_m
    return (B_l + B_h) / k ** 3


def elfouhaily_spread(k, theta, U_10, fetch):
    k_0 = G / U_10 ** 2
    X = k_0 * fetch
    Omega_c = 0.84 * np.tanh((X / X_0) ** 0.4) ** (-0.75)
    cK = np.sqrt(G / k + S_TENSION / RHO * k)
    k_p = k_0 * Omega_c ** 2
    cK_p = np.sqrt(G / k_p + S_TENSION / RHO * k_p)
    k_m = np.sqrt(RHO * G / S_TENSION)
    cK_m = np.sqrt(G / k_m + S_TENSION / RHO * k_m)
    C_10 = (0.8 + 0.065 * U_10) * 1e-3
    ustar = np.sqrt(C_10) * U_10
    a_0 = np.log(2.) / 4.
    a_p = 4.
    a_m = 0.13 * ustar / cK_m
    Delta = np.tanh(a_0 + a_p * (cK / cK_p) ** 2.5 + a_m * (cK_m / cK) ** 2.5)
    return np.where((theta > -np.pi / 2.) & (theta < np.pi / 2.),
                    (1. + Delta * np.cos(2. * theta)) / np.pi, 0)


def cos2s(k, theta, U_10, fetch):
    theta = np.asarray(theta)
    g = np.cos(theta) ** 2 / np.pi
    return np.where((theta < -np.pi / 2.0) | (theta > np.pi / 2.0), 0.0, g)


def ardhuin_swell_spec(k_axis, theta_axis, dir_swell_dir, freq_r=0.068, sigf=0.007, sigs=8,
                       Hs=1.45):
    f_k = 1 / 2 / np.pi * np.sqrt(G * k_axis)
    fac_f_k = 1 / 4 / np.pi * np.sqrt(G / k_axis)
    amp = (Hs / 4) ** 2 / sigf / np.sqrt(2 * np.pi)
    efs = (amp * np.exp(-(f_k - freq_r) ** 2 / (2 * sigf ** 2)) + 1E-5) * fac_f_k
    ang = np.angle(np.exp(1j * (theta_axis - np.radians(dir_swell_dir))))
    dirss = np.exp(-ang ** 2 / (2 * np.radians(sigs) ** 2))
    factor = np.sqrt(2 * np.pi) * np.radians(sigs)
    return efs * dirss / factor


SPEC_MODELS = {'elfouhaily': elfouhaily_spec}
SPREAD_MODELS = {'elfouhaily': elfouhaily_spread, 'cos2s': cos2s}
