"""Oracle (test infrastructure only): geometry helpers and FFT-size selection.

* ``inc_to_sr`` / ``inc_to_gr`` / ``inc_to_look`` / ``look_to_inc`` / ``max_look_angle`` /
  ``gr_to_geo`` / ``orbit_to_vel`` -- ``oceansar/utils/geometry.py:9-173``
* ``optimize_fftsize`` / ``factorize`` -- ``oceansar/utils/misc.py:39-83``
* ``db2lin`` -- ``oceansar/utils/misc.py:209-214``
"""
import numpy as np
from scipy import interpolate

R_EARTH = 6378.137e3
M_EARTH = 5.9742e24


def inc_to_look(theta_i, orbit_alt, r_planet=R_EARTH):
    return np.arcsin(np.sin(theta_i) / (r_planet + orbit_alt) * r_planet)


def look_to_inc(theta_l, orbit_alt, r_planet=R_EARTH):
    return np.arcsin(np.sin(theta_l) * (r_planet + orbit_alt) / r_planet)


def inc_to_sr(theta_i, orbit_alt, r_planet=R_EARTH):
    theta_l = inc_to_look(theta_i, orbit_alt, r_planet=r_planet)
    delta_theta = theta_i - theta_l
    return np.sqrt((orbit_alt + r_planet - r_planet * np.cos(delta_theta)) ** 2 +
                   (r_planet * np.sin(delta_theta)) ** 2)


def inc_to_gr(theta_i, orbit_alt, r_planet=R_EARTH):
    return r_planet * (theta_i - inc_to_look(theta_i, orbit_alt, r_planet=r_planet))


def max_look_angle(orbit_alt, r_planet=R_EARTH):
    return np.arcsin(r_planet / (r_planet + orbit_alt))


def sr_to_geo(slant_range, orbit_alt, r_planet=R_EARTH, m_planet=M_EARTH):
    """Ground range, incidence, look angle and b = v_orb^2 r_track / (r_planet + h) at the
    given slant ranges (geometry.py:101-133): quadratic splines through 2500 look angles."""
    theta_l = np.linspace(0, max_look_angle(orbit_alt, r_planet=r_planet), 2500)
    theta_i = look_to_inc(theta_l, orbit_alt, r_planet=r_planet)
    delta_theta = theta_i - theta_l
    r_track = np.cos(delta_theta) * r_planet
    v_orb = orbit_to_vel(orbit_alt, r_planet=r_planet, m_planet=m_planet)
    b = v_orb ** 2 * r_track / (r_planet + orbit_alt)
    gr = r_planet * delta_theta
    sr = np.sqrt((orbit_alt + r_planet - r_planet * np.cos(delta_theta)) ** 2 + (r_planet * np.sin(delta_theta)) ** 2)
    spl = interpolate.InterpolatedUnivariateSpline
    return (spl(sr, gr, k=2)(slant_range), spl(sr, theta_i, k=2)(slant_range),
            spl(sr, theta_l, k=2)(slant_range), spl(sr, b, k=2)(slant_range))


def gr_to_geo(ground_range, orbit_alt, r_planet=R_EARTH):
    theta_l = np.linspace(0, max_look_angle(orbit_alt), 500)
    theta_i = look_to_inc(theta_l, orbit_alt, r_planet=r_planet)
    delta_theta = theta_i - theta_l
    gr = r_planet * delta_theta
    sr = np.sqrt((orbit_alt + R_EARTH - r_planet * np.cos(delta_theta)) ** 2 +
                 (r_planet * np.sin(delta_theta)) ** 2)
    theta_l_interp = interpolate.InterpolatedUnivariateSpline(gr, theta_l, k=2)(ground_range)
    theta_i_interp = interpolate.InterpolatedUnivariateSpline(gr, theta_i, k=2)(ground_range)
    sr_interp = interpolate.InterpolatedUnivariateSpline(gr, sr, k=2)(ground_range)
    return sr_interp, theta_i_interp, theta_l_interp


def orbit_to_vel(orbit_alt, ground=False, r_planet=R_EARTH, m_planet=M_EARTH):
    from scipy.constants import G
    v = np.sqrt(G * m_planet / (r_planet + orbit_alt))
    if ground:
        v = r_planet / (r_planet + orbit_alt) * v
    return v


def factorize(n):
    result = np.array([])
    for i in np.append(2, np.arange(3, n + 1, 2)):
        s = 0
        while np.mod(n, i) == 0:
            n /= i
            s += 1
        result = np.append(result, [i] * s)
        if n == 1:
            return result


def _max_prime_factor(n):
    n = int(n)
    best = 1
    p = 2
    while p * p <= n:
        while n % p == 0:
            best = max(best, p)
            n //= p
        p += 1 if p == 2 else 2
    return max(best, n) if n > 1 else best


def optimize_fftsize(values, max_prime=2):
    """Next power of two for ``max_prime == 2``; otherwise the smallest value >= the
    input whose largest prime factor is <= ``max_prime`` (``misc.py:60-83``)."""
    scalar = np.isscalar(values)
    vals = np.atleast_1d(np.array(values, dtype=int))
    if max_prime == 2:
        good = (2 ** np.ceil(np.log2(vals))).astype(int)
    else:
        good = []
        for v in vals:
            b = int(v)
            while _max_prime_factor(b) > max_prime:
                b += 1
            good.append(b)
        good = np.array(good, dtype=int)
    return good[0] if (scalar or good.size == 1) else good


def db2lin(a, amplitude=False):
    return 10 ** (a / 20) if amplitude else 10 ** (a / 10)
