"""Spherical-Earth SAR geometry (``oceansar/utils/geometry.py:9-173``), host side.

Used once per scene to place the facet columns in slant range and incidence angle
(``gr_to_geo``: quadratic splines through 500 look angles, as the reference does).
"""
import numpy as np
from scipy import interpolate

R_EARTH = 6378.137e3
M_EARTH = 5.9742e24


def orbit_to_vel(orbit_alt, ground=False, r_planet=R_EARTH, m_planet=M_EARTH):
    from scipy.constants import G
    v = np.sqrt(G * m_planet / (r_planet + orbit_alt))
    return r_planet / (r_planet + orbit_alt) * v if ground else v


def inc_to_look(theta_i, orbit_alt, r_planet=R_EARTH):
    return np.arcsin(np.sin(theta_i) / (r_planet + orbit_alt) * r_planet)


def look_to_inc(theta_l, orbit_alt, r_planet=R_EARTH):
    return np.arcsin(np.sin(theta_l) * (r_planet + orbit_alt) / r_planet)


def inc_to_sr(theta_i, orbit_alt, r_planet=R_EARTH):
    dt = theta_i - inc_to_look(theta_i, orbit_alt, r_planet=r_planet)
    return np.sqrt((orbit_alt + r_planet - r_planet * np.cos(dt)) ** 2 + (r_planet * np.sin(dt)) ** 2)


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
    dt = theta_i - theta_l
    gr = r_planet * dt
    sr = np.sqrt((orbit_alt + R_EARTH - r_planet * np.cos(dt)) ** 2 + (r_planet * np.sin(dt)) ** 2)
    spl = interpolate.InterpolatedUnivariateSpline
    return (spl(gr, sr, k=2)(ground_range), spl(gr, theta_i, k=2)(ground_range),
            spl(gr, theta_l, k=2)(ground_range))
