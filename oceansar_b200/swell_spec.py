"""Directional swell spectrum (``oceansar/swell_spec/dir_swell_spec.py:24-39``).

Gaussian in frequency around ``freq_r`` (width ``sigf``) and Gaussian in direction around
``dir_swell_dir`` degrees (width ``sigs`` degrees), normalised so that the directional
integral is one, with significant wave height ``Hs``; evaluated on the host at set-up.
"""
import numpy as np

from .spec import G


def ardhuin_swell_spec(k_axis, theta_axis, dir_swell_dir, freq_r=0.068, sigf=0.007, sigs=8, Hs=1.45):
    f_k = 1 / 2 / np.pi * np.sqrt(G * k_axis)
    fac_f_k = 1 / 4 / np.pi * np.sqrt(G / k_axis)
    amp = (Hs / 4) ** 2 / sigf / np.sqrt(2 * np.pi)
    efs = (amp * np.exp(-(f_k - freq_r) ** 2 / (2 * sigf ** 2)) + 1E-5) * fac_f_k
    ang = np.angle(np.exp(1j * (theta_axis - np.radians(dir_swell_dir))))
    dirss = np.exp(-ang ** 2 / (2 * np.radians(sigs) ** 2))
    return efs * dirss / (np.sqrt(2 * np.pi) * np.radians(sigs))
