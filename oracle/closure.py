"""Oracle (test infrastructure only): sub-grid closure.

* ``grid_coherence`` -- ``oceansar/closure/coherence_times.py:7-18``
* ``RandomScatTS``   -- ``oceansar/closure/random_scatterers.py:6-31`` (``randomscat_ts``):
  a unit-power complex series with a Gaussian spectrum, a per-facet random start index
  ``ind0`` (drawn with the *un-optimised* length N, ``:25``) and
  ``scats(t) = s[(ind0 + int(t*Fs)) mod N_opt]``.
"""
import numpy as np
from scipy import special

from .geometry import optimize_fftsize

C_LIGHT = 2.99792458e8


def grid_coherence(U, res, f0):
    return 3.29 * C_LIGHT / f0 / U / np.sqrt(special.erf(2.688 * res / U ** 2))


class RandomScatTS:
    def __init__(self, tau, dim, Fs, N=None, seed=None):
        if seed is not None:
            np.random.seed(seed)
        if N is None:
            N = int(tau * Fs * 200)
        self.N = optimize_fftsize(N, max_prime=5)
        f = np.fft.fftfreq(self.N, 1. / Fs)
        a = 1 / (tau ** 2)
        spec = np.sqrt(np.pi / a) * np.exp(-np.pi ** 2 * f ** 2 / a)
        s_f = (np.random.normal(size=self.N) + 1j * np.random.normal(size=self.N))
        s = np.fft.ifft(s_f * np.sqrt(spec))
        self.s = s / np.sqrt(np.mean(np.abs(s) ** 2))
        self.ind0 = (N * np.random.uniform(size=dim)).astype(int)
        self.Fs = Fs

    def tind(self, t):
        return int(t * self.Fs)

    def scats(self, t):
        inds = np.mod(self.ind0 + int(t * self.Fs), self.N)
        return self.s[inds]
