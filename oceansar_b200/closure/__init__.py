"""Sub-grid closure (``oceansar/closure``): coherence time and random scatterer series.

``grid_coherence`` restates ``coherence_times.py:7-18``; ``randomscat_ts`` builds the
unit-power Gaussian-spectrum series and the per-facet start indices on the host with the
global numpy RNG (``random_scatterers.py:11-26``) and keeps device copies for the pulse
kernel, which gathers ``s[(ind0 + int(t*Fs)) mod N]`` (``:28-31``) per facet.
"""
import numpy as np
from scipy import special

from ..utils.misc import optimize_fftsize

C_LIGHT = 2.99792458e8


def grid_coherence(U, res, f0, model='Pierson-Moskowitz'):
    return 3.29 * C_LIGHT / f0 / U / np.sqrt(special.erf(2.688 * res / U ** 2))


class randomscat_ts(object):
    def __init__(self, tau, dim, Fs, N=None, seed=None):
        if seed is not None:
            np.random.seed(seed)
        if N is None:
            N = int(tau * Fs * 200)
        self.N = optimize_fftsize(N, max_prime=5)
        f = np.fft.fftfreq(self.N, 1. / Fs)
        a = 1 / (tau ** 2)
        spec = np.sqrt(np.pi / a) * np.exp(-np.pi ** 2 * f ** 2 / a)
        s_f = np.random.normal(size=self.N) + 1j * np.random.normal(size=self.N)
        s = np.fft.ifft(s_f * np.sqrt(spec))
        self.s = s / np.sqrt(np.mean(np.abs(s) ** 2))
        self.ind0 = (N * np.random.uniform(size=dim)).astype(int)
        self.Fs = Fs
        self._dev = None

    def tind(self, t):
        return int(t * self.Fs)

    def scats(self, t):
        return self.s[np.mod(self.ind0 + int(t * self.Fs), self.N)]

    def device(self):
        """(series complex128, ind0 int32) device tensors, uploaded once."""
        if self._dev is None:
            from .. import _device
            if self.ind0.size and self.ind0.max() >= 2 ** 31:
                raise ValueError('scatterer start index exceeds int32')
            self._dev = (_device.to_device(self.s, np.complex128),
                         _device.to_device(self.ind0.astype(np.int32), np.int32))
        return self._dev

    def device32(self):
        """The series as a complex64 device tensor (the mixed form's gathers), uploaded once."""
        if getattr(self, '_dev32', None) is None:
            from .. import _device
            self._dev32 = _device.to_device(self.s, np.complex64)
        return self._dev32
