"""Range-Doppler focusing (CPU restatement for the tests).

Test infrastructure only (see ``oracle/__init__.py``).  Restates ``sar_focus``
(oceansar/radarsim/sar_processor.py:30-274) with numpy's complex128 FFTs: zero padding to
powers of two (:143-149), 2-D FFT, range-cell-migration phase ramp (:150-176), range IFFT,
azimuth compression with the hyperbolic phase, the raised-cosine weighting over the
Doppler bandwidth and the antenna-pattern compensation (:180-217), azimuth IFFT, crop and
valid-aperture selection (:220-232).
"""
import numpy as np

from .geometry import optimize_fftsize

C = 299792458.0


def _sinc_bp(sin_angle, L, f0):
    return np.sinc(L / (C / f0) * sin_angle)


def focus_cube(raw, sar, proc, sr0):
    f0, prf, num_ch, v_ground = sar['f0'], sar['prf'], sar['num_ch'], sar['v_ground']
    l0 = C / f0
    rg_sampling = sar['rg_bw'] * sar['over_fs']
    sr0 = float(np.asarray(sr0))
    out = []
    for ch in range(num_ch):
        az0, rg0 = raw[0, ch].shape
        az_size, rg_size = [int(v) for v in optimize_fftsize(raw[0, ch].shape)]
        data = np.zeros([raw.shape[0], az_size, rg_size], dtype=complex)
        data[:, :az0, :rg0] = raw[:, ch, :, :]
        fr = np.fft.fftfreq(rg_size, 1 / rg_sampling)
        fa = np.fft.fftfreq(az_size, 1 / prf)
        sin_az = fa * l0 / (2 * v_ground)
        beam = _sinc_bp(sin_az, sar['ant_L_tx'], f0) * _sinc_bp(sin_az, sar['ant_L_rx'], f0)
        rcmc = sr0 / np.sqrt(1 - (fa * (l0 / 2.) / v_ground) ** 2.) - sr0
        data = np.fft.fft(np.fft.fft(data, axis=-1), axis=-2)
        data = data * np.exp(4j * np.pi * rcmc.reshape((1, az_size, 1)) / C * fr.reshape((1, 1, rg_size)))
        data = np.fft.ifft(data, axis=2)
        n_samp = 2 * (int(proc['doppler_bw'] / (fa[1] - fa[0])) / 2)
        w = proc['az_weighting'] - (1. - proc['az_weighting']) * np.cos(2 * np.pi * np.linspace(0, 1., int(n_samp)))
        w /= np.sqrt(np.sum(np.abs(w) ** 2) / w.size)
        if fa.size > n_samp:
            z = np.zeros(az_size)
            z[0:int(n_samp)] = w
            w = np.roll(z, int(-n_samp / 2))
        with np.errstate(divide='ignore', invalid='ignore'):
            w = np.where(np.abs(beam) > 0, w / beam, 0)
        ph = 4. * np.pi / l0 * sr0 * (np.sqrt(1. - (fa * l0 / 2. / v_ground) ** 2.) - 1.)
        data = data * (np.exp(1j * ph) * w).reshape((1, az_size, 1))
        data = np.fft.ifft(data, axis=1)[:, :az0, :rg0]
        nv = np.floor(proc['doppler_bw'] / 2. / (2. * v_ground ** 2. / l0 / sr0) * prf / 2.) * 2.
        out.append(data[:, int(nv):int(az0 - nv - 1), :])
    return np.array(out, dtype=complex)
