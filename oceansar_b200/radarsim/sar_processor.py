"""``sar_focus`` (``oceansar/radarsim/sar_processor.py:30-274``): range-Doppler focusing of
the raw data cube on the GPU.

Per channel, as the reference: zero-pad to power-of-two sizes, 2-D FFT, range-cell-
migration correction by a range-frequency phase ramp per Doppler bin, range IFFT, azimuth
compression (hyperbolic phase, amplitude weighting over the Doppler bandwidth, antenna-
pattern compensation), azimuth IFFT, crop, and removal of the azimuth samples outside the
valid aperture.  The transforms are the library's own complex128 power-of-two FFTs
(``ocs_fft64_rows``; the azimuth ones on the cube's transpose, ``ocs_transpose_c128``);
the two phase multiplications between them are the fused kernels ``ocs_rd_rcmc`` and
``ocs_rd_azfilter``, which form the phase of each sample on the fly.  The filter
vectors are computed on the host exactly as the reference computes them.  The SLC file is
a netCDF classic ``ProcFile``.  Plot options of the [processing] section are accepted and
ignored (no plotting here).
"""
import ctypes

import numpy as np
import torch

from .. import _capi, _device
from ..ocs_io import ConfigFile, ProcFile, RawFile
from ..utils import geometry as geo
from ..utils.misc import optimize_fftsize
from .sar_raw_nompi import C_LIGHT, sinc_bp


def sinc_1tx_nrx(sin_angle, L, f0, num_chan, field=False, sin_squint=0):
    """One transmitter, N receivers (``radarsim/antenna.py:28-42``): as in the reference the
    ``field`` flag is passed on positionally and ignored, so both patterns are in power
    units."""
    bp_tx = sinc_bp(sin_angle - sin_squint, L, f0)
    bp_rx = sinc_bp(sin_angle - sin_squint, L / num_chan, f0)
    return bp_tx * bp_rx


def _fft_rows(t, inverse):
    """In-place complex128 FFT along the last (contiguous) dimension of t (``ocs_fft64_rows``)."""
    n = int(t.shape[-1])
    nrows = t.numel() // n
    ws = int(_capi.load().ocs_fft64_workspace_bytes(nrows, n))
    if ws < 0:
        raise ValueError('FFT length %d is not a power of two' % n)
    scratch = torch.empty(ws // 16, dtype=torch.complex128, device=t.device) if ws else None
    _capi.call("ocs_fft64_rows", t.data_ptr(), nrows, n, int(inverse),
               scratch.data_ptr() if scratch is not None else None, _device.stream_ptr())


def _fft_az(t, inverse):
    """In-place complex128 FFT along dimension 1 of a contiguous [pol][az][rg] cube: row
    transforms of its [pol][rg][az] transpose (``ocs_transpose_c128``)."""
    p, a, r = (int(v) for v in t.shape)
    tt = torch.empty((p, r, a), dtype=t.dtype, device=t.device)
    sp = _device.stream_ptr()
    _capi.call("ocs_transpose_c128", t.data_ptr(), tt.data_ptr(), p, a, r, sp)
    _fft_rows(tt, inverse)
    _capi.call("ocs_transpose_c128", tt.data_ptr(), t.data_ptr(), p, r, a, sp)


def focus_cube(raw, cfg, sr0):
    """SLC of every channel: complex128 [ch, pol, az_valid, rg] from a raw cube
    [pol, ch, az, rg] (sar_processor.py:95-236)."""
    pr, sar = cfg.processing, cfg.sar
    f0, prf, num_ch, alt, v_ground = sar.f0, sar.prf, sar.num_ch, sar.alt, sar.v_ground
    rg_bw, over_fs = sar.rg_bw, sar.over_fs
    l0 = C_LIGHT / f0
    if v_ground == 'auto':
        v_ground = geo.orbit_to_vel(alt, ground=True)
    rg_sampling = rg_bw * over_fs
    sr0 = float(np.asarray(sr0))
    dev = _device.device()
    sp = _device.stream_ptr()
    lib = _capi.load()
    slc = []
    for ch in np.arange(num_ch):
        az_size_orig, rg_size_orig = raw[0, ch].shape
        opt = optimize_fftsize(raw[0, ch].shape)
        az_size, rg_size = int(opt[0]), int(opt[1])
        data = torch.zeros((raw.shape[0], az_size, rg_size), dtype=torch.complex128, device=dev)
        data[:, :az_size_orig, :rg_size_orig] = torch.from_numpy(
            np.ascontiguousarray(raw[:, ch].astype(np.complex128))).to(dev)
        fr = np.fft.fftfreq(rg_size, 1 / rg_sampling)
        fa = np.fft.fftfreq(az_size, 1 / prf)
        sin_az = fa * l0 / (2 * v_ground)
        if hasattr(sar, 'ant_L'):
            if sar.L_total:
                beam_pattern = sinc_1tx_nrx(sin_az, sar.ant_L * num_ch, f0, num_ch, field=True)
            else:
                beam_pattern = sinc_1tx_nrx(sin_az, sar.ant_L, f0, 1, field=True)
        else:
            beam_pattern = (sinc_bp(sin_az, sar.ant_L_tx, f0, field=True) *
                            sinc_bp(sin_az, sar.ant_L_rx, f0, field=True))
        rcmc_fa = sr0 / np.sqrt(1 - (fa * (l0 / 2.) / v_ground) ** 2.) - sr0
        _fft_rows(data, False)
        _fft_az(data, False)
        rcmc_d = torch.from_numpy(np.ascontiguousarray(rcmc_fa, dtype=np.float64)).to(dev)
        fr_d = torch.from_numpy(np.ascontiguousarray(fr, dtype=np.float64)).to(dev)
        _capi.call("ocs_rd_rcmc", data.data_ptr(), data.shape[0], az_size, rg_size, rcmc_d.data_ptr(),
                   fr_d.data_ptr(), float(C_LIGHT), sp)
        _fft_rows(data, True)
        # azimuth compression filter (sar_processor.py:180-215)
        n_samp = 2 * (int(pr.doppler_bw / (fa[1] - fa[0])) / 2)
        weighting = (pr.az_weighting -
                     (1. - pr.az_weighting) * np.cos(2 * np.pi * np.linspace(0, 1., int(n_samp))))
        L_win = np.sum(np.abs(weighting) ** 2) / weighting.size
        weighting /= np.sqrt(L_win)
        if fa.size > n_samp:
            zeros = np.zeros(az_size)
            zeros[0:int(n_samp)] = weighting
            weighting = np.roll(zeros, int(-n_samp / 2))
        with np.errstate(divide='ignore', invalid='ignore'):
            weighting = np.where(np.abs(beam_pattern) > 0, weighting / beam_pattern, 0)
        ph_ac = 4. * np.pi / l0 * sr0 * (np.sqrt(1. - (fa * l0 / 2. / v_ground) ** 2.) - 1.)
        h = np.ascontiguousarray(np.exp(1j * ph_ac) * weighting, dtype=np.complex128)
        h_d = torch.from_numpy(h).to(dev)
        _capi.call("ocs_rd_azfilter", data.data_ptr(), data.shape[0], az_size, rg_size, h_d.data_ptr(), sp)
        _fft_az(data, True)
        data = data[:, :int(az_size_orig), :int(rg_size_orig)]
        n_val_az_2 = np.floor(pr.doppler_bw / 2. / (2. * v_ground ** 2. / l0 / sr0) * prf / 2.) * 2.
        data = data[:, int(n_val_az_2):int(az_size_orig - n_val_az_2 - 1), :]
        slc.append(data.cpu().numpy())
    return np.array(slc, dtype=complex)


def sar_focus(cfg_file, raw_output_file, output_file):
    """Drop-in for ``sar_processor.sar_focus``: read the raw file, focus it, write the SLC."""
    cfg = ConfigFile(cfg_file)
    raw_file = RawFile(raw_output_file, 'r')
    raw_data = raw_file.get('raw_data*')
    sr0 = raw_file.get('sr0')
    inc_angle = raw_file.get('inc_angle')
    b_ati = raw_file.get('b_ati')
    b_xti = raw_file.get('b_xti')
    raw_file.close()
    slc = focus_cube(raw_data, cfg, sr0)
    sar = cfg.sar
    v_ground = sar.v_ground
    if v_ground == 'auto':
        v_ground = geo.orbit_to_vel(sar.alt, ground=True)
    proc_file = ProcFile(output_file, 'w', slc.shape)
    proc_file.set('slc*', slc)
    for k, v in (('inc_angle', inc_angle), ('f0', sar.f0), ('num_ch', sar.num_ch),
                 ('ant_L', getattr(sar, 'ant_L_tx', getattr(sar, 'ant_L', 0.0))), ('prf', sar.prf),
                 ('v_ground', v_ground), ('orbit_alt', sar.alt), ('sr0', sr0),
                 ('rg_sampling', sar.rg_bw * sar.over_fs), ('rg_bw', sar.rg_bw), ('b_ati', b_ati),
                 ('b_xti', b_xti)):
        proc_file.set(k, v)
    proc_file.close()
    return slc
