"""Drop-in for ``oceansar/radarsim/range_profile.py`` on the GPU.

``calc_sinc_vec`` builds the oversampled sinc table (``range_profile.py:15-19``, a 161-entry
host table).  ``chan_profile_numba`` has the reference's signature and semantics
(``range_profile.py:83-116``): it accumulates in place into ``output`` and returns None.
The accumulation runs in the sm_100a kernel behind ``ocs_chan_profile_f64`` /
``ocs_chan_profile_rows_f64``; numpy arguments are copied to the GPU and the result copied
back into ``output``, CUDA tensors are used in place.
"""
import numpy as np
import torch

from .. import _capi, _device


def calc_sinc_vec(n_sinc_samples=6, sinc_ovs=10, Fs=1.0):
    n_sinc_bins = int(sinc_ovs * n_sinc_samples + 1)
    sinc_bins = np.arange(n_sinc_bins) * 1. / sinc_ovs - n_sinc_samples / 2
    return np.array(np.sinc(sinc_bins / Fs), dtype=np.float32)


def chan_profile_numba(srg, scene, binsize, min_sr, sinc_vec, n_sinc_samples, sinc_ovs, output,
                       rg_only=False, stream=None):
    """``output += range profile of (srg, scene)``; see ``include/oceansar_b200.h``.

    ``srg``/``scene``: float64 / complex128 of the same shape: flattened, or a 2-D
    [ny, nx] surface (summed column-wise by ``ocs_chan_profile_2d_f64``; same result up to
    summation order), or [naz, npts] rows with ``rg_only``; ``output``: complex128 [nbins]
    (or [naz, nbins]) numpy array or CUDA tensor, updated in place.
    """
    n_sinc_samples = int(n_sinc_samples)
    sinc_ovs = int(sinc_ovs)
    if np.size(sinc_vec) < n_sinc_samples * sinc_ovs + 1:
        raise ValueError("sinc_vec needs n_sinc_samples*sinc_ovs + 1 entries")
    if isinstance(output, torch.Tensor):
        if output.dtype != torch.complex128 or not output.is_contiguous() or not output.is_cuda:
            raise TypeError("output tensor must be a contiguous complex128 CUDA tensor")
        out_d = output
    else:
        if output.dtype != np.complex128:
            raise TypeError("output must be complex128 (the reference's c16 signature)")
        out_d = _device.to_device(output, np.complex128)
    srg_d = _device.to_device(srg, np.float64)
    scene_d = _device.to_device(scene, np.complex128)
    sinc_d = _device.to_device(sinc_vec, np.float32)
    if srg_d.shape != scene_d.shape:
        raise ValueError("srg and scene must have the same shape")
    sp = _device.stream_ptr(stream)
    if rg_only:
        if srg_d.dim() != 2 or out_d.dim() != 2 or out_d.shape[0] != srg_d.shape[0]:
            raise ValueError("rg_only needs srg/scene [naz, npts] and output [naz, nbins]")
        naz, npts = srg_d.shape
        _capi.call("ocs_chan_profile_rows_f64", _device.ptr(srg_d), _device.ptr(scene_d), naz, npts,
                   float(binsize), float(min_sr), _device.ptr(sinc_d), n_sinc_samples, sinc_ovs,
                   _device.ptr(out_d), out_d.shape[1], sp)
    elif srg_d.dim() == 2:
        # a [ny][nx] surface: the column-walking kernel (same sum, other summation order)
        _capi.call("ocs_chan_profile_2d_f64", _device.ptr(srg_d), _device.ptr(scene_d), srg_d.shape[0],
                   srg_d.shape[1], float(binsize), float(min_sr), _device.ptr(sinc_d), n_sinc_samples,
                   sinc_ovs, _device.ptr(out_d), out_d.numel(), sp)
    else:
        _capi.call("ocs_chan_profile_f64", _device.ptr(srg_d), _device.ptr(scene_d), srg_d.numel(),
                   float(binsize), float(min_sr), _device.ptr(sinc_d), n_sinc_samples, sinc_ovs,
                   _device.ptr(out_d), out_d.numel(), sp)
    if not isinstance(output, torch.Tensor):
        output[...] = out_d.cpu().numpy().reshape(output.shape)
    return None

