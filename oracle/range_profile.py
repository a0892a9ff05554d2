"""Oracle (test infrastructure only): sinc table and facet-to-range-bin accumulation.

``calc_sinc_vec`` restates ``oceansar/radarsim/range_profile.py:15-19``.
``chan_profile`` restates ``chan_profile_numba`` (``range_profile.py:83-116``) by calling
the C loop in ``range_profile.c`` (``profile_integrator``, ``:22-49``), built on first
use into ``oracle/_build/`` with ``-O2 -ffp-contract=off`` so that no multiply-add is
fused and the serial sums match numba's bit for bit.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_SO = os.path.join(_BUILD, "liboracle_rp.so")
_lib = None


def build(force=False):
    """Compile ``range_profile.c`` into ``oracle/_build/liboracle_rp.so``."""
    src = os.path.join(_HERE, "range_profile.c")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        os.makedirs(_BUILD, exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                               "-shared", "-o", _SO, src, "-lm"])
    return _SO


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build())
        dp = ctypes.POINTER(ctypes.c_double)
        fp = ctypes.POINTER(ctypes.c_float)
        lib.oracle_chan_profile.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                            fp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int64]
        lib.oracle_chan_profile.restype = None
        lib.oracle_chan_profile_rows.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64,
                                                 ctypes.c_double, ctypes.c_double, fp, ctypes.c_int,
                                                 ctypes.c_int, dp, ctypes.c_int64]
        lib.oracle_chan_profile_rows.restype = None
        _lib = lib
    return _lib


def calc_sinc_vec(n_sinc_samples=6, sinc_ovs=10, Fs=1.0):
    """``range_profile.py:15-19``: float32 np.sinc sampled at (i/ovs - n/2)/Fs, i <= n*ovs."""
    n_sinc_bins = int(sinc_ovs * n_sinc_samples + 1)
    sinc_bins = np.arange(n_sinc_bins) * 1. / sinc_ovs - n_sinc_samples / 2
    return np.array(np.sinc(sinc_bins / Fs), dtype=np.float32)


def chan_profile(srg, scene, binsize, min_sr, sinc_vec, n_sinc_samples, sinc_ovs, output,
                 rg_only=False):
    """In-place ``output += profile(srg, scene)`` exactly as ``range_profile.py:83-116``."""
    lib = _load()
    srg = np.ascontiguousarray(srg, dtype=np.float64)
    scene = np.ascontiguousarray(scene, dtype=np.complex128)
    pulse = np.ascontiguousarray(sinc_vec, dtype=np.float32)
    if output.dtype != np.complex128 or not output.flags.c_contiguous:
        raise TypeError("output must be a C-contiguous complex128 array")
    dp = ctypes.POINTER(ctypes.c_double)
    fp = ctypes.POINTER(ctypes.c_float)
    if rg_only:
        naz, npts = scene.shape
        lib.oracle_chan_profile_rows(srg.ctypes.data_as(dp), scene.ctypes.data_as(dp), naz, npts,
                                     float(binsize), float(min_sr), pulse.ctypes.data_as(fp),
                                     int(n_sinc_samples), int(sinc_ovs),
                                     output.ctypes.data_as(dp), output.shape[-1])
    else:
        lib.oracle_chan_profile(srg.ctypes.data_as(dp), scene.ctypes.data_as(dp), srg.size,
                                float(binsize), float(min_sr), pulse.ctypes.data_as(fp),
                                int(n_sinc_samples), int(sinc_ovs),
                                output.ctypes.data_as(dp), output.size)
