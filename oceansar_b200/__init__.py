"""oceansar_b200: B200-native (sm_100a) raw-data generation for OCEANSAR.

A drop-in for the reference's raw-generation path: ``surfaces.OceanSurface``,
``nrcs`` models, ``radarsim.range_profile`` and ``radarsim.sar_raw_nompi.sar_raw`` with the
reference's ``.cfg`` files.  Host code is Python; all per-pulse work runs in hand-written
CUDA kernels reached through the C ABI of ``include/oceansar_b200.h``.
"""
__version__ = "0.1.0"
