"""``sarraw``: the entry of the reference's MPI raw-data generator
(``oceansar/radarsim/sar_raw.py:53-618``).

That script differs from ``sar_raw_nompi`` in how it gets the surface: an
``OceanSurfaceBalancer`` synthesises it at multiples of the ocean time step ``dt`` of the
.cfg and interpolates the fields linearly for every pulse in between, and the surface rows
are scattered over MPI processes.  Here one GPU holds the whole surface, so ``sarraw`` is
the GPU generator with the balancer's time interpolation at ``ocean.dt``; the pulse
physics, the noise and the raw file are those of ``sar_raw_nompi.sar_raw``.
"""
from ..ocs_io.cfg import ConfigFile
from .sar_raw_nompi import sar_raw


def sarraw(cfg_file, output_file, ocean_file, reuse_ocean_file, errors_file, reuse_errors_file,
           plot_save=True, precision='f64'):
    cfg = ConfigFile(cfg_file)
    return sar_raw(cfg, output_file, ocean_file, reuse_ocean_file, errors_file, reuse_errors_file,
                   plot_save=plot_save, precision=precision, surface_dt=cfg.ocean.dt)
