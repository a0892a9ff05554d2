"""``ProcFile`` (oceansar/ocs_io/processed.py): the SLC file written by sar_focus, with the
reference's dimensions (ch, pol, az, rg), variables and units, in the netCDF classic
format (``netcdf3.Dataset``)."""
import time

from .netcdf import NETCDFHandler
from .netcdf3 import Dataset

_SCALARS = (('inc_angle', '[deg]'), ('f0', '[Hz]'), ('ant_L', '[m]'), ('prf', '[Hz]'), ('v_ground', '[m/s]'),
            ('orbit_alt', '[m]'), ('sr0', '[m]'), ('rg_sampling', '[Hz]'), ('rg_bw', '[Hz]'))


class ProcFile(NETCDFHandler):
    def __init__(self, file_name, mode, proc_dim=None, format='NETCDF4'):
        self.__file__ = Dataset(file_name, mode, format)
        if mode != 'w':
            return
        f = self.__file__
        f.description = 'OCEANSAR Processed SLC Data File'
        f.history = 'Created ' + time.ctime(time.time())
        f.source = 'OCEANSAR Simulator'
        if not proc_dim:
            raise ValueError('Processed raw data dimensions are needed when creating a new file!')
        for n, size in zip(('ch_dim', 'pol_dim', 'az_dim', 'rg_dim'), proc_dim):
            f.createDimension(n, size)
        f.createVariable('num_ch', 'i4')
        for part in ('slc_r', 'slc_i'):
            f.createVariable(part, 'f8', ('ch_dim', 'pol_dim', 'az_dim', 'rg_dim')).units = '[]'
        for n, units in _SCALARS:
            f.createVariable(n, 'f8').units = units
        for n in ('b_ati', 'b_xti'):
            f.createVariable(n, 'f8', ('ch_dim',)).units = '[m]'
