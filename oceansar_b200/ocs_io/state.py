"""``OceanStateFile`` (oceansar/ocs_io/state.py): the ocean state file of OceanSurface.save.

Same dimensions (y, x), variables, units and global attributes as the reference; written
in the netCDF classic format (``netcdf3.Dataset``).  Nx / Ny, unsigned 32-bit in the
reference, are stored as 32-bit integers (the classic format has no unsigned types).
"""
import time

from .netcdf import NETCDFHandler
from .netcdf3 import Dataset

_FLOATS = (('Lx', '[m]'), ('Ly', '[m]'), ('dx', '[m]'), ('dy', '[m]'), ('wind_dir', '[deg]'),
           ('wind_dir_eff', '[deg]'), ('wind_fetch', '[m]'), ('wind_U', '[m/s]'), ('wind_U_eff', '[m/s]'),
           ('current_mag', '[]'), ('current_dir', '[deg]'), ('swell_enable', '[]'), ('swell_ampl', '[m]'),
           ('swell_dir', '[deg]'), ('swell_wl', '[m]'), ('swell_ph0', '[rad]'), ('choppy_enable', '[]'))


class OceanStateFile(NETCDFHandler):
    def __init__(self, file_name, mode, ocean_dim=None, format='NETCDF4'):
        self.__file__ = Dataset(file_name, mode, format)
        if mode != 'w':
            return
        f = self.__file__
        f.description = 'OCEANSAR Library Ocean State File'
        f.history = 'Created ' + time.ctime(time.time())
        f.source = 'OCEANSAR Library'
        if not ocean_dim:
            raise ValueError('Ocean dimensions are needed when creating new file!')
        f.createDimension('y_dim', ocean_dim[0])
        f.createDimension('x_dim', ocean_dim[1])
        f.createVariable('Nx', 'u4').units = '[]'
        f.createVariable('Ny', 'u4').units = '[]'
        for n, units in _FLOATS:
            f.createVariable(n, 'f4').units = units
        for n in ('kx', 'ky'):
            f.createVariable(n, 'f4', ('y_dim', 'x_dim')).units = '[rad/m]'
        for n in ('wave_coefs_r', 'wave_coefs_i'):
            f.createVariable(n, 'f8', ('y_dim', 'x_dim')).units = '[]'
