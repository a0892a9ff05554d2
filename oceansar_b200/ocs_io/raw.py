"""``RawFile`` (oceansar/ocs_io/raw.py:160-250): the raw data file of sar_raw.

Same dimensions (pol, ch, az, rg), variables, units and global attributes as the
reference; written in the netCDF classic format by ``netcdf3.Dataset`` (the reference's
default NETCDF4/HDF5 format needs the netCDF4 library, absent here; every netCDF reader
opens the classic format).
"""
import time

from .netcdf import NETCDFHandler
from .netcdf3 import Dataset

_SCALARS = (('inc_angle', '[deg]'), ('f0', '[Hz]'), ('ant_L', '[m]'), ('prf', '[Hz]'), ('v_ground', '[m/s]'),
            ('orbit_alt', '[m]'), ('sr0', '[m]'), ('rg_sampling', '[Hz]'), ('rg_bw', '[Hz]'))


class RawFile(NETCDFHandler):
    def __init__(self, file_name, mode, raw_dim=None, format='NETCDF4'):
        self.__file__ = Dataset(file_name, mode, format)
        if mode != 'w':
            return
        f = self.__file__
        f.description = 'OCEANSAR SAR Raw Data File'
        f.history = 'Created ' + time.ctime(time.time())
        f.source = 'OCEANSAR Simulator'
        if not raw_dim:
            raise ValueError('Raw data dimensions are needed when creating a new file!')
        if len(raw_dim) == 4:
            for n, size in zip(('pol_dim', 'ch_dim', 'az_dim', 'rg_dim'), raw_dim):
                f.createDimension(n, size)
            f.createVariable('num_ch', 'i4').units = '[]'
            dims = ('pol_dim', 'ch_dim', 'az_dim', 'rg_dim')
        else:
            for n, size in zip(('pol_dim', 'az_dim', 'rg_dim'), raw_dim):
                f.createDimension(n, size)
            dims = ('pol_dim', 'az_dim', 'rg_dim')
        for part in ('raw_data_r', 'raw_data_i'):
            f.createVariable(part, 'f8', dims).units = '[]'
        for n, units in _SCALARS:
            f.createVariable(n, 'f8').units = units
        if len(raw_dim) == 4:
            for n in ('b_ati', 'b_xti'):
                f.createVariable(n, 'f8', ('ch_dim',)).units = '[m]'
        f.createVariable('NRCS_avg', 'f8', ('pol_dim', 'az_dim')).units = '[]'


class DopscaRawFile(NETCDFHandler):
    """``DopscaRawFile`` (oceansar/ocs_io/raw.py:81-157): the DopSCA generator's raw file,
    dimensions (pol, az, rg), with the reference's variables and units."""

    def __init__(self, file_name, mode, raw_dim=None, format='NETCDF4'):
        self.__file__ = Dataset(file_name, mode, format)
        if mode != 'w':
            return
        f = self.__file__
        f.description = 'OCEANSAR SAR Raw Data File'
        f.history = 'Created ' + time.ctime(time.time())
        f.source = 'OCEANSAR Dopsca Simulator'
        if not raw_dim:
            raise ValueError('Raw data dimensions are needed when creating a new file!')
        for n, size in zip(('pol_dim', 'az_dim', 'rg_dim'), raw_dim):
            f.createDimension(n, size)
        for part in ('raw_data_r', 'raw_data_i'):
            f.createVariable(part, 'f8', ('pol_dim', 'az_dim', 'rg_dim')).units = '[]'
        f.createVariable('dop_ref', 'f8', ('rg_dim',)).units = '[Hz]'
        for n, units in (('inc_angle', '[deg]'), ('f0', '[Hz]'), ('ant_L', '[m]'), ('prf', '[Hz]'),
                         ('v_ground', '[m/s]'), ('orbit_alt', '[m]'), ('sr0', '[m]'), ('rg_sampling', '[Hz]'),
                         ('rg_bw', '[Hz]'), ('azimuth', '[deg]'), ('subpulse_length', '[s]'),
                         ('subpulse_bandwidth', '[Hz]')):
            f.createVariable(n, 'f8').units = units
        f.createVariable('NRCS_avg', 'f8', ('pol_dim', 'az_dim')).units = '[]'


class SkimRawFile(NETCDFHandler):
    """``SkimRawFile`` (oceansar/ocs_io/raw.py:6-78): the SKIM generator's raw file,
    dimensions (pol, az, rg), with the reference's variables and units."""

    def __init__(self, file_name, mode, raw_dim=None, format='NETCDF4'):
        self.__file__ = Dataset(file_name, mode, format)
        if mode != 'w':
            return
        f = self.__file__
        f.description = 'OCEANSAR SAR Raw Data File'
        f.history = 'Created ' + time.ctime(time.time())
        f.source = 'OCEANSAR Simulator'
        if not raw_dim:
            raise ValueError('Raw data dimensions are needed when creating a new file!')
        for n, size in zip(('pol_dim', 'az_dim', 'rg_dim'), raw_dim):
            f.createDimension(n, size)
        for part in ('raw_data_r', 'raw_data_i'):
            f.createVariable(part, 'f8', ('pol_dim', 'az_dim', 'rg_dim')).units = '[]'
        f.createVariable('dop_ref', 'f8', ('rg_dim',)).units = '[Hz]'
        for n, units in (('inc_angle', '[deg]'), ('f0', '[Hz]'), ('ant_L', '[m]'), ('prf', '[Hz]'),
                         ('v_ground', '[m/s]'), ('orbit_alt', '[m]'), ('sr0', '[m]'), ('rg_sampling', '[Hz]'),
                         ('rg_bw', '[Hz]'), ('azimuth', '[deg]')):
            f.createVariable(n, 'f8').units = units
        f.createVariable('NRCS_avg', 'f8', ('pol_dim', 'az_dim')).units = '[]'
