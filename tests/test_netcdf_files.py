"""netCDF classic raw / ocean-state files (no GPU): structure read back by an independent
reader (scipy.io.netcdf_file), our reader on scipy-written files, the reference's variable
sets, units and complex get / set convention."""
import os

import numpy as np
from scipy.io import netcdf_file


def test_rawfile_roundtrip_and_independent_reader(tmp_path):
    from oceansar_b200.ocs_io import RawFile
    p = str(tmp_path / "raw.nc")
    raw = np.random.RandomState(0).randn(2, 3, 5, 7) + 1j * np.random.RandomState(1).randn(2, 3, 5, 7)
    f = RawFile(p, 'w', raw_dim=raw.shape)
    f.set('raw_data*', raw)
    f.set('NRCS_avg', np.arange(10.).reshape(2, 5))
    f.set('inc_angle', 35.0)
    f.set('num_ch', 3)
    f.set('b_ati', [0., 5., 10.])
    f.close()
    with open(p, 'rb') as fh:
        assert fh.read(4) == b'CDF\x02'
    g = netcdf_file(p, 'r', mmap=False)
    assert g.dimensions == {'pol_dim': 2, 'ch_dim': 3, 'az_dim': 5, 'rg_dim': 7}
    np.testing.assert_array_equal(g.variables['raw_data_r'][:], raw.real)
    np.testing.assert_array_equal(g.variables['raw_data_i'][:], raw.imag)
    assert g.variables['raw_data_r'].dimensions == ('pol_dim', 'ch_dim', 'az_dim', 'rg_dim')
    assert g.variables['inc_angle'].getValue() == 35.0 and g.variables['inc_angle'].units == b'[deg]'
    assert int(g.variables['num_ch'].getValue()) == 3
    np.testing.assert_array_equal(g.variables['b_ati'][:], [0., 5., 10.])
    assert g.description == b'OCEANSAR SAR Raw Data File'
    for v in ('f0', 'ant_L', 'prf', 'v_ground', 'orbit_alt', 'sr0', 'rg_sampling', 'rg_bw', 'b_xti', 'NRCS_avg'):
        assert v in g.variables
    g.close()
    r = RawFile(p, 'r')
    np.testing.assert_array_equal(r.get('raw_data*'), raw.astype(np.complex64))
    assert r.get('inc_angle') == 35.0
    r.close()


def test_reader_on_scipy_file(tmp_path):
    from oceansar_b200.ocs_io.netcdf3 import Dataset
    p = str(tmp_path / "s.nc")
    g = netcdf_file(p, 'w')
    g.createDimension('x', 4)
    g.createDimension('y', 2)
    v = g.createVariable('v', 'f4', ('y', 'x'))
    v[:] = np.arange(8, dtype=np.float32).reshape(2, 4)
    v.units = 'm'
    w = g.createVariable('n', 'i4', ('y',))
    w[:] = [7, 8]
    g.title = 'scipy'
    g.close()
    d = Dataset(p, 'r')
    np.testing.assert_array_equal(d.variables['v'][:], np.arange(8, dtype=np.float32).reshape(2, 4))
    assert d.variables['v'].units == 'm' and d.title == 'scipy' and list(d.variables['n'][:]) == [7, 8]


def test_ocean_state_file_variables(tmp_path):
    from oceansar_b200.ocs_io import OceanStateFile
    p = str(tmp_path / "ocean.nc")
    f = OceanStateFile(p, 'w', ocean_dim=(3, 4))
    coefs = (np.arange(12) + 1j * np.arange(12)).reshape(3, 4)
    f.set('wave_coefs*', coefs)
    f.set('Nx', 4)
    f.set('Ny', 3)
    f.set('kx', np.ones((3, 4)))
    f.close()
    g = netcdf_file(p, 'r', mmap=False)
    assert g.dimensions == {'y_dim': 3, 'x_dim': 4}
    np.testing.assert_array_equal(g.variables['wave_coefs_r'][:], coefs.real)
    assert g.variables['kx'].typecode() == 'f' and g.variables['wave_coefs_r'].typecode() == 'd'
    assert int(g.variables['Nx'].getValue()) == 4
    for v in ('Lx', 'Ly', 'dx', 'dy', 'wind_dir', 'wind_dir_eff', 'wind_fetch', 'wind_U', 'wind_U_eff', 'current_mag',
              'current_dir', 'swell_enable', 'swell_ampl', 'swell_dir', 'swell_wl', 'swell_ph0', 'ky',
              'choppy_enable'):
        assert v in g.variables, v
    g.close()
