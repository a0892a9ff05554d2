"""The drop-in writes the reference's file formats: sar_raw's raw file and the ocean state
file as netCDF classic files (read back with scipy's independent reader)."""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_sar_raw_writes_netcdf_raw_and_state(tmp_path):
    from oceansar_b200.radarsim.sar_raw_nompi import sar_raw
    raw_p, ocean_p = str(tmp_path / "raw.nc"), str(tmp_path / "ocean.nc")
    np.random.seed(0)
    total_raw, nrcs = sar_raw(os.path.join(G, "cfg", "c1small.cfg"), raw_p, ocean_p, False, None, False)
    g = netcdf_file(raw_p, 'r', mmap=False)
    got = g.variables['raw_data_r'][:] + 1j * g.variables['raw_data_i'][:]
    np.testing.assert_array_equal(got, total_raw)
    np.testing.assert_array_equal(g.variables['NRCS_avg'][:], nrcs)
    ref = np.load(os.path.join(G, "sar_raw_c1small.npz"))
    assert float(g.variables['sr0'].getValue()) == pytest.approx(float(ref['sr0']), rel=1e-15)
    assert np.linalg.norm(got - ref['raw']) / np.linalg.norm(ref['raw']) < 1e-4
    g.close()
    s = netcdf_file(ocean_p, 'r', mmap=False)
    coefs = s.variables['wave_coefs_r'][:] + 1j * s.variables['wave_coefs_i'][:]
    np.testing.assert_allclose(coefs, ref['wave_coefs'], rtol=0, atol=1e-3)
    s.close()


def test_surface_state_roundtrip(tmp_path):
    from oceansar_b200.surfaces import OceanSurface
    np.random.seed(4)
    s = OceanSurface()
    s.init(128., 96., 1., 1., 'auto', 'elfouhaily', 'elfouhaily', 0.4, 500e3, 9., 0.1, 0.2,
           compute=['D', 'Diff', 'Diff2'])
    p = str(tmp_path / "state.nc")
    s.save(p)
    r = OceanSurface()
    r.load(p, compute=['D', 'Diff', 'Diff2'])
    assert (r.Nx, r.Ny) == (s.Nx, s.Ny)
    np.testing.assert_array_equal(r.wave_coefs, s.wave_coefs)
    s.t = 1.3
    r.t = 1.3
    for f in ('Dz', 'Diffx', 'Diffxy'):
        assert np.linalg.norm(getattr(r, f) - getattr(s, f)) <= 1e-5 * np.linalg.norm(getattr(s, f))
