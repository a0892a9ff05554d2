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


def test_sar_focus_against_reference(tmp_path):
    """sar_focus on the GPU (own complex128 FFTs + fused phase kernels) against the reference's SLC
    of the same raw cube, through the raw and SLC files."""
    from oceansar_b200.ocs_io import ProcFile, RawFile
    from oceansar_b200.radarsim.sar_processor import sar_focus
    d = np.load(os.path.join(G, "sar_focus.npz"))
    raw_p, slc_p = str(tmp_path / "raw.nc"), str(tmp_path / "slc.nc")
    f = RawFile(raw_p, 'w', raw_dim=d["raw"].shape)
    f.set('raw_data*', d["raw"])
    f.set('sr0', float(d["sr0"]))
    f.set('inc_angle', 35.0)
    f.set('b_ati', [0., 10.])
    f.set('b_xti', [0., 0.])
    f.close()
    slc = sar_focus(os.path.join(G, "cfg", "proc.cfg"), raw_p, slc_p)
    ref = d["slc"]
    assert slc.shape == ref.shape
    assert np.linalg.norm(slc - ref) / np.linalg.norm(ref) < 1e-10
    p = ProcFile(slc_p, 'r')
    np.testing.assert_array_equal(p.get('slc*'), slc.astype(np.complex64))
    g = netcdf_file(slc_p, 'r', mmap=False)
    assert g.dimensions == {'ch_dim': 2, 'pol_dim': 1, 'az_dim': ref.shape[2], 'rg_dim': ref.shape[3]}
    g.close()
