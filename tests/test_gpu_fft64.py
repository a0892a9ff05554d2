"""Complex128 power-of-two FFTs of the SAR processor (``ocs_fft64_rows``) and the batched
transpose (``ocs_transpose_c128``) against numpy.fft.

Lengths cover the single-CTA shared-memory transform (2 .. 8192, every radix-8 / 4 / 2
pass split) and the four-step path (16384, 65536, 2^18), forward and inverse; bar 1e-13
of the spectrum's largest magnitude (float64 rounding grows like log n).
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run(x, inverse):
    from oceansar_b200 import _capi
    lib = _capi.load()
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    n = x.shape[-1]
    nrows = x.size // n
    ws = int(lib.ocs_fft64_workspace_bytes(nrows, n))
    assert ws >= 0
    scratch = torch.empty(max(ws // 16, 1), dtype=torch.complex128, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_fft64_rows", t.data_ptr(), nrows, n, int(inverse), scratch.data_ptr() if ws else None, st)
    return t.cpu().numpy()


@pytest.mark.parametrize("n,rows", [(1, 3), (2, 5), (4, 3), (8, 7), (16, 2), (32, 3), (64, 9), (128, 4), (512, 3),
                                    (1024, 5), (2048, 3), (4096, 2), (8192, 3), (16384, 2), (65536, 2),
                                    (1 << 18, 1)])
@pytest.mark.parametrize("inverse", [False, True], ids=["fwd", "inv"])
def test_rows_against_numpy(n, rows, inverse):
    rs = np.random.default_rng(n + rows)
    x = rs.standard_normal((rows, n)) + 1j * rs.standard_normal((rows, n))
    got = _run(x, inverse)
    ref = np.fft.ifft(x, axis=-1) if inverse else np.fft.fft(x, axis=-1)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-13, (n, rows, inverse, err)


def test_transpose_and_azimuth_transform():
    """A [pol][az][rg] cube transformed along az through its transpose equals numpy's
    FFT along axis 1; ragged (non-multiple-of-32) matrix sizes."""
    from oceansar_b200 import _capi
    from oceansar_b200.radarsim.sar_processor import _fft_az
    rs = np.random.default_rng(7)
    x = rs.standard_normal((2, 45, 77)) + 1j * rs.standard_normal((2, 45, 77))
    t = torch.from_numpy(x).cuda()
    tt = torch.empty((2, 77, 45), dtype=torch.complex128, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.call("ocs_transpose_c128", t.data_ptr(), tt.data_ptr(), 2, 45, 77, st)
    assert np.array_equal(tt.cpu().numpy(), x.transpose(0, 2, 1))
    y = rs.standard_normal((2, 256, 64)) + 1j * rs.standard_normal((2, 256, 64))
    ty = torch.from_numpy(y).cuda()
    _fft_az(ty, False)
    ref = np.fft.fft(y, axis=1)
    assert np.abs(ty.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-13
    _fft_az(ty, True)
    assert np.abs(ty.cpu().numpy() - y).max() < 1e-13


def test_rejects_non_power_of_two_and_missing_scratch():
    from oceansar_b200 import _capi
    lib = _capi.load()
    t = torch.zeros(3 * 100, dtype=torch.complex128, device="cuda")
    assert lib.ocs_fft64_workspace_bytes(3, 100) == -1
    assert lib.ocs_fft64_rows(ctypes.c_void_p(t.data_ptr()), 3, 100, 0, None, None) == -1
    big = torch.zeros(16384, dtype=torch.complex128, device="cuda")
    assert lib.ocs_fft64_rows(ctypes.c_void_p(big.data_ptr()), 1, 16384, 0, None, None) == -1
