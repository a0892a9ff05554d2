"""Device-buffer plumbing: PyTorch tensors as CUDA buffers for the C ABI.

Kernels only ever see raw device pointers.  Host (numpy) inputs are copied to the current
CUDA device; CUDA tensors are used in place.  No CPU execution path exists.
"""
import numpy as np
import torch

_NP2TORCH = {
    np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
    np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128,
    np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
    np.dtype(np.uint16): torch.uint16 if hasattr(torch, "uint16") else torch.int16,
}


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("oceansar_b200 needs a CUDA device (B200, sm_100a); none is available")
    return torch.device("cuda", torch.cuda.current_device())


def device():
    return require_cuda()


def stream_ptr(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes_void(s.cuda_stream)


def ctypes_void(v):
    import ctypes
    return ctypes.c_void_p(int(v))


def ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


def to_device(a, dtype, contiguous=True):
    """Return a CUDA tensor of numpy ``dtype`` holding ``a`` (numpy, scalar or tensor)."""
    dev = require_cuda()
    tdt = _NP2TORCH[np.dtype(dtype)]
    if isinstance(a, torch.Tensor):
        t = a.to(device=dev, dtype=tdt)
    else:
        arr = np.ascontiguousarray(np.asarray(a, dtype=dtype))
        t = torch.from_numpy(arr).to(dev, non_blocking=False)
    return t.contiguous() if contiguous else t


def is_cuda_tensor(a):
    return isinstance(a, torch.Tensor) and a.is_cuda


def empty(shape, dtype):
    return torch.empty(shape, dtype=_NP2TORCH[np.dtype(dtype)], device=require_cuda())


def zeros(shape, dtype):
    return torch.zeros(shape, dtype=_NP2TORCH[np.dtype(dtype)], device=require_cuda())
