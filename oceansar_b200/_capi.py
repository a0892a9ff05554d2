"""ctypes binding of the C ABI in ``include/oceansar_b200.h``.

The shared library is built in-tree (``oceansar_b200/_lib/liboceansar_b200.so``) by
``oceansar_b200.build``.  There is no fallback: if the library is missing or cannot be
loaded, every entry point raises ``RuntimeError``.
"""
import ctypes
import os

# OCEANSAR_B200_LIB selects another build of the same library (e.g. a debug build).
_LIB_PATH = os.environ.get("OCEANSAR_B200_LIB") or os.path.join(
    os.path.dirname(os.path.abspath(__file__)), "_lib", "liboceansar_b200.so")

OK = 0
ERRORS = {
    -1: (ValueError, "invalid argument"),
    -2: (RuntimeError, "CUDA launch or runtime error"),
    -3: (ValueError, "size beyond the supported range"),
    -4: (NotImplementedError, "option not supported by this build"),
    -5: (TimeoutError, "a bounded device-side wait gave up"),
}

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_flt = ctypes.c_float
c_ptr = ctypes.c_void_p

# name -> argtypes (every function returns int status unless listed in _RESTYPE)
SIGNATURES = {
    "ocs_version": [],
    "ocs_chan_profile_f64": [c_ptr, c_ptr, c_i64, c_dbl, c_dbl, c_ptr, c_int, c_int, c_ptr, c_i64, c_ptr],
    "ocs_chan_profile_rows_f64": [c_ptr, c_ptr, c_i64, c_i64, c_dbl, c_dbl, c_ptr, c_int, c_int, c_ptr,
                                  c_i64, c_ptr],
    "ocs_chan_profile_c64": [c_ptr, c_ptr, c_i64, c_dbl, c_dbl, c_ptr, c_int, c_int, c_ptr, c_i64, c_ptr],
    "ocs_chan_profile_2d_f64": [c_ptr, c_ptr, c_i64, c_i64, c_dbl, c_dbl, c_ptr, c_int, c_int, c_ptr, c_i64,
                                c_ptr],
    "ocs_chan_profile_2d_c64": [c_ptr, c_ptr, c_i64, c_i64, c_dbl, c_dbl, c_ptr, c_int, c_int, c_ptr, c_i64,
                                c_ptr],
    "ocs_surface_workspace_bytes": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
    "ocs_surface_prepare": [ctypes.c_int32, ctypes.c_int32, c_ptr, c_ptr],
    "ocs_surface_update": [c_ptr, c_flt, c_ptr],
    "ocs_surface_update_passes": [c_ptr, c_flt, c_int, c_ptr],
    "ocs_surface_choppy": [c_ptr, c_ptr],
    "ocs_surface_update_noalloc": [c_ptr, c_flt, c_ptr],
    "ocs_surface_blend": [c_i64, ctypes.c_int32, c_ptr, c_ptr, c_ptr, c_flt, c_flt, c_ptr],
    "ocs_pulse": [c_ptr, c_int, c_ptr],
    "ocs_pulse_reset": [c_ptr, c_ptr],
    "ocs_pulse_flush": [c_ptr, c_ptr],
    "ocs_pulse_error": [c_ptr],
    "ocs_pulse_workspace_bytes": [ctypes.c_int32, ctypes.c_int32],
    "ocs_rcs_romeiser": [c_ptr, c_ptr],
    "ocs_field_kodis": [c_ptr, c_ptr],
    "ocs_field_ka": [c_ptr, c_ptr],
    "ocs_skim_upsample": [c_ptr, c_ptr, c_ptr, c_ptr, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                          ctypes.c_int32, c_dbl, c_ptr],
    "ocs_fma_rate": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_ptr, c_ptr],
    "ocs_fft64_workspace_bytes": [c_i64, c_i64],
    "ocs_fft64_rows": [c_ptr, c_i64, c_i64, ctypes.c_int32, c_ptr, c_ptr],
    "ocs_transpose_c128": [c_ptr, c_ptr, c_i64, c_i64, c_i64, c_ptr],
    "ocs_rd_rcmc": [c_ptr, c_i64, ctypes.c_int32, ctypes.c_int32, c_ptr, c_ptr, c_dbl, c_ptr],
    "ocs_rd_azfilter": [c_ptr, c_i64, ctypes.c_int32, ctypes.c_int32, c_ptr, c_ptr],
    "ocs_batch_create": [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(c_ptr)],
    "ocs_batch_destroy": [c_ptr],
    "ocs_batch_set": [c_ptr, ctypes.c_int32, c_ptr, c_ptr],
    "ocs_batch_clear": [c_ptr, ctypes.c_int32, c_ptr],
    "ocs_batch_step": [c_ptr, ctypes.c_int32, c_ptr],
    "ocs_batch_launches_per_step": [c_ptr],
    "ocs_batch_counters": [c_ptr, c_ptr, c_ptr],
}
_RESTYPE = {"ocs_version": ctypes.c_char_p, "ocs_surface_workspace_bytes": ctypes.c_int64,
            "ocs_pulse_workspace_bytes": ctypes.c_int64, "ocs_fft64_workspace_bytes": ctypes.c_int64}

_lib = None


def lib_path():
    return _LIB_PATH


def load():
    """Load the library (once).  Raises RuntimeError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise RuntimeError("oceansar_b200 CUDA library not built (%s); run `python -m "
                           "oceansar_b200.build`" % _LIB_PATH)
    lib = ctypes.CDLL(_LIB_PATH)
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = _RESTYPE.get(name, ctypes.c_int)
    _lib = lib
    return lib


def call(name, *args):
    """Call an entry point and raise on a non-zero status."""
    fn = getattr(load(), name)
    st = fn(*args)
    if st != OK:
        exc, msg = ERRORS.get(st, (RuntimeError, "unknown status"))
        raise exc("%s: %s (status %d)" % (name, msg, st))
    return st
