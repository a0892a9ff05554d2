"""Import-time shims that let the unmodified OCEANSAR reference run in this container.

Used ONLY by ``make_golden.py`` (fixture generation). Nothing here is imported by the
package, the GPU tests, ``smoke()`` or ``bench.py``: the reference tree does not exist on
GPU machines.

The reference needs a few modules that are absent from this image; each shim below
replaces one of them without touching the reference sources:

1. ``matplotlib`` / ``matplotlib.pyplot``: a no-op object (plots are side effects only).
2. ``netCDF4.Dataset``: an in-memory variable store; files written by
   ``RawFile`` / ``OceanStateFile`` are kept in ``NC_STORE`` keyed by path.
3. ``numexpr.evaluate``: the same expression evaluated by numpy in the caller's frame
   (``exp``, ``arctan``, ``ones_like``, ``sum(..., axis=0)``); FP64 throughout, so the
   result only differs from numexpr by rounding order.
4. ``np.complex`` / ``np.float`` / ``np.int`` aliases that numpy 2 removed
   (used e.g. by ``oceansar/nrcs/kodis.py:55``).
5. ``spread.models['cos2s']``: the reference's ``oceansar/spread/cos2s.py:13-19`` raises on
   arrays (``or`` between boolean arrays).  Its evident intent, G = cos^2(theta)/pi inside
   |theta| <= pi/2 and 0 outside, is registered in its place; the product implements the
   same function.
7. ``drama.io.cfg``: the DopSCA generator reads its .cfg through the (absent) drama
   package; the reference's own ``oceansar.ocs_io.cfg`` module parses the same format and
   is registered as ``drama.io.cfg``.
6. ``mpi4py.MPI``: a one-process communicator (rank 0 of 1) for
   ``surfaces/balancer.py``; ``bcast`` returns its argument and ``Scatterv`` copies the
   root's float32 buffer into the receive buffer (with one process the whole surface is
   the root's share); ``Reduce`` copies (the sum over one process).
"""
import os
import sys
import types

import numpy as np

# where the reference source tree is checked out (read-only); set OCEANSAR_REF_ROOT
REF_ROOT = os.environ.get("OCEANSAR_REF_ROOT", "/root/reference")

NC_STORE = {}


class _NoOp:
    def __getattr__(self, name):
        return self

    def __call__(self, *args, **kwargs):
        return self

    def __iter__(self):
        return iter(())


class _NCVar:
    def __init__(self, dtype, dims, ds):
        self.dtype = np.dtype(dtype)
        self.dims = tuple(dims) if isinstance(dims, (tuple, list)) else (dims,)
        shape = tuple(ds.dims[d] for d in self.dims)
        self.data = np.zeros(shape, dtype=self.dtype)

    @property
    def shape(self):
        return self.data.shape

    def __setitem__(self, key, value):
        if self.data.shape == ():
            self.data = np.asarray(value, dtype=self.dtype).reshape(())
        else:
            self.data[key] = value

    def __getitem__(self, key):
        if self.data.shape == ():
            return self.data.copy()
        return self.data[key]


class _Dataset:
    def __init__(self, file_name, mode="r", format=None):
        if mode == "r":
            if file_name not in NC_STORE:
                raise RuntimeError("no such in-memory file: %s" % file_name)
            src = NC_STORE[file_name]
            self.dims = dict(src.dims)
            self.variables = dict(src.variables)
        else:
            self.dims = {}
            self.variables = {}
            NC_STORE[file_name] = self

    def createDimension(self, name, size):
        self.dims[name] = int(size)

    def createVariable(self, name, dtype, dims=()):
        v = _NCVar(dtype, dims, self)
        self.variables[name] = v
        return v

    def close(self):
        pass


def _ne_evaluate(expr, local_dict=None, global_dict=None, **kw):
    frame = sys._getframe(1)
    ns = {}
    ns.update(frame.f_globals if global_dict is None else global_dict)
    ns.update(frame.f_locals if local_dict is None else local_dict)
    ns.update({"exp": np.exp, "arctan": np.arctan, "ones_like": np.ones_like,
               "sum": lambda a, axis=None: np.sum(a, axis=axis),
               "sin": np.sin, "cos": np.cos, "sqrt": np.sqrt, "abs": np.abs,
               "real": np.real, "imag": np.imag})
    return eval(expr, {"__builtins__": {}}, ns)


def cos2s_restated(k, theta, U_10, fetch):
    """Intended cos^2 spreading of ``oceansar/spread/cos2s.py:13-19``."""
    theta = np.asarray(theta)
    g = np.cos(theta) ** 2 / np.pi
    return np.where((theta < -np.pi / 2.0) | (theta > np.pi / 2.0), 0.0, g)


class _Comm:
    def Get_size(self):
        return 1

    def Get_rank(self):
        return 0

    def bcast(self, obj, root=0):
        return obj

    def Scatterv(self, sendbuf, recvbuf, root=0):
        src = np.asarray(sendbuf[0])
        if src.dtype != np.float32:
            raise TypeError("MPI.FLOAT scatter of a %s buffer" % src.dtype)
        dst = recvbuf[0]
        dst.reshape(-1)[:] = src.reshape(-1)[:dst.size]

    def Reduce(self, sendbuf, recvbuf, op=None, root=0):
        recvbuf[...] = sendbuf


def install():
    """Install the shims and put the reference on ``sys.path``; returns the package."""
    if "matplotlib" not in sys.modules or not isinstance(sys.modules["matplotlib"], types.ModuleType):
        pass
    mpl = types.ModuleType("matplotlib")
    plt = _NoOp()
    mpl.pyplot = plt
    mpl.cm = _NoOp()
    mpl.mlab = _NoOp()
    mpl.use = lambda *a, **k: None
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    sys.modules["matplotlib.cm"] = mpl.cm
    sys.modules["matplotlib.mlab"] = mpl.mlab

    nc = types.ModuleType("netCDF4")
    nc.Dataset = _Dataset
    sys.modules["netCDF4"] = nc

    ne = types.ModuleType("numexpr")
    ne.evaluate = _ne_evaluate
    sys.modules["numexpr"] = ne

    for alias, typ in (("complex", complex), ("float", float), ("int", int)):
        if not hasattr(np, alias):
            setattr(np, alias, typ)
    if not hasattr(np, "trapz"):
        np.trapz = np.trapezoid

    mpi = types.ModuleType("mpi4py")
    mpi.MPI = types.SimpleNamespace(COMM_WORLD=_Comm(), FLOAT="MPI_FLOAT", SUM="MPI_SUM")
    sys.modules["mpi4py"] = mpi
    sys.modules["mpi4py.MPI"] = mpi.MPI

    if REF_ROOT not in sys.path:
        sys.path.insert(0, REF_ROOT)
    import oceansar  # noqa: F401
    from oceansar.ocs_io import cfg as ocs_cfg
    drama = types.ModuleType("drama")
    drama_io = types.ModuleType("drama.io")
    drama_io.cfg = ocs_cfg
    drama.io = drama_io
    sys.modules["drama"] = drama
    sys.modules["drama.io"] = drama_io
    sys.modules["drama.io.cfg"] = ocs_cfg
    from oceansar import spread
    spread.models["cos2s"] = cos2s_restated
    return oceansar
