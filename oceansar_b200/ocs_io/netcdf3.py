"""netCDF classic files (64-bit offset format, "CDF-2") in numpy.

The reference writes its raw and ocean-state files with the netCDF4 library
(``ocs_io/raw.py``, ``ocs_io/state.py``), which is not available here.  This module writes
and reads the netCDF classic data model, which every netCDF reader (netCDF4-python,
netCDF-C, scipy.io.netcdf_file, xarray) opens: fixed-size dimensions, variables of type
byte / char / short / int / float / double, global and per-variable attributes.  The
format follows the published netCDF classic specification: a big-endian header (magic
``CDF\\x02``, dimension list, global attributes, variable list with 8-byte data offsets)
followed by each variable's data, padded to 4 bytes.  No record (unlimited) dimension.

The API is the subset of ``netCDF4.Dataset`` the reference uses: ``Dataset(path, mode)``,
``createDimension``, ``createVariable(name, dtype, dims)``, attribute assignment on the
dataset and on variables, ``variables[name][:] = value`` / ``[:]`` and ``close``.
"""
import struct

import numpy as np

NC_BYTE, NC_CHAR, NC_SHORT, NC_INT, NC_FLOAT, NC_DOUBLE = 1, 2, 3, 4, 5, 6
_TAG_DIM, _TAG_VAR, _TAG_ATT = 10, 11, 12
_NP = {NC_BYTE: '>i1', NC_CHAR: 'S1', NC_SHORT: '>i2', NC_INT: '>i4', NC_FLOAT: '>f4', NC_DOUBLE: '>f8'}
_SIZE = {NC_BYTE: 1, NC_CHAR: 1, NC_SHORT: 2, NC_INT: 4, NC_FLOAT: 4, NC_DOUBLE: 8}


def _nc_type(dtype):
    """netCDF classic type of a numpy dtype (unsigned 32-bit integers are stored as int)."""
    d = np.dtype(dtype)
    if d.kind == 'f':
        return NC_DOUBLE if d.itemsize == 8 else NC_FLOAT
    if d.kind in 'iu':
        return {1: NC_BYTE, 2: NC_SHORT}.get(d.itemsize, NC_INT)
    if d.kind in 'SU':
        return NC_CHAR
    if d.kind == 'b':
        return NC_BYTE
    raise TypeError('no netCDF classic type for %s' % d)


def _pad4(n):
    return (4 - n % 4) % 4


def _name(s):
    b = s.encode('utf-8')
    return struct.pack('>i', len(b)) + b + b'\0' * _pad4(len(b))


def _att_bytes(value):
    if isinstance(value, (str, bytes)):
        b = value.encode('utf-8') if isinstance(value, str) else value
        return struct.pack('>ii', NC_CHAR, len(b)) + b + b'\0' * _pad4(len(b))
    a = np.atleast_1d(np.asarray(value))
    t = _nc_type(a.dtype)
    raw = a.astype(_NP[t]).tobytes()
    return struct.pack('>ii', t, a.size) + raw + b'\0' * _pad4(len(raw))


def _att_list(atts):
    if not atts:
        return struct.pack('>ii', 0, 0)
    out = struct.pack('>ii', _TAG_ATT, len(atts))
    for k, v in atts.items():
        out += _name(k) + _att_bytes(v)
    return out


class Variable(object):
    def __init__(self, ds, name, nc_type, dims):
        object.__setattr__(self, '_ds', ds)
        object.__setattr__(self, 'name', name)
        object.__setattr__(self, '_type', nc_type)
        object.__setattr__(self, 'dimensions', tuple(dims))
        object.__setattr__(self, '_atts', {})
        shape = tuple(ds.dimensions[d] for d in dims)
        object.__setattr__(self, '_data', np.zeros(shape, dtype=_NP[nc_type]).astype(_NP[nc_type].replace('>', '=')))

    @property
    def shape(self):
        return self._data.shape

    @property
    def dtype(self):
        return self._data.dtype

    def ncattrs(self):
        return list(self._atts)

    def __setattr__(self, k, v):
        self._atts[k] = v

    def __getattr__(self, k):
        try:
            return self.__dict__['_atts'][k]
        except KeyError:
            raise AttributeError(k)

    def __setitem__(self, key, value):
        if self._ds._mode == 'r':
            raise IOError('dataset opened read-only')
        if self._data.ndim == 0:                   # scalar variables take var[:] = value
            self._data[()] = np.asarray(value).reshape(())
        else:
            self._data[key] = value

    def __getitem__(self, key):
        return self._data[()] if self._data.ndim == 0 else self._data[key]

    def getValue(self):
        return self._data[()]


class Dataset(object):
    """A netCDF classic file; ``mode`` 'w' (create, written at ``close``) or 'r'.

    ``format`` is accepted for call compatibility; every file is written as
    NETCDF3_64BIT_OFFSET."""

    def __init__(self, filename, mode='r', format='NETCDF3_64BIT_OFFSET'):
        object.__setattr__(self, '_path', filename)
        object.__setattr__(self, '_mode', mode)
        object.__setattr__(self, 'dimensions', {})
        object.__setattr__(self, 'variables', {})
        object.__setattr__(self, '_atts', {})
        object.__setattr__(self, 'file_format', 'NETCDF3_64BIT_OFFSET')
        if mode == 'r':
            self._read()
        elif mode != 'w':
            raise ValueError("mode must be 'r' or 'w'")

    # ---- attributes ------------------------------------------------------------------
    def __setattr__(self, k, v):
        self._atts[k] = v

    def __getattr__(self, k):
        try:
            return self.__dict__['_atts'][k]
        except KeyError:
            raise AttributeError(k)

    def ncattrs(self):
        return list(self._atts)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    # ---- definition ------------------------------------------------------------------
    def createDimension(self, name, size):
        if size is None or int(size) < 0:
            raise ValueError('only fixed-size dimensions are supported')
        self.dimensions[name] = int(size)
        return name

    def createVariable(self, name, datatype, dimensions=()):
        if isinstance(dimensions, str):
            dimensions = (dimensions,)
        for d in dimensions:
            if d not in self.dimensions:
                raise KeyError('unknown dimension %s' % d)
        v = Variable(self, name, _nc_type(datatype), dimensions)
        self.variables[name] = v
        return v

    # ---- writing -----------------------------------------------------------------------
    def close(self):
        if self._mode == 'w':
            self._write()
            object.__setattr__(self, '_mode', 'closed')

    def _write(self):
        dims = list(self.dimensions.items())
        dim_index = {n: i for i, (n, _) in enumerate(dims)}
        head = b'CDF\x02' + struct.pack('>i', 0)
        if dims:
            head += struct.pack('>ii', _TAG_DIM, len(dims))
            for n, size in dims:
                head += _name(n) + struct.pack('>i', size)
        else:
            head += struct.pack('>ii', 0, 0)
        head += _att_list(self._atts)
        variables = list(self.variables.values())

        def var_entries(offsets):
            out = b''
            if not variables:
                return struct.pack('>ii', 0, 0)
            out += struct.pack('>ii', _TAG_VAR, len(variables))
            for v, off in zip(variables, offsets):
                nbytes = int(np.prod(v.shape, dtype=np.int64)) * _SIZE[v._type]
                vsize = min(nbytes + _pad4(nbytes), 0xFFFFFFFF)
                out += _name(v.name) + struct.pack('>i', len(v.dimensions))
                out += b''.join(struct.pack('>i', dim_index[d]) for d in v.dimensions)
                out += _att_list(v._atts) + struct.pack('>iIq', v._type, vsize, off)
            return out

        header_len = len(head) + len(var_entries([0] * len(variables)))
        offsets, pos = [], header_len
        for v in variables:
            offsets.append(pos)
            nbytes = int(np.prod(v.shape, dtype=np.int64)) * _SIZE[v._type]
            pos += nbytes + _pad4(nbytes)
        with open(self._path, 'wb') as f:
            f.write(head + var_entries(offsets))
            for v in variables:
                raw = np.ascontiguousarray(v._data).astype(_NP[v._type]).tobytes()
                f.write(raw + b'\0' * _pad4(len(raw)))

    # ---- reading -----------------------------------------------------------------------
    def _read(self):
        with open(self._path, 'rb') as f:
            buf = f.read()
        if buf[:3] != b'CDF' or buf[3] not in (1, 2):
            raise IOError('%s is not a netCDF classic file' % self._path)
        off_fmt = '>q' if buf[3] == 2 else '>i'
        pos = [8]

        def take(fmt):
            v = struct.unpack_from(fmt, buf, pos[0])
            pos[0] += struct.calcsize(fmt)
            return v[0] if len(v) == 1 else v

        def name():
            n = take('>i')
            s = buf[pos[0]:pos[0] + n].decode('utf-8')
            pos[0] += n + _pad4(n)
            return s

        def atts():
            tag, n = take('>ii')
            out = {}
            for _ in range(n):
                k = name()
                t, cnt = take('>ii')
                raw = buf[pos[0]:pos[0] + cnt * _SIZE[t]]
                pos[0] += cnt * _SIZE[t] + _pad4(cnt * _SIZE[t])
                if t == NC_CHAR:
                    out[k] = raw.decode('utf-8')
                else:
                    a = np.frombuffer(raw, dtype=_NP[t]).astype(_NP[t].replace('>', '='))
                    out[k] = a[0] if a.size == 1 else a
            return out

        tag, n = take('>ii')
        dims = []
        for _ in range(n):
            nm = name()
            dims.append((nm, take('>i')))
            self.dimensions[nm] = dims[-1][1]
        self._atts.update(atts())
        tag, n = take('>ii')
        for _ in range(n):
            nm = name()
            nd = take('>i')
            ids = [take('>i') for _ in range(nd)]
            vatts = atts()
            t, vsize = take('>ii')
            begin = take(off_fmt)
            v = Variable(self, nm, t, [dims[i][0] for i in ids])
            count = int(np.prod(v.shape, dtype=np.int64))
            data = np.frombuffer(buf, dtype=_NP[t], count=count, offset=begin).reshape(v.shape)
            object.__setattr__(v, '_data', data.astype(_NP[t].replace('>', '=')))
            v._atts.update(vatts)
            self.variables[nm] = v


def is_netcdf3(path):
    with open(path, 'rb') as f:
        head = f.read(4)
    return head[:3] == b'CDF' and len(head) == 4 and head[3] in (1, 2)
