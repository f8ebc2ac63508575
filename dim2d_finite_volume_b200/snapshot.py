"""Snapshots and restarts in the reference's netCDF layout, written on the
host from the device state.

The reference writes one netCDF file per output time
(src/io_operators/nf90_operators/nf90_operators_module.f:979-1353): dimensions
time(1), x(nx), y(ny); coordinate variables time, x, y (with units, axis and
long_name); the conservative variables mass, momentum_x, momentum_y and
energy (nodes(:,:,k), with units and long_name) over Fortran dimensions
(time, x, y) -- (y, x, time) in the file's C order -- and global attributes
describing the run; restarts read these files back
(nf90_operators_read_module.f).  This module writes and reads that layout
itself, in the classic 64-bit-offset netCDF format (published format
specification: magic "CDF\\x02", big-endian header of dimension, attribute
and variable lists, then the variables' data), so no netCDF library is
needed; any netCDF reader opens the files.

`Snapshotter` overlaps output with stepping: it queues an asynchronous copy
of the state into pinned host memory (Field.download_async), keeps stepping,
and writes the file from a background thread once the copy has landed.
"""
import struct
import threading

import numpy as np

NC_DIMENSION, NC_VARIABLE, NC_ATTRIBUTE = 10, 11, 12
NC_BYTE, NC_CHAR, NC_SHORT, NC_INT, NC_FLOAT, NC_DOUBLE = 1, 2, 3, 4, 5, 6
_NP = {NC_BYTE: ">i1", NC_CHAR: "S1", NC_SHORT: ">i2", NC_INT: ">i4", NC_FLOAT: ">f4",
       NC_DOUBLE: ">f8"}
_SIZE = {NC_BYTE: 1, NC_CHAR: 1, NC_SHORT: 2, NC_INT: 4, NC_FLOAT: 4, NC_DOUBLE: 8}

# nf90_operators_module.f:993-1005 and pmodel_eq_class.f get_var_name /
# get_var_longname / get_var_unit
VARIABLES = (("mass", "mass density", "(kg/m3)/(kg/m3)"),
             ("momentum_x", "momentum density along the x-axis", "(kg/(m2.s))/(kg/(m2.s))"),
             ("momentum_y", "momentum density along the y-axis", "(kg/(m2.s))/(kg/(m2.s))"),
             ("energy", "total energy density", "(J/m3)/(J.m3)"))
COORDS = (("time", "s/s", None, "reduced time"),
          ("x", "m/m", "X", "reduced x-coordinate"),
          ("y", "m/m", "Y", "reduced y-coordinate"))


def _pad(b):
    return b + b"\0" * (-len(b) % 4)


def _name(s):
    b = s.encode()
    return struct.pack(">i", len(b)) + _pad(b)


def _attr_value(v):
    if isinstance(v, str):
        b = v.encode()
        return NC_CHAR, struct.pack(">i", len(b)) + _pad(b)
    a = np.atleast_1d(np.asarray(v))
    if a.dtype.kind in "iub":
        return NC_INT, struct.pack(">i", a.size) + _pad(a.astype(">i4").tobytes())
    return NC_DOUBLE, struct.pack(">i", a.size) + a.astype(">f8").tobytes()


def _attr_list(attrs):
    if not attrs:
        return b"\0" * 8
    out = struct.pack(">ii", NC_ATTRIBUTE, len(attrs))
    for k, v in attrs.items():
        t, payload = _attr_value(v)
        out += _name(k) + struct.pack(">i", t) + payload
    return out


def write_netcdf(path, nodes, x_map, y_map, time, global_attrs=None):
    """One snapshot: nodes (4, ny, nx) FP64 (the memory of nodes(nx,ny,4)),
    x_map (nx), y_map (ny), time; global_attrs: extra run description."""
    nodes = np.asarray(nodes, dtype=np.float64)
    ny, nx = nodes.shape[1], nodes.shape[2]
    dims = [("time", 1), ("x", nx), ("y", ny)]
    # (name, dim ids, attributes, data)
    vars_ = []
    for (name, units, axis, long_name), dim, data in zip(
            COORDS, (0, 1, 2), (np.array([time]), np.asarray(x_map), np.asarray(y_map))):
        att = {"units": units}
        if axis:
            att["axis"] = axis
        att["long_name"] = long_name
        vars_.append((name, [dim], att, np.asarray(data, dtype=np.float64)))
    for k, (name, long_name, units) in enumerate(VARIABLES):
        vars_.append((name, [2, 1, 0], {"long_name": long_name, "units": units},
                      nodes[k].reshape(ny, nx, 1)))

    def header(begins):
        h = b"CDF\x02" + struct.pack(">i", 0)
        h += struct.pack(">ii", NC_DIMENSION, len(dims))
        for n, l in dims:
            h += _name(n) + struct.pack(">i", l)
        h += _attr_list(global_attrs or {})
        h += struct.pack(">ii", NC_VARIABLE, len(vars_))
        for (name, dimids, att, data), begin in zip(vars_, begins):
            h += _name(name) + struct.pack(">i", len(dimids))
            h += b"".join(struct.pack(">i", d) for d in dimids)
            h += _attr_list(att)
            h += struct.pack(">ii", NC_DOUBLE, data.size * 8) + struct.pack(">q", begin)
        return h

    hlen = len(header([0] * len(vars_)))
    begins, off = [], hlen
    for v in vars_:
        begins.append(off)
        off += v[3].size * 8
    with open(path, "wb") as fh:
        fh.write(header(begins))
        for v in vars_:
            fh.write(np.ascontiguousarray(v[3], dtype=">f8").tobytes())


def read_netcdf(path):
    """Classic / 64-bit-offset netCDF (non-record variables): returns
    dict(dims, attrs, vars: name -> (dim names, attrs, array))."""
    buf = open(path, "rb").read()
    if buf[:3] != b"CDF" or buf[3] not in (1, 2):
        raise ValueError("%s: not a classic netCDF file" % path)
    off_size = 8 if buf[3] == 2 else 4
    pos = 8

    def i4():
        nonlocal pos
        v = struct.unpack_from(">i", buf, pos)[0]
        pos += 4
        return v

    def name():
        nonlocal pos
        n = i4()
        s = buf[pos:pos + n].decode()
        pos += n + (-n % 4)
        return s

    def attrs():
        nonlocal pos
        tag, n = i4(), i4()
        out = {}
        for _ in range(n if tag == NC_ATTRIBUTE else 0):
            k = name()
            t, cnt = i4(), i4()
            nb = cnt * _SIZE[t]
            raw = buf[pos:pos + nb]
            pos += nb + (-nb % 4)
            if t == NC_CHAR:
                out[k] = raw.decode()
            else:
                a = np.frombuffer(raw, dtype=_NP[t]).astype(_NP[t][1:])
                out[k] = a[0] if a.size == 1 else a
        return out

    tag, ndims = i4(), i4()
    dims = []
    for _ in range(ndims if tag == NC_DIMENSION else 0):
        dims.append((name(), i4()))
    gatts = attrs()
    tag, nvars = i4(), i4()
    vars_ = {}
    for _ in range(nvars if tag == NC_VARIABLE else 0):
        vn = name()
        nd = i4()
        dimids = [i4() for _ in range(nd)]
        va = attrs()
        t = i4()
        i4()  # vsize
        begin = struct.unpack_from(">q" if off_size == 8 else ">i", buf, pos)[0]
        pos += off_size
        shape = tuple(dims[d][1] for d in dimids)
        n = int(np.prod(shape)) if shape else 1
        a = np.frombuffer(buf, dtype=_NP[t], count=n, offset=begin).reshape(shape)
        vars_[vn] = ([dims[d][0] for d in dimids], va, a.astype(_NP[t][1:]))
    return dict(dims=dict(dims), attrs=gatts, vars=vars_)


def read_snapshot(path):
    """(nodes (4, ny, nx), x_map, y_map, time, global attrs) of a snapshot,
    ready for Field.ini -- the restart path (nf90_operators_read_module.f)."""
    d = read_netcdf(path)
    v = d["vars"]
    nodes = np.stack([v[name][2][:, :, 0] for name, _, _ in VARIABLES])
    return (np.ascontiguousarray(nodes), v["x"][2].copy(), v["y"][2].copy(),
            float(v["time"][2][0]), d["attrs"])


def run_attrs(field, dt=None, title="dim2d-b200 snapshot"):
    """Global attributes in the reference's header (nf90_write_header:
    title, source, domain extent, dt) for a Field."""
    p = field.params
    a = {"title": title, "source": "dim2d-b200 (sm_100a)",
         "x_min": float(field.x_map[2]), "x_max": float(field.x_map[-3]),
         "y_min": float(field.y_map[2]), "y_max": float(field.y_map[-3]),
         "Re": p.re, "We": p.we, "Pr": p.pr, "cv_r": p.cv_r, "viscous_r": p.viscous_r}
    if dt is not None:
        a["dt"] = float(dt)
    return a


class Snapshotter:
    """Overlapped output: snapshot(path) queues an asynchronous copy of the
    field's state into one of two pinned host buffers and returns at once;
    the caller keeps stepping.  Copies that have landed (checked by
    snapshot() and poll(), on the caller's thread -- the only thread that
    touches the field) are written to their files by background threads.
    close() waits for the copies and the writes."""

    def __init__(self, field, attrs=None):
        from .field import pinned_empty
        self.field = field
        self.attrs = attrs or {}
        self.bufs = [pinned_empty((4, field.ny, field.nx)) for _ in range(2)]
        self.turn = 0
        self.pending = []              # (buffer, path, time): copy queued
        self.threads = [None, None]    # file writers per buffer
        self.errors = []

    def _write(self, k, path, t):
        try:
            write_netcdf(path, self.bufs[k], self.field.x_map, self.field.y_map, t, self.attrs)
        except Exception as e:  # reported by close()
            self.errors.append(e)

    def poll(self, wait=False):
        """Start the writers of landed copies (wait: sync the field first)."""
        if not self.pending:
            return
        if wait:
            self.field.sync()
        elif not self.field.copy_done():  # the latest copy; earlier ones precede it
            return
        for k, path, t in self.pending:
            th = threading.Thread(target=self._write, args=(k, path, t), daemon=True)
            th.start()
            self.threads[k] = th
        self.pending = []

    def snapshot(self, path):
        self.poll()
        k = self.turn
        self.turn ^= 1
        if any(p[0] == k for p in self.pending):  # that buffer's copy must land first
            self.poll(wait=True)
        if self.threads[k] is not None:  # and its file be written
            self.threads[k].join()
            self.threads[k] = None
        t = self.field.download_async(self.bufs[k])
        self.pending.append((k, path, t))
        return t

    def close(self):
        self.poll(wait=True)
        for th in self.threads:
            if th is not None:
                th.join()
        self.threads = [None, None]
        if self.errors:
            raise self.errors[0]
