"""ctypes loader for the oracle library (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke()
and the CPU-baseline legs of bench.py.  The product never imports this.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_dp = ctypes.POINTER(ctypes.c_double)

# parameters_constant.f:145-176
PERIODIC_X, PERIODIC_Y, REFLECTION_X, REFLECTION_Y, HEDSTROM, WALL = 0, 1, 2, 3, 4, 7
BC_NODES, BC_FLUXES, BC_TIMEDEV, BC_FLUX_AND_NODE = 0, 1, 2, 3
SW_CORNER, SE_CORNER, NW_CORNER, NE_CORNER, S_EDGE, E_EDGE, W_EDGE, N_EDGE = range(1, 9)


class Params(ctypes.Structure):
    _fields_ = [
        ("re", ctypes.c_double), ("we", ctypes.c_double), ("pr", ctypes.c_double),
        ("cv_r", ctypes.c_double), ("viscous_r", ctypes.c_double),
        ("gravity_ac", ctypes.c_int), ("gravity", ctypes.c_double),
        ("wall_micro_contact_angle", ctypes.c_double),
        ("wall_heat_source_choice", ctypes.c_int),
        ("wall_maximum_heat_flux", ctypes.c_double),
        ("wall_heat_source_center", ctypes.c_double),
        ("wall_heat_source_variance", ctypes.c_double),
        ("obc_eigenqties_strategy", ctypes.c_int),
        ("obc_edge_flux_strategy", ctypes.c_int),
        ("T0", ctypes.c_double), ("flow_velocity", ctypes.c_double),
    ]


class Cfg(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("periodic", ctypes.c_int),
        ("bc_choice", ctypes.c_int * 8), ("bc_type", ctypes.c_int * 8),
        ("bc_order", ctypes.c_int * 8),
    ]


def build():
    """Compile the oracle (make in this directory)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None
_fast = None


def _cpu_key():
    """Short key of this host's CPU model (a -march=native build is only
    valid on the CPU it was built for)."""
    import hashlib
    import platform
    model = platform.machine()
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith(("model name", "flags")):
                    model += line
    except OSError:
        pass
    return hashlib.sha1(model.encode()).hexdigest()[:12]


def fast_lib():
    """The timing build of the same sources (-O3 -march=native, same
    rounding order), compiled on first use for this host's CPU.  Used only
    to time the CPU baseline; the -O2 build (lib()) is the checker."""
    global _fast
    if _fast is None:
        path = os.path.join(HERE, "_build", "fast_" + _cpu_key(), "liboracle_fast.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", HERE, "fast",
                                   "FAST_LIB=" + os.path.relpath(path, HERE)])
        _fast = _declare(ctypes.CDLL(path))
        p = get_params()  # the constants set on the checker build
        _fast.orc_set_params(ctypes.byref(p))
    return _fast


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def _declare(L):
    """Declare the C signatures on a loaded oracle library."""
    L.orc_sd_operator.restype = ctypes.c_double
    L.orc_sd_operator.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    L.orc_flux_function.restype = ctypes.c_double
    L.orc_flux_function.argtypes = [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double]
    L.orc_classical_pressure_local.restype = ctypes.c_double
    L.orc_classical_pressure_local.argtypes = [_dp]
    L.orc_speed_of_sound.restype = ctypes.c_double
    L.orc_speed_of_sound.argtypes = [_dp]
    L.orc_compute_time_dev.restype = None
    L.orc_compute_time_dev.argtypes = [ctypes.POINTER(Cfg), ctypes.c_double, _dp, _dp, _dp, _dp]
    L.orc_apply_bc_on_nodes.restype = None
    L.orc_apply_bc_on_nodes.argtypes = [ctypes.POINTER(Cfg), ctypes.c_double, _dp, _dp, _dp, _dp]
    L.orc_integrate.restype = ctypes.c_int
    L.orc_integrate.argtypes = [ctypes.POINTER(Cfg), _dp, _dp, _dp,
                                ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int]
    L.orc_ini_coordinates.restype = None
    L.orc_ini_coordinates.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [_dp, _dp]
    L.orc_set_params.argtypes = [ctypes.POINTER(Params)]
    L.orc_get_params.argtypes = [ctypes.POINTER(Params)]
    L.orc_set_threads.argtypes = [ctypes.c_int]
    L.orc_debug_real.restype = ctypes.c_double
    _ip = ctypes.POINTER(ctypes.c_int)
    L.orc_compute_time_dev_masked.restype = None
    L.orc_compute_time_dev_masked.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _ip,
                                              ctypes.c_double, ctypes.c_double, _ip, _ip, _dp]
    L.orc_rk_stage_masked.restype = None
    L.orc_rk_stage_masked.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                      _ip, ctypes.c_double, _ip, _ip]
    return L


def ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def get_params():
    p = Params()
    lib().orc_get_params(ctypes.byref(p))
    return p


def set_params(**kw):
    p = get_params()
    for k, v in kw.items():
        setattr(p, k, v)
    lib().orc_set_params(ctypes.byref(p))
    if _fast is not None:
        _fast.orc_set_params(ctypes.byref(p))
    return p


def set_threads(n):
    lib().orc_set_threads(int(n))


def make_cfg(nx, ny, periodic=False, bc_choice=None, bc_type=None, bc_order=None):
    c = Cfg()
    c.nx, c.ny, c.periodic = nx, ny, int(bool(periodic))
    for k in range(8):
        c.bc_choice[k] = (bc_choice or [0] * 8)[k]
        c.bc_type[k] = (bc_type or [0] * 8)[k]
        c.bc_order[k] = (bc_order or list(range(1, 9)))[k]
    return c


def ini_coordinates(nx, ny, x_min, x_max, y_min, y_max):
    x = np.zeros(nx)
    y = np.zeros(ny)
    lib().orc_ini_coordinates(nx, ny, x_min, x_max, y_min, y_max, ptr(x), ptr(y))
    return x, y


def compute_time_dev(cfg, t, nodes, x_map, y_map):
    """nodes: C array [4][ny][nx] (Fortran nodes(nx,ny,4))."""
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    td = np.empty_like(nodes)
    lib().orc_compute_time_dev(ctypes.byref(cfg), t, ptr(nodes), ptr(x_map), ptr(y_map), ptr(td))
    return td


def apply_bc_on_nodes(cfg, t, x_map, y_map, nodes_tmp, nodes):
    lib().orc_apply_bc_on_nodes(ctypes.byref(cfg), t, ptr(x_map), ptr(y_map), ptr(nodes_tmp),
                                ptr(nodes))


def integrate(cfg, nodes, x_map, y_map, t, dt, nsteps, fast=False):
    """Advance nodes in place by nsteps RK3 steps; returns the new time.
    fast: on the -O3 -march=native timing build (same results)."""
    tt = ctypes.c_double(t)
    L = fast_lib() if fast else lib()
    rc = L.orc_integrate(ctypes.byref(cfg), ptr(nodes), ptr(x_map), ptr(y_map),
                         ctypes.byref(tt), dt, nsteps)
    if rc != 0:
        raise RuntimeError("oracle integrate failed: %d" % rc)
    return tt.value


def _iptr(a):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def compute_time_dev_masked(nodes, grdpts_id, dx, dy, x_borders, y_borders, time_dev):
    """Masked interior time derivative of a buffer-layer grid, written into
    time_dev at its interior_pt points (nodes [4][ny][nx], grdpts_id
    [ny][nx] int32, borders 1-based inclusive)."""
    ny, nx = grdpts_id.shape
    xb = np.array(x_borders, dtype=np.int32)
    yb = np.array(y_borders, dtype=np.int32)
    lib().orc_compute_time_dev_masked(nx, ny, ptr(nodes), _iptr(grdpts_id), dx, dy, _iptr(xb),
                                      _iptr(yb), ptr(time_dev))


def rk_stage_masked(stage, nodes, nodes_tmp, time_dev, grdpts_id, dt, x_borders, y_borders):
    ny, nx = grdpts_id.shape
    xb = np.array(x_borders, dtype=np.int32)
    yb = np.array(y_borders, dtype=np.int32)
    lib().orc_rk_stage_masked(stage, nx, ny, ptr(nodes), ptr(nodes_tmp), ptr(time_dev),
                              _iptr(grdpts_id), dt, _iptr(xb), _iptr(yb))


def sd_operator(set_id, op, nodes, i, j, dx, dy):
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    ny, nx = nodes.shape[1], nodes.shape[2]
    return lib().orc_sd_operator(set_id, op, ptr(nodes), nx, ny, i, j, dx, dy)


def flux_function(which, nodes, i, j, dx, dy):
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    ny, nx = nodes.shape[1], nodes.shape[2]
    return lib().orc_flux_function(which, ptr(nodes), nx, ny, i, j, dx, dy)


def pressure(q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_classical_pressure_local(ptr(q))


def speed_of_sound(q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_speed_of_sound(ptr(q))


def timedev_with_openbc(nodes, i, j, dir_y, oneside_right, dn, side_right, obc_prim=None):
    """hedstrom_xy_module.f:445-558 at node (i,j) (1-based)."""
    L = lib()
    fn = L.orc_timedev_with_openbc
    fn.restype = None
    fn.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp]
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    ny, nx = nodes.shape[1], nodes.shape[2]
    td = np.zeros(4)
    pp = None
    if obc_prim is not None:
        pp = np.ascontiguousarray(obc_prim, dtype=np.float64)
    fn(ptr(nodes), nx, ny, i, j, int(dir_y), int(oneside_right), dn, int(side_right),
       ptr(pp) if pp is not None else None, ptr(td))
    return td
