"""Host-side mirror of the reference's `field` API over the C ABI.

The reference owns the state in a Fortran `field` object and advances it
with `field%integrate(dt)` (src/field/field_class.f:61-72), whose body is
`td_integrator%integrate` (src/td_integrator/rungekutta3rdtvd/
td_integrator_class.f:103-161).  `Field` keeps the same names and argument
meanings, but the state lives in HBM and every operation is a call into
libdim2d.so (include/dim2d.h).  There is no CPU fallback: if the library
or a CUDA device is missing, construction raises.

Boundary presets follow src/config/library_config.py:41-230 (choices,
types, order); 'periodic_xy' selects the legacy periodic operator
(src/boundary_conditions/periodic_xy/bc_operators_class.f) and
'wall_xy' puts the wall operator on all four sides.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_dp = ctypes.POINTER(ctypes.c_double)

# include/dim2d.h
PERIODIC_X, PERIODIC_Y, REFLECTION_X, REFLECTION_Y, HEDSTROM, WALL = 0, 1, 2, 3, 4, 7
BC_NODES, BC_FLUXES, BC_TIMEDEV, BC_FLUX_AND_NODE = 0, 1, 2, 3
SW_CORNER, SE_CORNER, NW_CORNER, NE_CORNER, S_EDGE, E_EDGE, W_EDGE, N_EDGE = range(1, 9)
SIDES = ("N", "S", "E", "W", "NE", "NW", "SE", "SW")
_SECTION = {"SW": SW_CORNER, "SE": SE_CORNER, "NW": NW_CORNER, "NE": NE_CORNER,
            "S": S_EDGE, "E": E_EDGE, "W": W_EDGE, "N": N_EDGE}
FP64, MIXED = 0, 1

ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "unsupported configuration",
          4: "device allocation refused", 5: "wall root not bracketed/converged",
          6: "device wait timed out", 7: "state not uploaded",
          8: "state not finite"}


class Dim2dError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("dim2d error %d (%s): %s" % (code, ERRORS.get(code, "?"), msg))
        self.code = code


class Params(ctypes.Structure):
    """dim2d_params (include/dim2d.h)."""
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

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _preset(name):
    """(bc_choice[8], bc_type[8], bc_order[8]) indexed N,S,E,W,NE,NW,SE,SW."""
    if name == "periodic_xy":
        ch = dict(N=PERIODIC_Y, S=PERIODIC_Y, E=PERIODIC_X, W=PERIODIC_X, NE=PERIODIC_X,
                  NW=PERIODIC_X, SE=PERIODIC_X, SW=PERIODIC_X)
        order = ["S", "N", "SW", "SE", "W", "E", "NW", "NE"]
    elif name == "wall_xy":
        ch = {s: WALL for s in SIDES}
        order = ["SW", "S", "SE", "W", "E", "NW", "N", "NE"]
    elif name == "hedstrom_xy":
        ch = {s: HEDSTROM for s in SIDES}
        order = ["SW", "S", "SE", "W", "E", "NW", "N", "NE"]
    elif name == "wall_S_reflection":  # library_config.py:102-115
        ch = dict(N=REFLECTION_Y, S=WALL, E=REFLECTION_X, W=REFLECTION_X, NE=REFLECTION_X,
                  NW=REFLECTION_X, SE=REFLECTION_X, SW=REFLECTION_X)
        order = ["W", "E", "S", "N", "SW", "SE", "NW", "NE"]
    elif name == "wall_S_open":  # library_config.py:118-131
        ch = dict(N=HEDSTROM, S=WALL, E=HEDSTROM, W=HEDSTROM, NE=HEDSTROM, NW=HEDSTROM,
                  SE=WALL, SW=WALL)
        order = ["SW", "S", "SE", "W", "E", "NW", "N", "NE"]
    elif name == "half_wall_S_open":  # library_config.py:134-150, the reference's default
        ch = dict(N=HEDSTROM, S=WALL, E=HEDSTROM, W=REFLECTION_X, NE=HEDSTROM,
                  NW=REFLECTION_X, SE=WALL, SW=REFLECTION_X)
        order = ["W", "S", "SE", "SW", "E", "N", "NE", "NW"]
    elif name == "reflection_xy":
        ch = dict(N=REFLECTION_Y, S=REFLECTION_Y, E=REFLECTION_X, W=REFLECTION_X,
                  NE=REFLECTION_Y, NW=REFLECTION_Y, SE=REFLECTION_Y, SW=REFLECTION_Y)
        order = ["W", "E", "SW", "S", "SE", "NW", "N", "NE"]
    else:
        raise ValueError("unknown boundary preset %r" % name)
    bc_choice = [ch[s] for s in SIDES]
    bc_type = [bc_type_of(c) for c in bc_choice]
    bc_order = [_SECTION[s] for s in order]
    return bc_choice, bc_type, bc_order


def bc_type_of(choice):
    """library_config.py:256-282 get_bc_type."""
    if choice in (REFLECTION_X, REFLECTION_Y, PERIODIC_X, PERIODIC_Y):
        return BC_NODES
    if choice == WALL:
        return BC_FLUX_AND_NODE
    if choice == HEDSTROM:
        return BC_TIMEDEV
    raise ValueError("unknown bc choice %r" % choice)


_lib = None


def library():
    """Load libdim2d.so (built in-tree).  Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        raise ImportError("libdim2d.so not built (%s); run python -m dim2d_finite_volume_b200.build"
                          % path)
    L = ctypes.CDLL(path)
    H = ctypes.c_void_p
    sig = {
        "dim2d_default_params": (None, [ctypes.POINTER(Params)]),
        "dim2d_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                        ctypes.POINTER(H)]),
        "dim2d_upload": (ctypes.c_int, [H, _dp, _dp, _dp, ctypes.c_double]),
        "dim2d_step": (ctypes.c_int, [H, ctypes.c_double, ctypes.c_int]),
        "dim2d_time_dev": (ctypes.c_int, [H, _dp]),
        "dim2d_apply_bc_on_nodes": (ctypes.c_int, [H]),
        "dim2d_download": (ctypes.c_int, [H, _dp, ctypes.POINTER(ctypes.c_double)]),
        "dim2d_download_async": (ctypes.c_int, [H, _dp, ctypes.POINTER(ctypes.c_double)]),
        "dim2d_copy_done": (ctypes.c_int, [H]),
        "dim2d_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
        "dim2d_host_free": (ctypes.c_int, [ctypes.c_void_p]),
        "dim2d_cfl_dt": (ctypes.c_int, [H, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
        "dim2d_set_stream": (ctypes.c_int, [H, ctypes.c_void_p]),
        "dim2d_sync": (ctypes.c_int, [H]),
        "dim2d_device_state": (ctypes.c_int, [H, ctypes.POINTER(_dp), ctypes.POINTER(ctypes.c_int)]),
        "dim2d_launch_count": (ctypes.c_longlong, [H]),
        "dim2d_profile": (ctypes.c_int, [H, ctypes.c_int]),
        "dim2d_profile_read": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_longlong)]),
        "dim2d_set_variant": (ctypes.c_int, [H, ctypes.c_int]),
        "dim2d_set_graphs": (ctypes.c_int, [H, ctypes.c_int]),
        "dim2d_get_variant": (ctypes.c_int, [H]),
        "dim2d_autotune": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_int), _dp]),
        "dim2d_destroy": (ctypes.c_int, [H]),
        "dim2d_ini_coordinates": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4
                                  + [_dp, _dp]),
        "dim2d_last_error": (ctypes.c_char_p, []),
        "dim2d_version": (ctypes.c_char_p, []),
        "dim2d_time_dev_masked": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_double, ctypes.c_double,
                                                 ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_int), ctypes.c_void_p,
                                                 ctypes.c_void_p]),
        "dim2d_rk_stage_masked": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise Dim2dError(rc, library().dim2d_last_error().decode())


def default_params(**overrides):
    p = Params()
    library().dim2d_default_params(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def pinned_empty(shape):
    """float64 array in pinned (page-locked) host memory, for
    Field.download_async and fast uploads; freed with the array."""
    import weakref
    n = int(np.prod(shape))
    p = ctypes.c_void_p()
    _check(library().dim2d_host_alloc(max(8, n * 8), ctypes.byref(p)))
    buf = (ctypes.c_double * max(1, n)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=np.float64, count=n).reshape(shape)
    weakref.finalize(arr, library().dim2d_host_free, p)
    return arr


# ---- buffer-layer grids (bf_layer): masked interior operators on device
# arrays the caller owns (addresses as integers, e.g. torch.Tensor.data_ptr())
NO_PT, INTERIOR_PT, BC_INTERIOR_PT, BC_PT = 0, 1, 2, 3  # parameters_bf_layer.f:41-44


def time_dev_masked(params, nx, ny, nodes_ptr, grdpts_id_ptr, dx, dy, x_borders, y_borders,
                    time_dev_ptr, stream=0):
    """td_operators%compute_time_dev_nopt's interior part on the device:
    time_dev at the interior_pt points inside the (1-based) borders."""
    arr = ctypes.c_int * 2
    _check(library().dim2d_time_dev_masked(ctypes.byref(params), nx, ny, nodes_ptr,
                                           grdpts_id_ptr, dx, dy, arr(*x_borders),
                                           arr(*y_borders), time_dev_ptr, stream))


def rk_stage_masked(stage, nx, ny, nodes_ptr, nodes_tmp_ptr, time_dev_ptr, grdpts_id_ptr, dt,
                    x_borders, y_borders, stream=0):
    """compute_1st/2nd/3rd_step_nopt on the device, in place."""
    arr = ctypes.c_int * 2
    _check(library().dim2d_rk_stage_masked(stage, nx, ny, nodes_ptr, nodes_tmp_ptr,
                                           time_dev_ptr, grdpts_id_ptr, dt, arr(*x_borders),
                                           arr(*y_borders), stream))


def _ptr(a):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


class Field:
    """One DIM field resident in HBM; mirrors field_abstract / field.

    nodes are numpy arrays shaped (4, ny, nx) -- the memory of the Fortran
    nodes(nx,ny,4)."""

    def __init__(self, nx, ny, bc="periodic_xy", params=None, precision=FP64,
                 bc_choice=None, bc_type=None, bc_order=None):
        L = library()
        if bc is not None and bc_choice is None:
            bc_choice, bc_type, bc_order = _preset(bc)
        self.nx, self.ny = int(nx), int(ny)
        self.params = params if params is not None else default_params()
        self.bc_choice, self.bc_type, self.bc_order = list(bc_choice), list(bc_type), list(bc_order)
        arr = ctypes.c_int * 8
        h = ctypes.c_void_p()
        _check(L.dim2d_create(ctypes.byref(self.params), self.nx, self.ny, arr(*self.bc_choice),
                              arr(*self.bc_type), arr(*self.bc_order), int(precision),
                              ctypes.byref(h)))
        self._h = h
        self.x_map = None
        self.y_map = None

    # --- field_abstract_class.f:148-198 / 286-315 -----------------------
    def ini(self, nodes, x_map, y_map, time=0.0):
        """Upload the initial nodes (ghosts as the reference's ini leaves them)."""
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        if nodes.shape != (4, self.ny, self.nx):
            raise ValueError("nodes must be shaped (4, ny, nx) = (4, %d, %d)" % (self.ny, self.nx))
        self.x_map = np.ascontiguousarray(x_map, dtype=np.float64)
        self.y_map = np.ascontiguousarray(y_map, dtype=np.float64)
        _check(library().dim2d_upload(self._h, _ptr(nodes), _ptr(self.x_map), _ptr(self.y_map),
                                      float(time)))

    upload = ini

    # --- field_class.f:61-72 ---------------------------------------------
    def integrate(self, dt, nsteps=1):
        _check(library().dim2d_step(self._h, float(dt), int(nsteps)))

    # --- field_abstract_class.f:360-379 ----------------------------------
    def compute_time_dev(self):
        out = np.empty((4, self.ny, self.nx))
        _check(library().dim2d_time_dev(self._h, _ptr(out)))
        return out

    # --- field_abstract_class.f:447-463 ----------------------------------
    def apply_bc_on_nodes(self):
        _check(library().dim2d_apply_bc_on_nodes(self._h))

    def download_async(self, out):
        """Queue a copy of the state into `out` (a pinned (4, ny, nx) array,
        see pinned_empty) and return the state's time at once; the copy
        overlaps the next integrate().  Read `out` after copy_done() or
        sync()."""
        if out.shape != (4, self.ny, self.nx):
            raise ValueError("out must have shape (4, ny, nx)")
        t = ctypes.c_double()
        _check(library().dim2d_download_async(self._h, _ptr(out), ctypes.byref(t)))
        return t.value

    def copy_done(self):
        rc = library().dim2d_copy_done(self._h)
        if rc < 0:
            _check(-rc)
        return rc == 1

    def download(self, out=None):
        out = np.empty((4, self.ny, self.nx)) if out is None else out
        t = ctypes.c_double()
        _check(library().dim2d_download(self._h, _ptr(out), ctypes.byref(t)))
        self._time = t.value
        return out

    @property
    def nodes(self):
        return self.download()

    @property
    def time(self):
        t = ctypes.c_double()
        tmp = np.empty((4, self.ny, self.nx))
        _check(library().dim2d_download(self._h, _ptr(tmp), ctypes.byref(t)))
        return t.value

    def cfl_dt(self, cfl):
        dt = ctypes.c_double()
        _check(library().dim2d_cfl_dt(self._h, float(cfl), ctypes.byref(dt)))
        return dt.value

    def set_stream(self, stream_ptr):
        _check(library().dim2d_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def sync(self):
        _check(library().dim2d_sync(self._h))

    def device_state(self):
        p = _dp()
        pitch = ctypes.c_int()
        _check(library().dim2d_device_state(self._h, ctypes.byref(p), ctypes.byref(pitch)))
        return ctypes.cast(p, ctypes.c_void_p).value, pitch.value

    def profile(self, enable=True):
        _check(library().dim2d_profile(self._h, int(bool(enable))))

    def profile_read(self):
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        _check(library().dim2d_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    @property
    def launches(self):
        return library().dim2d_launch_count(self._h)

    NUM_VARIANTS = 7

    @property
    def variant(self):
        """Stage-kernel variant in use (0 = CTA tiles, 1..5 = warp strips)."""
        return library().dim2d_get_variant(self._h)

    @variant.setter
    def variant(self, v):
        _check(library().dim2d_set_variant(self._h, int(v)))

    def set_graphs(self, enable):
        """Replay pairs of steps from a captured CUDA graph (default on)."""
        _check(library().dim2d_set_graphs(self._h, 1 if enable else 0))

    def autotune(self, measure=False):
        """Time every stage-kernel variant on the resident field and keep
        the fastest; returns (variant, per-variant ms or None)."""
        chosen = ctypes.c_int()
        times = np.zeros(self.NUM_VARIANTS) if measure else None
        ptr = times.ctypes.data_as(_dp) if measure else None
        _check(library().dim2d_autotune(self._h, ctypes.byref(chosen), ptr))
        return chosen.value, times

    def close(self):
        if getattr(self, "_h", None):
            library().dim2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
