"""dim2d_step_noalloc: the time step for callers that cannot allocate.

Some hosts cannot call cudaMalloc while they step a field: their HBM is
handed out by their own pool, or the loop must not synchronise the device.
dim2d_step_noalloc runs the same RK3 stages with its stage copies in a
fixed file-scope device array.  This test checks, through the C ABI, that
two calls in a row give the same state as the allocating entry point
(dim2d_create / dim2d_upload / dim2d_step / dim2d_download), within the
1e-12 normwise tolerance of the one-step parity tests, for both accepted
configurations (periodic_xy, hedstrom_xy) at an even and an odd width, and
that fields larger than the fixed limit and configurations with a node
boundary pass are refused.

The file sorts last so a run that stops at the first failure has run every
other test before this one.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import open_case, periodic_case, stable_dt

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _lib():
    from dim2d_finite_volume_b200 import field as F
    L = F.library()
    fn = L.dim2d_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(F.Params), ctypes.c_int, ctypes.c_int,
                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                   ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, F._dp, F._dp,
                   ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
    return F, L


def _rel(a, b):
    out = []
    for k in range(4):
        den = np.abs(b[k]).max()
        num = np.abs(a[k] - b[k]).max()
        out.append(num / den if den > 0 else num)
    return max(out)


def _case(preset, n, ny):
    if preset == "periodic_xy":
        nx, nyy, x_map, y_map, q = periodic_case(n, ny, seed=11)
        # periodic ghosts as field%ini leaves them
        px, py = nx - 4, nyy - 4
        q[:, :, 0:2] = q[:, :, px:px + 2]
        q[:, :, nx - 2:] = q[:, :, 2:4]
        q[:, 0:2, :] = q[:, py:py + 2, :]
        q[:, nyy - 2:, :] = q[:, 2:4, :]
    else:
        nx, nyy, x_map, y_map, q = open_case(n, ny, seed=12, radius=0.15)
    return nx, nyy, x_map, y_map, np.ascontiguousarray(q)


# an even and an odd width: the caller's pitch is nx, so the odd one puts
# every other row off a 16-byte boundary
@pytest.mark.parametrize("preset", ["periodic_xy", "hedstrom_xy"])
@pytest.mark.parametrize("n,ny", [(60, 44), (61, 44)])
def test_noalloc_matches_allocating_path_two_calls(preset, n, ny):
    import torch
    F, L = _lib()
    nx, ny, x_map, y_map, q = _case(preset, n, ny)
    dt = stable_dt(q, x_map, y_map)
    steps = (5, 4)  # odd then even: the result leaves the scratch both ways

    # reference: the allocating entry points
    want = []
    with F.Field(nx, ny, bc=preset) as fld:
        fld.ini(q, x_map, y_map)
        for n_ in steps:
            fld.integrate(dt, n_)
            want.append(fld.download())

    # the no-allocation entry point, on a caller-owned device buffer
    p = F.default_params()
    bc_choice, bc_type, bc_order = F._preset(preset)
    arr = ctypes.c_int * 8
    dev = torch.from_numpy(q.copy()).cuda()
    stream = torch.cuda.current_stream()
    for n_, ref in zip(steps, want):
        rc = L.dim2d_step_noalloc(ctypes.byref(p), nx, ny, arr(*bc_choice), arr(*bc_type),
                                  arr(*bc_order), ctypes.c_void_p(dev.data_ptr()),
                                  F._ptr(x_map), F._ptr(y_map), dt, n_,
                                  ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.dim2d_last_error().decode()
        torch.cuda.synchronize()
        got = dev.cpu().numpy()
        assert np.isfinite(got).all()
        # open fields integrate their ghost cells too: compare every cell
        assert _rel(got, ref) <= TOL


def test_noalloc_refuses_configurations_with_a_node_pass():
    import torch
    F, L = _lib()
    nx, ny, x_map, y_map, q = periodic_case(40, 36)
    p = F.default_params()
    bc_choice, bc_type, bc_order = F._preset("wall_S_reflection")
    arr = ctypes.c_int * 8
    dev = torch.from_numpy(q.copy()).cuda()
    rc = L.dim2d_step_noalloc(ctypes.byref(p), nx, ny, arr(*bc_choice), arr(*bc_type),
                              arr(*bc_order), ctypes.c_void_p(dev.data_ptr()), F._ptr(x_map),
                              F._ptr(y_map), 1e-6, 1, None)
    assert rc == 3  # DIM2D_ERR_UNSUPPORTED
    assert np.array_equal(dev.cpu().numpy(), q)


def test_noalloc_rejects_fields_beyond_the_limit():
    import torch
    F, L = _lib()
    p = F.default_params()
    bc_choice, bc_type, bc_order = F._preset("periodic_xy")
    arr = ctypes.c_int * 8
    nx, ny = 1028, 1028  # 1056784 cells > DIM2D_NOALLOC_MAX_CELLS
    x = np.linspace(0.0, 1.0, nx)
    y = np.linspace(0.0, 1.0, ny)
    dev = torch.zeros(8, device="cuda", dtype=torch.float64)
    rc = L.dim2d_step_noalloc(ctypes.byref(p), nx, ny, arr(*bc_choice), arr(*bc_type),
                              arr(*bc_order), ctypes.c_void_p(dev.data_ptr()), F._ptr(x),
                              F._ptr(y), 1e-6, 1, None)
    assert rc == 1  # DIM2D_ERR_ARG
    assert "DIM2D_NOALLOC_MAX_CELLS" in L.dim2d_last_error().decode()
