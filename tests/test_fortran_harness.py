"""The Fortran drop-in's call sequence, driven from C.

dim2d_finite_volume_b200/fortran/td_integrator_class.f is the reference's
td_integrator_class rebuilt over the C ABI; this image has no Fortran
compiler, so tests/harness/fortran_sequence.c makes the same calls, in the
same order, under the reference driver's loop (sim_dim2d.f:50-92): default
params overwritten with the run's constants, dim2d_create, dim2d_upload,
dim2d_step once per integrate, dim2d_download at the output steps of
detail_print and at the last step.  Every downloaded state is compared
with the oracle advanced from the same initial state (bar 1e-10 normwise).

CPU: the harness compiles and links against include/dim2d.h, libdim2d.so
and the oracle, and without a GPU it fails cleanly (exit 2, the library's
CUDA message).  GPU: the reference's default preset half_wall_S_open with
its default wall heat source, hedstrom_xy and periodic_xy."""
import os
import struct
import subprocess

import numpy as np
import pytest

from tests.helpers import open_case, periodic_case, stable_dt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "harness", "fortran_sequence.c")


@pytest.fixture(scope="module")
def harness(tmp_path_factory, oracle):
    from dim2d_finite_volume_b200 import build as B
    lib_dir = os.path.dirname(B.LIB)
    if not os.path.exists(B.LIB):
        pytest.skip("libdim2d.so not built")
    orc_dir = os.path.dirname(oracle.LIB_PATH)
    exe = str(tmp_path_factory.mktemp("harness") / "fortran_sequence")
    subprocess.check_call(
        ["gcc", "-O2", "-std=c11", "-Wall", "-Werror", SRC, "-I", os.path.join(ROOT, "include"),
         "-I", os.path.join(ROOT, "oracle"), "-L", lib_dir, "-ldim2d", "-L", orc_dir, "-loracle",
         "-Wl,-rpath," + lib_dir, "-Wl,-rpath," + orc_dir, "-lm", "-o", exe])
    return exe


def write_case(path, nodes, x_map, y_map, bc, nt, dt, detail_print, params, precision=0,
               tol=1e-10, time=0.0):
    from dim2d_finite_volume_b200 import field as F
    ch, ty, od = F._preset(bc)
    ny, nx = nodes.shape[1], nodes.shape[2]
    pv = [params.re, params.we, params.pr, params.cv_r, params.viscous_r, params.gravity_ac,
          params.gravity, params.wall_micro_contact_angle, params.wall_heat_source_choice,
          params.wall_maximum_heat_flux, params.wall_heat_source_center,
          params.wall_heat_source_variance, params.obc_eigenqties_strategy,
          params.obc_edge_flux_strategy, params.T0, params.flow_velocity]
    with open(path, "wb") as fh:
        fh.write(struct.pack("<4i", nx, ny, nt, precision))
        fh.write(struct.pack("<8i", *ch) + struct.pack("<8i", *ty) + struct.pack("<8i", *od))
        fh.write(struct.pack("<4d", dt, detail_print, time, tol))
        fh.write(struct.pack("<16d", *[float(v) for v in pv]))
        fh.write(np.ascontiguousarray(x_map, np.float64).tobytes())
        fh.write(np.ascontiguousarray(y_map, np.float64).tobytes())
        fh.write(np.ascontiguousarray(nodes, np.float64).tobytes())


def _params(bc):
    """The test constant set; for the wall preset the reference's default
    wall parameters (parameters_input.f:542-600: 90 degree contact angle,
    Gaussian heat source, maximum flux 0.02, centre 0, variance half the
    heater length 0.0712945354)."""
    from dim2d_finite_volume_b200 import field as F
    p = F.default_params()
    if bc == "half_wall_S_open":
        p.wall_heat_source_choice = 2
        p.wall_maximum_heat_flux = 0.02
        p.wall_heat_source_center = 0.0
        p.wall_heat_source_variance = 0.5 * 0.0712945354
    return p


def _initial(oracle, bc, p):
    """nodes after field%ini (node boundary pass on the oracle)."""
    from dim2d_finite_volume_b200 import field as F
    if bc == "hedstrom_xy":
        nx, ny, x_map, y_map, q = open_case(70, 52, seed=21, radius=0.15)
        return x_map, y_map, q
    nx, ny, x_map, y_map, q = periodic_case(70, 52, radius=0.15, seed=22)
    if bc == "periodic_xy":
        cfg = oracle.make_cfg(nx, ny, periodic=True)
    else:
        ch, ty, od = F._preset(bc)
        cfg = oracle.make_cfg(nx, ny, periodic=False, bc_choice=ch, bc_type=ty, bc_order=od)
    import ctypes
    saved = oracle.get_params()
    op = oracle.Params()
    for name, _ in oracle.Params._fields_:
        setattr(op, name, getattr(p, name))
    oracle.lib().orc_set_params(ctypes.byref(op))
    try:
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)
    finally:
        oracle.lib().orc_set_params(ctypes.byref(saved))
    return x_map, y_map, q


def test_harness_builds_and_fails_cleanly_without_a_gpu(harness, oracle, tmp_path):
    """CPU only: the harness links, and with no CUDA device dim2d_create
    returns an error that the harness reports (exit status 2)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU tests run the harness")
    x_map, y_map, q = _initial(oracle, "periodic_xy", _params("periodic_xy"))
    case = str(tmp_path / "case.bin")
    write_case(case, q, x_map, y_map, "periodic_xy", 2, 1e-6, 0.5, _params("periodic_xy"))
    r = subprocess.run([harness, case], capture_output=True, text=True, timeout=120)
    assert r.returncode == 2, (r.returncode, r.stdout, r.stderr)
    assert "dim2d_create failed" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("bc", ["half_wall_S_open", "hedstrom_xy", "periodic_xy"])
def test_fortran_call_sequence_matches_oracle(harness, oracle, tmp_path, bc):
    p = _params(bc)
    x_map, y_map, q = _initial(oracle, bc, p)
    dt = stable_dt(q, x_map, y_map)
    case = str(tmp_path / "case.bin")
    # 30 steps, output every 4 (detail_print 0.25) and at the last step
    write_case(case, q, x_map, y_map, bc, 30, dt, 0.25, p)
    r = subprocess.run([harness, case], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, (r.stdout, r.stderr)
    assert "8 states compared" in r.stdout
