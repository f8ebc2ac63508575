"""CPU check of the open-boundary kernel's per-cell code (no GPU needed).

tests/emu/emu_open.cu compiles dim2d_open.cu for the host and runs
open_ghost_cell() -- the body of k_open_ghosts -- for every thread index of
the launch and a margin of out-of-range ones, with checked reads and guard
zones around the output.  This pins the index arithmetic (reads in bounds,
writes exactly the ghost ring) and the values (against the oracle) before
the kernel ever runs on a device.
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from tests.helpers import open_case

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def emu():
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "emu_open")
    subprocess.check_call([NVCC, "-std=c++17", "-O1", "-w", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-I", os.path.join(ROOT, "include"),
                           "-o", exe, os.path.join(HERE, "emu", "emu_open.cu")])
    yield exe, d
    shutil.rmtree(d, ignore_errors=True)


@pytest.mark.parametrize("n,ny,seed", [(64, 64, None), (37, 53, 3), (130, 20, 4), (8, 9, 5)])
def test_open_ghost_cells_host_emulation(oracle, emu, n, ny, seed):
    from dim2d_finite_volume_b200 import field as F
    exe, d = emu
    nx, nyy, x_map, y_map, q = open_case(n, ny, seed=seed, radius=0.15)
    bc = F._preset("hedstrom_xy")
    cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                          bc_order=bc[2])
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
    with open(fin, "wb") as fh:
        np.array([nx, nyy], dtype=np.int32).tofile(fh)
        np.array([x_map[1] - x_map[0], y_map[1] - y_map[0], 5.0, 10.0, 20.0, 2.5, -1.5]).tofile(fh)
        q.tofile(fh)
    out = subprocess.check_output([exe, fin, fout]).decode()
    stats = dict(kv.split("=") for kv in out.split())
    assert stats["bad_reads"] == "0" and stats["guard_writes"] == "0", out
    assert stats["written"] == stats["expected"], out
    got = np.fromfile(fout).reshape(4, nyy, nx)
    ghost = np.zeros((nyy, nx), bool)
    ghost[:2] = ghost[-2:] = True
    ghost[:, :2] = ghost[:, -2:] = True
    assert np.array_equal(got[0] != -777.0, ghost)
    for k in range(4):
        den = np.abs(ref[k]).max()
        num = np.abs(got[k][ghost] - ref[k][ghost]).max()
        assert num / den <= 1e-12, (k, num / den)


# open sections (StageArgs::open bits S, N, W, E, SW, SE, NW, NE) of the
# presets with a south wall
MIXED = {"wall_S_open": 2 | 4 | 8 | 64 | 128, "half_wall_S_open": 2 | 8 | 128}


def open_cells(nx, ny, mask):
    g = np.zeros((ny, nx), bool)
    edges = [(slice(0, 2), slice(2, -2)), (slice(-2, None), slice(2, -2)),
             (slice(2, -2), slice(0, 2)), (slice(2, -2), slice(-2, None)),
             (slice(0, 2), slice(0, 2)), (slice(0, 2), slice(-2, None)),
             (slice(-2, None), slice(0, 2)), (slice(-2, None), slice(-2, None))]
    for s, sl in enumerate(edges):
        if mask >> s & 1:
            g[sl] = True
    return g


@pytest.mark.parametrize("preset,n,ny,seed,q", [("wall_S_open", 64, 48, None, 0.0),
                                                ("wall_S_open", 37, 29, 3, 0.02),
                                                ("half_wall_S_open", 64, 48, None, 0.0),
                                                ("half_wall_S_open", 9, 11, 5, 0.01)])
def test_mixed_open_ghost_cells_host_emulation(oracle, emu, preset, n, ny, seed, q):
    """Open sections beside a south wall: only the masked sections are
    written, and the first interior row of an open W/E edge takes the wall
    corner flux as its bottom face (compared with the oracle's
    compute_time_dev, which applies the wall flux sections first)."""
    from dim2d_finite_volume_b200 import field as F
    exe, d = emu
    nx, nyy, x_map, y_map, st = open_case(n, ny, seed=seed, radius=0.15, center=(0.0, -0.1))
    bc = F._preset(preset)
    cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                          bc_order=bc[2])
    p0 = oracle.get_params()
    p = oracle.set_params(wall_heat_source_choice=1 if q else 0, wall_maximum_heat_flux=q)
    try:
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, st.copy(), st)  # wall ghosts as ini sets
        assert oracle.lib().orc_status() == 0
        ref = oracle.compute_time_dev(cfg, 0.0, st, x_map, y_map)
    finally:
        oracle.set_params(**{name: getattr(p0, name) for name, _ in p0._fields_})
    mask = MIXED[preset]
    fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
    with open(fin, "wb") as fh:
        np.array([nx, nyy], dtype=np.int32).tofile(fh)
        np.array([x_map[1] - x_map[0], y_map[1] - y_map[0], 5.0, 10.0, 20.0, 2.5, -1.5]).tofile(fh)
        st.tofile(fh)
    cos_a = np.cos(p.wall_micro_contact_angle * np.arccos(-1.0) / 180.0)
    out = subprocess.check_output([exe, fin, fout, str(mask), "1", repr(float(x_map[0])),
                                   repr(float(q)), repr(float(cos_a))]).decode()
    stats = dict(kv.split("=") for kv in out.split())
    assert stats["bad_reads"] == "0" and stats["guard_writes"] == "0", out
    assert stats["written"] == stats["expected"], out
    got = np.fromfile(fout).reshape(4, nyy, nx)
    cells = open_cells(nx, nyy, mask)
    assert np.array_equal(got[0] != -777.0, cells)
    inner = np.zeros_like(cells)
    inner[2:-2, 2:-2] = True
    for k in range(4):
        den = np.abs(ref[k][cells | inner]).max()
        num = np.abs(got[k][cells] - ref[k][cells]).max()
        assert num / den <= 1e-12, (preset, k, num / den)
    # the cells whose bottom face is the wall corner flux
    if mask & 4:
        assert np.isfinite(got[:, 2, :2]).all()
