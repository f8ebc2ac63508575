"""CPU check of the node boundary kernel's per-thread code (no GPU needed).

tests/emu/emu_nodebc.cu compiles dim2d_nodebc.cu for the host and runs
node_bc_cell() -- the body of k_node_bc -- for every thread index, with
checked reads and writes and a race detector (a read of a cell written by
another thread index).  Its ghost cells are compared with the oracle's
apply_bc_on_nodes: the mirror sides bit-exactly, the wall ghost cells to
1e-12 (root tolerance of Ridders' method)."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def emu():
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "emu_nodebc")
    subprocess.check_call([NVCC, "-std=c++17", "-O1", "-w", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-I", os.path.join(ROOT, "include"),
                           "-o", exe, os.path.join(HERE, "emu", "emu_nodebc.cu")])
    yield exe, d
    shutil.rmtree(d, ignore_errors=True)


def defined_ghost_mask(nx, ny, south_wall):
    """Ghost entries the reference's node operators define (the wall leaves
    the energy of its first ghost row and the momenta/energy of the second
    undefined; its corners mirror those)."""
    m = np.zeros((4, ny, nx), bool)
    m[:, :2, :] = m[:, -2:, :] = True
    m[:, :, :2] = m[:, :, -2:] = True
    if south_wall:
        m[3, 1, :] = False
        m[1:, 0, :] = False
    return m


# (south_wall, corners_y, open_w, open_e, open_n) of the node pass per preset
FLAGS = {"wall_S_reflection": (1, 0, 0, 0, 0), "reflection_xy": (0, 1, 0, 0, 0),
         "wall_S_open": (1, 0, 1, 1, 1), "half_wall_S_open": (1, 0, 0, 1, 1)}


def node_ghosts(nx, ny, preset):
    """Ghost cells that have node work (the others are stage output)."""
    g = np.zeros((ny, nx), bool)
    south_wall, _, open_w, open_e, open_n = FLAGS[preset]
    g[:2, :] = True  # S side: wall or mirror, corners included
    if not open_n:
        g[-2:, :] = True
    if not open_w:
        g[:, :2] = True
    if not open_e:
        g[:, -2:] = True
    return g


@pytest.mark.parametrize("preset,n,ny,seed", [("wall_S_reflection", 40, 30, 1),
                                               ("wall_S_reflection", 9, 12, 2),
                                               ("reflection_xy", 33, 21, 3),
                                               ("wall_S_open", 40, 30, 4),
                                               ("wall_S_open", 9, 12, 5),
                                               ("half_wall_S_open", 40, 30, 6),
                                               ("half_wall_S_open", 11, 9, 7)])
def test_node_bc_host_emulation(oracle, emu, preset, n, ny, seed):
    from dim2d_finite_volume_b200 import field as F, ic
    exe, d = emu
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    un = ic.bubbles(x_map, y_map, 0.95, [(0.05, 0.02, 0.15)], li=4.0 * dx)
    bc = F._preset(preset)
    cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1], bc_order=bc[2])
    oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, un.copy(), un)  # u^n as ini leaves it
    rng = np.random.default_rng(seed)
    u = un * (1.0 + 1e-3 * rng.standard_normal(un.shape))       # a stage state
    u[:, node_ghosts(nx, nyy, preset)] = 1e31                     # ghosts: stage-1 garbage
    want = u.copy()
    oracle.lib().orc_clear_status()
    oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, un, want)
    assert oracle.lib().orc_status() == 0
    south_wall = FLAGS[preset][0]
    p = oracle.get_params()
    fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
    with open(fin, "wb") as fh:
        np.array([nx, nyy, *FLAGS[preset]], dtype=np.int32).tofile(fh)
        np.array([dx, y_map[1] - y_map[0], p.re, p.we, p.pr, p.cv_r, p.viscous_r,
                  np.cos(p.wall_micro_contact_angle * np.arccos(-1.0) / 180.0), x_map[0],
                  0.0]).tofile(fh)
        un.tofile(fh)
        u.tofile(fh)
    out = subprocess.check_output([exe, fin, fout]).decode()
    stats = dict(kv.split("=") for kv in out.split())
    assert stats["bad"] == "0" and stats["race"] == "0" and stats["status"] == "0", out
    got = np.fromfile(fout).reshape(4, nyy, nx)
    mask = defined_ghost_mask(nx, nyy, south_wall)
    assert np.array_equal(got[:, 2:-2, 2:-2], u[:, 2:-2, 2:-2])  # interior untouched
    stage_cells = ~node_ghosts(nx, nyy, preset)
    assert np.array_equal(got[:, stage_cells], u[:, stage_cells])  # open sections untouched
    wall_rows = np.zeros_like(mask)
    if south_wall:
        wall_rows[:, :2, :] = True
    exact = mask & ~wall_rows
    assert np.array_equal(got[exact], want[exact])
    if south_wall:
        wm = mask & wall_rows
        assert np.abs(got[wm] - want[wm]).max() <= 1e-12 * np.abs(want[wm]).max()
