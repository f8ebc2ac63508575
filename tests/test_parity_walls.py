"""GPU parity of the mirror and wall configurations through the C ABI:
reflection_xy (mirrors on all sides) and wall_S_reflection (contact-angle
wall at the bottom, mirrors elsewhere; library_config.py:58-115).

Compared: interior cells, and the ghost entries the reference's node
operators define (the wall leaves the energy of its first ghost row and the
momenta/energy of the second undefined -- the reference fills them with its
debug value and never reads them).  Bar (FP64): normwise <= 1e-12 for one
time derivative / step, <= 1e-10 after 100 RK3 steps."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err, stable_dt
from tests.test_nodebc_emulation import defined_ghost_mask

pytestmark = pytest.mark.gpu
PRESETS = ["reflection_xy", "wall_S_reflection"]


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _case(oracle, F, preset, n, ny, seed=None, center=(0.05, -0.05), r=0.15):
    from dim2d_finite_volume_b200 import ic
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    q = ic.bubbles(x_map, y_map, 0.95, [(center[0], center[1], r)], li=4.0 * dx)
    if seed is not None:
        rng = np.random.default_rng(seed)
        q[1] += 0.02 * rng.standard_normal(q[0].shape) * q[0]
        q[2] += 0.02 * rng.standard_normal(q[0].shape) * q[0]
        q[3] += 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0]
    bc = F._preset(preset)
    cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1], bc_order=bc[2])
    oracle.lib().orc_clear_status()
    oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)  # field%ini
    return cfg, nx, nyy, x_map, y_map, q


def _compare(got, ref, preset, tol):
    nx, ny = got.shape[2], got.shape[1]
    err = normwise_rel_err(got, ref)
    assert np.all(err <= tol), ("interior", err)
    m = defined_ghost_mask(nx, ny, preset == "wall_S_reflection")
    for k in range(4):
        den = np.abs(ref[k][2:-2, 2:-2]).max()
        num = np.abs(got[k][m[k]] - ref[k][m[k]]).max()
        assert num / den <= tol, ("ghost", k, num / den)


@pytest.mark.parametrize("preset", PRESETS)
@pytest.mark.parametrize("n,ny,seed", [(64, 48, 1), (37, 29, 2)])
def test_time_dev(oracle, F, preset, n, ny, seed):
    cfg, nx, nyy, x_map, y_map, q = _case(oracle, F, preset, n, ny, seed)
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    with F.Field(nx, nyy, bc=preset) as fld:
        fld.ini(q, x_map, y_map)
        got = fld.compute_time_dev()
    err = normwise_rel_err(got, ref)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("preset", PRESETS)
def test_one_step(oracle, F, preset):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 72, 56, seed=3)
    dt = stable_dt(q, x_map, y_map)
    ref = q.copy()
    assert oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 1) == dt
    with F.Field(nx, ny, bc=preset) as fld:
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 1)
        got = fld.download()
    _compare(got, ref, preset, 1e-12)


@pytest.mark.parametrize("preset", PRESETS)
def test_100_steps(oracle, F, preset):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 96, 80)
    dt = stable_dt(q, x_map, y_map)
    ref = q.copy()
    oracle.set_threads(8)
    oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 100)
    with F.Field(nx, ny, bc=preset) as fld:
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 100)
        got = fld.download()
    assert np.isfinite(got[:, 2:-2, 2:-2]).all()
    _compare(got, ref, preset, 1e-10)


def test_apply_bc_on_nodes_matches_oracle(oracle, F):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, "wall_S_reflection", 50, 40, seed=5)
    state = q * 1.0001
    ref = state.copy()
    oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, ref.copy(), ref)
    with F.Field(nx, ny, bc="wall_S_reflection") as fld:
        fld.ini(state, x_map, y_map)
        fld.apply_bc_on_nodes()
        got = fld.download()
    m = defined_ghost_mask(nx, ny, True)
    assert np.abs(got[m] - ref[m]).max() <= 1e-12 * np.abs(ref).max()
