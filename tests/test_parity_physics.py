"""GPU parity of the optional physics, through the C ABI: gravity (the body
forces of pmodel_eq_class.f:1840-1918, -rho g on the y-momentum and -rho v g
on the energy, added to the interior and to the open ghost cells,
openbc_operators_module.f:354-372) and the wall's Gaussian heat source with
a non-neutral contact angle (wall_xy_equilibrium_module.f:1645-1707 and
:2238-2270).

Bars (FP64, normwise relative to the interior maximum): <= 1e-12 for one
time derivative, <= 1e-10 after 20 RK3 steps, on the tile kernel (variant 0)
and a strip shape (variant 4)."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err, stable_dt
from tests.test_nodebc_emulation import defined_ghost_mask
from tests.test_open_emulation import MIXED, open_cells

pytestmark = pytest.mark.gpu
DEBUG_REAL = 9.9692099683868690e+36


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _with_oracle_params(oracle, **kw):
    """Set oracle constants, return a restore callable."""
    p0 = oracle.get_params()
    oracle.set_params(**kw)
    return lambda: oracle.set_params(**{n: getattr(p0, n) for n, _ in p0._fields_})


def _case(oracle, F, preset, n, ny, seed, mach):
    from dim2d_finite_volume_b200 import ic
    from tests.helpers import liquid_sound_speed
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    q = ic.bubbles(x_map, y_map, 0.95, [(0.05, -0.05, 0.15)], li=4.0 * dx,
                   velocity=(mach * liquid_sound_speed(0.95), 0.0))
    rng = np.random.default_rng(seed)
    q[2] += 0.01 * rng.standard_normal(q[0].shape) * q[0]
    q[3] += 0.5 * (q[2] ** 2) / q[0]
    q = np.ascontiguousarray(q)
    if preset == "periodic_xy":
        cfg = oracle.make_cfg(nx, nyy, periodic=True)
    else:
        bc = F._preset(preset)
        cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                              bc_order=bc[2])
    if preset != "hedstrom_xy":
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)  # field%ini
        assert oracle.lib().orc_status() == 0
    return cfg, nx, nyy, x_map, y_map, q


def _td_err(got, ref, preset):
    """Interior, plus the time-integrated ghost cells of open sections."""
    ny, nx = got.shape[1], got.shape[2]
    cells = np.zeros((ny, nx), bool)
    cells[2:-2, 2:-2] = True
    if preset == "hedstrom_xy":
        cells[:] = True
    elif preset in MIXED:
        cells |= open_cells(nx, ny, MIXED[preset])
    e = []
    for k in range(4):
        den = np.abs(ref[k][2:-2, 2:-2]).max()
        e.append(np.abs(got[k][cells] - ref[k][cells]).max() / den)
    return np.array(e)


def _state_err(got, ref, preset):
    ny, nx = got.shape[1], got.shape[2]
    e = list(normwise_rel_err(got, ref))
    if preset in ("periodic_xy", "hedstrom_xy"):
        m = np.ones((4, ny, nx), bool)
    else:
        m = defined_ghost_mask(nx, ny, preset != "reflection_xy")
    for k in range(4):
        den = np.abs(ref[k][2:-2, 2:-2]).max()
        e.append(np.abs(got[k][m[k]] - ref[k][m[k]]).max() / den)
    return np.array(e)


@pytest.mark.parametrize("variant", [0, 4])
@pytest.mark.parametrize("preset,mach", [("periodic_xy", 0.0), ("hedstrom_xy", 0.05),
                                         ("wall_S_reflection", 0.0),
                                         ("half_wall_S_open", 0.0)])
def test_gravity(oracle, F, preset, mach, variant):
    g = 0.5
    restore = _with_oracle_params(oracle, gravity_ac=1, gravity=g)
    try:
        cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 61, 47, 11, mach)
        dt = stable_dt(q, x_map, y_map)
        ref_td = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
        ref = q.copy()
        oracle.lib().orc_clear_status()
        oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 20)
        assert oracle.lib().orc_status() == 0
    finally:
        restore()
    params = F.default_params()
    params.gravity_ac = 1
    params.gravity = g
    with F.Field(nx, ny, bc=preset, params=params) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        td = fld.compute_time_dev()
        fld.integrate(dt, 20)
        got = fld.download()
    assert np.all(_td_err(td, ref_td, preset) <= 1e-12), (preset, variant, _td_err(td, ref_td, preset))
    assert np.isfinite(got[:, 2:-2, 2:-2]).all()
    err = _state_err(got, ref, preset)
    assert np.all(err <= 1e-10), (preset, variant, err)
    # gravity changes the answer (the test is not vacuous)
    with F.Field(nx, ny, bc=preset) as fld0:
        fld0.variant = variant
        fld0.ini(q, x_map, y_map)
        td0 = fld0.compute_time_dev()
    assert np.abs(td0[2][2:-2, 2:-2] - td[2][2:-2, 2:-2]).max() > 1e-3


@pytest.mark.parametrize("variant", [0, 4])
def test_gaussian_heat_source_and_contact_angle(oracle, F, variant):
    preset = "wall_S_reflection"
    kw = dict(wall_heat_source_choice=2, wall_maximum_heat_flux=0.05,
              wall_heat_source_center=0.1, wall_heat_source_variance=0.2,
              wall_micro_contact_angle=75.0)
    restore = _with_oracle_params(oracle, **kw)
    try:
        cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 57, 45, 12, 0.0)
        dt = stable_dt(q, x_map, y_map)
        ref_td = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
        ref = q.copy()
        oracle.lib().orc_clear_status()
        oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 20)
        assert oracle.lib().orc_status() == 0
    finally:
        restore()
    params = F.default_params()
    for k, v in kw.items():
        setattr(params, k, v)
    with F.Field(nx, ny, bc=preset, params=params) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        td = fld.compute_time_dev()
        fld.integrate(dt, 20)
        got = fld.download()
    assert np.all(_td_err(td, ref_td, preset) <= 1e-12)
    err = _state_err(got, ref, preset)
    assert np.all(err <= 1e-10), (variant, err)
