"""GPU parity of the presets that put open (Hedstrom) sides beside a south
wall, through the C ABI: wall_S_open (S, SW, SE wall; N, E, W, NE, NW open)
and half_wall_S_open, the reference's default preset (S, SE wall; W, SW, NW
reflection_x; N, E, NE open), library_config.py:118-150.

The open sections are time-integrated (their ghost cells get a time
derivative, bc_operators_hedstrom_xy_class.f:182-496); the bottom face of
the first interior row of an open W/E edge carries the wall corner flux
(bc_operators_wall_xy_class.f:702-854); the node pass solves the wall
columns, the wall corner columns with one-sided tangential gradients, and
the mirrors.

Compared: the interior, the ghost cells of the open sections and the ghost
entries the node operators define (the wall leaves the energy of its two
ghost rows and the momenta of the second undefined; the reference fills
them with its debug value and never reads them).  Bars (FP64, normwise
relative to the interior maximum): <= 1e-12 for one time derivative and one
step, <= 1e-10 after 60 RK3 steps; mixed precision: <= 1e-4 for the time
derivative, <= 1e-5 for the state after 1 and 60 steps."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err, stable_dt
from tests.test_nodebc_emulation import defined_ghost_mask
from tests.test_open_emulation import MIXED, open_cells

pytestmark = pytest.mark.gpu
PRESETS = ["wall_S_open", "half_wall_S_open"]
VARIANTS = list(range(7))
DEBUG_REAL = 9.9692099683868690e+36  # td_operators_class.f:150-154


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _case(oracle, F, preset, n, ny, seed=None, center=(0.05, -0.1), r=0.15, flow=0.05):
    """A bubble near the wall in a slow x-flow (so that waves leave through
    the open sides), ghost cells set as field%ini leaves them."""
    from dim2d_finite_volume_b200 import ic
    from tests.helpers import liquid_sound_speed
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    q = ic.bubbles(x_map, y_map, 0.95, [(center[0], center[1], r)], li=4.0 * dx,
                   velocity=(flow * liquid_sound_speed(0.95), 0.0))
    if seed is not None:
        rng = np.random.default_rng(seed)
        q[1] += 0.02 * rng.standard_normal(q[0].shape) * q[0]
        q[2] += 0.02 * rng.standard_normal(q[0].shape) * q[0]
        q[3] += 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0]
    bc = F._preset(preset)
    cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1], bc_order=bc[2])
    oracle.lib().orc_clear_status()
    oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)  # field%ini
    assert oracle.lib().orc_status() == 0
    return cfg, nx, nyy, x_map, y_map, np.ascontiguousarray(q)


def _td_err(got, ref, preset):
    """Interior and open ghost cells; every other cell keeps the debug value."""
    ny, nx = got.shape[1], got.shape[2]
    cells = open_cells(nx, ny, MIXED[preset])
    inner = np.zeros_like(cells)
    inner[2:-2, 2:-2] = True
    e = []
    for k in range(4):
        den = np.abs(ref[k][inner]).max()
        e.append(np.abs(got[k][cells | inner] - ref[k][cells | inner]).max() / den)
        assert np.all(got[k][~(cells | inner)] == DEBUG_REAL)
        assert np.all(ref[k][~(cells | inner)] == DEBUG_REAL)
    return np.array(e)


def _state_err(got, ref):
    """Interior, and every ghost entry the reference defines."""
    ny, nx = got.shape[1], got.shape[2]
    e = list(normwise_rel_err(got, ref))
    m = defined_ghost_mask(nx, ny, True)
    for k in range(4):
        den = np.abs(ref[k][2:-2, 2:-2]).max()
        e.append(np.abs(got[k][m[k]] - ref[k][m[k]]).max() / den)
    return np.array(e)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("preset", PRESETS)
@pytest.mark.parametrize("n,ny,seed", [(67, 45, 1), (33, 70, 2)])
def test_time_dev(oracle, F, preset, variant, n, ny, seed):
    cfg, nx, nyy, x_map, y_map, q = _case(oracle, F, preset, n, ny, seed)
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    with F.Field(nx, nyy, bc=preset) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        got = fld.compute_time_dev()
    err = _td_err(got, ref, preset)
    assert np.all(err <= 1e-12), (variant, err)


@pytest.mark.parametrize("variant", [0, 2, 4])
@pytest.mark.parametrize("preset", PRESETS)
def test_steps(oracle, F, preset, variant):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 72, 56, seed=3)
    dt = stable_dt(q, x_map, y_map)
    ref1 = q.copy()
    oracle.lib().orc_clear_status()
    assert oracle.integrate(cfg, ref1, x_map, y_map, 0.0, dt, 1) == dt
    ref60 = q.copy()
    oracle.set_threads(8)
    oracle.integrate(cfg, ref60, x_map, y_map, 0.0, dt, 60)
    assert oracle.lib().orc_status() == 0
    with F.Field(nx, ny, bc=preset) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 1)
        got1 = fld.download()
        fld.integrate(dt, 59)
        got60 = fld.download()
    assert np.all(_state_err(got1, ref1) <= 1e-12), (variant, _state_err(got1, ref1))
    assert np.isfinite(got60[:, 2:-2, 2:-2]).all()
    assert np.all(_state_err(got60, ref60) <= 1e-10), (variant, _state_err(got60, ref60))


@pytest.mark.parametrize("preset", PRESETS)
def test_heat_flux_and_contact_angle(oracle, F, preset):
    """A heated wall (constant heat flux) with a 60 degree contact angle:
    the wall corner fluxes carry the heat flux, the corner roots the angle."""
    p0 = oracle.get_params()
    p = oracle.set_params(wall_heat_source_choice=1, wall_maximum_heat_flux=0.02,
                          wall_micro_contact_angle=60.0)
    try:
        cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 50, 40, seed=4)
        dt = stable_dt(q, x_map, y_map)
        ref_td = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
        ref = q.copy()
        oracle.lib().orc_clear_status()
        oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 5)
        assert oracle.lib().orc_status() == 0
    finally:
        oracle.set_params(**{name: getattr(p0, name) for name, _ in p0._fields_})
    params = F.default_params()
    params.wall_heat_source_choice = 1
    params.wall_maximum_heat_flux = 0.02
    params.wall_micro_contact_angle = 60.0
    with F.Field(nx, ny, bc=preset, params=params) as fld:
        fld.variant = 2
        fld.ini(q, x_map, y_map)
        td = fld.compute_time_dev()
        fld.integrate(dt, 5)
        got = fld.download()
    assert np.all(_td_err(td, ref_td, preset) <= 1e-12)
    assert np.all(_state_err(got, ref) <= 1e-11)


@pytest.mark.parametrize("preset", PRESETS)
def test_mixed_precision(oracle, F, preset):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 70, 52, seed=5)
    dt = stable_dt(q, x_map, y_map)
    ref_td = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    ref1 = q.copy()
    oracle.integrate(cfg, ref1, x_map, y_map, 0.0, dt, 1)
    ref = q.copy()
    oracle.set_threads(8)
    oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 60)
    for variant in (0, 2):
        with F.Field(nx, ny, bc=preset, precision=F.MIXED) as fld:
            fld.variant = variant
            fld.ini(q, x_map, y_map)
            td = fld.compute_time_dev()
            fld.integrate(dt, 1)
            got1 = fld.download()
            fld.integrate(dt, 59)
            got = fld.download()
        e_td = _td_err(td, ref_td, preset)
        assert np.all(e_td <= 1e-4), (variant, e_td)
        assert e_td.max() > 1e-13  # the FP32 face pass really ran
        assert np.all(_state_err(got1, ref1) <= 1e-5), (variant, _state_err(got1, ref1))
        assert np.all(_state_err(got, ref) <= 1e-5), (variant, _state_err(got, ref))


@pytest.mark.parametrize("preset", PRESETS)
def test_graph_steps_match_stream_steps(F, oracle, preset):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 64, 48, seed=6)
    dt = stable_dt(q, x_map, y_map)
    out = []
    for graphs in (True, False):
        with F.Field(nx, ny, bc=preset) as fld:
            fld.variant = 3
            fld.set_graphs(graphs)
            fld.ini(q, x_map, y_map)
            fld.integrate(dt, 7)
            out.append(fld.download())
    m = defined_ghost_mask(nx, ny, True)
    m[:, 2:-2, 2:-2] = True
    assert np.array_equal(out[0][m], out[1][m])
