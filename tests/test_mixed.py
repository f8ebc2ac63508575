"""Mixed precision (DIM2D_MIXED): FP32 face pass, FP64 node pass (EOS
inversion), FP64 third-derivative capillary term and FP64 RK accumulation.

Stated bars against the FP64 oracle (normwise relative error per
conservative variable): <= 1e-4 for one time derivative (the divergence of
FP32 fluxes loses digits to cancellation), <= 1e-5 for the state after 1
and after 200 RK3 steps.  The path must also differ from the FP64 path by
more than FP64 rounding (it really runs the face pass in FP32)."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err, normwise_rel_err_all, open_case, periodic_case, stable_dt

pytestmark = pytest.mark.gpu
PRESETS = ["periodic_xy", "hedstrom_xy", "wall_S_reflection", "reflection_xy"]


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _case(oracle, F, preset, n=70, ny=52, seed=3):
    if preset == "hedstrom_xy":
        nx, nyy, x_map, y_map, q = open_case(n, ny, seed=seed, radius=0.15)
    else:
        nx, nyy, x_map, y_map, q = periodic_case(n, ny, radius=0.15, seed=seed)
    if preset == "periodic_xy":
        cfg = oracle.make_cfg(nx, nyy, periodic=True)
    else:
        bc = F._preset(preset)
        cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                              bc_order=bc[2])
    if preset != "hedstrom_xy":
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)  # field%ini
    return cfg, nx, nyy, x_map, y_map, q


def _err(got, ref, preset):
    if preset == "hedstrom_xy":
        return normwise_rel_err_all(got, ref)
    return normwise_rel_err(got, ref)


@pytest.mark.parametrize("preset", PRESETS)
def test_time_dev_within_1e4(oracle, F, preset):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset)
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    with F.Field(nx, ny, bc=preset, precision=F.MIXED) as fld:
        fld.ini(q, x_map, y_map)
        got = fld.compute_time_dev()
    err = _err(got, ref, preset)
    assert np.all(err <= 1e-4), err
    assert err.max() > 1e-13  # not the FP64 path


@pytest.mark.parametrize("preset", PRESETS)
def test_steps_within_1e5(oracle, F, preset):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset)
    dt = stable_dt(q, x_map, y_map)
    ref1 = q.copy()
    oracle.integrate(cfg, ref1, x_map, y_map, 0.0, dt, 1)
    ref = q.copy()
    oracle.set_threads(8)
    oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 200)
    for variant in (0, 2, 5):
        with F.Field(nx, ny, bc=preset, precision=F.MIXED) as fld:
            fld.variant = variant
            fld.ini(q, x_map, y_map)
            fld.integrate(dt, 1)
            got1 = fld.download()
            fld.integrate(dt, 199)
            got = fld.download()
        e1 = _err(got1, ref1, preset)
        e = _err(got, ref, preset)
        assert np.isfinite(got).all()
        assert np.all(e1 <= 1e-5), (variant, e1)
        assert np.all(e <= 1e-5), (variant, e)
        assert e.max() > 1e-13


def test_mixed_graph_steps_match_stream_steps(F):
    nx, ny, x_map, y_map, q = open_case(80, 64, seed=8)
    dt = stable_dt(q, x_map, y_map)
    out = []
    for graphs in (True, False):
        with F.Field(nx, ny, bc="hedstrom_xy", precision=F.MIXED) as fld:
            fld.set_graphs(graphs)
            fld.ini(q, x_map, y_map)
            fld.integrate(dt, 5)
            out.append(fld.download())
    assert np.array_equal(out[0], out[1])
