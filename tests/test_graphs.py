"""Step graphs (dim2d_step replays a captured CUDA graph per buffer parity):
the replayed steps launch the same kernels with the same arguments as the
stream path, so the states must be bit-identical; the graphs must follow
dt changes, variant changes and re-uploads with a different grid."""
import numpy as np
import pytest

from tests.helpers import open_case, periodic_case, stable_dt

pytestmark = pytest.mark.gpu
PRESETS = ["periodic_xy", "hedstrom_xy", "reflection_xy", "wall_S_reflection"]


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _case(preset, n=70, ny=52, seed=3):
    if preset == "hedstrom_xy":
        return open_case(n, ny, seed=seed, radius=0.15)
    return periodic_case(n, ny, radius=0.15, seed=seed)


def _run(F, preset, graphs, schedule, variant=None):
    nx, ny, x_map, y_map, q = _case(preset)
    dt = stable_dt(q, x_map, y_map)
    with F.Field(nx, ny, bc=preset) as fld:
        fld.set_graphs(graphs)
        if variant is not None:
            fld.variant = variant
        fld.ini(q, x_map, y_map)
        n0 = fld.launches
        for item in schedule:
            if item[0] == "step":
                fld.integrate(dt * item[1], item[2])
            elif item[0] == "variant":
                fld.variant = item[1]
        return fld.download(), fld.time, fld.launches - n0


@pytest.mark.parametrize("preset", PRESETS)
def test_graph_steps_bit_identical(F, preset):
    sched = [("step", 1.0, 1)] * 3 + [("step", 1.0, 4), ("step", 0.5, 1), ("step", 1.0, 3)]
    a, ta, na = _run(F, preset, True, sched)
    b, tb, nb = _run(F, preset, False, sched)
    assert np.array_equal(a, b)
    assert ta == tb
    assert na == nb  # the graph reports the launches it replays


@pytest.mark.parametrize("preset", ["periodic_xy", "hedstrom_xy"])
def test_graphs_follow_variant_changes(F, preset):
    sched = [("step", 1.0, 2), ("variant", 0), ("step", 1.0, 3), ("variant", 2),
             ("step", 1.0, 1)]
    a, _, na = _run(F, preset, True, sched, variant=1)
    b, _, nb = _run(F, preset, False, sched, variant=1)
    assert np.array_equal(a, b)
    assert na == nb


def test_reupload_same_grid_keeps_results_and_new_grid_recaptures(F):
    nx, ny, x_map, y_map, q = _case("periodic_xy")
    dt = stable_dt(q, x_map, y_map)
    x2 = x_map * 1.1  # another grid step: dx changes
    outs = {}
    for graphs in (True, False):
        with F.Field(nx, ny, bc="periodic_xy") as fld:
            fld.set_graphs(graphs)
            fld.ini(q, x_map, y_map)
            fld.integrate(dt, 3)
            fld.ini(q, x_map, y_map)  # same grid: graphs stay valid
            fld.integrate(dt, 2)
            r1 = fld.download()
            fld.ini(q, x2, y_map)  # new dx: graphs must be recaptured
            fld.integrate(dt, 2)
            outs[graphs] = (r1, fld.download())
    assert np.array_equal(outs[True][0], outs[False][0])
    assert np.array_equal(outs[True][1], outs[False][1])
    assert not np.array_equal(outs[True][0], outs[True][1])
