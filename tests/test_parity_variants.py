"""GPU parity of every stage-kernel variant (the 32x8 CTA-tile kernel and
the five warp-strip shapes) through the C ABI, on all provided boundary
configurations, plus the autotuner.

Sizes are ragged so that partial strips, partial CTAs and one-warp-wide
domains occur.  Bar (FP64): normwise <= 1e-12 for one time derivative /
step, <= 1e-10 after 30 RK3 steps, against the oracle."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err, normwise_rel_err_all, open_case, periodic_case, stable_dt
from tests.test_nodebc_emulation import defined_ghost_mask

pytestmark = pytest.mark.gpu
VARIANTS = list(range(7))
PRESETS = ["periodic_xy", "hedstrom_xy", "reflection_xy", "wall_S_reflection"]


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _case(oracle, F, preset, n, ny, seed):
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
    if preset in ("reflection_xy", "wall_S_reflection"):
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)  # field%ini
    elif preset == "periodic_xy":
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)
    return cfg, nx, nyy, x_map, y_map, q


def _err(got, ref, preset):
    if preset == "hedstrom_xy":
        return normwise_rel_err_all(got, ref)
    if preset == "periodic_xy":
        return normwise_rel_err_all(got, ref)
    e = list(normwise_rel_err(got, ref))
    nx, ny = got.shape[2], got.shape[1]
    m = defined_ghost_mask(nx, ny, preset == "wall_S_reflection")
    for k in range(4):
        den = np.abs(ref[k][2:-2, 2:-2]).max()
        e.append(np.abs(got[k][m[k]] - ref[k][m[k]]).max() / den)
    return np.array(e)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("preset", PRESETS)
@pytest.mark.parametrize("n,ny,seed", [(67, 45, 1), (33, 97, 2)])
def test_time_dev(oracle, F, preset, variant, n, ny, seed):
    cfg, nx, nyy, x_map, y_map, q = _case(oracle, F, preset, n, ny, seed)
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    with F.Field(nx, nyy, bc=preset) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        got = fld.compute_time_dev()
    # open fields: every cell has a time derivative; others: the interior
    err = normwise_rel_err_all(got, ref) if preset == "hedstrom_xy" else normwise_rel_err(got, ref)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("variant", VARIANTS[1:])
@pytest.mark.parametrize("preset", PRESETS)
def test_steps(oracle, F, preset, variant):
    cfg, nx, ny, x_map, y_map, q = _case(oracle, F, preset, 70, 52, 3)
    dt = stable_dt(q, x_map, y_map)
    ref1 = q.copy()
    oracle.integrate(cfg, ref1, x_map, y_map, 0.0, dt, 1)
    ref30 = q.copy()
    oracle.set_threads(8)
    oracle.integrate(cfg, ref30, x_map, y_map, 0.0, dt, 30)
    with F.Field(nx, ny, bc=preset) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 1)
        got1 = fld.download()
        fld.integrate(dt, 29)
        got30 = fld.download()
    assert np.all(_err(got1, ref1, preset) <= 1e-12)
    assert np.isfinite(got30[:, 2:-2, 2:-2]).all()
    assert np.all(_err(got30, ref30, preset) <= 1e-10)


def test_variants_agree_with_each_other(F):
    """All variants on a 300x260 periodic field: same state after 5 steps
    to rounding (the variants differ only in work distribution)."""
    nx, ny, x_map, y_map, q = periodic_case(300, 260, seed=11)
    dt = stable_dt(q, x_map, y_map)
    outs = []
    for v in VARIANTS:
        with F.Field(nx, ny, bc="periodic_xy") as fld:
            fld.variant = v
            fld.ini(q, x_map, y_map)
            fld.integrate(dt, 5)
            outs.append(fld.download())
    for v in VARIANTS[1:]:
        assert np.all(normwise_rel_err(outs[v], outs[0]) <= 1e-13), v


def test_autotune_picks_a_variant_and_keeps_state(F):
    nx, ny, x_map, y_map, q = open_case(200, 150, seed=4)
    with F.Field(nx, ny, bc="hedstrom_xy") as fld:
        fld.ini(q, x_map, y_map)
        before = fld.download()
        v, times = fld.autotune(measure=True)
        assert 0 <= v < F.Field.NUM_VARIANTS
        assert fld.variant == v
        assert np.all(np.isfinite(times)) and np.all(times > 0)
        assert times[v] == times.min()
        assert np.array_equal(fld.download(), before)
        # cached: a second call on the same shape returns the same choice
        v2, _ = fld.autotune()
        assert v2 == v


def test_set_variant_rejects_out_of_range(F):
    nx, ny, x_map, y_map, q = periodic_case(24, 20)
    with F.Field(nx, ny, bc="periodic_xy") as fld:
        with pytest.raises(F.Dim2dError):
            fld.variant = 7
        with pytest.raises(F.Dim2dError):
            fld.variant = -1
        assert fld.variant == 0
