"""GPU parity, periodic_xy domain: CUDA path through the C ABI vs the oracle.

Bar (FP64): max_cells |gpu - oracle| / max_cells |oracle| <= 1e-10 for every
conservative variable over the interior, after 100 RK3 steps.
"""
import numpy as np
import pytest

from tests.helpers import interior, normwise_rel_err, periodic_case, stable_dt

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


def _prep(oracle, n, ny=None, seed=None):
    nx, nyy, x_map, y_map, q = periodic_case(n, ny, seed=seed)
    cfg = oracle.make_cfg(nx, nyy, periodic=True)
    oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)  # field%ini
    return cfg, x_map, y_map, q


@pytest.mark.parametrize("n,ny", [(128, 128), (12, 10), (37, 53), (64, 200)])
def test_time_dev_matches_oracle(oracle, F, n, ny):
    cfg, x_map, y_map, q = _prep(oracle, n, ny, seed=1)
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    with F.Field(q.shape[2], q.shape[1], bc="periodic_xy") as fld:
        fld.ini(q, x_map, y_map)
        got = fld.compute_time_dev()
    err = normwise_rel_err(got, ref)
    assert np.all(err <= 1e-12), err
    # cells outside the interior keep debug_real like the reference
    assert np.all(got[:, :2, :] == ref[:, :2, :])


def test_one_step_matches_oracle_all_cells(oracle, F):
    cfg, x_map, y_map, q = _prep(oracle, 64, 48, seed=2)
    dt = stable_dt(q, x_map, y_map)
    ref = q.copy()
    oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 1)
    with F.Field(q.shape[2], q.shape[1]) as fld:
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 1)
        got = fld.download()
    # ghosts included: the periodic images are exact copies
    err = [np.abs(got[k] - ref[k]).max() / np.abs(ref[k]).max() for k in range(4)]
    assert max(err) <= 1e-12, err


def test_100_steps_config1_parity(oracle, F):
    """128^2 periodic static bubble, T0=0.95, r=0.1, 100 RK3 steps."""
    cfg, x_map, y_map, q = _prep(oracle, 128)
    dt = stable_dt(q, x_map, y_map)
    ref = q.copy()
    oracle.set_threads(8)
    t_ref = oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 100)
    with F.Field(q.shape[2], q.shape[1]) as fld:
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 100)
        got = fld.download()
        assert abs(fld.time - t_ref) < 1e-15
    assert np.isfinite(got).all()
    err = normwise_rel_err(got, ref)
    assert np.all(err <= TOL), err


def test_ragged_small_grids_many_steps(oracle, F):
    for (n, ny) in [(8, 8), (33, 17)]:
        cfg, x_map, y_map, q = _prep(oracle, n, ny, seed=3)
        dt = stable_dt(q, x_map, y_map)
        ref = q.copy()
        oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 20)
        with F.Field(q.shape[2], q.shape[1]) as fld:
            fld.ini(q, x_map, y_map)
            fld.integrate(dt, 20)
            got = fld.download()
        err = normwise_rel_err(got, ref)
        assert np.all(err <= TOL), (n, ny, err)


def test_deterministic_bitwise(F):
    nx, ny, x_map, y_map, q = periodic_case(96, seed=4)
    outs = []
    for _ in range(2):
        with F.Field(nx, ny) as fld:
            fld.ini(q, x_map, y_map)
            fld.apply_bc_on_nodes()
            fld.integrate(2e-5, 7)
            outs.append(fld.download())
    assert np.array_equal(outs[0], outs[1])


def test_cfl_dt_matches_host(F):
    from dim2d_finite_volume_b200 import ic
    nx, ny, x_map, y_map, q = periodic_case(100, seed=5)
    want = ic.cfl_dt(q, x_map[1] - x_map[0], y_map[1] - y_map[0], 0.1)
    with F.Field(nx, ny) as fld:
        fld.ini(q, x_map, y_map)
        got = fld.cfl_dt(0.1)
    assert abs(got - want) <= 1e-13 * want


def test_launch_count_is_three_per_step(F):
    nx, ny, x_map, y_map, q = periodic_case(32)
    with F.Field(nx, ny) as fld:
        fld.ini(q, x_map, y_map)
        n0 = fld.launches
        fld.integrate(1e-5, 5)
        assert fld.launches - n0 == 15
