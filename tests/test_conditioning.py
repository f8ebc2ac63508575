"""How the reference's own FP64 algorithm responds to rounding-sized
perturbations, measured with the oracle alone (no GPU).

A GPU path that evaluates the same formulas in another order (or a face pass
in FP32) differs from the oracle by rounding in every operation.  How far
such differences travel depends on the problem, not on the implementation:

* on the smallest open (hedstrom_xy) domain of the batched workload, a
  relative perturbation of 1e-14 of the initial state moves the oracle's own
  rho v by more than the 1e-10 FP64 bar after the workload's 2039 steps,
  and the difference grows over the run: the open boundary
  (hedstrom_xy_module.f:445-558, obc_eigenqties_bc, no buffer layer)
  amplifies it;
* on the wall (wall_S_reflection) domain the same perturbation decays
  (viscous damping), so differences stay at their rounding size.

The bars of the long GPU parity tests (tests/test_long_parity.py) are
stated against this response.  The error metric is the parity tests' own:
per conservative variable, max|a - b| / max|b| over the interior."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err

# the bench's batched workload: seed 1234 + 77, 64 domains; domain 11 is
# the first 132^2 open domain, domain 1 the first 132^2 wall domain
BATCH_SEED = 1311
OPEN_DOMAIN = 11
WALL_DOMAIN = 1
BATCH_STEPS = 2039  # 3 + 3 + 33 warm-up steps + 2000 timed steps of the bench


def _domain(oracle, index):
    from dim2d_finite_volume_b200 import field as F
    from dim2d_finite_volume_b200 import workloads
    spec = workloads.batched_specs(BATCH_SEED, 64)[index]
    d = workloads.batched_domain(spec)
    nx, ny = d["nx"], d["ny"]
    ch, ty, od = F._preset(d["bc"])
    cfg = oracle.make_cfg(nx, ny, periodic=False, bc_choice=ch, bc_type=ty, bc_order=od)
    q = d["nodes"].copy()
    if d["bc"] != "hedstrom_xy":  # field%ini: node boundary pass
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, d["x_map"], d["y_map"], q.copy(), q)
    return d, cfg, q


def response(oracle, d, cfg, q, eps, checkpoints):
    """Normwise error of the oracle started from q * (1 + eps * noise)
    against the oracle started from q, at each checkpoint step."""
    a = q.copy()
    b = q * (1.0 + eps * np.random.default_rng(0).standard_normal(q.shape))
    out, done = [], 0
    for n in checkpoints:
        oracle.integrate(cfg, a, d["x_map"], d["y_map"], 0.0, d["dt"], n - done)
        oracle.integrate(cfg, b, d["x_map"], d["y_map"], 0.0, d["dt"], n - done)
        done = n
        assert np.isfinite(a).all() and np.isfinite(b).all()
        out.append(normwise_rel_err(b, a))
    return out


@pytest.fixture(scope="module")
def batch_oracle(oracle):
    from dim2d_finite_volume_b200 import workloads
    import ctypes
    import os
    oracle.set_threads(os.cpu_count() or 1)
    saved = oracle.get_params()
    oracle.set_params(we=workloads.BATCH_WE)
    yield oracle
    oracle.lib().orc_set_params(ctypes.byref(saved))


def test_open_domain_amplifies_rounding_past_the_fp64_bar(batch_oracle):
    d, cfg, q = _domain(batch_oracle, OPEN_DOMAIN)
    assert d["bc"] == "hedstrom_xy" and d["nx"] == 132
    e100, e_end = response(batch_oracle, d, cfg, q, 1e-14, (100, BATCH_STEPS))
    # rho v (its maximum is ~3 % of rho u's) moves past 1e-10 ...
    assert e_end[2] > 1e-10, e_end
    # ... because the difference grows along the run, in every variable
    assert np.all(e_end > 10.0 * e100), (e100, e_end)


def test_wall_domain_damps_rounding(batch_oracle):
    d, cfg, q = _domain(batch_oracle, WALL_DOMAIN)
    assert d["bc"] == "wall_S_reflection" and d["nx"] == 132
    e100, e1000 = response(batch_oracle, d, cfg, q, 1e-14, (100, 1000))
    assert np.all(e1000 < e100), (e100, e1000)
    assert np.all(e1000 < 1e-10), e1000
