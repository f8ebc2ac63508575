"""Seeded workloads (CPU): the equilibrium interface width and the long-run
configurations built on it.

The served stream, the batched configuration and the 2048^2 mixed-precision
configuration start from bubbles with the equilibrium interface width at T0
(dim2d_state_eq_module.f:90-125), the width the reference's own bubble
initial conditions use, for one Weber number per configuration.  These
tests pin the width formula and check with the oracle that small requests
of those configurations run thousands of steps without the wall root
failing or the state blowing up (the 4-dx interfaces at We = 10 fail within
a few hundred)."""
import math

import numpy as np
import pytest

from dim2d_finite_volume_b200 import ic, workloads


def test_interface_length_formula():
    # 1/sqrt(2 We) * 1.6309400153322933/sqrt(1-T)
    assert ic.interface_length(0.95, 10.0) == pytest.approx(
        1.0 / math.sqrt(20.0) * 1.6309400153322933 / math.sqrt(0.05), rel=1e-15)
    assert ic.interface_length(0.95, 10.0) > 1.0  # wider than the [-0.5, 0.5] box
    w = [ic.interface_length(T, workloads.SERVED_WE) for T in (0.90, 0.99)]
    assert 0.08 < w[0] < w[1] < 0.26


def test_long_run_configurations_share_their_weber_number():
    assert workloads.served_params().we == workloads.SERVED_WE
    assert workloads.batch_params().we == workloads.BATCH_WE
    assert workloads.mixed_params().we == workloads.MIXED_WE
    reqs = workloads.served_requests(5, 6, n_range=(64, 80), steps_range=(10, 20))
    for r in reqs:
        assert r["dt"] > 0 and np.isfinite(r["nodes"]).all()
        # the interface spans several cells on every grid of the stream
        dx = r["x_map"][1] - r["x_map"][0]
        assert ic.interface_length(r["T0"], workloads.SERVED_WE) > 4 * dx


# steps: the open preset stops short of t ~ 0.45, where the open boundary's
# own growth (the reference's Hedstrom formulation) sets in on small grids
@pytest.mark.parametrize("bc,T0,r,steps", [("wall_S_reflection", 0.99, 0.05, 3000),
                                           ("wall_S_reflection", 0.90, 0.2, 3000),
                                           ("half_wall_S_open", 0.95, 0.15, 800)])
def test_equilibrium_bubbles_run_long(oracle, bc, T0, r, steps):
    from dim2d_finite_volume_b200 import field as F
    we = workloads.SERVED_WE
    d = workloads.domain(48, T0=T0, bubbles=[(0.0, 0.0, r)], bc=bc,
                         li=ic.interface_length(T0, we), we=we)
    p0 = oracle.get_params()
    oracle.set_params(we=we)
    try:
        ch, ty, od = F._preset(bc)
        cfg = oracle.make_cfg(d["nx"], d["ny"], periodic=False, bc_choice=ch, bc_type=ty,
                              bc_order=od)
        q = d["nodes"].copy()
        oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, d["x_map"], d["y_map"], q.copy(), q)
        oracle.set_threads(4)
        oracle.integrate(cfg, q, d["x_map"], d["y_map"], 0.0, d["dt"], steps)
        assert oracle.lib().orc_status() == 0
        assert np.isfinite(q[:, 2:-2, 2:-2]).all()
    finally:
        oracle.set_params(**{name: getattr(p0, name) for name, _ in p0._fields_})
