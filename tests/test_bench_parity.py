"""The error against the oracle that bench.py states with every run
(cpu_baseline.parity): the checker itself, on the CPU.  A state equal to the
oracle's reports zero error; a mistake planted in one conservative variable
shows up in that variable alone, at its size."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("bc", ["hedstrom_xy", "periodic_xy", "wall_S_reflection"])
def test_parity_check_reports_planted_error(oracle, bc):
    sys.path.insert(0, ROOT)
    import bench

    w = bench.workload(64, 1234, 0, bc=bc)
    nx, ny = w["nx"], w["ny"]
    q = np.ascontiguousarray(w["nodes"], dtype=np.float64).copy()
    cfg = bench.oracle_cfg(oracle, bc, nx, ny)
    if bc not in ("periodic_xy", "hedstrom_xy"):
        oracle.apply_bc_on_nodes(cfg, 0.0, w["x_map"], w["y_map"], q.copy(), q)
    oracle.integrate(cfg, q, w["x_map"], w["y_map"], 0.0, w["dt"], bench.PARITY_STEPS)

    same = bench.parity_vs_oracle(oracle, w, q.copy())
    assert same["max_rel"] == [0.0] * 4 and same["l2_rel"] == [0.0] * 4

    planted = q.copy()
    j, i = ny // 2, nx // 3
    planted[3, j, i] += 1e-8 * np.abs(q[3, 2:ny - 2, 2:nx - 2]).max()
    got = bench.parity_vs_oracle(oracle, w, planted)
    assert got["max_rel"][:3] == [0.0] * 3
    assert got["max_rel"][3] == pytest.approx(1e-8, rel=1e-6)
    assert 0.0 < got["l2_rel"][3] < 1e-8
