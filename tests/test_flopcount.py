"""FP64 operation count of the oracle per cell-update (oracle/flopcount.cpp).

The counting build compiles the oracle's own C sources as C++ with a double
that counts its arithmetic.  These tests check that it computes exactly what
the oracle computes (so the count is the oracle's work, not a variant's),
that its figures are the ones committed beside the kernel's ncu counts in
profiles/fp64_ops.json (which bench.py reports), and that the counts add up
(an RK3 step is three time derivatives plus three stage updates).
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_build", "flopcount")


@pytest.fixture(scope="module")
def counted(tmp_path_factory):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "flopcount"], check=True)
    pre = str(tmp_path_factory.mktemp("flops") / "periodic")
    out = subprocess.run([EXE, pre], check=True, capture_output=True, text=True).stdout
    return json.loads(out), pre


def test_counting_build_computes_the_oracle(oracle, counted):
    """Bit-identical time derivative from the counting build and the oracle."""
    _, pre = counted
    n = 132
    nodes = np.fromfile(pre + ".nodes").reshape(4, n, n)
    td = np.fromfile(pre + ".td").reshape(4, n, n)
    p0 = oracle.get_params()
    try:
        oracle.set_params(re=5.0, we=10.0, pr=20.0, cv_r=2.5, viscous_r=-1.5, gravity_ac=0)
        x, y = oracle.ini_coordinates(n, n, -0.5, 0.5, -0.5, 0.5)
        from dim2d_finite_volume_b200 import field
        ch, ty, od = field._preset("periodic_xy")
        cfg = oracle.make_cfg(n, n, periodic=True, bc_choice=ch, bc_type=ty, bc_order=od)
        ref = oracle.compute_time_dev(cfg, 0.0, nodes, x, y)
    finally:
        oracle.set_params(**{name: getattr(p0, name) for name, _ in p0._fields_})
    inner = (slice(None), slice(2, n - 2), slice(2, n - 2))
    assert np.array_equal(td[inner], ref[inner])


def test_counts_match_the_committed_figures(counted):
    d, _ = counted
    committed = json.load(open(os.path.join(ROOT, "profiles", "fp64_ops.json")))
    assert committed["oracle"] == d


def test_counts_add_up(counted):
    d, _ = counted
    for bc in ("periodic_xy", "hedstrom_xy"):
        td = d["%s_time_dev" % bc]
        step = d["%s_rk3_step" % bc]
        assert td["flops"] > 500  # flux formulas, operators and primitives per cell
        # three time derivatives plus the stage arithmetic (a few dozen per cell)
        assert 3 * td["flops"] < step["flops"] < 3 * td["flops"] + 100
        parts = step["add"] + step["mul"] + step["div"] + step["sqrt"] + step["transcendental"]
        assert abs(parts - step["flops"]) < 0.5
    # the open boundary adds its ghost-cell work to the interior's
    assert d["hedstrom_xy_rk3_step"]["flops"] > d["periodic_xy_rk3_step"]["flops"]
