"""Pin the oracle (CPU restatement) to the reference's own known answers.

Fixtures in tests/golden/ were extracted from the reference's test programs
by tests/golden/make_golden.py:
  * Mattsson operators  -- test_augeanstables/test_mattsson_operators.f
  * DIM face fluxes     -- test_lernaeanhydra/test_dim2d_fluxes.f
Tolerance per value: half a unit of the last printed digit for rounded
literals (>= 6 significant digits), 1e-9 relative for exact ones.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")

# operator sets the oracle restates (diagonal n1/n2 sets are out of scope:
# they serve only the buffer-layer extension)
SETS = {"sd_interior": 0, "sd_x_oneside_L0": 1, "sd_x_oneside_L1": 2, "sd_x_oneside_R1": 3,
        "sd_x_oneside_R0": 4, "sd_y_oneside_L0": 5, "sd_y_oneside_L1": 6,
        "sd_y_oneside_R1": 7, "sd_y_oneside_R0": 8}


def _mattsson():
    return json.load(open(os.path.join(GOLD, "mattsson_operators.json")))


def _init_nodes(spec, n=7):
    a = np.zeros((4, n, n))
    for i, j, v in spec["nodes"]:
        a[0, j - 1, i - 1] = v
    return a


def _cases():
    d = _mattsson()
    out = []
    for c in d["cases"]:
        if c["set"] not in SETS:
            continue
        for k in sorted(c["expected"], key=int):
            out.append((c["name"], c["set"], int(k)))
    return out


@pytest.mark.parametrize("name,set_name,idx", _cases())
def test_mattsson_known_answers(oracle, name, set_name, idx):
    d = _mattsson()
    c = next(c for c in d["cases"] if c["name"] == name and c["set"] == set_name)
    ini = d["inits"][c["init"]]
    nodes = _init_nodes(ini)
    op = idx - 1
    if op in (0, 1, 2, 3, 4, 5, 6, 14):
        if c["test_only_g"]:
            pytest.skip("value not checked by the reference test")
        i, j = c["i1"], c["j1"]
    else:
        if c["test_only_f"]:
            pytest.skip("value not checked by the reference test")
        i, j = c["i2"], c["j2"]
    set_id = SETS[set_name]
    v = oracle.sd_operator(set_id, op, nodes, i, j, ini["dx"], ini["dy"])
    if np.isnan(v):
        pytest.skip("operator set %s not restated yet" % set_name)
    e = c["expected"][str(idx)]
    assert abs(v - e["value"]) <= e["tol"], (name, d["ops"][op], v, e["literal"])


def test_dim2d_flux_known_answers(oracle):
    f = json.load(open(os.path.join(GOLD, "dim2d_fluxes.json")))
    p = f["params"]
    oracle.set_params(re=p["re"], we=p["we"], pr=p["pr"], cv_r=p["cv_r"], viscous_r=p["viscous_r"])
    nodes = np.array(f["nodes"]).reshape(4, 5, 5)  # Fortran (5,5,4) -> [k][j][i]
    bad = []
    for k, e in sorted(f["expected"].items(), key=lambda kv: int(kv[0])):
        v = oracle.flux_function(int(k), nodes, f["i"], f["j"], f["dx"], f["dy"])
        if not abs(v - e["value"]) <= e["tol"]:
            bad.append((k, v, e["literal"]))
    assert not bad, bad
    assert len(f["expected"]) == 26


def _fortran_array(block):
    """reshape((/values/),(/a,b,c/)) -> C array [c][b][a]."""
    a, b, c = block["shape"]
    return np.array(block["values"]).reshape(c, b, a)


def test_hedstrom_characteristic_known_answers(oracle):
    """compute_timedev_with_openbc at an L0 and an R0 node
    (test_bc_operators/test_hedstrom_xy.f:54-136), far-field eigen-quantities."""
    h = json.load(open(os.path.join(GOLD, "hedstrom_xy.json")))
    oracle.set_params(cv_r=h["cv_r"])
    nL = _fortran_array(h["nodes_L0"])
    nR = _fortran_array(h["nodes_R0"])
    tdL = oracle.timedev_with_openbc(nL, h["i_L0"], h["j"], 0, 0, h["dx"], 0, h["obc_prim"])
    tdR = oracle.timedev_with_openbc(nR, h["i_R0"], h["j"], 0, 1, h["dx"], 1, h["obc_prim"])
    np.testing.assert_allclose(tdL, h["timedev_L0"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(tdR, h["timedev_R0"], rtol=0, atol=1e-10)


def test_periodic_ghost_known_answers(oracle):
    """periodic_xy legacy operator on nodes(i,j,k) = (i-1)+8(j-1)+100(k-1)
    (test_bc_operators/test_periodic_xy.f:94-190): ghosts bit-exact."""
    p = json.load(open(os.path.join(GOLD, "periodic_xy.json")))
    nx, ny = p["nx"], p["ny"]
    k, j, i = np.meshgrid(np.arange(4), np.arange(ny), np.arange(nx), indexing="ij")
    nodes = (i + 8 * j + 100 * k).astype(np.float64)
    cfg = oracle.make_cfg(nx, ny, periodic=True)
    x = np.arange(nx, dtype=np.float64)
    y = np.arange(ny, dtype=np.float64)
    oracle.apply_bc_on_nodes(cfg, 0.0, x, y, nodes.copy(), nodes)
    for b in p["expected_blocks"]:
        want = _fortran_array(b)  # [k][j][i] for the block
        got = nodes[:3, b["j"][0] - 1:b["j"][1], b["i"][0] - 1:b["i"][1]]
        assert np.array_equal(got, want), b


def test_wall_known_answers(oracle):
    """wall_xy_equilibrium_module.f unit functions and the capillarity parts
    of the wall x-flux (test_bc_operators/test_wall_xy_equilibrium.f)."""
    import ctypes
    w = json.load(open(os.path.join(GOLD, "wall_xy_equilibrium.json")))
    oracle.set_params(re=5.0, we=10.0, pr=20.0, cv_r=2.5, viscous_r=-1.5)
    L = oracle.lib()
    d, dp = ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    L.orc_dwall_internal_energy_dmd.restype = d
    L.orc_dwall_internal_energy_dmd.argtypes = [d, d, d]
    L.orc_wall_temperature.restype = d
    L.orc_wall_temperature.argtypes = [d] * 5
    L.orc_dmddx.restype = d
    L.orc_dmddx.argtypes = [d, dp, ctypes.c_int]
    L.orc_wall_capillarity_x.restype = d
    L.orc_wall_capillarity_x.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, d, d, ctypes.c_int]
    e = w["dwallInternalEnergy_dmd"]
    assert abs(L.orc_dwall_internal_energy_dmd(*e["args"]) - e["value"]) < 5e-10
    e = w["temperature"]
    assert abs(L.orc_wall_temperature(*e["args"]) - e["value"]) < 1e-12
    e = w["dmddx"]
    tab = np.array(e["args"][1:])
    assert L.orc_dmddx(e["args"][0], oracle.ptr(tab), 0) == e["value"]
    e = w["md_average"]
    assert 0.5 * (e["args"][0] + e["args"][1]) == e["value"]
    fn = w["flux_nodes"]
    nodes = np.full((4, 5, 5), fn["fill"])
    for a in fn["assign"]:
        i0, i1 = a["i"]
        nodes[a["k"] - 1, a["j"] - 1, i0 - 1:i1] = a["values"]
    i, j = fn["face"]
    got_x = L.orc_wall_capillarity_x(oracle.ptr(nodes), 5, 5, i, j, fn["dx"], fn["dy"], 0)
    got_y = L.orc_wall_capillarity_x(oracle.ptr(nodes), 5, 5, i, j, fn["dx"], fn["dy"], 1)
    assert abs(got_x - w["flux_x_capillarity_momentum_x"]) < 1e-9
    assert abs(got_y - w["flux_x_capillarity_momentum_y"]) < 1e-10


def test_timing_build_matches_checker_build(oracle):
    """The -O3 -march=native timing build of the oracle (the CPU baseline)
    gives the checker build's results bit for bit: same sources, same
    rounding order (no FMA contraction), per-cell loops without reductions."""
    import numpy as np
    from dim2d_finite_volume_b200 import field as F
    from tests.helpers import open_case, stable_dt
    nx, ny, x_map, y_map, q = open_case(40, 30, seed=3)
    ch, ty, od = F._preset("hedstrom_xy")
    cfg = oracle.make_cfg(nx, ny, bc_choice=ch, bc_type=ty, bc_order=od)
    dt = stable_dt(q, x_map, y_map)
    a, b = q.copy(), q.copy()
    oracle.integrate(cfg, a, x_map, y_map, 0.0, dt, 5)
    oracle.integrate(cfg, b, x_map, y_map, 0.0, dt, 5, fast=True)
    assert np.array_equal(a, b)
