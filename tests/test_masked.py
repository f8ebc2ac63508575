"""Masked ("_nopt") interior operators of buffer-layer grids:
dim2d_time_dev_masked and dim2d_rk_stage_masked against the oracle's
restatement of compute_time_dev_nopt's interior part
(td_operators_class.f:293-417, pmodel_eq_class.f:1215-1360) and of
compute_1st/2nd/3rd_step_nopt (rk3tvd_steps_module.f:130-614).

Grids are laid out as the reference's buffer layers: an L-shaped interior_pt
region, one ring of bc_interior_pt around it, one ring of bc_pt, no_pt
elsewhere (parameters_bf_layer.f:41-44).  Points outside the mask must keep
their values.  Bars (FP64): <= 1e-12 normwise for the time derivative,
<= 1e-11 after a masked RK3 step."""
import numpy as np
import pytest

from dim2d_finite_volume_b200.workloads import layer_map
from tests.helpers import periodic_case


def _case(n=44, ny=36, seed=3):
    nx, nyy, x_map, y_map, q = periodic_case(n, ny, radius=0.15, seed=seed)
    # an L-shaped interior at least bc_size + 2 points from the edges
    g = layer_map(nx, nyy, [(4, nx - 5, 4, nyy // 2), (4, nx // 2, nyy // 2, nyy - 5)])
    return nx, nyy, x_map, y_map, np.ascontiguousarray(q), g


def test_layer_map_rings():
    g = layer_map(12, 10, [(4, 7, 3, 6)])
    assert (g == 1).sum() == 16 and (g == 2).sum() == 20 and (g == 3).sum() == 28
    assert g[0].tolist() == [0] * 12           # nothing wraps around the grid
    assert g[3, 2] == 3 and g[3, 3] == 2 and g[3, 4] == 1


def test_oracle_masked_matches_full_grid_on_interior_points(oracle):
    nx, ny, x_map, y_map, q, g = _case()
    dx, dy = x_map[1] - x_map[0], y_map[1] - y_map[0]
    td = np.full_like(q, 7.0)
    oracle.compute_time_dev_masked(q, g, dx, dy, (3, nx - 2), (3, ny - 2), td)
    cfg = oracle.make_cfg(nx, ny, periodic=True)
    ref = oracle.compute_time_dev(cfg, 0.0, q, x_map, y_map)
    m = g == 1
    assert np.array_equal(td[:, m], ref[:, m])  # same faces, same formulas
    assert np.all(td[:, ~m] == 7.0)             # nothing written elsewhere


def test_oracle_masked_stages_leave_no_pt_alone(oracle):
    nx, ny, x_map, y_map, q, g = _case()
    rng = np.random.default_rng(1)
    td = rng.standard_normal(q.shape)
    u = q.copy()
    tmp = np.zeros_like(q)
    oracle.rk_stage_masked(1, u, tmp, td, g, 1e-3, (3, nx - 2), (3, ny - 2))
    assert np.array_equal(u[:, g == 0], q[:, g == 0])
    assert np.array_equal(tmp[:, g != 0], q[:, g != 0])
    assert np.array_equal(u[:, g != 0], q[:, g != 0] + 1e-3 * td[:, g != 0])


def _gpu_time_dev(F, torch, params, q, g, dx, dy, xb, yb, fill):
    qd = torch.from_numpy(q).cuda()
    gd = torch.from_numpy(g).cuda()
    td = torch.from_numpy(fill.copy()).cuda()
    ny, nx = g.shape
    F.time_dev_masked(params, nx, ny, qd.data_ptr(), gd.data_ptr(), dx, dy, xb, yb, td.data_ptr())
    torch.cuda.synchronize()
    return td.cpu().numpy()


BORDERS = {"full": lambda nx, ny: ((3, nx - 2), (3, ny - 2)),
           "narrow": lambda nx, ny: ((9, nx - 8), (6, ny - 10)),
           # first border column 8: the box starts at the odd column 7
           "odd": lambda nx, ny: ((8, nx - 7), (5, ny - 9))}


# even nx: the warp-strip kernel (rows copied as 16-byte pairs), 8-row strips
# where 16-row ones would not fill the GPU (2048 x 600 takes 16-row strips);
# odd nx: the tile kernel; 100 x 83 spans several strips and row blocks, the
# last ones partial
@pytest.mark.gpu
@pytest.mark.parametrize("n,ny,borders", [(44, 36, "full"), (44, 36, "narrow"), (44, 36, "odd"),
                                          (43, 36, "full"), (43, 36, "odd"),
                                          (100, 83, "odd"), (100, 83, "full"),
                                          (2048, 600, "odd")])
def test_time_dev_masked_matches_oracle(oracle, n, ny, borders):
    import torch

    from dim2d_finite_volume_b200 import field as F
    nx, ny, x_map, y_map, q, g = _case(n, ny)
    dx, dy = x_map[1] - x_map[0], y_map[1] - y_map[0]
    xb, yb = BORDERS[borders](nx, ny)
    fill = np.full_like(q, 7.0)
    ref = fill.copy()
    oracle.compute_time_dev_masked(q, g, dx, dy, xb, yb, ref)
    got = _gpu_time_dev(F, torch, F.default_params(), q, g, dx, dy, xb, yb, fill)
    m = np.zeros_like(g, bool)
    m[yb[0] - 1:yb[1], xb[0] - 1:xb[1]] = True
    m &= g == 1
    assert m.sum() > 100
    for k in range(4):
        den = np.abs(ref[k][m]).max()
        assert np.abs(got[k][m] - ref[k][m]).max() <= 1e-12 * den, k
    assert np.all(got[:, ~m] == 7.0)  # the other points are untouched


@pytest.mark.gpu
@pytest.mark.parametrize("n", [44, 43])
def test_time_dev_masked_with_gravity(oracle, n):
    """The body force (pmodel_eq_class.f:1840-1918) in the masked time
    derivative: strip kernel (even nx) and tile kernel (odd nx)."""
    import torch

    from dim2d_finite_volume_b200 import field as F
    nx, ny, x_map, y_map, q, g = _case(n, 36, seed=7)
    dx, dy = x_map[1] - x_map[0], y_map[1] - y_map[0]
    xb, yb = BORDERS["odd"](nx, ny)
    fill = np.full_like(q, 7.0)
    ref = fill.copy()
    p0 = oracle.get_params()
    try:
        oracle.set_params(gravity_ac=1, gravity=0.7)
        oracle.compute_time_dev_masked(q, g, dx, dy, xb, yb, ref)
    finally:
        oracle.set_params(**{name: getattr(p0, name) for name, _ in p0._fields_})
    got = _gpu_time_dev(F, torch, F.default_params(gravity_ac=1, gravity=0.7), q, g, dx, dy,
                        xb, yb, fill)
    m = np.zeros_like(g, bool)
    m[yb[0] - 1:yb[1], xb[0] - 1:xb[1]] = True
    m &= g == 1
    for k in range(4):
        den = np.abs(ref[k][m]).max()
        assert np.abs(got[k][m] - ref[k][m]).max() <= 1e-12 * den, k
    # the body force changes the momentum_y and energy derivatives
    plain = fill.copy()
    oracle.compute_time_dev_masked(q, g, dx, dy, xb, yb, plain)
    assert np.abs(ref[2][m] - plain[2][m]).max() > 5e-4 * np.abs(plain[2][m]).max()
    assert np.all(got[:, ~m] == 7.0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [44, 43])
def test_masked_rk3_step_matches_oracle(oracle, n):
    """A whole masked step: time derivative, stage, three times; the layer's
    boundary points take a fixed time derivative, as its boundary sections
    would supply."""
    import torch

    from dim2d_finite_volume_b200 import field as F
    nx, ny, x_map, y_map, q, g = _case(n, seed=5)
    dx, dy = x_map[1] - x_map[0], y_map[1] - y_map[0]
    xb, yb = (3, nx - 2), (3, ny - 2)
    dt = 2e-6
    bc_td = np.random.default_rng(2).standard_normal(q.shape) * 1e-2
    # oracle
    u, tmp = q.copy(), np.zeros_like(q)
    for st in (1, 2, 3):
        td = bc_td.copy()
        oracle.compute_time_dev_masked(u, g, dx, dy, xb, yb, td)
        oracle.rk_stage_masked(st, u, tmp, td, g, dt, xb, yb)
    # GPU
    ud = torch.from_numpy(q.copy()).cuda()
    tmpd = torch.zeros_like(ud)
    gd = torch.from_numpy(g).cuda()
    p = F.default_params()
    for st in (1, 2, 3):
        tdd = torch.from_numpy(bc_td.copy()).cuda()
        F.time_dev_masked(p, nx, ny, ud.data_ptr(), gd.data_ptr(), dx, dy, xb, yb, tdd.data_ptr())
        F.rk_stage_masked(st, nx, ny, ud.data_ptr(), tmpd.data_ptr(), tdd.data_ptr(), gd.data_ptr(),
                          dt, xb, yb)
    torch.cuda.synchronize()
    got = ud.cpu().numpy()
    for k in range(4):
        den = np.abs(u[k][g != 0]).max()
        assert np.abs(got[k] - u[k]).max() <= 1e-11 * den, k
    assert np.array_equal(got[:, g == 0], q[:, g == 0])


@pytest.mark.gpu
def test_masked_calls_reject_bad_arguments():
    from dim2d_finite_volume_b200 import field as F
    p = F.default_params()
    with pytest.raises(F.Dim2dError):
        F.time_dev_masked(p, 40, 30, 8, 8, 0.1, 0.1, (0, 40), (3, 28), 8)  # border below 1
    with pytest.raises(F.Dim2dError):
        F.rk_stage_masked(4, 40, 30, 8, 8, 8, 8, 1e-3, (3, 38), (3, 28))   # no stage 4
