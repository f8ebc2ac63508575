"""Batched fields (dim2d_batch_*): uneven domains of every boundary kind
advanced together must give each field's own result -- the same as the
field stepped alone through dim2d_step, and the oracle's.

The batched launch runs the same device code per domain as the single-field
strip kernel, compiled into another kernel, so results agree to rounding:
normwise <= 1e-12 against the field alone, <= 1e-10 against the oracle."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err_all, open_case, periodic_case, stable_dt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


@pytest.fixture(scope="module")
def B():
    from dim2d_finite_volume_b200 import batch
    return batch


# (preset, interior n, ny, seed)
MIX = [("periodic_xy", 64, 48, 1), ("hedstrom_xy", 70, 52, 2), ("wall_S_reflection", 56, 40, 3),
       ("reflection_xy", 48, 64, 4), ("periodic_xy", 33, 97, 5), ("hedstrom_xy", 100, 40, 6),
       ("wall_S_reflection", 90, 72, 7), ("half_wall_S_open", 66, 50, 8),
       ("wall_S_open", 45, 61, 9)]


def _case(preset, n, ny, seed):
    if preset == "hedstrom_xy":
        return open_case(n, ny, seed=seed, radius=0.15)
    return periodic_case(n, ny, radius=0.15, seed=seed)


def _prepared(oracle, F, preset, n, ny, seed):
    nx, nyy, x_map, y_map, q = _case(preset, n, ny, seed)
    if preset != "hedstrom_xy":  # field%ini applies the node boundary pass
        if preset == "periodic_xy":
            cfg = oracle.make_cfg(nx, nyy, periodic=True)
        else:
            bc = F._preset(preset)
            cfg = oracle.make_cfg(nx, nyy, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                                  bc_order=bc[2])
            oracle.lib().orc_clear_status()
        oracle.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)
    return nx, nyy, x_map, y_map, q, stable_dt(q, x_map, y_map)


def _alone(F, preset, nx, ny, x_map, y_map, q, dt, nsteps, variant=2):
    with F.Field(nx, ny, bc=preset) as fld:
        fld.variant = variant
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, nsteps)
        return fld.download(), fld.time


def _err(a, b, preset):
    if preset in ("periodic_xy", "hedstrom_xy"):
        return normwise_rel_err_all(a, b)
    return normwise_rel_err_all(a[:, 2:-2, 2:-2], b[:, 2:-2, 2:-2])


@pytest.mark.parametrize("graphs", [True, False])
def test_mixed_batch_matches_fields_alone(oracle, F, B, graphs):
    cases = [(p,) + _prepared(oracle, F, p, n, ny, s) for p, n, ny, s in MIX]
    fields = []
    with B.Batch() as bt:
        bt.set_graphs(graphs)
        for p, nx, ny, x_map, y_map, q, dt in cases:
            fld = F.Field(nx, ny, bc=p)
            fld.ini(q, x_map, y_map)
            bt.add(fld, dt)
            fields.append(fld)
        assert bt.size == len(MIX)
        assert bt.cells == sum((c[1] - 4) * (c[2] - 4) for c in cases)
        bt.step(7)
        bt.step(5)
        bt.sync()
        for (p, nx, ny, x_map, y_map, q, dt), fld in zip(cases, fields):
            got = fld.download()
            ref, t_ref = _alone(F, p, nx, ny, x_map, y_map, q, dt, 12)
            assert np.isfinite(got).all()
            assert np.all(_err(got, ref, p) <= 1e-12), (p, nx, ny)
            assert abs(fld.time - t_ref) <= 1e-15 * max(1.0, abs(t_ref))
    for fld in fields:
        fld.close()


def test_batch_matches_oracle(oracle, F, B):
    picks = [MIX[0], MIX[1], MIX[2], MIX[7], MIX[8]]
    cases = [(p,) + _prepared(oracle, F, p, n, ny, s) for p, n, ny, s in picks]
    fields = []
    with B.Batch() as bt:
        for p, nx, ny, x_map, y_map, q, dt in cases:
            fld = F.Field(nx, ny, bc=p)
            fld.ini(q, x_map, y_map)
            bt.add(fld, dt)
            fields.append(fld)
        bt.step(30)
        bt.sync()
        oracle.set_threads(8)
        for (p, nx, ny, x_map, y_map, q, dt), fld in zip(cases, fields):
            if p == "periodic_xy":
                cfg = oracle.make_cfg(nx, ny, periodic=True)
            else:
                bc = F._preset(p)
                cfg = oracle.make_cfg(nx, ny, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                                      bc_order=bc[2])
            ref = q.copy()
            oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 30)
            assert np.all(_err(fld.download(), ref, p) <= 1e-10), p
    for fld in fields:
        fld.close()


def test_membership_changes_between_steps(oracle, F, B):
    cases = [(p,) + _prepared(oracle, F, p, n, ny, s) for p, n, ny, s in MIX[:4]]
    f = []
    with B.Batch() as bt:
        for p, nx, ny, x_map, y_map, q, dt in cases:
            fld = F.Field(nx, ny, bc=p)
            fld.ini(q, x_map, y_map)
            f.append(fld)
        bt.add(f[0], cases[0][-1])
        bt.add(f[1], cases[1][-1])
        bt.step(3)
        bt.add(f[2], cases[2][-1])   # joins after 3 steps
        bt.step(2)
        bt.remove(f[0])              # leaves after 5 steps
        bt.add(f[3], cases[3][-1])
        bt.step(4)
        bt.sync()
        n_steps = [5, 9, 6, 4]
        for c, fld, n in zip(cases, f, n_steps):
            p, nx, ny, x_map, y_map, q, dt = c
            ref, _ = _alone(F, p, nx, ny, x_map, y_map, q, dt, n)
            assert np.all(_err(fld.download(), ref, p) <= 1e-12), p
    for fld in f:
        fld.close()


def test_group_larger_than_one_launch(F, B):
    """70 periodic domains: the group is split over two launches."""
    nx, ny, x_map, y_map, q = periodic_case(20, 16, seed=9)
    dt = stable_dt(q, x_map, y_map)
    ref, _ = _alone(F, "periodic_xy", nx, ny, x_map, y_map, q, dt, 3)
    fields = []
    with B.Batch() as bt:
        for i in range(70):
            fld = F.Field(nx, ny, bc="periodic_xy")
            fld.ini(q, x_map, y_map)
            bt.add(fld, dt)
            fields.append(fld)
        bt.step(3)
        bt.sync()
        for fld in fields:
            assert np.all(normwise_rel_err_all(fld.download(), ref) <= 1e-12)
    for fld in fields:
        fld.close()


def test_autotune_keeps_state_and_picks_shapes(oracle, F, B):
    cases = [(p,) + _prepared(oracle, F, p, n, ny, s) for p, n, ny, s in MIX[:3]]
    fields = []
    with B.Batch() as bt:
        for p, nx, ny, x_map, y_map, q, dt in cases:
            fld = F.Field(nx, ny, bc=p)
            fld.ini(q, x_map, y_map)
            bt.add(fld, dt)
            fields.append(fld)
        before = [fld.download() for fld in fields]
        shapes, times = bt.autotune()
        assert all(0 <= s < B.NSHAPES for s in shapes)
        for g in range(3):  # non-empty groups have measured times
            assert np.all(times[g] > 0)
            assert times[g][shapes[g]] == times[g].min()
        bt.sync()
        for b0, fld in zip(before, fields):
            assert np.array_equal(fld.download(), b0)
    for fld in fields:
        fld.close()


def test_member_rules(oracle, F, B):
    p, nx, ny, x_map, y_map, q, dt = ("periodic_xy",) + _prepared(oracle, F, "periodic_xy",
                                                                  24, 20, 1)
    with B.Batch() as bt, F.Field(nx, ny) as fld, F.Field(nx, ny) as other:
        fld.ini(q, x_map, y_map)
        bt.add(fld, dt)
        with pytest.raises(F.Dim2dError):
            bt.add(fld, dt)          # already a member
        with pytest.raises(F.Dim2dError):
            fld.integrate(dt, 1)     # advanced by its batch only
        with pytest.raises(F.Dim2dError):
            bt.add(other, dt)        # no state uploaded
        odd = F.Field(nx, ny, params=F.default_params(re=7.0))
        odd.ini(q, x_map, y_map)
        with pytest.raises(F.Dim2dError):
            bt.add(odd, dt)          # other physical constants
        odd.close()
        bt.remove(fld)
        fld.integrate(dt, 1)         # free again


def test_fp64_and_mixed_members_in_one_batch(oracle, F, B):
    """Mixed-precision members form their own groups; each member's result
    equals the field alone: FP64 to 1e-12, mixed to 1e-6 (the FP32 face
    pass of the batched kernel against the single-field kernel)."""
    picks = [MIX[0], MIX[1], MIX[2], MIX[3], MIX[7]]
    cases = [(p,) + _prepared(oracle, F, p, n, ny, s) for p, n, ny, s in picks]
    fields, precs = [], []
    with B.Batch() as bt:
        for k, (p, nx, ny, x_map, y_map, q, dt) in enumerate(cases):
            for prec in (F.FP64, F.MIXED):
                fld = F.Field(nx, ny, bc=p, precision=prec)
                fld.ini(q, x_map, y_map)
                bt.add(fld, dt)
                fields.append((k, fld))
                precs.append(prec)
        bt.step(6)
        bt.sync()
        for (k, fld), prec in zip(fields, precs):
            p, nx, ny, x_map, y_map, q, dt = cases[k]
            with F.Field(nx, ny, bc=p, precision=prec) as alone:
                alone.variant = 2
                alone.ini(q, x_map, y_map)
                alone.integrate(dt, 6)
                ref = alone.download()
            bar = 1e-6 if prec == F.MIXED else 1e-12
            assert np.all(_err(fld.download(), ref, p) <= bar), (p, prec)
    for _, fld in fields:
        fld.close()
