"""The persistent batched kernel (dim2d_batch_set_persistent): one launch
per precision advances every member by n steps, work items taken in
dependency order, per-field completion counters instead of grid barriers.

Checked against the graph mode of the same batch (same per-cell code:
FP64 normwise <= 1e-13, and equal bit for bit is reported; mixed precision
<= 1e-6, as FP32 face arithmetic compiled into another kernel may round
differently), against the oracle (<= 1e-10 after 30 steps), across odd and
even step counts (the A/B buffer parity), ragged sizes whose last row band
would hold a single row, with the autotuner, and the bounded waits:
a work item whose completion is withheld makes the waits of the items
after it run out, the launch stops, dim2d_batch_sync returns
DIM2D_ERR_TIMEOUT, and the device stays usable."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err_all
from tests.test_batch import MIX, _err, _prepared

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


@pytest.fixture(scope="module")
def B():
    from dim2d_finite_volume_b200 import batch
    return batch


def _run(F, B, cases, steps, persistent, precision=0, rows=None, autotune=False):
    fields = []
    with B.Batch() as bt:
        bt.set_persistent(persistent)
        if rows:
            bt.set_rows(rows)
        for p, nx, ny, x_map, y_map, q, dt in cases:
            fld = F.Field(nx, ny, bc=p, precision=precision)
            fld.ini(q, x_map, y_map)
            bt.add(fld, dt)
            fields.append(fld)
        if autotune:
            chosen, times = bt.autotune()
        for n in steps:
            bt.step(n)
        bt.sync()
        out = [(fld.download(), fld.time) for fld in fields]
    for fld in fields:
        fld.close()
    return (out, chosen, times) if autotune else out


@pytest.fixture(scope="module")
def cases(oracle, F):
    return [(p,) + _prepared(oracle, F, p, n, ny, s) for p, n, ny, s in MIX]


@pytest.mark.parametrize("rows", [8, 16, 32])
def test_persistent_matches_graph_mode(F, B, cases, rows):
    ref = _run(F, B, cases, (7, 5), persistent=False)
    got = _run(F, B, cases, (7, 5), persistent=True, rows=rows)
    identical = 0
    for (p, *_), (g, tg), (r, tr) in zip(cases, got, ref):
        assert np.isfinite(g).all(), p
        assert np.all(_err(g, r, p) <= 1e-13), (p, _err(g, r, p))
        assert tg == tr
        identical += int(np.array_equal(g, r))
    print("persistent rows=%d: %d of %d fields bit-identical to the graph mode"
          % (rows, identical, len(cases)))


def test_persistent_matches_oracle(oracle, F, B, cases):
    got = _run(F, B, cases, (30,), persistent=True)
    oracle.set_threads(8)
    for (p, nx, ny, x_map, y_map, q, dt), (g, _) in zip(cases, got):
        if p == "periodic_xy":
            cfg = oracle.make_cfg(nx, ny, periodic=True)
        else:
            bc = F._preset(p)
            cfg = oracle.make_cfg(nx, ny, periodic=False, bc_choice=bc[0], bc_type=bc[1],
                                  bc_order=bc[2])
        ref = q.copy()
        oracle.integrate(cfg, ref, x_map, y_map, 0.0, dt, 30)
        assert np.all(_err(g, ref, p) <= 1e-10), (p, _err(g, ref, p))


MIXED_TOL = 1e-6


def test_persistent_mixed_precision_matches_graph_mode(F, B, cases):
    ref = _run(F, B, cases, (6,), persistent=False, precision=F.MIXED)
    got = _run(F, B, cases, (6,), persistent=True, precision=F.MIXED)
    for (p, *_), (g, _), (r, _) in zip(cases, got, ref):
        assert np.all(_err(g, r, p) <= MIXED_TOL), (p, _err(g, r, p))


def test_persistent_both_precisions_in_one_batch(F, B, cases):
    """FP64 and mixed members in one batch: one launch each, on their own
    streams; each matches its precision's graph-mode result."""
    fields = []
    with B.Batch() as bt:
        bt.set_persistent(True)
        for i, (p, nx, ny, x_map, y_map, q, dt) in enumerate(cases):
            fld = F.Field(nx, ny, bc=p, precision=F.MIXED if i % 2 else F.FP64)
            fld.ini(q, x_map, y_map)
            bt.add(fld, dt)
            fields.append(fld)
        bt.step(5)
        bt.sync()
        got = [fld.download() for fld in fields]
    for fld in fields:
        fld.close()
    ref64 = _run(F, B, cases, (5,), persistent=False)
    refmx = _run(F, B, cases, (5,), persistent=False, precision=F.MIXED)
    for i, (p, *_) in enumerate(cases):
        r = (refmx if i % 2 else ref64)[i][0]
        assert np.all(_err(got[i], r, p) <= (MIXED_TOL if i % 2 else 1e-13)), (i, p)


@pytest.mark.parametrize("rows", [16, 32])
def test_persistent_long_run_matches_graph_mode(F, B, rows):
    """300 steps in 6 launches on twelve of the batched workload's domains
    (the smallest four of each kind, which stay physical that long): races
    between bands or stages would show as differences growing with the run;
    FP64 stays at amplified rounding (the open boundary's: ~3e-11 in rho v
    after 300 steps)."""
    from dim2d_finite_volume_b200 import workloads
    specs = workloads.batched_specs(1311, 64)
    idx = []
    for kind in ("hedstrom_xy", "wall_S_reflection", "periodic_xy"):
        idx += [i for _, i in sorted((s["n"], i) for i, s in enumerate(specs)
                                     if s["bc"] == kind)[:4]]
    doms = [workloads.batched_domain(specs[i]) for i in idx]
    outs = []
    for persistent in (False, True):
        fields = []
        with B.Batch() as bt:
            bt.set_persistent(persistent)
            if persistent:
                bt.set_rows(rows)
            for d in doms:
                fld = F.Field(d["nx"], d["ny"], bc=d["bc"], params=workloads.batch_params())
                fld.ini(d["nodes"], d["x_map"], d["y_map"])
                if d["bc"] not in ("periodic_xy", "hedstrom_xy"):
                    fld.apply_bc_on_nodes()
                bt.add(fld, d["dt"])
                fields.append(fld)
            for _ in range(6):
                bt.step(50)
            bt.sync()
            outs.append([fld.download() for fld in fields])
        for fld in fields:
            fld.close()
    for d, r, g in zip(doms, outs[0], outs[1]):
        err = _err(g, r, d["bc"])
        assert np.isfinite(g).all(), d["bc"]
        assert np.all(err <= 1e-9), (d["bc"], d["nx"], err)


WALL_PRESETS = ("wall_S_reflection", "half_wall_S_open", "wall_S_open")


def test_unwritten_ghost_cells_keep_uploaded_values(F, B, cases):
    """Ghost cells that no boundary operator writes -- on a south wall the
    energy of both ghost rows and the momenta of the outer one (the wall
    pass sets the density ghosts and the inner momenta) -- keep the uploaded
    values whichever of the ping-pong buffers holds the state: after an odd
    number of steps, alone, in the graph mode and in the persistent mode;
    and the two batch modes then agree over all cells, ghosts included."""
    walls = [c for c in cases if c[0] in WALL_PRESETS]
    graph = _run(F, B, walls, (7,), persistent=False)
    pers = _run(F, B, walls, (7,), persistent=True)
    for (p, nx, ny, x_map, y_map, q, dt), (g, _), (r, _) in zip(walls, graph, pers):
        assert np.all(normwise_rel_err_all(r, g) <= 1e-13), (p, normwise_rel_err_all(r, g))
        for out in (g, r):
            assert np.array_equal(out[3, :2, 2:-2], q[3, :2, 2:-2]), p  # energy, both rows
            assert np.array_equal(out[1:3, 0, 2:-2], q[1:3, 0, 2:-2]), p  # momenta, outer row
    p, nx, ny, x_map, y_map, q, dt = walls[0]
    with F.Field(nx, ny, bc=p) as fld:
        fld.ini(q, x_map, y_map)
        fld.apply_bc_on_nodes()  # field%ini
        fld.variant = 2
        fld.integrate(dt, 7)
        out = fld.download()
    assert np.array_equal(out[3, :2, 2:-2], q[3, :2, 2:-2])
    assert np.array_equal(out[1:3, 0, 2:-2], q[1:3, 0, 2:-2])


def test_persistent_autotune_keeps_state(F, B, cases):
    (out, chosen, times) = _run(F, B, cases[:4], (3,), persistent=True, autotune=True)
    assert all(c in (8, 16, 32) for c in chosen)
    assert np.all(times[:, :3] > 0)
    ref = _run(F, B, cases[:4], (3,), persistent=False)
    for (p, *_), (g, _), (r, _) in zip(cases[:4], out, ref):
        assert np.all(_err(g, r, p) <= 1e-13), p


def test_withheld_item_times_out_and_device_stays_usable(F, B, cases):
    p, nx, ny, x_map, y_map, q, dt = cases[0]
    fld = F.Field(nx, ny, bc=p)
    fld.ini(q, x_map, y_map)
    with B.Batch() as bt:
        bt.set_persistent(True)
        bt.add(fld, dt)
        bt.set_wait_limit(0.05)
        bt.withhold_item(0)  # the field's first item never reports completion
        bt.step(2)
        with pytest.raises(F.Dim2dError) as ex:
            bt.sync()
        assert ex.value.code == 6  # DIM2D_ERR_TIMEOUT
        # the launch stopped; the context is fine: a normal batch step works
        bt.withhold_item(-1)
        bt.remove(fld)
    fld.ini(q, x_map, y_map)
    fld.integrate(dt, 2)
    assert np.isfinite(fld.download()).all()
    fld.close()
