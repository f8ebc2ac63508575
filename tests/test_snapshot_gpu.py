"""Overlapped snapshots and restarts on the GPU: the asynchronous copy
(dim2d_download_async) must capture exactly the state of its step while the
following steps run -- including the step that overwrites the copied buffer,
which must wait for the copy -- and a restart from a written file must
continue bit-identically to an uninterrupted run."""
import numpy as np
import pytest

from dim2d_finite_volume_b200 import snapshot as S
from tests.helpers import open_case, periodic_case, stable_dt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


@pytest.mark.parametrize("bc,graphs", [("periodic_xy", True), ("hedstrom_xy", True),
                                       ("periodic_xy", False)])
def test_snapshots_match_synchronous_downloads(F, tmp_path, bc, graphs):
    case = open_case if bc == "hedstrom_xy" else periodic_case
    nx, ny, x_map, y_map, q = case(90, 70, seed=4)
    dt = stable_dt(q, x_map, y_map)
    plan = [3, 1, 4, 2]  # steps before each snapshot
    with F.Field(nx, ny, bc=bc) as fld, F.Field(nx, ny, bc=bc) as ref:
        for f in (fld, ref):
            f.set_graphs(graphs)
            f.variant = 2
            f.ini(q, x_map, y_map)
        snap = S.Snapshotter(fld, S.run_attrs(fld, dt))
        expect = []
        for i, n in enumerate(plan):
            fld.integrate(dt, n)
            snap.snapshot(tmp_path / ("s%d.nc" % i))
            ref.integrate(dt, n)
            expect.append((ref.download(), ref.time))
        fld.integrate(dt, 5)  # keeps stepping over the copied buffers
        snap.close()
        for i, (want, t) in enumerate(expect):
            got, gx, gy, gt, att = S.read_snapshot(tmp_path / ("s%d.nc" % i))
            assert np.array_equal(got, want), i
            assert gt == t and np.array_equal(gx, x_map) and att["dt"] == dt


def test_restart_continues_bit_identically(F, tmp_path):
    nx, ny, x_map, y_map, q = periodic_case(80, 64, seed=6)
    dt = stable_dt(q, x_map, y_map)
    with F.Field(nx, ny) as fld:
        fld.variant = 2
        fld.ini(q, x_map, y_map)
        fld.integrate(dt, 3)
        snap = S.Snapshotter(fld)
        snap.snapshot(tmp_path / "r.nc")
        fld.integrate(dt, 5)
        snap.close()
        straight = fld.download()
        t_straight = fld.time
    nodes, xr, yr, tr, _ = S.read_snapshot(tmp_path / "r.nc")
    with F.Field(nx, ny) as fld:
        fld.variant = 2
        fld.ini(nodes, xr, yr, tr)
        fld.integrate(dt, 5)
        assert np.array_equal(fld.download(), straight)
        assert fld.time == t_straight


def test_async_download_refused_for_batch_members(F):
    from dim2d_finite_volume_b200 import batch as B
    nx, ny, x_map, y_map, q = periodic_case(40, 32, seed=2)
    with B.Batch() as bt, F.Field(nx, ny) as fld:
        fld.ini(q, x_map, y_map)
        bt.add(fld, 1e-6)
        buf = F.pinned_empty((4, ny, nx))
        with pytest.raises(F.Dim2dError):
            fld.download_async(buf)
