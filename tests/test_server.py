"""Serving loop (dim2d_server_*): requests arriving over time are admitted
by free memory and advanced together in batched chunks; every result must
be the same alone and in the mix.

"Alone" is the request's field stepped by itself through dim2d_step; in
the mix it shares batched launches with other requests, joining and
leaving between chunks.  Bar (FP64): normwise <= 1e-12 over all cells of
open fields and the interior of wall fields."""
import numpy as np
import pytest

from tests.helpers import normwise_rel_err_all

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


@pytest.fixture(scope="module")
def S():
    from dim2d_finite_volume_b200 import server
    return server


def _requests(count, seed, n_range=(36, 110), kinds=None):
    from dim2d_finite_volume_b200 import workloads
    return workloads.served_requests(seed, count, rate=200.0, n_range=n_range,
                                     steps_range=(20, 90),
                                     kinds=kinds or workloads.SERVED_KINDS)


def _params():
    from dim2d_finite_volume_b200 import workloads
    return workloads.served_params()


def _alone(F, r):
    with F.Field(r["nx"], r["ny"], bc=r["bc"], precision=r.get("precision", 0),
                 params=_params()) as fld:
        fld.variant = 2
        fld.ini(r["nodes"], r["x_map"], r["y_map"])
        if r["bc"] != "hedstrom_xy":
            fld.apply_bc_on_nodes()  # field%ini
        fld.integrate(r["dt"], r["nsteps"])
        return fld.download(), fld.time


def _err(a, b, bc):
    if bc == "hedstrom_xy":
        return normwise_rel_err_all(a, b)
    return normwise_rel_err_all(a[:, 2:-2, 2:-2], b[:, 2:-2, 2:-2])


def _bar(r):
    """FP64 requests: 1e-12; mixed-precision requests (FP32 face pass in a
    batched kernel vs the single-field kernel): 1e-6."""
    return 1e-6 if r.get("precision", 0) else 1e-12


def test_results_same_alone_and_in_the_mix(F, S):
    reqs = _requests(8, seed=21)
    with S.Server(params=_params(), chunk_steps=16) as srv:
        run = S.serve(srv, reqs, keep_results=True)
    assert run["stats"]["completed"] == len(reqs)
    assert run["failed"] == []
    assert run["stats"]["max_active"] >= 2  # requests overlapped on the device
    for i, r in enumerate(reqs):
        got, t = run["results"][i]
        ref, t_ref = _alone(F, r)
        assert np.isfinite(got).all()
        assert np.all(_err(got, ref, r["bc"]) <= _bar(r)), (i, r["nx"], r["bc"], r["precision"])
        assert abs(t - t_ref) <= 1e-12 * t_ref
        assert run["latencies"][i] > 0


def test_open_wall_presets_same_alone_and_in_the_mix(F, S):
    """Requests of the reference's default preset (half_wall_S_open) and of
    wall_S_open share the wall chain of the batched launches with
    wall_S_reflection requests."""
    reqs = _requests(8, seed=33, kinds=("half_wall_S_open", "wall_S_open", "wall_S_reflection",
                                        "hedstrom_xy"))
    assert {r["bc"] for r in reqs} >= {"half_wall_S_open", "wall_S_open"}
    with S.Server(params=_params(), chunk_steps=16) as srv:
        run = S.serve(srv, reqs, keep_results=True)
    assert run["stats"]["completed"] == len(reqs)
    assert run["failed"] == []
    for i, r in enumerate(reqs):
        got, t = run["results"][i]
        ref, t_ref = _alone(F, r)
        assert np.isfinite(got[:, 2:-2, 2:-2]).all()
        assert np.all(_err(got, ref, r["bc"]) <= _bar(r)), (i, r["nx"], r["bc"], r["precision"])


def test_admission_by_memory_budget(F, S):
    reqs = _requests(6, seed=5, n_range=(60, 60))  # equal sizes
    for r in reqs:
        r["arrival"] = 0.0  # all at once
    one = 3 * 4 * reqs[0]["ny"] * ((reqs[0]["nx"] + 15) // 16 * 16) * 8
    with S.Server(params=_params(), mem_budget=2 * one + 65536, chunk_steps=10) as srv:
        run = S.serve(srv, reqs, keep_results=True)
        st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["max_active"] == 2  # the budget holds two fields
    assert st["bytes_in_use"] == 0
    for i, r in enumerate(reqs):
        ref, _ = _alone(F, r)
        assert np.all(_err(run["results"][i][0], ref, r["bc"]) <= _bar(r))


def test_result_protocol(F, S):
    reqs = _requests(1, seed=2)
    r = reqs[0]
    with S.Server(params=_params(), chunk_steps=8) as srv:
        rid = srv.submit(r["nodes"], r["x_map"], r["y_map"], r["dt"], r["nsteps"], r["bc"])
        assert srv.result(rid) is None  # not run yet
        while srv.stats()["completed"] < 1:
            srv.poll(wait=True)
        nodes, t, lat, status = srv.result(rid)
        assert status == 0
        assert lat > 0 and np.isfinite(nodes).all()
        with pytest.raises(F.Dim2dError):
            srv.result(rid)  # forgotten once read
        with pytest.raises(F.Dim2dError):  # larger than the whole budget
            big = np.zeros((4, 600, 600))
            S.Server(params=_params(), mem_budget=1 << 20).submit(big, np.linspace(0, 1, 600),
                                                np.linspace(0, 1, 600), 1e-6, 10)


def test_diverged_request_stops_early(F, S):
    """A request whose state is not finite (a NaN planted in one interior
    cell of an open field's initial state) is stopped at a chunk boundary
    soon after the server's check sees it -- not stepped to its 4000th
    step -- and reported as NONFINITE with the time it reached; the request
    beside it ends as it does when served without the diverged one (same
    batched kernel and shape: <= 1e-14 normwise, rounding of the contraction
    at most)."""
    reqs = _requests(2, seed=8, kinds=("hedstrom_xy",))
    bad = dict(reqs[1])
    bad["nodes"] = reqs[1]["nodes"].copy()
    bad["nodes"][0, bad["ny"] // 2, bad["nx"] // 2] = np.nan
    bad["nsteps"] = 4000
    chunk = 16
    with S.Server(params=_params(), chunk_steps=chunk) as srv:
        run = S.serve(srv, [reqs[0], bad], keep_results=True)
    assert run["nonfinite"] == [1] and run["failed"] == []
    # flagged after the first chunk, seen by the host at most two chunks
    # later (two chunks stay queued), stopped at the next boundary
    assert run["end_time"][1] <= 4 * chunk * bad["dt"] * (1 + 1e-12), run["end_time"][1]
    with S.Server(params=_params(), chunk_steps=chunk) as srv:
        solo = S.serve(srv, [reqs[0]], keep_results=True)
    got, t = run["results"][0]
    ref, t_ref = solo["results"][0]
    assert np.isfinite(got).all()
    assert np.all(_err(got, ref, reqs[0]["bc"]) <= 1e-14)
    assert abs(t - t_ref) <= 1e-12 * t_ref


def test_wall_root_failure_stops_early(F, S):
    """A 64^2 wall bubble with a 4-dx interface under the test constants
    (We = 10) collapses and its wall ghost-cell root stops being bracketed
    after about 136 steps (the oracle fails at that step, where the reference
    stops); the server's check sees the wall status word and stops the
    request at a chunk boundary shortly after, with DIM2D_ERR_WALL_ROOT,
    instead of stepping it to its 4000th step."""
    from dim2d_finite_volume_b200 import workloads
    d = workloads.domain(64, T0=0.95, bubbles=[(0.0, 0.0, 0.2)], bc="wall_S_reflection")
    req = dict(d, arrival=0.0, nsteps=4000, precision=0)
    with S.Server(params=F.default_params(), chunk_steps=16) as srv:
        run = S.serve(srv, [req])
    assert run["failed"] == [0], run
    steps = run["end_time"][0] / d["dt"]
    assert 100 <= steps <= 400, steps  # failure near step 136, then at most a few chunks
