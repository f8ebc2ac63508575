"""GPU parity at the lengths and sizes of the benchmarked configurations,
through the C ABI, against the oracle.

* The plain FP64 configurations with stage-kernel variant 4 (k_strip<16,2,8>),
  the one the autotuner picks and the persistent kernel (variant 6, the 100
  steps as one launch), 100 RK3 steps:
  the 128^2 periodic bubble (132^2 nodes) and the 1024^2 open-boundary
  bubble of the headline workload (1028^2 nodes, whole field) -- bar 1e-10
  normwise, the north star's -- and mixed precision on it (bar 1e-5).
* The reference's default preset half_wall_S_open and reflection_xy at the
  same size with a bubble touching the S boundary, 100 steps, FP64 and
  mixed: the symmetric bubble at rest leaves rho u near zero, and there the
  bar is 10x the oracle's own response to a rounding-sized perturbation of
  the initial state where that exceeds 1e-10 (1e-5 mixed).
* Batches of the batched workload's domains (seeded sizes, temperatures,
  radii, Mach numbers; wall / periodic / open), autotuned shapes, 100 steps
  -- bar 1e-10.
* The batched workload's full length, 2039 steps, on its smallest open,
  wall and periodic domains, FP64 and mixed precision.  Wall and periodic
  domains damp rounding differences and keep the bars 1e-10 (FP64) and
  1e-5 (mixed).  The open boundary amplifies them (tests/test_conditioning.py):
  there the bar is 10x the oracle's own response to a perturbation of the
  initial state of the size of the path's rounding (1e-14 relative for
  FP64, 6e-8 = FP32 unit roundoff for mixed), or the plain bar where that is
  larger.

Error metric: per conservative variable, max|a - b| / max|b| (all cells for
periodic and open fields, whose ghosts are time-integrated or images;
interior cells for wall fields)."""
import os

import numpy as np
import pytest

from tests.helpers import normwise_rel_err, normwise_rel_err_all, periodic_case, stable_dt

pytestmark = pytest.mark.gpu

BENCH_VARIANT = 4
PERSISTENT_VARIANT = 6  # the persistent kernel: all 100 steps in one launch
BATCH_SEED = 1311  # the bench's batched workload (seed 1234 + 77)


@pytest.fixture(scope="module")
def F():
    from dim2d_finite_volume_b200 import field
    return field


@pytest.fixture(scope="module")
def B():
    from dim2d_finite_volume_b200 import batch
    return batch


@pytest.fixture(scope="module")
def orc(oracle):
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


def _cfg(O, F, bc, nx, ny):
    if bc == "periodic_xy":
        return O.make_cfg(nx, ny, periodic=True)
    ch, ty, od = F._preset(bc)
    return O.make_cfg(nx, ny, periodic=False, bc_choice=ch, bc_type=ty, bc_order=od)


def _err(a, b, bc):
    if bc in ("periodic_xy", "hedstrom_xy"):
        return normwise_rel_err_all(a, b)
    return normwise_rel_err(a, b)


def _run_field(F, bc, q, x_map, y_map, dt, nsteps, variant, params=None, precision=0):
    nx, ny = q.shape[2], q.shape[1]
    with F.Field(nx, ny, bc=bc, params=params, precision=precision) as fld:
        fld.ini(q, x_map, y_map)
        if bc not in ("periodic_xy", "hedstrom_xy"):
            fld.apply_bc_on_nodes()  # field%ini
        if variant == "auto":
            variant, _ = fld.autotune(measure=True)
        else:
            fld.variant = variant
        fld.integrate(dt, nsteps)
        return fld.download(), variant


@pytest.mark.parametrize("variant", [BENCH_VARIANT, "auto", PERSISTENT_VARIANT])
def test_periodic_128_100_steps(orc, F, variant):
    nx, ny, x_map, y_map, q = periodic_case(128)
    cfg = _cfg(orc, F, "periodic_xy", nx, ny)
    orc.apply_bc_on_nodes(cfg, 0.0, x_map, y_map, q.copy(), q)
    dt = stable_dt(q, x_map, y_map)
    ref = q.copy()
    orc.integrate(cfg, ref, x_map, y_map, 0.0, dt, 100)
    got, v = _run_field(F, "periodic_xy", q, x_map, y_map, dt, 100, variant)
    err = _err(got, ref, "periodic_xy")
    print("periodic 128^2, variant %s, 100 steps:" % v, err)
    assert np.isfinite(got).all()
    assert np.all(err <= 1e-10), (v, err)


@pytest.fixture(scope="module")
def open_1024(orc, F):
    """The headline workload (bench seed 1234) and the oracle's state after
    100 steps of it (whole 1028^2 field, all host cores)."""
    from dim2d_finite_volume_b200 import workloads
    w = workloads.plain_1024(1234, 1024, "hedstrom_xy")
    ref = w["nodes"].copy()
    orc.integrate(_cfg(orc, F, "hedstrom_xy", w["nx"], w["ny"]), ref, w["x_map"], w["y_map"],
                  0.0, w["dt"], 100)
    return w, ref


@pytest.mark.parametrize("variant", [BENCH_VARIANT, "auto", PERSISTENT_VARIANT])
def test_open_1024_100_steps(open_1024, F, variant):
    w, ref = open_1024
    got, v = _run_field(F, "hedstrom_xy", w["nodes"], w["x_map"], w["y_map"], w["dt"], 100,
                        variant)
    err = _err(got, ref, "hedstrom_xy")
    print("open 1024^2, variant %s, 100 steps:" % v, err)
    assert np.isfinite(got).all()
    assert np.all(err <= 1e-10), (v, err)


WALL_PRESETS = ("half_wall_S_open", "reflection_xy")


@pytest.fixture(scope="module", params=WALL_PRESETS)
def wall_1024(request, orc, F):
    """The reference's default preset half_wall_S_open (S wall, W mirror, N
    and E open) and reflection_xy (mirrors) on a 1024^2 field with a bubble
    (radius 0.15, equilibrium interface width at T0 = 0.95) touching the S
    side, as the reference's bubble-next-to-wall set-up, so the S boundary
    operator (wall root solve or mirror) works on the interface from the
    first step; the batched workload's constants (We = 2000; no wall heat
    source, 90 degree contact angle).  After field%ini's node pass: the
    oracle's state after 100 steps (whole 1028^2 field, all host cores) and
    its responses to relative perturbations of the initial state of 1e-14
    (FP64 rounding) and 6e-8 (FP32): the bubble at rest is symmetric, rho u
    is near zero (max ~2e-4) and its normwise error amplifies rounding (the
    oracle's own rho u moves by ~2e-9 for 1e-14).
    Returns (preset, workload, state, {eps: response})."""
    import ctypes
    from dim2d_finite_volume_b200 import ic, workloads
    preset = request.param
    w = workloads.domain(1024, T0=0.95, bubbles=[(0.0, -0.35, 0.15)], bc=preset,
                         li=ic.interface_length(0.95, workloads.BATCH_WE), we=workloads.BATCH_WE)
    saved = orc.get_params()
    orc.set_params(we=workloads.BATCH_WE)
    try:
        cfg = _cfg(orc, F, preset, w["nx"], w["ny"])
        q = w["nodes"].copy()
        orc.lib().orc_clear_status()
        orc.apply_bc_on_nodes(cfg, 0.0, w["x_map"], w["y_map"], q.copy(), q)
        ref = q.copy()
        orc.integrate(cfg, ref, w["x_map"], w["y_map"], 0.0, w["dt"], 100)
        resp = {}
        for eps in (1e-14, 6e-8):
            p = q * (1.0 + eps * np.random.default_rng(0).standard_normal(q.shape))
            orc.integrate(cfg, p, w["x_map"], w["y_map"], 0.0, w["dt"], 100)
            resp[eps] = _err(p, ref, preset)
    finally:
        orc.lib().orc_set_params(ctypes.byref(saved))
    return preset, w, ref, resp


@pytest.mark.parametrize("variant", [BENCH_VARIANT, "auto"])
def test_wall_presets_1024_100_steps(wall_1024, F, variant):
    """Bar: 1e-10, or 10x the oracle's response to an FP64-rounding
    perturbation of the initial state where that is larger."""
    from dim2d_finite_volume_b200 import workloads
    preset, w, ref, resp = wall_1024
    got, v = _run_field(F, preset, w["nodes"], w["x_map"], w["y_map"], w["dt"], 100, variant,
                        params=workloads.batch_params())
    err = _err(got, ref, preset)
    bar = np.maximum(1e-10, 10.0 * resp[1e-14])
    print("%s 1024^2, variant %s, 100 steps: err" % (preset, v), err, "bar", bar)
    assert np.isfinite(got[:, 2:-2, 2:-2]).all()
    assert np.all(err <= bar), (v, err, bar)


def _mixed_check(F, bc, w, ref, params=None, resp=None):
    got, v = _run_field(F, bc, w["nodes"], w["x_map"], w["y_map"], w["dt"], 100, "auto",
                        params=params, precision=F.MIXED)
    err = _err(got, ref, bc)
    bar = np.full(4, 1e-5) if resp is None else np.maximum(1e-5, 10.0 * resp)
    print("mixed %s 1024^2, variant %s, 100 steps: err" % (bc, v), err, "bar", bar)
    assert np.all(err <= bar), (bc, v, err, bar)


def test_mixed_open_1024_100_steps(open_1024, F):
    """Mixed precision at the headline size against the FP64 oracle, on the
    autotuned shape: the north star's 1e-5 bar."""
    w, ref = open_1024
    _mixed_check(F, "hedstrom_xy", w, ref)


def test_mixed_wall_presets_1024_100_steps(wall_1024, F):
    """The same on the wall-touching bubble; bar 1e-5, or 10x the oracle's
    response to an FP32-rounding perturbation where that is larger."""
    from dim2d_finite_volume_b200 import workloads
    preset, w, ref, resp = wall_1024
    _mixed_check(F, preset, w, ref, params=workloads.batch_params(), resp=resp[6e-8])


def _batch_domains(indices):
    from dim2d_finite_volume_b200 import workloads
    specs = workloads.batched_specs(BATCH_SEED, 64)
    return [workloads.batched_domain(specs[i]) for i in indices]


def _smallest(kind, count):
    from dim2d_finite_volume_b200 import workloads
    specs = workloads.batched_specs(BATCH_SEED, 64)
    idx = sorted((s["n"], i) for i, s in enumerate(specs) if s["bc"] == kind)
    return [i for _, i in idx[:count]]


def _batch_run(F, B, doms, nsteps, precision=0):
    from dim2d_finite_volume_b200 import workloads
    fields = []
    with B.Batch() as bt:
        for d in doms:
            fld = F.Field(d["nx"], d["ny"], bc=d["bc"], params=workloads.batch_params(),
                          precision=precision)
            fld.ini(d["nodes"], d["x_map"], d["y_map"])
            if d["bc"] not in ("periodic_xy", "hedstrom_xy"):
                fld.apply_bc_on_nodes()  # field%ini
            bt.add(fld, d["dt"])
            fields.append(fld)
        shapes, _ = bt.autotune()
        bt.step(nsteps)
        bt.sync()
        out = [fld.download() for fld in fields]
    for fld in fields:
        fld.close()
    return out, shapes


def _oracle_run(O, F, d, nsteps, eps=0.0):
    from dim2d_finite_volume_b200 import workloads
    saved = O.get_params()
    O.set_params(we=workloads.BATCH_WE)
    try:
        cfg = _cfg(O, F, d["bc"], d["nx"], d["ny"])
        q = d["nodes"].copy()
        if d["bc"] not in ("periodic_xy", "hedstrom_xy"):
            O.lib().orc_clear_status()
            O.apply_bc_on_nodes(cfg, 0.0, d["x_map"], d["y_map"], q.copy(), q)
        if eps:
            q *= 1.0 + eps * np.random.default_rng(0).standard_normal(q.shape)
        O.integrate(cfg, q, d["x_map"], d["y_map"], 0.0, d["dt"], nsteps)
        return q
    finally:
        import ctypes
        O.lib().orc_set_params(ctypes.byref(saved))


def test_batch_domains_100_steps(orc, F, B):
    """Three of each kind (the smallest), one batch, autotuned shapes."""
    idx = _smallest("hedstrom_xy", 3) + _smallest("wall_S_reflection", 3) + \
        _smallest("periodic_xy", 3)
    doms = _batch_domains(idx)
    got, shapes = _batch_run(F, B, doms, 100)
    for i, d, g in zip(idx, doms, got):
        ref = _oracle_run(orc, F, d, 100)
        err = _err(g, ref, d["bc"])
        print("batched domain %d (%s %d^2), 100 steps:" % (i, d["bc"], d["nx"] - 4), err)
        assert np.isfinite(g).all()
        assert np.all(err <= 1e-10), (i, d["bc"], err)


LONG_STEPS = 2039


@pytest.fixture(scope="module")
def long_runs(orc, F, B):
    """The smallest open, wall and periodic domains, 2039 batched steps in
    FP64 and in mixed precision; the oracle's states, and for the open
    domain its responses to 1e-14 and 6e-8 perturbations."""
    idx = [_smallest("hedstrom_xy", 1)[0], _smallest("wall_S_reflection", 1)[0],
           _smallest("periodic_xy", 1)[0]]
    doms = _batch_domains(idx)
    fp64, _ = _batch_run(F, B, doms, LONG_STEPS)
    mixed, _ = _batch_run(F, B, doms, LONG_STEPS, precision=F.MIXED)
    refs = [_oracle_run(orc, F, d, LONG_STEPS) for d in doms]
    d_open = doms[0]
    resp = {eps: _err(_oracle_run(orc, F, d_open, LONG_STEPS, eps), refs[0], "hedstrom_xy")
            for eps in (1e-14, 6e-8)}
    return doms, fp64, mixed, refs, resp


def test_long_fp64(long_runs):
    doms, fp64, _, refs, resp = long_runs
    for d, g, ref in zip(doms, fp64, refs):
        err = _err(g, ref, d["bc"])
        bar = np.full(4, 1e-10)
        if d["bc"] == "hedstrom_xy":
            bar = np.maximum(bar, 10.0 * resp[1e-14])
        print("FP64 %s %d^2, %d steps: err" % (d["bc"], d["nx"] - 4, LONG_STEPS), err,
              "bar", bar)
        assert np.isfinite(g).all()
        assert np.all(err <= bar), (d["bc"], err, bar)


def test_long_mixed(long_runs):
    doms, _, mixed, refs, resp = long_runs
    for d, g, ref in zip(doms, mixed, refs):
        err = _err(g, ref, d["bc"])
        bar = np.full(4, 1e-5)
        if d["bc"] == "hedstrom_xy":
            bar = np.maximum(bar, 10.0 * resp[6e-8])
        print("mixed %s %d^2, %d steps: err" % (d["bc"], d["nx"] - 4, LONG_STEPS), err,
              "bar", bar)
        assert np.isfinite(g).all()
        assert np.all(err <= bar), (d["bc"], err, bar)
