"""Benchmark of the DIM RK3 time step on B200 (one JSON line on rank 0).

Workload (N=1): the plain FP64 1024^2 DIM field -- a vapour bubble (seeded
radius in [0.05, 0.15]) in saturated liquid at T0 = 0.95, Re=5, We=10,
Pr=20, cv_r=2.5 -- advanced by RK3-TVD steps.  A "step" is one full RK3
time step (3 stages, boundary passes included) of the whole field.  The
metric is interior cell-updates per second (1 cell-update = one RK3 step of
one interior cell).  Inputs are seeded synthetic arrays of that shape.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--gpus N > 1 runs under torchrun, one rank per GPU, each rank advancing
its own field (replicas: the north-star domain is never sharded), so the
scaling is weak; value = all ranks' cell-updates / max-over-ranks time.

--impl reference times the reference algorithm's CPU restatement (the
oracle, all host threads) on the same workload, each step a bounded
sample of rows of that field (the reference's Fortran cannot be built on
this image: no Fortran compiler, no netCDF).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_INTERIOR = 1024
BYTES_PER_CELL_UPDATE = 256  # 3 stage writes + 3 stage reads + 2 reads of u^n, 32 B each
L2_BYTES = 126 * 1024 * 1024
# stage-kernel variants of the library (dim2d_set_variant)
STAGE_KERNELS = ["k_interior<1> 32x8 tiles", "k_strip<8,4,4>", "k_strip<16,4,4>",
                 "k_strip<16,4,5>", "k_strip<16,2,8>", "k_strip<16,8,2>",
                 "k_batch_persistent (a whole RK3 step per launch)"]


# presets with a wall on S: their CPU samples are the bottom rows (the wall)
WALL_PRESETS = ("wall_S_reflection", "wall_S_open", "half_wall_S_open")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", dest="n", type=int, default=N_INTERIOR,
                    help="interior cells per side of the plain workload")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--bc", default="hedstrom_xy",
                    choices=["hedstrom_xy", "periodic_xy", "wall_S_reflection", "wall_S_open",
                             "half_wall_S_open"])
    ap.add_argument("--threads", type=int, default=0,
                    help="host threads of the reference arm (0: all)")
    ap.add_argument("--variant", default="auto",
                    help="stage-kernel variant 0..5, or 'auto' (the library's autotuner)")
    ap.add_argument("--batch-domains", type=int, default=64,
                    help="domains of the batched workload (0: skip it)")
    ap.add_argument("--batch-steps", type=int, default=2000,
                    help="timed steps of the batched workload (its configuration: 2000)")
    ap.add_argument("--batch-mixed", type=int, default=1,
                    help="also time the batched workload in mixed precision (0: skip it)")
    ap.add_argument("--mixed-steps", type=int, default=10000,
                    help="steps of the mixed-precision configuration (0: skip it)")
    ap.add_argument("--mixed-n", type=int, default=2048)
    ap.add_argument("--buffer-layer", type=int, default=1,
                    help="also time the masked buffer-layer operators (0: skip)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="precision of the plain workload")
    ap.add_argument("--served", type=int, default=32,
                    help="requests of the served stream (0: skip it)")
    ap.add_argument("--cpu-budget", type=float, default=None,
                    help="no effect (the CPU legs time --steps steps of their sample); "
                         "accepted so that older profiling command lines still run")
    return ap.parse_args()


def workload(n, seed, rank=0, bc="hedstrom_xy"):
    """The 1024^2 plain FP64 configuration (workloads.plain_1024): a bubble
    of seeded radius in [0.05, 0.15] at T0 = 0.95, carried by a uniform
    x-flow at Mach 0.1 of the liquid sound speed, open (Hedstrom)
    boundaries on all sides.  With bc='periodic_xy' the same bubble sits
    still in a periodic box."""
    from dim2d_finite_volume_b200 import workloads
    return workloads.plain_1024(seed + rank, n, bc)


def oracle_cfg(O, bc, nx, ny):
    if bc == "periodic_xy":
        return O.make_cfg(nx, ny, periodic=True)
    from dim2d_finite_volume_b200 import field as F
    bc_choice, bc_type, bc_order = F._preset(bc)
    return O.make_cfg(nx, ny, periodic=False, bc_choice=bc_choice, bc_type=bc_type,
                      bc_order=bc_order)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per launch of the interior stage kernel from the committed
    ncu summary (profiles/interior_stage_traffic.json), per interior cell."""
    p = os.path.join(ROOT, "profiles", "interior_stage_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("dram_bytes_per_cell_per_launch")
    return None


def fp64_figures(bc):
    """FP64 operations per cell-update from the committed counts
    (profiles/fp64_ops.json): the stage kernel's executed FP64 thread
    instructions from ncu, and the oracle's FP64 flops (the reference's
    serial algorithm) from the counting build of oracle/flopcount.cpp."""
    p = os.path.join(ROOT, "profiles", "fp64_ops.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    key = "%s_rk3_step" % (bc if bc == "periodic_xy" else "hedstrom_xy")
    return {"kernel_inst": d["kernel_fp64_inst_per_cell_update"],
            "kernel_flops": d["kernel_fp64_flops_per_cell_update"],
            "oracle_flops": d["oracle"][key]["flops"], "oracle_key": key,
            "kernel_workload": d["workload"]}


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="dim2d_clocks_", suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        try:
            lines = open(self.path).read().splitlines()
        finally:
            os.unlink(self.path)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def band_sample(w, rows, bottom=False):
    """Rows [c - rows/2, c + rows/2) of the field around its centre line
    (bottom: the first rows, which hold the S wall), plus ghosts: the same
    per-cell work as the full field, bounded."""
    ny = w["ny"]
    c = ny // 2
    lo = 0 if bottom else max(0, c - rows // 2 - 2)
    hi = lo + rows + 4
    q = np.ascontiguousarray(w["nodes"][:, lo:hi, :])
    return q, np.ascontiguousarray(w["y_map"][lo:hi])


PARITY_STEPS = 3


def parity_vs_oracle(O, w, q_gpu):
    """Error of the GPU field after PARITY_STEPS RK3 steps against the
    oracle's on the same initial state (the oracle as the checker): per
    conservative variable, max|a - b| / max|b| and the L2 relative error
    over the interior cells."""
    nx, ny = w["nx"], w["ny"]
    q = np.ascontiguousarray(w["nodes"], dtype=np.float64).copy()
    cfg = oracle_cfg(O, w["bc"], nx, ny)
    if w["bc"] not in ("periodic_xy", "hedstrom_xy"):
        O.apply_bc_on_nodes(cfg, 0.0, w["x_map"], w["y_map"], q.copy(), q)
    t0 = time.perf_counter()
    O.integrate(cfg, q, w["x_map"], w["y_map"], 0.0, w["dt"], PARITY_STEPS)
    el = time.perf_counter() - t0
    a, b = q_gpu[:, 2:ny - 2, 2:nx - 2], q[:, 2:ny - 2, 2:nx - 2]
    linf = [float(np.abs(a[k] - b[k]).max() / np.abs(b[k]).max()) for k in range(4)]
    l2 = [float(np.sqrt(((a[k] - b[k]) ** 2).sum() / (b[k] ** 2).sum())) for k in range(4)]
    return {"steps": PARITY_STEPS, "max_rel": linf, "l2_rel": l2, "oracle_s": round(el, 2),
            "note": "GPU field vs the oracle after %d RK3 steps of the whole %dx%d field from "
                    "the same initial state; per conservative variable (rho, rho u, rho v, "
                    "rho E), interior cells: max|a-b|/max|b| and sqrt(sum (a-b)^2 / sum b^2)"
                    % (PARITY_STEPS, nx, ny)}


CPU_SAMPLE_ROWS = 256  # interior rows of the CPU legs' sample of the field


def cpu_sample(w):
    """The sample both CPU legs time: a band of CPU_SAMPLE_ROWS interior
    rows of the field (through its centre, or at the S wall for the wall
    presets), or the whole field when it is not larger than that."""
    if w["ny"] - 4 <= CPU_SAMPLE_ROWS:
        return np.ascontiguousarray(w["nodes"]).copy(), w["y_map"], "all %dx%d nodes" % (
            w["nx"], w["ny"])
    q, y_map = band_sample(w, CPU_SAMPLE_ROWS, bottom=w["bc"] in WALL_PRESETS)
    return q, y_map, "a %dx%d band (interior %dx%d) %s" % (
        w["nx"], q.shape[1], w["nx"] - 4, q.shape[1] - 4,
        "at the S wall" if w["bc"] in WALL_PRESETS else "through the centre")


def host_cpu():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_measure(w, steps, warmup, threads):
    """The reference algorithm on the host cores: the oracle's timing build
    (-O3 -march=native, the checker's results bit for bit) with `threads`
    OpenMP threads advances the sample by `warmup` untimed RK3 steps, then
    `steps` RK3 steps each timed on its own (steady clock).  value = sample
    cell-updates / median step time; best = over the fastest step."""
    from oracle import oracle as O
    O.set_threads(threads)
    O.fast_lib()
    q, y_map, what = cpu_sample(w)
    cfg = oracle_cfg(O, w["bc"], w["nx"], q.shape[1])
    if w["bc"] != "hedstrom_xy":  # field%ini: node boundary pass
        O.lib().orc_clear_status()
        O.apply_bc_on_nodes(cfg, 0.0, w["x_map"], y_map, q.copy(), q)
    cells = (w["nx"] - 4) * (q.shape[1] - 4)
    t = 0.0
    for _ in range(warmup):
        t = O.integrate(cfg, q, w["x_map"], y_map, t, w["dt"], 1, fast=True)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        t = O.integrate(cfg, q, w["x_map"], y_map, t, w["dt"], 1, fast=True)
        times.append(time.perf_counter() - t0)
    med, best = float(np.median(times)), float(min(times))
    return {"value": cells / med, "best": cells / best, "median_ms": 1e3 * med,
            "best_ms": 1e3 * best, "steps": steps, "warmup": warmup, "cells": cells,
            "threads": threads, "sample": what, "finite": bool(np.isfinite(q).all())}


def cpu_baseline(w, steps, warmup, gpu_state=None):
    """The CPU baseline on the line: the same measurement as the reference
    arm (cpu_measure on all host threads, same sample, steps and warm-up),
    the serial rate beside it (1 thread, 3 steps), and with gpu_state (the
    GPU field after PARITY_STEPS steps) the error of that state against the
    oracle's."""
    from oracle import oracle as O
    nth = os.cpu_count() or 1
    O.set_threads(nth)
    parity = parity_vs_oracle(O, w, gpu_state) if gpu_state is not None else None
    m = cpu_measure(w, steps, warmup, nth)
    serial = cpu_measure(w, 3, 1, 1)
    out = {"value": m["value"], "unit": "cell-updates/s", "cores": nth, "kind": "port",
           "host": host_cpu(), "nproc": os.cpu_count(),
           "sample": "each step: one RK3 step of %s of the %d^2 field; %d warm-up steps, then "
                     "%d steps timed one by one; value over the median step, best over the "
                     "fastest" % (m["sample"], w["nx"] - 4, warmup, steps),
           "best": m["best"], "median_ms": m["median_ms"], "best_ms": m["best_ms"],
           "build": "oracle timing build: gcc -O3 -march=native -ffp-contract=off -fopenmp "
                    "(bit-identical to the -O2 checker build)",
           "serial": {"value": serial["value"], "best": serial["best"], "cores": 1,
                      "steps": 3}}
    if parity is not None:
        out["parity"] = parity
    return out


def bench_config(a, w, nx, ny, dt):
    """The `config` of both arms' lines (identical by construction)."""
    return {"workload": "plain FP64 DIM %d^2 (+2 ghosts) bubble, T0=0.95, Mach %.1f flow, RK3 "
                        "step" % (a.n, 0.1 if a.bc == "hedstrom_xy" else 0.0),
            "bc": a.bc, "nx": nx, "ny": ny, "dt": dt, "seed": a.seed,
            "l2": "GPU arm: flushed between timed steps (2x L2 write, outside the events); "
                  "CPU arm: host arrays, no flush"}


def run_reference(a, rank, world):
    """The reference arm: the reference's CPU algorithm (the oracle's timing
    build, all host threads) on this arm's workload, config and metric;
    rank 0 only."""
    if rank != 0:
        return
    w = workload(a.n, a.seed, bc=a.bc)
    nth = a.threads or os.cpu_count() or 1
    m = cpu_measure(w, a.steps, a.warmup, nth)
    line = {
        "metric": "cell-updates/s", "value": m["value"], "unit": "cell-updates/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": m["median_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": bench_config(a, w, w["nx"], w["ny"], w["dt"]),
        "cpu_baseline": {"value": m["value"], "unit": "cell-updates/s", "cores": nth,
                         "kind": "port", "host": host_cpu(), "nproc": os.cpu_count(),
                         "best": m["best"], "median_ms": m["median_ms"],
                         "best_ms": m["best_ms"],
                         "sample": "each step: one RK3 step of %s of the %d^2 field; value over "
                                   "the median step" % (m["sample"], a.n)},
        "e2e": {"value": m["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference is Fortran and cannot be built on this image (no Fortran "
                "compiler, no netCDF-Fortran): this arm times the oracle, the C restatement of "
                "its algorithm, in its -O3 -march=native timing build",
    }
    print(json.dumps(line), flush=True)


def reduce_max(values, dist, device):
    """Element-wise maximum over all ranks (every rank gets it): the
    multi-rank timing rule -- the job takes as long as its slowest rank."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def whole_job_rate(units_per_rank, world, steps, max_ms):
    """Units per second of the whole job: every rank processed
    units_per_rank per step (weak scaling) in at most max_ms."""
    return units_per_rank * world * steps / (max_ms * 1e-3)


def run_batched(a, stream, barrier, F, torch, flush):
    """Batched FP64 (64 seeded domains, n in {128..512}^2, wall / periodic /
    open mix): the batch advanced by graph-replayed batched steps, against
    the same fields stepped one field per launch.  Returns a dict."""
    from dim2d_finite_volume_b200 import batch as Bm
    from dim2d_finite_volume_b200 import workloads
    doms = workloads.batched_domains(a.seed + 77, count=a.batch_domains)
    fields = []
    for d in doms:
        fld = F.Field(d["nx"], d["ny"], bc=d["bc"], params=workloads.batch_params())
        fld.set_stream(stream.cuda_stream)
        fld.ini(d["nodes"], d["x_map"], d["y_map"])
        if d["bc"] not in ("periodic_xy", "hedstrom_xy"):
            fld.apply_bc_on_nodes()  # field%ini
        fields.append(fld)
    # plain form first: each field its own launches (its step graph), each
    # with the stage-kernel variant the per-field autotuner picks for it
    plain_variants = [fld.autotune()[0] for fld in fields]
    for _ in range(3):
        for fld, d in zip(fields, doms):
            fld.integrate(d["dt"], 1)
    barrier()
    steps = max(3, a.steps // 2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain_ms = 0.0
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(float(k))
            e0.record(stream)
            for fld, d in zip(fields, doms):
                fld.integrate(d["dt"], 1)
            e1.record(stream)
            e1.synchronize()
            plain_ms += e0.elapsed_time(e1)
    barrier()
    total_steps = 3 + steps + 3 + a.batch_steps  # every step the FP64 fields take
    modes = {}
    for mode in ("graph", "persistent"):
        if mode == "persistent":
            graph_state = [fld.download() for fld in fields]
        reinit(fields, doms)  # both modes take the same steps from the initial state
        modes[mode] = batch_mode_run(a, Bm, fields, doms, mode, stream, barrier, torch,
                                     warm=total_steps - a.batch_steps)
    # same per-cell code in both modes: the states after the same steps agree
    # (normwise per field and variable; the open boundary amplifies rounding)
    diff = 0.0
    for fld, g in zip(fields, graph_state):
        q = fld.download()
        for v in range(4):
            diff = max(diff, float(np.abs(q[v] - g[v]).max() / np.abs(g[v]).max()))
    best = min(modes, key=lambda m: modes[m]["ms"])
    cells = modes[best]["cells"]
    batch_ms, per_block, bclocks = modes[best]["ms"], modes[best]["blocks"], modes[best]["clocks"]
    out = {"cells_per_step": int(cells), "steps": a.batch_steps, "batch_ms": batch_ms,
           "mode": best, "mode_ms": {m: modes[m]["ms"] for m in modes},
           "mode_launches": {m: modes[m]["launches"] for m in modes},
           "persistent_rows": modes["persistent"]["shapes"][0],
           "persistent_vs_graph_max_abs_diff": diff,
           "we": workloads.BATCH_WE, "clocks": bclocks,
           "block_ms_per_step": [round(min(per_block), 4), round(max(per_block), 4)],
           "plain_ms": plain_ms, "plain_steps": steps,
           "launches": int(modes[best]["launches"]),
           "plain_variants": {str(v): plain_variants.count(v) for v in sorted(set(plain_variants))},
           "domains": len(doms), "shapes": modes["graph"]["shapes"],
           "kinds": {k: sum(1 for d in doms if d["bc"] == k) for k in workloads.BATCH_KINDS}}
    if a.batch_mixed:
        out["mixed"] = run_batched_mixed(a, stream, barrier, F, Bm, torch, flush, doms, fields,
                                         total_steps)
    for fld in fields:
        fld.close()
    return out


def reinit(fields, doms):
    """Every field back to its initial state (field%ini)."""
    for fld, d in zip(fields, doms):
        fld.ini(d["nodes"], d["x_map"], d["y_map"])
        if d["bc"] not in ("periodic_xy", "hedstrom_xy"):
            fld.apply_bc_on_nodes()


def batch_mode_run(a, Bm, fields, doms, mode, stream, barrier, torch, warm):
    """One batch of `fields` in `mode` (graph: a captured graph of batched
    launches per step; persistent: one persistent-kernel launch per step
    call), autotuned, `warm` untimed steps, then the timed steps."""
    bt = Bm.Batch()
    bt.set_stream(stream.cuda_stream)
    bt.set_persistent(mode == "persistent")
    for fld, d in zip(fields, doms):
        bt.add(fld, d["dt"])
    shapes, _ = bt.autotune()
    bt.step(warm)
    barrier()
    n0 = bt.launches
    # NVTX range "batched_<mode>" around the timed steps: profilers select
    # this mode's timed launches by it (ncu --nvtx --nvtx-include)
    torch.cuda.nvtx.range_push("batched_" + mode)
    ms, per_block, clocks = timed_batch_steps(bt, a.batch_steps, stream, torch)
    torch.cuda.nvtx.range_pop()
    barrier()
    bt.sync()
    out = {"ms": ms, "blocks": per_block, "clocks": clocks, "shapes": shapes,
           "launches": bt.launches - n0, "cells": bt.cells}
    bt.close()
    return out


def timed_batch_steps(bt, nsteps, stream, torch, block=100):
    """nsteps graph-replayed batched steps, CUDA events around blocks of
    `block` steps on the batch's stream, SM clocks sampled meanwhile.
    Returns (summed milliseconds, per-block ms per step, clocks).  No L2
    flush: the batch's state (64 domains, three buffers each) is several
    times larger than L2."""
    ev = []
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    with torch.cuda.stream(stream):
        done = 0
        while done < nsteps:
            k = min(block, nsteps - done)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            bt.step(k)
            e1.record(stream)
            ev.append((e0, e1, k))
            done += k
    stream.synchronize()
    clocks = sampler.stop()
    per_block = [x.elapsed_time(y) / k for x, y, k in ev]
    return sum(x.elapsed_time(y) for x, y, _ in ev), per_block, clocks


def run_batched_mixed(a, stream, barrier, F, Bm, torch, flush, doms, fields64, total_steps):
    """The same domains as DIM2D_MIXED fields in one batch: timed like the
    FP64 batch, then advanced to the FP64 fields' step count and compared
    with them (normwise over each interior, max over domains; the FP64
    batch matches the oracle to 1e-10 in the parity tests)."""
    from dim2d_finite_volume_b200 import workloads
    fields = []
    for d in doms:
        fld = F.Field(d["nx"], d["ny"], bc=d["bc"], precision=F.MIXED,
                      params=workloads.batch_params())
        fld.set_stream(stream.cuda_stream)
        fld.ini(d["nodes"], d["x_map"], d["y_map"])
        if d["bc"] not in ("periodic_xy", "hedstrom_xy"):
            fld.apply_bc_on_nodes()  # field%ini
        fields.append(fld)
    modes = {}
    for mode in ("graph", "persistent"):
        reinit(fields, doms)
        modes[mode] = batch_mode_run(a, Bm, fields, doms, mode, stream, barrier, torch,
                                     warm=total_steps - a.batch_steps)
    best = min(modes, key=lambda m: modes[m]["ms"])
    ms, per_block, mclocks = modes[best]["ms"], modes[best]["blocks"], modes[best]["clocks"]
    shapes, launches = modes[best]["shapes"], modes[best]["launches"]
    err = np.zeros(4)
    abs_err = np.zeros(4)
    scale = np.zeros(4)
    by_kind = {}
    for fm, f64, d in zip(fields, fields64, doms):
        qm, qd = fm.download(), f64.download()
        kind = by_kind.setdefault(d["bc"], np.zeros(4))
        for v in range(4):
            b_ = qd[v, 2:-2, 2:-2]
            d_ = float(np.abs(qm[v, 2:-2, 2:-2] - b_).max())
            r_ = d_ / float(np.abs(b_).max())
            err[v] = max(err[v], r_)
            kind[v] = max(kind[v], r_)
            abs_err[v] = max(abs_err[v], d_)
            scale[v] = max(scale[v], float(np.abs(b_).max()))
        fm.close()
    return {"batch_ms": ms, "steps": a.batch_steps, "launches": int(launches), "shapes": shapes,
            "mode": best, "mode_ms": {m: modes[m]["ms"] for m in modes},
            "steps_compared": total_steps, "rel_err_vs_fp64": [float(e) for e in err],
            "abs_err_vs_fp64": [float(e) for e in abs_err],
            "max_abs_fp64": [float(e) for e in scale], "clocks": mclocks,
            "rel_err_by_kind": {k: [float(e) for e in v] for k, v in by_kind.items()},
            "block_ms_per_step": [round(min(per_block), 4), round(max(per_block), 4)]}


def run_served(a):
    """Served stream: seeded Poisson arrivals (rate 50/s) of FP64 or mixed
    requests, n log-uniform in [64, 1024], steps in [500, 20000], wall / open;
    replayed in real time through the serving loop."""
    from dim2d_finite_volume_b200 import server as Sm
    from dim2d_finite_volume_b200 import workloads
    reqs = workloads.served_requests(a.seed + 99, a.served, rate=50.0)
    with Sm.Server(params=workloads.served_params(), chunk_steps=500) as srv:
        run = Sm.serve(srv, reqs)
    lat_all = np.array(run["latencies"])
    fin = run["finished"]
    lat = lat_all[fin] if fin else lat_all[:0]
    # steps each request actually ran (the server stops diverged ones early)
    done = {i: min(r["nsteps"], int(round(run["end_time"][i] / r["dt"])))
            for i, r in enumerate(reqs)}
    def cells(r):
        return (r["nodes"].shape[1] - 4) * (r["nodes"].shape[2] - 4)
    ran = sum(done[i] * cells(r) for i, r in enumerate(reqs))
    stopped = {int(i): [done[i], int(reqs[i]["nsteps"])] for i in sorted(done)
               if done[i] < reqs[i]["nsteps"]}
    return {
        "workload": "served stream: %d requests, Poisson arrivals at 50/s, n log-uniform in "
                    "[64,1024], steps uniform in [500,20000], T0 in [0.90,0.99], wall "
                    "(wall_S_reflection) / open, FP64 or mixed precision per request (%d mixed); "
                    "one bubble per request with the equilibrium interface width at T0, "
                    "We = %g for the whole stream"
                    % (len(reqs), sum(r["precision"] for r in reqs), workloads.SERVED_WE),
        "value": run["cell_updates_finished"] / run["wall_s"], "unit": "cell-updates/s",
        "value_note": "cell-updates of the requests that finished with a finite state (failed "
                      "and non-finite requests excluded) / wall time of the whole stream; "
                      "latencies likewise over the finished requests",
        "wall_s": run["wall_s"], "cell_updates": int(run["cell_updates_finished"]),
        "finished_requests": len(fin),
        "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
        "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
        "latency_max_s": float(lat.max()) if len(lat) else None,
        "all_requests": {"value": ran / run["wall_s"],
                         "cell_updates": int(ran),
                         "latency_p50_s": float(np.percentile(lat_all, 50)),
                         "latency_p99_s": float(np.percentile(lat_all, 99)),
                         "note": "every request counted with the steps it ran, failed and "
                                 "non-finite ones included"},
        "requests": len(reqs), "arrival_span_s": float(reqs[-1]["arrival"]),
        "max_active": int(run["stats"]["max_active"]),
        "failed_requests": len(run["failed"]),
        "nonfinite_requests": len(run["nonfinite"]),
        "stopped_early": stopped,
        "failed_note": "failed = the wall ghost-cell root was not found (where the reference "
                       "stops); non-finite = the solve blew up.  The server checks every "
                       "member after each chunk and stops such requests at the next chunk "
                       "boundary (stopped_early: request -> [steps run, steps requested]).  "
                       "Both are left out of value and of the latency percentiles "
                       "(all_requests keeps them)",
        "timing": "host wall clock from the first arrival to the last completion (the "
                  "stream is replayed in real time); latency = submit to completion",
    }


def run_mixed(a, stream, F, torch):
    """Mixed precision at 2048^2 (4 bubbles, T0 = 0.97, wall): the mixed
    field and the FP64 field advanced side by side in blocks of 1000 steps;
    after every block, the L2 and Linf errors of rho and rho E of the mixed
    state relative to the FP64 state.  The FP64 path is the error reference
    (it matches the oracle to 1e-10 in the parity tests)."""
    from dim2d_finite_volume_b200 import workloads
    d = workloads.mixed_2048(a.seed + 4, n=a.mixed_n)
    nx, ny, dt = d["nx"], d["ny"], d["dt"]
    cells = (nx - 4) * (ny - 4)
    flds = {}
    for prec in (F.MIXED, F.FP64):
        fld = F.Field(nx, ny, bc="wall_S_reflection", precision=prec,
                      params=workloads.mixed_params())
        fld.set_stream(stream.cuda_stream)
        fld.ini(d["nodes"], d["x_map"], d["y_map"])
        fld.apply_bc_on_nodes()  # field%ini
        flds[prec] = fld
    # each field on the stage-kernel shape its own autotuner picks (dry
    # steps: the state is untouched)
    variants = {("mixed" if prec == F.MIXED else "fp64"): fld.autotune()[0]
                for prec, fld in flds.items()}
    block = 1000 if a.mixed_steps >= 1000 else a.mixed_steps
    ms = {F.MIXED: 0.0, F.FP64: 0.0}
    errors = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for fld in flds.values():  # warm-up (graph capture), then restart from the IC
        fld.integrate(dt, 3)
        fld.ini(d["nodes"], d["x_map"], d["y_map"])
        fld.apply_bc_on_nodes()
    done = 0
    status = "ok"
    with torch.cuda.stream(stream):
        while done < a.mixed_steps:
            k = min(block, a.mixed_steps - done)
            for prec, fld in flds.items():
                e0.record(stream)
                fld.integrate(dt, k)
                e1.record(stream)
                e1.synchronize()
                ms[prec] += e0.elapsed_time(e1)
            done += k
            try:
                qm = flds[F.MIXED].download()
                qd = flds[F.FP64].download()
            except F.Dim2dError as ex:  # wall root failure: where the reference stops
                status = "stopped after %d steps: %s" % (done, ex)
                break
            row = {"step": done}
            for name, v in (("rho", 0), ("rhoE", 3)):
                a_, b_ = qm[v, 2:-2, 2:-2], qd[v, 2:-2, 2:-2]
                row[name + "_linf"] = float(np.abs(a_ - b_).max() / np.abs(b_).max())
                row[name + "_l2"] = float(np.sqrt(((a_ - b_) ** 2).sum() / (b_ ** 2).sum()))
            errors.append(row)
    for fld in flds.values():
        fld.close()
    vm = cells * done / (ms[F.MIXED] * 1e-3) if done else None
    vd = cells * done / (ms[F.FP64] * 1e-3) if done else None
    return {
        "workload": "mixed precision %d^2: %d bubbles r in [0.05,0.1], T0=0.97, wall "
                    "(wall_S_reflection), %d steps; equilibrium interface width at T0, We = %g"
                    % (a.mixed_n, len(d["bubbles"]), a.mixed_steps, workloads.MIXED_WE),
        "value": vm, "unit": "cell-updates/s", "fp64_value": vd,
        "vs_fp64": (vm / vd) if vm and vd else None, "steps_run": done, "status": status,
        "variants": variants,
        "errors_vs_fp64": errors, "error_bar": 1e-5,
        "error_reference": "the FP64 path (matches the oracle to <= 1e-10 in the parity tests)",
        "timing": "CUDA events around each 1000-step block of graph-replayed steps; downloads "
                  "for the error check outside the timed blocks; each field on the "
                  "stage-kernel variant its autotuner picked (variants)",
    }


def run_buffer_layer(a, stream, F, torch, flush, peak):
    """The masked (buffer-layer) operators on a 2048 x 256 edge band: a
    RK3 step = 3 x (dim2d_time_dev_masked + dim2d_rk_stage_masked), on the
    caller's device arrays (boundary points keep a zero time derivative).
    Each step and each launch is bracketed by CUDA events on the launching
    stream, L2 flushed before each.  Algorithmic bytes per layer point:
    time derivative 32 (nodes) + 4 (grdpts_id) + 32 (time_dev) = 68;
    stage 32 (nodes in) + 32 (time_dev) + 32 (nodes_tmp) + 32 (nodes out)
    + 4 = 132; step 3 x (68 + 132) = 600."""
    from dim2d_finite_volume_b200 import workloads
    d = workloads.buffer_layer(a.seed + 5)
    nx, ny, dt = d["nx"], d["ny"], d["dt"]
    xb, yb = d["x_borders"], d["y_borders"]
    g = d["grdpts_id"]
    points = int((g != 0).sum())
    u = torch.from_numpy(d["nodes"]).cuda()
    tmp = torch.empty_like(u)
    td = torch.zeros_like(u)
    gid = torch.from_numpy(g).cuda()
    p = F.default_params()
    s = stream.cuda_stream

    def td_call():
        F.time_dev_masked(p, nx, ny, u.data_ptr(), gid.data_ptr(), d["dx"], d["dy"], xb, yb,
                          td.data_ptr(), s)

    def st_call(st):
        F.rk_stage_masked(st, nx, ny, u.data_ptr(), tmp.data_ptr(), td.data_ptr(),
                          gid.data_ptr(), dt, xb, yb, s)

    def step():
        for st in (1, 2, 3):
            td_call()
            st_call(st)

    steps = max(5, a.steps)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
    with torch.cuda.stream(stream):
        # at least W steps and ~0.3 s of work, so the clocks have ramped up
        t0, n = time.perf_counter(), 0
        while n < max(3, a.warmup) or time.perf_counter() - t0 < 0.3:
            step()
            n += 1
            if n % 50 == 0:
                torch.cuda.synchronize()
        torch.cuda.synchronize()
        for e in ev:
            flush.zero_()
            e[0].record(stream)
            step()
            e[1].record(stream)
        torch.cuda.synchronize()
        step_ms = float(np.median([e[0].elapsed_time(e[1]) for e in ev]))
        launch_ms = {}
        for name, call in (("time_dev_masked", td_call), ("rk_stage_masked", lambda: st_call(2))):
            for e in ev:
                flush.zero_()
                e[0].record(stream)
                call()
                e[1].record(stream)
            torch.cuda.synchronize()
            launch_ms[name] = float(np.median([e[0].elapsed_time(e[1]) for e in ev]))
    finite = bool(torch.isfinite(u).all().item())
    per_kernel = {}
    for name, b in (("time_dev_masked", 68), ("rk_stage_masked", 132)):
        gbs = b * points / (launch_ms[name] * 1e-3) / 1e9
        per_kernel[name] = {"launch_ms": launch_ms[name], "algorithmic_bytes": b * points,
                            "achieved_gbs": gbs, "frac": gbs / peak}
    return {
        "workload": "buffer layer: 2048 x 256 edge band of a 2048^2 domain (%d x %d grid, "
                    "%d layer points), bubble crossing it in a Mach 0.1 flow" % (nx, ny, points),
        "value": points / (step_ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": step_ms,
        "steps": steps, "launches_per_step": 6, "finite": finite,
        "roofline": {"bound": "hbm", "bytes_per_point_step": 600,
                     "achieved_gbs": 600 * points / (step_ms * 1e-3) / 1e9,
                     "frac": 600 * points / (step_ms * 1e-3) / 1e9 / peak,
                     "per_kernel": per_kernel},
        "timing": "median of CUDA-event brackets per step and per launch, L2 flushed before each",
    }


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference(a, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from dim2d_finite_volume_b200 import field as F

    w = workload(a.n, a.seed, rank, bc=a.bc)
    nx, ny = w["nx"], w["ny"]
    cells = (nx - 4) * (ny - 4)
    dt = w["dt"]
    stream = torch.cuda.Stream()
    fld = F.Field(nx, ny, bc=a.bc, precision=F.MIXED if a.precision == "mixed" else F.FP64)
    fld.set_stream(stream.cuda_stream)
    fld.ini(w["nodes"], w["x_map"], w["y_map"])
    if a.bc not in ("periodic_xy", "hedstrom_xy"):
        fld.apply_bc_on_nodes()  # field%ini
    tune_ms = None
    if a.variant == "auto":
        _, tune_ms = fld.autotune(measure=True)  # before the timed region
    else:
        fld.variant = int(a.variant)
    variant = fld.variant
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing (value) --------------------------------
    for _ in range(max(3, a.warmup)):
        fld.integrate(dt, 1)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    n_launch0 = fld.launches
    barrier()
    with torch.cuda.stream(stream):
        for k in range(a.steps):
            flush.fill_(float(k))  # L2 flush between timed steps (outside the events)
            ev[k][0].record(stream)
            fld.integrate(dt, 1)  # one step: replay of the captured step graph
            ev[k][1].record(stream)
    barrier()
    launches = fld.launches - n_launch0
    step_ms = sum(s.elapsed_time(e) for s, e in ev)
    # ---- stage-kernel time for the roofline: the same K steps again with
    # CUDA events around every stage launch (stream launches, same kernels)
    fld.profile(True)
    with torch.cuda.stream(stream):
        for k in range(a.steps):
            flush.fill_(float(k))
            fld.integrate(dt, 1)
    barrier()
    prof_ms, prof_n = fld.profile_read()
    fld.profile(False)
    # ---- end-to-end through the public API with host buffers ----------
    host_in = torch.empty((4, ny, nx), dtype=torch.float64, pin_memory=True)
    host_in.copy_(torch.from_numpy(w["nodes"]))
    host_out = torch.empty((4, ny, nx), dtype=torch.float64, pin_memory=True)
    hin = host_in.numpy()
    hout = host_out.numpy()
    e2e_steps = max(10, a.steps)
    for _ in range(2):
        fld.ini(hin, w["x_map"], w["y_map"])
        fld.integrate(dt, 1)
        fld.download(hout)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        fld.ini(hin, w["x_map"], w["y_map"])  # H2D of the step's input nodes
        fld.integrate(dt, 1)
        fld.download(hout)                    # D2H of the step's result nodes
    e1.record(stream)
    barrier()
    e2e_serial_ms = e0.elapsed_time(e1)
    # ---- the same steps pipelined over two fields: each step still uploads
    # its input and reads its result back, but the step's device-to-host copy
    # (dim2d_download_async, side stream) overlaps the next step's
    # host-to-device copy on the other field (PCIe carries both directions)
    fld2 = F.Field(nx, ny, bc=a.bc, precision=F.MIXED if a.precision == "mixed" else F.FP64)
    stream2 = torch.cuda.Stream()
    fld2.set_stream(stream2.cuda_stream)
    fld2.variant = variant
    xm = torch.empty(nx, dtype=torch.float64, pin_memory=True).numpy()
    ym = torch.empty(ny, dtype=torch.float64, pin_memory=True).numpy()
    xm[:] = w["x_map"]
    ym[:] = w["y_map"]
    host_out2 = torch.empty((4, ny, nx), dtype=torch.float64, pin_memory=True)
    pipe = [(fld, hout), (fld2, host_out2.numpy())]
    for k in range(4):  # warm-up: captures fld2's step graph
        g, out = pipe[k % 2]
        g.ini(hin, xm, ym)
        g.integrate(dt, 1)
        g.download_async(out)
    fld.sync()
    fld2.sync()
    barrier()
    e0.record(stream)
    stream2.wait_event(e0)
    for k in range(e2e_steps):
        g, out = pipe[k % 2]
        g.ini(hin, xm, ym)        # H2D of the step's input nodes
        g.integrate(dt, 1)
        g.download_async(out)     # D2H of the step's result nodes
    fld.sync()                    # both fields' streams and copies have landed
    fld2.sync()
    e1.record(stream)
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    fld2.close()
    # ---- the headline field after PARITY_STEPS steps from its initial
    # state, for the error against the oracle stated on the line
    fld.ini(w["nodes"], w["x_map"], w["y_map"])
    if a.bc not in ("periodic_xy", "hedstrom_xy"):
        fld.apply_bc_on_nodes()  # field%ini
    fld.integrate(dt, PARITY_STEPS)
    q_gpu = fld.download()
    fld.close()
    bres = None
    if a.batch_domains > 0:
        bres = run_batched(a, stream, barrier, F, torch, flush)
    served = run_served(a) if a.served > 0 else None
    mixed = run_mixed(a, stream, F, torch) if a.mixed_steps > 0 else None
    layer = (run_buffer_layer(a, stream, F, torch, flush, measured_peaks()[0])
             if a.buffer_layer else None)

    step_ms, e2e_ms, e2e_serial_ms = reduce_max([step_ms, e2e_ms, e2e_serial_ms], dist, "cuda")
    batched = None
    if bres is not None:
        tb = reduce_max([bres["batch_ms"], bres["plain_ms"]], dist, "cuda")
        bv = whole_job_rate(bres["cells_per_step"], world, bres["steps"], tb[0])
        pv = whole_job_rate(bres["cells_per_step"], world, bres["plain_steps"], tb[1])
        peak_b, _ = measured_peaks()
        batched = {
            "workload": "batched FP64: %d seeded domains, n in {128,...,512}^2, T0 in "
                        "[0.90,0.99], r in [0.05,0.2], wall (wall_S_reflection) / periodic / "
                        "open mix, Mach in [0,0.1] on open domains; equilibrium interface "
                        "width at T0, We = %g; %d timed steps"
                        % (bres["domains"], bres["we"], bres["steps"]),
            "value": bv, "unit": "cell-updates/s", "ms_per_step": tb[0] / bres["steps"],
            "steps": bres["steps"], "cells_per_step": bres["cells_per_step"],
            "kinds": bres["kinds"], "shapes": bres["shapes"],
            "gpu_launches": bres["launches"],
            "mode": bres["mode"],
            "mode_values": {m: whole_job_rate(bres["cells_per_step"], world, bres["steps"],
                                              reduce_max([v], dist, "cuda")[0])
                            for m, v in bres["mode_ms"].items()},
            "mode_launches": bres["mode_launches"],
            "persistent_rows": bres["persistent_rows"],
            "persistent_vs_graph_max_abs_diff": bres["persistent_vs_graph_max_abs_diff"],
            "plain_per_field_value": pv,
            "plain_variants": bres["plain_variants"],
            "vs_plain_per_field": bv / pv,
            "roofline": {"bound": "hbm", "achieved": bv * BYTES_PER_CELL_UPDATE / 1e9,
                         "peak": peak_b, "unit": "GB/s",
                         "frac": bv * BYTES_PER_CELL_UPDATE / 1e9 / peak_b},
            "timing": "CUDA events around blocks of 100 batched steps, no L2 flush: the "
                      "batch's state is several times larger than L2.  Two modes from the same "
                      "initial state, the faster one in value: graph = one replay of the "
                      "batch's step graph (batched launches per stage and boundary kind) per "
                      "step; persistent = one persistent-kernel launch per block (a dependency-"
                      "ordered work queue over all domains).  plain: the same fields stepped "
                      "one after another, "
                      "each by its own step graph with the stage-kernel variant its own "
                      "autotuner picked (plain_variants: variant -> fields), L2 flushed "
                      "between steps (outside the events)",
            "clocks": bres["clocks"], "block_ms_per_step": bres["block_ms_per_step"],
        }
        if "mixed" in bres:
            bm = bres["mixed"]
            tm = reduce_max([bm["batch_ms"]], dist, "cuda")[0]
            mv = whole_job_rate(bres["cells_per_step"], world, bm["steps"], tm)
            batched["mixed"] = {
                "workload": "the same domains as DIM2D_MIXED fields (FP32 face pass, FP64 node "
                            "pass / capillary third derivative / RK accumulation), one batch",
                "value": mv, "unit": "cell-updates/s", "ms_per_step": tm / bm["steps"],
                "steps": bm["steps"], "gpu_launches": bm["launches"], "shapes": bm["shapes"],
                "mode": bm["mode"],
                "mode_values": {m: whole_job_rate(bres["cells_per_step"], world, bm["steps"],
                                                  reduce_max([v], dist, "cuda")[0])
                                for m, v in bm["mode_ms"].items()},
                "vs_fp64_batched": mv / bv, "vs_plain_per_field": mv / pv,
                "roofline": {"bound": "hbm", "achieved": mv * BYTES_PER_CELL_UPDATE / 1e9,
                             "peak": peak_b, "unit": "GB/s",
                             "frac": mv * BYTES_PER_CELL_UPDATE / 1e9 / peak_b},
                "rel_err_vs_fp64": bm["rel_err_vs_fp64"],
                "abs_err_vs_fp64": bm["abs_err_vs_fp64"],
                "max_abs_fp64": bm["max_abs_fp64"],
                "rel_err_by_kind": bm["rel_err_by_kind"],
                "error_bar": 1e-5,
                "error_note": "per conservative variable (rho, rho u, rho v, rho E): max over "
                              "domains of max|mixed - FP64| / max|FP64| over each interior, after "
                              "%d steps of both (the FP64 batch matches the oracle to <= 1e-10 in "
                              "the parity tests); abs_err / max_abs: the same numerators and the "
                              "largest |FP64| per variable.  The momenta of the domains at rest "
                              "stay small, so their ratio is large for a small absolute error"
                              % bm["steps_compared"],
                "clocks": bm["clocks"], "block_ms_per_step": bm["block_ms_per_step"],
            }
    value = whole_job_rate(cells, world, a.steps, step_ms)
    e2e_value = whole_job_rate(cells, world, e2e_steps, e2e_ms)

    if rank == 0:
        peak, peak_kind = measured_peaks()
        ev_launch_ms = prof_ms / max(1, prof_n)
        # stage launches per step: 3, or 1 for the persistent kernel (a
        # whole RK3 step per launch)
        per_step = 1 if variant == 6 else 3
        if launches == per_step * a.steps:
            # every launch of the timed steps is a stage-kernel launch: the
            # average launch duration over the timed region is at most step
            # time / launches per step
            per_launch_ms = step_ms / launches
            launch_timing = ("timed steps / kernel launches (each timed step is exactly %d "
                             "launch%s of the kernel; inter-launch gaps included)"
                             % (per_step, "es" if per_step > 1 else ""))
        else:
            per_launch_ms = ev_launch_ms
            launch_timing = ("CUDA events around each stage launch over %d further steps "
                             "(stream launches of the same kernels)" % a.steps)
        bytes_per_launch = cells * BYTES_PER_CELL_UPDATE / float(per_step)
        achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
        tr = profile_traffic()
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": max(3, a.warmup),
            "ms_per_step": step_ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f32 face pass + f64 (mixed)",
            "data": "synthetic",
            "config": bench_config(a, w, nx, ny, dt),
            "stage_kernel": STAGE_KERNELS[variant],
            "autotune_ms": None if tune_ms is None else [round(float(x), 5) for x in tune_ms],
            "replicas_per_gpu": 1,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "kernel": STAGE_KERNELS[variant] + (" (fused RK3 stage)" if variant != 6
                                                             else ""),
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "launch_ms": per_launch_ms, "launch_timing": launch_timing,
                         "launch_ms_events": ev_launch_ms,
                         "traffic": (tr * cells * 3 / per_step if tr is not None else None)},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": int(hin.nbytes + w["x_map"].nbytes + w["y_map"].nbytes),
                    "d2h_bytes_per_step": int(hout.nbytes),
                    "serial_value": whole_job_rate(cells, world, e2e_steps, e2e_serial_ms),
                    "note": "each step: dim2d_upload (pinned host nodes) + dim2d_step(1) + "
                            "dim2d_download_async of the result, alternating over two fields "
                            "so that one step's D2H copy overlaps the next step's H2D copy; "
                            "timed from an event before the first upload to an event after "
                            "both fields' copies have landed (dim2d_sync).  serial_value: the "
                            "same steps on one field with the blocking dim2d_download"},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        f64 = fp64_figures(a.bc) if a.precision == "fp64" else None
        if f64 is not None:
            # FP64 lanes: 148 SMs x 64 per clock; DFMA counts as one instruction
            mhz = float((clocks or {}).get("sm_max_mhz") or 1965.0)
            peak_inst = 148 * 64 * mhz * 1e6
            ach_inst = value * f64["kernel_inst"]
            line["fp64"] = {
                "kernel_inst_per_cell_update": f64["kernel_inst"],
                "kernel_flops_per_cell_update": f64["kernel_flops"],
                "oracle_flops_per_cell_update": f64["oracle_flops"],
                "achieved_tinst_per_s": ach_inst / 1e12,
                "peak_tinst_per_s": peak_inst / 1e12, "frac": ach_inst / peak_inst,
                "note": ("FP64-ALU utilisation: the value's cell-updates/s x the stage kernel's "
                         "FP64 thread instructions per cell-update (ncu, %s) / (148 SMs x 64 FP64 "
                         "lanes x %.0f MHz); oracle: %s" % (f64["kernel_workload"], mhz,
                                                           f64["oracle_key"]))}
        if batched is not None:
            line["batched"] = batched
        if mixed is not None:
            line["mixed"] = mixed
        if served is not None:
            if dist is None:
                line["served"] = served
            else:  # replicas: every rank served its own stream; report rank 0's
                line["served"] = dict(served, note="rank 0 of %d replicas" % world)
        if layer is not None:
            line["buffer_layer"] = layer if dist is None else dict(
                layer, note="rank 0 of %d replicas" % world)
        line["cpu_baseline"] = cpu_baseline(w, a.steps, a.warmup, gpu_state=q_gpu)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
