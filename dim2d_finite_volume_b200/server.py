"""Serving loop (include/dim2d.h, dim2d_server_*): requests of different
grid sizes arrive over time, are admitted by free device memory and
advanced together in batched chunks (continuous batching).

No counterpart in the reference (one solve per process there).  `serve`
replays a request stream with its arrival times in real time and reports
each request's latency (submit to completion) and the aggregate
cell-updates/s.
"""
import ctypes
import time

import numpy as np

from .field import FP64, _check, _preset, library

_bound = False


def _lib():
    global _bound
    L = library()
    if not _bound:
        H = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        sig = {
            "dim2d_server_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                                   ctypes.POINTER(H)]),
            "dim2d_server_submit": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int, ip, ip, ip,
                                                   ctypes.c_int, dp, dp, dp, ctypes.c_double,
                                                   ctypes.c_longlong,
                                                   ctypes.POINTER(ctypes.c_longlong)]),
            "dim2d_server_poll": (ctypes.c_int, [H, ctypes.c_int, ip]),
            "dim2d_server_result": (ctypes.c_int, [H, ctypes.c_longlong, dp, dp, dp]),
            "dim2d_server_stats": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_longlong)]),
            "dim2d_server_destroy": (ctypes.c_int, [H]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


NOT_READY = 7
WALL_ROOT = 5
NONFINITE = 8
STATS = ("pending", "active", "copying", "completed", "cell_updates", "bytes_in_use",
         "budget_bytes", "max_active")


class Server:
    def __init__(self, params=None, mem_budget=0, chunk_steps=500):
        from .field import default_params
        self.params = params if params is not None else default_params()
        h = ctypes.c_void_p()
        _check(_lib().dim2d_server_create(ctypes.byref(self.params), int(mem_budget),
                                          int(chunk_steps), ctypes.byref(h)))
        self._h = h
        self.shapes = {}

    def submit(self, nodes, x_map, y_map, dt, nsteps, bc="hedstrom_xy", precision=FP64):
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        ny, nx = nodes.shape[1], nodes.shape[2]
        ch, ty, od = _preset(bc)
        arr = ctypes.c_int * 8
        dp = ctypes.POINTER(ctypes.c_double)
        rid = ctypes.c_longlong()
        x_map = np.ascontiguousarray(x_map, dtype=np.float64)
        y_map = np.ascontiguousarray(y_map, dtype=np.float64)
        _check(_lib().dim2d_server_submit(self._h, nx, ny, arr(*ch), arr(*ty), arr(*od),
                                          int(precision), nodes.ctypes.data_as(dp),
                                          x_map.ctypes.data_as(dp), y_map.ctypes.data_as(dp),
                                          float(dt), int(nsteps), ctypes.byref(rid)))
        self.shapes[rid.value] = nodes.shape
        return rid.value

    def poll(self, wait=False):
        n = ctypes.c_int()
        _check(_lib().dim2d_server_poll(self._h, 1 if wait else 0, ctypes.byref(n)))
        return n.value

    def result(self, rid):
        """(nodes, time, latency_s, status), or None while the request runs.
        status 0; WALL_ROOT when a wall ghost-cell root failed during the
        solve -- where the reference stops; NONFINITE when the state stopped
        being finite.  The server stops such requests at the chunk boundary
        after its check saw them; nodes and time are then the state and time
        the solve ended with."""
        out = np.empty(self.shapes.get(rid, (4, 1, 1)))  # unknown ids: the library errors
        t = ctypes.c_double()
        lat = ctypes.c_double()
        dp = ctypes.POINTER(ctypes.c_double)
        rc = _lib().dim2d_server_result(self._h, rid, out.ctypes.data_as(dp), ctypes.byref(t),
                                        ctypes.byref(lat))
        if rc == NOT_READY:
            return None
        if rc not in (WALL_ROOT, NONFINITE):
            _check(rc)
        del self.shapes[rid]
        return out, t.value, lat.value, rc

    def stats(self):
        v = (ctypes.c_longlong * 8)()
        _check(_lib().dim2d_server_stats(self._h, v))
        return dict(zip(STATS, list(v)))

    def close(self):
        if getattr(self, "_h", None):
            _lib().dim2d_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def serve(server, requests, keep_results=False):
    """Replay `requests` (dicts with arrival (s), nodes, x_map, y_map, dt,
    nsteps, bc and optionally precision) in real time: each is submitted at
    its arrival time, the loop polls in between.  Returns dict(latencies, results (index ->
    (nodes, time) if keep_results), failed (indices of requests whose wall
    root failed), nonfinite (other requests whose state stopped being
    finite), finished (the other requests: finite solves), end_time (index
    -> the time each solve ended at; earlier than dt * nsteps for requests
    the server stopped), wall_s, cell_updates (all requests, as
    requested), cell_updates_finished (finished requests only), stats)."""
    order = sorted(range(len(requests)), key=lambda i: requests[i]["arrival"])
    ids = {}
    out, lat, failed, nonfinite, end_time = {}, {}, [], [], {}
    t0 = time.perf_counter()
    nxt = 0
    while len(lat) < len(requests):
        now = time.perf_counter() - t0
        while nxt < len(order) and requests[order[nxt]]["arrival"] <= now:
            r = requests[order[nxt]]
            ids[server.submit(r["nodes"], r["x_map"], r["y_map"], r["dt"], r["nsteps"],
                              r["bc"], r.get("precision", FP64))] = order[nxt]
            nxt += 1
        st = server.stats()
        busy = st["active"] + st["copying"] > 0
        server.poll(wait=busy)
        if not busy and nxt < len(order):  # idle until the next arrival
            time.sleep(max(0.0, min(0.002, requests[order[nxt]]["arrival"] - now)))
        for rid in list(ids):
            res = server.result(rid)
            if res is None:
                continue
            i = ids.pop(rid)
            lat[i] = res[2]
            end_time[i] = res[1]
            if res[3] == WALL_ROOT:
                failed.append(i)
            elif res[3] == NONFINITE or not np.isfinite(res[0]).all():
                nonfinite.append(i)
            if keep_results:
                out[i] = (res[0], res[1])
    wall = time.perf_counter() - t0
    def cells(r):
        return r["nsteps"] * (r["nodes"].shape[1] - 4) * (r["nodes"].shape[2] - 4)

    bad = set(failed) | set(nonfinite)
    return dict(latencies=[lat[i] for i in range(len(requests))], results=out,
                failed=sorted(failed), nonfinite=sorted(nonfinite), end_time=end_time,
                wall_s=wall,
                cell_updates=sum(cells(r) for r in requests),
                finished=[i for i in range(len(requests)) if i not in bad],
                cell_updates_finished=sum(cells(r) for i, r in enumerate(requests)
                                          if i not in bad),
                stats=server.stats())
