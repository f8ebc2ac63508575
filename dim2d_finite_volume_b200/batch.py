"""Batches of fields advanced together (include/dim2d.h, dim2d_batch_*).

No counterpart in the reference, which advances one field per process.
A Batch borrows the device state of Field objects (created and uploaded as
usual) and advances them with one launch per RK stage per boundary kind,
replaying a captured CUDA graph per step; fields keep their own dt.
"""
import ctypes

import numpy as np

from .field import Dim2dError, _check, library  # noqa: F401  (re-exported error type)

GROUPS = ("periodic_xy", "hedstrom_xy", "wall_S_reflection", "reflection_xy",
          "periodic_xy/mixed", "hedstrom_xy/mixed", "wall_S_reflection/mixed",
          "reflection_xy/mixed")
NSHAPES = 5
_bound = False


def _lib():
    global _bound
    L = library()
    if not _bound:
        H = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        sig = {
            "dim2d_batch_create": (ctypes.c_int, [ctypes.POINTER(H)]),
            "dim2d_batch_add": (ctypes.c_int, [H, H, ctypes.c_double]),
            "dim2d_batch_remove": (ctypes.c_int, [H, H]),
            "dim2d_batch_set_dt": (ctypes.c_int, [H, H, ctypes.c_double]),
            "dim2d_batch_step": (ctypes.c_int, [H, ctypes.c_int]),
            "dim2d_batch_sync": (ctypes.c_int, [H]),
            "dim2d_batch_set_shape": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int]),
            "dim2d_batch_set_graphs": (ctypes.c_int, [H, ctypes.c_int]),
            "dim2d_batch_set_persistent": (ctypes.c_int, [H, ctypes.c_int]),
            "dim2d_batch_set_rows": (ctypes.c_int, [H, ctypes.c_int]),
            "dim2d_batch_set_wait_limit": (ctypes.c_int, [H, ctypes.c_double]),
            "dim2d_batch_withhold_item": (ctypes.c_int, [H, ctypes.c_longlong]),
            "dim2d_batch_autotune": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_int), dp]),
            "dim2d_batch_size": (ctypes.c_int, [H]),
            "dim2d_batch_launch_count": (ctypes.c_longlong, [H]),
            "dim2d_batch_cells": (ctypes.c_longlong, [H]),
            "dim2d_batch_set_stream": (ctypes.c_int, [H, ctypes.c_void_p]),
            "dim2d_batch_destroy": (ctypes.c_int, [H]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


class Batch:
    """Many Field objects advanced together on one GPU."""

    def __init__(self):
        h = ctypes.c_void_p()
        _check(_lib().dim2d_batch_create(ctypes.byref(h)))
        self._h = h
        self.members = []

    def add(self, field, dt):
        _check(_lib().dim2d_batch_add(self._h, field._h, float(dt)))
        self.members.append(field)

    def remove(self, field):
        _check(_lib().dim2d_batch_remove(self._h, field._h))
        self.members.remove(field)

    def set_dt(self, field, dt):
        _check(_lib().dim2d_batch_set_dt(self._h, field._h, float(dt)))

    def step(self, nsteps=1):
        _check(_lib().dim2d_batch_step(self._h, int(nsteps)))

    def sync(self):
        _check(_lib().dim2d_batch_sync(self._h))

    def set_shape(self, group, shape):
        g = GROUPS.index(group) if isinstance(group, str) else int(group)
        _check(_lib().dim2d_batch_set_shape(self._h, g, int(shape)))

    def set_graphs(self, enable):
        _check(_lib().dim2d_batch_set_graphs(self._h, 1 if enable else 0))

    def set_persistent(self, enable=True):
        """Persistent mode: each step call is one persistent-kernel launch
        per precision that advances every member (include/dim2d.h)."""
        _check(_lib().dim2d_batch_set_persistent(self._h, int(bool(enable))))

    def set_rows(self, rows):
        _check(_lib().dim2d_batch_set_rows(self._h, int(rows)))

    def set_wait_limit(self, seconds):
        _check(_lib().dim2d_batch_set_wait_limit(self._h, float(seconds)))

    def withhold_item(self, item):
        """Tests of the bounded waits: never signal work item `item`."""
        _check(_lib().dim2d_batch_withhold_item(self._h, int(item)))

    def set_stream(self, stream):
        _check(_lib().dim2d_batch_set_stream(self._h, ctypes.c_void_p(stream)))

    def autotune(self):
        """Per group: the fastest strip shape; returns (shapes[8], times ms [8][5])."""
        ng = len(GROUPS)
        chosen = (ctypes.c_int * ng)()
        times = np.zeros(ng * NSHAPES)
        _check(_lib().dim2d_batch_autotune(self._h, chosen,
                                           times.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return list(chosen), times.reshape(ng, NSHAPES)

    @property
    def size(self):
        return _lib().dim2d_batch_size(self._h)

    @property
    def cells(self):
        """Interior cells of all members (cell-updates per step)."""
        return _lib().dim2d_batch_cells(self._h)

    @property
    def launches(self):
        return _lib().dim2d_batch_launch_count(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _lib().dim2d_batch_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
