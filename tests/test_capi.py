"""The C-ABI library builds for sm_100a, loads, and exports every symbol
that include/*.h declares (no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"DIM2D_API\s+[\w\s\*]*?\b(dim2d_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("dim2d_create", "dim2d_upload", "dim2d_step", "dim2d_time_dev",
              "dim2d_download", "dim2d_destroy", "dim2d_apply_bc_on_nodes", "dim2d_cfl_dt"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from dim2d_finite_volume_b200 import build
    lib = build.build()
    out = subprocess.check_output(["nm", "-D", "--defined-only", lib]).decode()
    exported = set(re.findall(r"\bT (dim2d_\w+)", out))
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, missing
    L = ctypes.CDLL(lib)
    for n in declared_symbols():
        getattr(L, n)


def test_library_is_sm100a():
    from dim2d_finite_volume_b200 import build
    lib = build.build()
    out = subprocess.check_output(["/usr/local/cuda/bin/cuobjdump", "--list-elf", lib]).decode()
    assert "sm_100a" in out


def test_host_only_calls_without_gpu():
    """Calls that need no device: defaults, coordinates, argument checks."""
    import numpy as np
    from dim2d_finite_volume_b200 import field as F
    p = F.default_params()
    assert (p.re, p.we, p.pr, p.cv_r, p.viscous_r) == (5.0, 10.0, 20.0, 2.5, -1.5)
    x = np.zeros(20)
    y = np.zeros(12)
    F._check(F.library().dim2d_ini_coordinates(20, 12, -0.5, 0.5, -1.0, 1.0, F._ptr(x), F._ptr(y)))
    assert x[2] == -0.5 and abs(x[-3] - 0.5) < 1e-15
    assert abs((y[1] - y[0]) - 2.0 / 7) < 1e-15
    with pytest.raises(F.Dim2dError) as e:
        F._check(F.library().dim2d_ini_coordinates(3, 12, 0, 1, 0, 1, F._ptr(x), F._ptr(y)))
    assert e.value.code == 1


def test_mixed_presets_classified_before_any_device_call():
    """wall_S_open and half_wall_S_open are provided configurations; a
    half_wall_S_open section order whose node pass the kernels do not
    reproduce (S wall before the W mirror) is refused with its own message.
    Classification happens before any CUDA call, so this runs without a GPU."""
    import ctypes

    from dim2d_finite_volume_b200 import field as F
    L = F.library()
    arr = ctypes.c_int * 8
    p = F.default_params()
    h = ctypes.c_void_p()
    for preset in ("wall_S_open", "half_wall_S_open"):
        ch, ty, order = F._preset(preset)
        rc = L.dim2d_create(ctypes.byref(p), 40, 30, arr(*ch), arr(*ty), arr(*order), 0,
                            ctypes.byref(h))
        msg = L.dim2d_last_error().decode()
        assert "not provided" not in msg and "half_wall_S_open needs" not in msg, (preset, msg)
        if rc == 0:  # a device is present
            L.dim2d_destroy(h)
    ch, ty, order = F._preset("half_wall_S_open")
    bad = list(order)
    i, j = bad.index(F._SECTION["W"]), bad.index(F._SECTION["S"])
    bad[i], bad[j] = bad[j], bad[i]
    rc = L.dim2d_create(ctypes.byref(p), 40, 30, arr(*ch), arr(*ty), arr(*bad), 0, ctypes.byref(h))
    assert rc != 0 and "half_wall_S_open needs" in L.dim2d_last_error().decode()
    # a W side that is neither open nor a mirror beside the open N/E sides
    ch2 = list(ch)
    ch2[3] = F.WALL
    ty2 = [F.bc_type_of(c) for c in ch2]
    rc = L.dim2d_create(ctypes.byref(p), 40, 30, arr(*ch2), arr(*ty2), arr(*order), 0,
                        ctypes.byref(h))
    assert rc != 0 and "not provided" in L.dim2d_last_error().decode()
