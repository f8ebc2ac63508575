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
