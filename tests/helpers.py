"""Shared helpers of the parity tests (error metric, case set-up)."""
import numpy as np

from dim2d_finite_volume_b200 import ic

BC = 2


def interior(a):
    return a[:, BC:-BC, BC:-BC]


def normwise_rel_err(a, b, sl=None):
    """Per conservative variable: max|a-b| / max|b| over the interior."""
    A = interior(a) if sl is None else a[sl]
    B = interior(b) if sl is None else b[sl]
    out = []
    for k in range(4):
        den = np.abs(B[k]).max()
        num = np.abs(A[k] - B[k]).max()
        out.append(num / den if den > 0 else num)
    return np.array(out)


def periodic_case(n=128, ny=None, T0=0.95, radius=0.1, seed=None):
    """128^2 periodic static bubble (or a smaller/ragged variant)."""
    ny = n if ny is None else ny
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    q = ic.bubbles(x_map, y_map, T0, [(0.0, 0.0, radius)], li=4.0 * dx)
    if seed is not None:
        rng = np.random.default_rng(seed)
        q[1] += 0.02 * rng.standard_normal(q[0].shape) * q[0]
        q[2] += 0.02 * rng.standard_normal(q[0].shape) * q[0]
        q[3] += 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0]
    return nx, nyy, x_map, y_map, np.ascontiguousarray(q)


def stable_dt(q, x_map, y_map, cfl=0.1, fourier=0.2, re=5.0, cv_r=2.5):
    """min(acoustic CFL step, viscous Fourier step) of the interior."""
    dx = x_map[1] - x_map[0]
    dy = y_map[1] - y_map[0]
    dt_a = ic.cfl_dt(q, dx, dy, cfl, cv_r)
    rho_min = float(interior(q)[0].min())
    return min(dt_a, fourier * re * rho_min * min(dx, dy) ** 2)


def liquid_sound_speed(T0, cv_r=2.5):
    rv, rl = ic.maxwell_densities(T0)
    e = rl * (8.0 / 3.0 * cv_r * T0 - 3.0 * rl)
    return float(ic.sound_speed(np.array(rl), np.array(0.0), np.array(0.0), np.array(e), cv_r))


def open_case(n=128, ny=None, T0=0.95, radius=0.12, mach=0.1, seed=None, center=(0.0, 0.0)):
    """Bubble transported by a uniform x-flow (Mach `mach` of the liquid
    sound speed) -- the open-boundary (hedstrom_xy) configuration."""
    ny = n if ny is None else ny
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    u0 = mach * liquid_sound_speed(T0)
    q = ic.bubbles(x_map, y_map, T0, [(center[0], center[1], radius)], li=4.0 * dx,
                   velocity=(u0, 0.0))
    if seed is not None:
        rng = np.random.default_rng(seed)
        q[2] += 0.01 * rng.standard_normal(q[0].shape) * q[0]
        q[3] += 0.5 * (q[2] ** 2) / q[0]
    return nx, nyy, x_map, y_map, np.ascontiguousarray(q)


def normwise_rel_err_all(a, b):
    """Per conservative variable over ALL cells (ghosts included)."""
    out = []
    for k in range(4):
        den = np.abs(b[k]).max()
        num = np.abs(a[k] - b[k]).max()
        out.append(num / den if den > 0 else num)
    return np.array(out)
