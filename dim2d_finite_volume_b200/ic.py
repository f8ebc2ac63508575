"""Seeded synthetic initial conditions for the DIM solver (set-up, host side).

These restate the reference's bubble initial condition so that the GPU path
and the oracle start from the same arrays:

* grid: vertex-centred, 2 ghost layers; dx = (x_max-x_min)/(nx-1-2*bc_size),
  x_map(i) = x_min + (i-1-bc_size)*dx (src/field/field_abstract_class.f:286-315),
  so an n x n interior is nx = n + 4 points.
* mass density: tanh profile (src/physical_models/dim2d/dim2d_ic/
  dim2d_dropbubble_module.f:180-210), vapour at the centre.
* total energy: rho*(8/3 cv_r T0 - 3 rho) + |grad rho|^2/(2 We)
  + rho |u|^2 / 2 (dim2d_dropbubble_module.f:266-386 and
  dim2d_ic/bubble_transported/ic_class.f:195-215).
* saturated densities: the van der Waals Maxwell construction (equal
  pressure, equal chemical potential) solved by Newton; the reference's
  sqrt(1-T) fits (dim2d_state_eq_module.f:145-227) are its starting guess.
* time step: dt = CFL * min(dx,dy) / max(c + |u|) over the interior, with the
  reference's speed of sound (dim2d_prim_module.f:1179-1215).

Arrays are C-ordered [4][ny][nx] (the Fortran nodes(nx,ny,4) in memory).
"""
import math

import numpy as np

BC_SIZE = 2


def grid(n_interior_x, n_interior_y=None, x_min=-0.5, x_max=0.5, y_min=-0.5, y_max=0.5):
    n_interior_y = n_interior_x if n_interior_y is None else n_interior_y
    nx = n_interior_x + 2 * BC_SIZE
    ny = n_interior_y + 2 * BC_SIZE
    dx = (x_max - x_min) / (nx - 1 - 2 * BC_SIZE)
    dy = (y_max - y_min) / (ny - 1 - 2 * BC_SIZE)
    x_map = x_min + (np.arange(1, nx + 1) - 1 - BC_SIZE) * dx
    y_map = y_min + (np.arange(1, ny + 1) - 1 - BC_SIZE) * dy
    return nx, ny, x_map, y_map


def saturation_fits(T):
    """dim2d_state_eq_module.f:145-227 (high-temperature branch)."""
    return 1.0 - 1.91 * math.sqrt(1.0 - T), 1.0 + 2.06 * math.sqrt(1.0 - T)


def vdw_pressure(rho, T):
    return 8.0 * rho * T / (3.0 - rho) - 3.0 * rho ** 2


def vdw_chemical_potential(rho, T):
    # derivative of the reduced vdW free energy density
    # rho*(8T/3)*ln(rho/(3-rho)) - 3 rho^2 with respect to rho
    return (8.0 * T / 3.0) * (math.log(rho / (3.0 - rho)) + 3.0 / (3.0 - rho)) - 6.0 * rho


def maxwell_densities(T, tol=1e-14, maxit=100):
    """(rho_vap, rho_liq) of the reduced vdW fluid at T < 1."""
    if not 0.0 < T < 1.0:
        raise ValueError("Maxwell construction needs 0 < T < 1")
    rv, rl = saturation_fits(T)
    for _ in range(maxit):
        f1 = vdw_pressure(rl, T) - vdw_pressure(rv, T)
        f2 = vdw_chemical_potential(rl, T) - vdw_chemical_potential(rv, T)
        # dP/drho and dmu/drho
        dp_l = 24.0 * T / (3.0 - rl) ** 2 - 6.0 * rl
        dp_v = 24.0 * T / (3.0 - rv) ** 2 - 6.0 * rv
        dm_l = dp_l / rl
        dm_v = dp_v / rv
        det = (-dp_v) * dm_l - dp_l * (-dm_v)
        drv = (-f1 * dm_l + dp_l * f2) / det
        drl = (-(-dp_v) * f2 + (-dm_v) * f1) / det
        rv += drv
        rl += drl
        if abs(drv) + abs(drl) < tol:
            break
    return rv, rl


def sound_speed(rho, mx, my, E, cv_r):
    """dim2d_prim_module.f:1179-1215, vectorised."""
    u2 = (mx / rho) ** 2 + (my / rho) ** 2
    P = 3.0 / ((3.0 - rho) * cv_r) * (E - 0.5 * rho * u2 + 3.0 * rho ** 2) - 3.0 * rho ** 2
    e = P + rho ** 2 * (-3.0 + 2.0 * rho)
    b = np.sqrt((P + 3.0 * rho ** 2) / (cv_r * e))
    a = 1.0 / np.sqrt(1.0 + b ** 2)
    d = np.sqrt(rho ** 3) * np.sqrt((3.0 - rho) / e)
    return np.sqrt(3.0) * rho / (a * d)


def interface_length(T, we):
    """Equilibrium width of the liquid-vapour interface at temperature T
    (dim2d_state_eq_module.f:90-125, high-temperature branch): the width the
    reference's own bubble initial conditions use (e.g.
    dim2d_ic/bubble_next_to_wall/ic_class.f:186)."""
    return 1.0 / math.sqrt(2.0 * we) * (1.6309400153322933 / math.sqrt(1.0 - T))


def bubbles(x_map, y_map, T0, bubbles_xyr, li, velocity=(0.0, 0.0), we=10.0, cv_r=2.5,
            densities=None):
    """Vapour bubbles (centre x, centre y, radius) in saturated liquid.

    Overlapping profiles combine by taking the minimum density, which for
    separated bubbles equals the single-bubble profile of the reference."""
    rv, rl = maxwell_densities(T0) if densities is None else densities
    X, Y = np.meshgrid(x_map, y_map)  # [ny][nx]
    rho = np.full(X.shape, rl)
    grad2 = np.zeros(X.shape)
    for (xc, yc, r) in bubbles_xyr:
        d = np.sqrt((X - xc) ** 2 + (Y - yc) ** 2)
        th = np.tanh(2.0 * (d - r) / li)
        rb = (rl + rv) / 2.0 + (rl - rv) / 2.0 * th
        g2 = ((rl - rv) / li) ** 2 * (1.0 - th ** 2) ** 2
        take = rb < rho
        rho = np.where(take, rb, rho)
        grad2 = np.where(take, g2, grad2)
    ux, uy = velocity
    q = np.empty((4,) + X.shape)
    q[0] = rho
    q[1] = rho * ux
    q[2] = rho * uy
    q[3] = rho * (8.0 / 3.0 * cv_r * T0 - 3.0 * rho) + 1.0 / (2.0 * we) * grad2 \
        + 0.5 * rho * (ux ** 2 + uy ** 2)
    return np.ascontiguousarray(q)


def cfl_dt(q, dx, dy, cfl, cv_r=2.5):
    """dt = CFL*min(dx,dy)/max(c+|u|) over the interior nodes.

    Nodes where the speed of sound is undefined (spinodal states, where
    the square roots of dim2d_prim_module.f:1197-1202 have negative
    arguments) are skipped, like fmax skips NaN in the device reduction."""
    s = (slice(None), slice(BC_SIZE, -BC_SIZE), slice(BC_SIZE, -BC_SIZE))
    qi = q[s]
    with np.errstate(invalid="ignore"):
        c = sound_speed(qi[0], qi[1], qi[2], qi[3], cv_r)
    u = np.sqrt((qi[1] / qi[0]) ** 2 + (qi[2] / qi[0]) ** 2)
    return cfl * min(dx, dy) / float(np.nanmax(c + u))


def config1(n=128, T0=0.95, radius=0.1, cfl=0.1, cv_r=2.5, we=10.0):
    """128^2 periodic static vapour bubble, width 4 dx, zero velocity."""
    nx, ny, x_map, y_map = grid(n)
    dx = x_map[1] - x_map[0]
    q = bubbles(x_map, y_map, T0, [(0.0, 0.0, radius)], li=4.0 * dx, we=we, cv_r=cv_r)
    dt = cfl_dt(q, dx, y_map[1] - y_map[0], cfl, cv_r)
    return dict(nx=nx, ny=ny, x_map=x_map, y_map=y_map, nodes=q, dt=dt, T0=T0)
