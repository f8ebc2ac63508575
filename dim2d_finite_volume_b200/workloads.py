"""Seeded synthetic workloads of the benchmark configurations.

Every domain is the DIM bubble set-up of ic.bubbles on [-0.5, 0.5]^2
(saturated densities from the van der Waals Maxwell construction, tanh
interface ~4 dx wide, uniform temperature T0), optionally carried by a
uniform x-flow at a given Mach number of the liquid sound speed.  The time
step is the smaller of the acoustic CFL step (CFL 0.1) and a viscous
Fourier step, both from the initial state.

"wall" domains use the reference's wall preset wall_S_reflection
(library_config.py:102-115: contact-angle wall on S, mirrors elsewhere);
the reference refuses wall_xy (library_config.py:93-99).
"""
import numpy as np

from . import ic

CV_R = 2.5
RE = 5.0


def liquid_sound_speed(T0, cv_r=CV_R):
    rv, rl = ic.maxwell_densities(T0)
    e = rl * (8.0 / 3.0 * cv_r * T0 - 3.0 * rl)
    return float(ic.sound_speed(np.array(rl), np.array(0.0), np.array(0.0), np.array(e), cv_r))


def stable_dt(q, dx, dy, cfl=0.1, fourier=0.2):
    """min(acoustic CFL step, viscous Fourier step) over the interior."""
    dt_a = ic.cfl_dt(q, dx, dy, cfl, CV_R)
    rho_min = float(q[0, 2:-2, 2:-2].min())
    return min(dt_a, fourier * RE * rho_min * min(dx, dy) ** 2)


def fill_periodic_ghosts(q):
    """Periodic ghost layers as field%ini leaves them
    (periodic_xy/bc_operators_class.f:156-199)."""
    ny, nx = q.shape[1], q.shape[2]
    px, py = nx - 4, ny - 4
    q[:, :, 0:2] = q[:, :, px:px + 2]
    q[:, :, nx - 2:] = q[:, :, 2:4]
    q[:, 0:2, :] = q[:, py:py + 2, :]
    q[:, ny - 2:, :] = q[:, 2:4, :]
    return q


def domain(n, ny=None, T0=0.95, bubbles=((0.0, 0.0, 0.1),), mach=0.0, bc="periodic_xy",
           li=None, we=10.0):
    """One field: dict(nx, ny, x_map, y_map, nodes (4, ny, nx), dt, bc, T0, mach).
    Interface width li (default 4 dx) and Weber number we of the initial
    energy.  Mirror and wall fields still need their node boundary pass
    (Field.apply_bc_on_nodes) after upload, as field%ini does."""
    ny = n if ny is None else ny
    nx, nyy, x_map, y_map = ic.grid(n, ny)
    dx = x_map[1] - x_map[0]
    dy = y_map[1] - y_map[0]
    u0 = mach * liquid_sound_speed(T0) if mach else 0.0
    q = ic.bubbles(x_map, y_map, T0, list(bubbles), li=4.0 * dx if li is None else li,
                   velocity=(u0, 0.0), we=we)
    if bc == "periodic_xy":
        fill_periodic_ghosts(q)
    q = np.ascontiguousarray(q)
    return dict(nx=nx, ny=nyy, x_map=x_map, y_map=y_map, nodes=q, dt=stable_dt(q, dx, dy),
                bc=bc, T0=T0, mach=mach)


def plain_1024(seed, n=1024, bc="hedstrom_xy"):
    """Plain FP64 at 1024^2: a bubble of seeded radius in [0.05, 0.15] at
    T0 = 0.95 carried by a Mach 0.1 x-flow with open boundaries on all
    sides (bc='periodic_xy': the same bubble at rest in a periodic box)."""
    rng = np.random.default_rng(seed)
    r = float(rng.uniform(0.05, 0.15))
    d = domain(n, T0=0.95, bubbles=[(0.0, 0.0, r)], mach=0.1 if bc == "hedstrom_xy" else 0.0,
               bc=bc)
    d["radius"] = r
    return d


BATCH_KINDS = ("wall_S_reflection", "periodic_xy", "hedstrom_xy")


# Weber number of the batched configuration (one constant set: the domains
# share batched launches); equilibrium interface widths 0.08-0.26 over T0 in
# [0.9, 0.99], so that every domain runs the configuration's 2000 steps
BATCH_WE = 2000.0


def batch_params():
    """dim2d_params of the batched configuration (We = BATCH_WE)."""
    from .field import default_params
    p = default_params()
    p.we = BATCH_WE
    return p


def batched_specs(seed, count=64, sizes=tuple(range(128, 513, 64))):
    """The seeded draws of batched_domains without building the fields: one
    dict(n, T0, radius, mach, bc) per domain, in order."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(sizes))
        T0 = float(rng.uniform(0.90, 0.99))
        r = float(rng.uniform(0.05, 0.2))
        mach = float(rng.uniform(0.0, 0.1))
        bc = BATCH_KINDS[int(rng.integers(0, len(BATCH_KINDS)))]
        out.append(dict(n=n, T0=T0, radius=r, mach=mach if bc == "hedstrom_xy" else 0.0, bc=bc))
    return out


def batched_domain(spec):
    """The field of one batched_specs entry."""
    d = domain(spec["n"], T0=spec["T0"], bubbles=[(0.0, 0.0, spec["radius"])],
               mach=spec["mach"], bc=spec["bc"], li=ic.interface_length(spec["T0"], BATCH_WE),
               we=BATCH_WE)
    d["radius"] = spec["radius"]
    return d


def batched_domains(seed, count=64, sizes=tuple(range(128, 513, 64))):
    """Batched FP64: `count` independent domains, n uniform in
    {128, 192, ..., 512} (square), T0 in U[0.90, 0.99], bubble radius in
    U[0.05, 0.2], boundary kind uniform over wall / periodic / open, flow
    Mach in U[0, 0.1] for open domains (wall and periodic domains at rest).
    The bubbles have the equilibrium interface width at T0 for We =
    BATCH_WE (ic.interface_length); solve them with batch_params()."""
    return [batched_domain(sp) for sp in batched_specs(seed, count, sizes)]


SERVED_KINDS = ("wall_S_reflection", "hedstrom_xy")
# Weber number of the served stream: one constant set for the whole stream
# (requests share batched launches), large enough that the equilibrium
# interface width (0.08-0.26 over T0 in [0.9, 0.99]) fits the bubbles
SERVED_WE = 2000.0


def served_params():
    """dim2d_params of the served stream: the test constant set with
    We = SERVED_WE."""
    from .field import default_params
    p = default_params()
    p.we = SERVED_WE
    return p


def served_requests(seed, count, rate=50.0, n_range=(64, 1024), steps_range=(500, 20000),
                    mixed_fraction=0.5, kinds=SERVED_KINDS):
    """Served stream: Poisson arrivals at `rate` per second; grid size n
    (square) log-uniform in n_range, step count uniform in steps_range,
    T0 in U[0.9, 0.99], wall or open boundaries, one bubble of radius in
    U[0.05, 0.2] (open fields: Mach in U[0, 0.1]), FP64 or mixed precision
    (a `mixed_fraction` share, drawn from a separate seeded stream).  Each
    request carries its arrival time (s) from the start of the stream.
    `kinds`: the boundary presets drawn from (uniformly).
    The bubbles have the equilibrium interface width at T0 for We =
    SERVED_WE (ic.interface_length), as the reference's bubble initial
    conditions do; solve them with served_params()."""
    rng = np.random.default_rng(seed)
    rng_p = np.random.default_rng(seed + 7919)
    t = 0.0
    out = []
    lo, hi = np.log(n_range[0]), np.log(n_range[1])
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        n = int(round(float(np.exp(rng.uniform(lo, hi)))))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        T0 = float(rng.uniform(0.90, 0.99))
        r = float(rng.uniform(0.05, 0.2))
        bc = kinds[int(rng.integers(0, len(kinds)))]
        mach = float(rng.uniform(0.0, 0.1)) if bc == "hedstrom_xy" else 0.0
        d = domain(n, T0=T0, bubbles=[(0.0, 0.0, r)], mach=mach, bc=bc,
                   li=ic.interface_length(T0, SERVED_WE), we=SERVED_WE)
        d.update(arrival=t, nsteps=steps, radius=r,
                 precision=1 if rng_p.uniform() < mixed_fraction else 0)
        out.append(d)
    return out


# Weber number of the mixed-precision configuration: equilibrium interface
# width 0.067 at T0 = 0.97, below the bubble radii
MIXED_WE = 1.0e4


def mixed_params():
    """dim2d_params of the mixed-precision configuration (We = MIXED_WE)."""
    from .field import default_params
    p = default_params()
    p.we = MIXED_WE
    return p


def mixed_2048(seed, n=2048, count=4):
    """Mixed-precision configuration: 2048^2, `count` bubbles of radius in
    U[0.05, 0.1] at seeded non-overlapping centres (clear of the walls), in
    liquid at T0 = 0.97, wall boundaries (wall_S_reflection), at rest.  The
    bubbles have the equilibrium interface width at T0 for We = MIXED_WE
    (ic.interface_length); solve them with mixed_params()."""
    rng = np.random.default_rng(seed)
    bub = []
    while len(bub) < count:
        r = float(rng.uniform(0.05, 0.1))
        cx, cy = (float(v) for v in rng.uniform(-0.5 + r + 0.05, 0.5 - r - 0.05, 2))
        if all((cx - x) ** 2 + (cy - y) ** 2 > (r + rr + 0.05) ** 2 for x, y, rr in bub):
            bub.append((cx, cy, r))
    d = domain(n, T0=0.97, bubbles=bub, mach=0.0, bc="wall_S_reflection",
               li=ic.interface_length(0.97, MIXED_WE), we=MIXED_WE)
    d["bubbles"] = bub
    return d


# grdpts_id values of buffer-layer grids (parameters_bf_layer.f:41-44)
NO_PT, INTERIOR_PT, BC_INTERIOR_PT, BC_PT = 0, 1, 2, 3


def layer_map(nx, ny, rects):
    """grdpts_id [ny][nx] int32 of a buffer layer: interior_pt over the
    union of the rectangles (0-based inclusive (x0, x1, y0, y1)), one ring
    of bc_interior_pt around it, one ring of bc_pt around that, no_pt
    elsewhere -- the layout the reference's layers keep around their
    interior points."""
    inner = np.zeros((ny, nx), bool)
    for x0, x1, y0, y1 in rects:
        inner[y0:y1 + 1, x0:x1 + 1] = True

    def grow(m):  # 8-neighbour dilation without wrap-around
        p = np.pad(m, 1)
        out = np.zeros_like(m)
        for sy in range(3):
            for sx in range(3):
                out |= p[sy:sy + ny, sx:sx + nx]
        return out

    ring1 = grow(inner) & ~inner
    ring2 = grow(inner | ring1) & ~(inner | ring1)
    g = np.zeros((ny, nx), np.int32)
    g[ring2] = BC_PT
    g[ring1] = BC_INTERIOR_PT
    g[inner] = INTERIOR_PT
    return g


def buffer_layer(seed, n=2048, width=256, T0=0.95, mach=0.1):
    """An edge band of a n^2 domain as a buffer layer grid: n x width
    interior points of the domain's y range [0.5 - width dx, 0.5] extended
    north, both boundary rings inside the (n + 4) x (width + 4) grid, and a
    seeded bubble crossing the band in a Mach-`mach` x-flow.  Returns
    dict(nx, ny, x_map, y_map, dx, dy, nodes, grdpts_id, dt, x_borders,
    y_borders) with the reference's 1-based borders."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / (n - 1)
    y0 = 0.5 - (width - 1) * dx
    nx, ny, x_map, y_map = ic.grid(n, width, y_min=y0, y_max=0.5)
    r = float(rng.uniform(0.05, 0.1))
    xc = float(rng.uniform(-0.3, 0.3))
    u0 = mach * liquid_sound_speed(T0) if mach else 0.0
    q = np.ascontiguousarray(ic.bubbles(x_map, y_map, T0, [(xc, y0 + 0.5 * r, r)],
                                        li=4.0 * dx, velocity=(u0, 0.0)))
    g = layer_map(nx, ny, [(2, nx - 3, 2, ny - 3)])
    return dict(nx=nx, ny=ny, x_map=x_map, y_map=y_map, dx=dx, dy=y_map[1] - y_map[0],
                nodes=q, grdpts_id=g, dt=stable_dt(q, dx, dx), x_borders=(3, nx - 2),
                y_borders=(3, ny - 2))
