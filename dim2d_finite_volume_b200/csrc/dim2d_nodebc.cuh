// dim2d_nodebc.cuh -- node boundary pass for mirror sides and the south
// wall on sm_100a: the per-cell work (node_bc_cell), shared by the node-pass
// launches (dim2d_nodebc.cu) and the persistent batched kernel
// (dim2d_strip.cu).
//
// Configurations (the reference's presets, library_config.py:58-150):
//   reflection_xy      N/S reflection_y, E/W reflection_x, corners reflection_y
//   wall_S_reflection  S wall, N reflection_y, E/W reflection_x, corners reflection_x
//   wall_S_open        S, SW, SE wall; N, E, W, NE, NW open (no node work)
//   half_wall_S_open   S, SE wall; W, SW, NW reflection_x; N, E, NE open
// Mirrors: bc_operators_reflection_{x,y}_class.f:178-296 (prefactor -1 on
// the normal momentum, reflection_xy_module.f:50-110).  Every mirror ghost
// is a signed copy of an interior node, so all of them are computed
// straight from the interior, in one launch, whatever the section order.
// The corners of wall_S_reflection (and the SW corner of half_wall_S_open)
// mirror the wall ghost cells; the thread that solves a wall column writes
// them too.  The wall corners next to an open side solve their ghost cells
// like the wall edge, with one-sided tangential gradients in the outer
// column.
//
// Wall ghost cell (wall_xy_equilibrium_module.f:948-1040, 1747-2461):
// density of the first ghost row = root in [rho_vap(T), rho_liq(T)] of the
// contact-angle equilibrium function (bracket scan of at most 99 steps,
// then Ridders' method with at most 60 iterations, xacc = 1e-12,
// ridders_method_module.f:112-216); second ghost row by extrapolation;
// ghost momenta from the first interior velocity.  Where the reference
// stops the program (no bracket, no convergence) the kernel writes NaN and
// sets a bit of the status word the host reads after the step.
#pragma once
#include "dim2d_kernels.cuh"

// Device loads go through the read-only (non-coherent) path, except in a
// translation unit that defines DIM2D_COHERENT_LOADS: the persistent kernel
// reads fields that other SMs rewrite during the same launch, so its loads
// must be coherent (ld.global.cg, ordered by the acquire of its waits).
#if defined(__CUDA_ARCH__) && defined(DIM2D_COHERENT_LOADS)
#define NBC_LDG(p) __ldcg(p)
#define NBC_ST(p, v) (*(p) = (v))
#elif defined(__CUDA_ARCH__)
#define NBC_LDG(p) __ldg(p)
#define NBC_ST(p, v) (*(p) = (v))
#elif defined(DIM2D_LDG_HOST)
#define NBC_LDG(p) DIM2D_LDG_HOST(p)  // host emulation: checked reads and writes
#define NBC_ST(p, v) DIM2D_ST_HOST(p, v)
#else
#define NBC_LDG(p) (*(p))
#define NBC_ST(p, v) (*(p) = (v))
#endif

namespace dim2d {

namespace {

__host__ __device__ __forceinline__ int mirror_lo_hi(int i, int n) {
  // ghost index -> mirrored interior index (bc_size = 2)
  return i < BC ? 2 * BC - 1 - i : 2 * n - 2 * BC - 1 - i;
}

// gradient type of a wall column along the wall (gradient_type of
// compute_wall_*_ghost_cell, parameters_constant.f): centred, or one-sided
// in the outer column of a wall corner
enum WallGrad : int { WG_CENTRED = 0, WG_L0 = 1, WG_R0 = 2 };

// wall root function context (wall_x_root_fct, :2016-2103)
struct WallRoot {
  double md1;  // md_x(2): first interior density
  double md2;  // md_x(1): second interior density
  double my0, my1;
  double vx, vy, Ed;
  double dxn, dyt;  // delta_x (normal), delta_y (tangential)
  double q;
  double cosang;
  int gt;  // WallGrad of the tangential density gradient (get_dmd_dx, :2433-2461)
};

// dim2d_state_eq_module.f:56-227 (high-temperature fits)
__host__ __device__ __forceinline__ double md_vap(double T) { return 1.0 - 1.91 * sqrt(1.0 - T); }
__host__ __device__ __forceinline__ double md_liq(double T) { return 1.0 + 2.06 * sqrt(1.0 - T); }

// wall_x_equilibrium_root_fct(md_x(2), [md_x(1), x], ...), :2151-2212,
// with its per-column constants computed once (WallRootFn) and the algebra
// reduced: with s = sqrt(1 - Tav), md_liq - md_vap = 3.97 s and the surface
// tension is a constant times s^3 (:2238-2270, dim2d_state_eq_module.f:
// 56-227), so the energy-derivative term is
//   6 cos(angle) (md_av - md_liq)(md_av - md_vap) st / (md_liq - md_vap)^3
//   = C (md_av - md_liq)(md_av - md_vap),   C = 6 cos(angle) 2 sqrt(2)/(3 sqrt(We)) 9.6917.../3.97^3
// and an evaluation is one square root and a dozen multiply-adds instead of
// four divisions and three square roots (the solve runs one thread per
// wall column, so its instruction chain is the kernel's duration).  The
// value differs from the reference's evaluation order by rounding only.
struct WallRootFn {
  double md1, md2;
  double a1;    // 1/(We delta_x): dmddx_half / We
  double a2;    // 1/(2 delta_x): interior gradient normal to the wall
  double gy2;   // square of the tangential density gradient (get_dmd_dx type of the column)
  double base;  // Ed/md - |v|^2/2 + 3 md, the temperature without its gradient term
  double cw;    // 1/(2 We md)
  double c38;   // 3/(8 cv_r)
  double tq;    // temperature jump of the heat flux, :2295-2315
  double C;
};

__host__ __device__ __forceinline__ WallRootFn wall_root_fn(const WallRoot& c, const DimConst& k) {
  WallRootFn w;
  double gy;
  if (c.gt == WG_L0) gy = (c.my1 - c.md1) / c.dyt;
  else if (c.gt == WG_R0) gy = (c.md1 - c.my0) / c.dyt;
  else gy = (c.my1 - c.my0) / (2.0 * c.dyt);
  w.md1 = c.md1;
  w.md2 = c.md2;
  w.a1 = 1.0 / (k.we * c.dxn);
  w.a2 = 0.5 / c.dxn;
  w.gy2 = gy * gy;
  w.base = c.Ed / c.md1 - 0.5 * (c.vx * c.vx + c.vy * c.vy) + 3.0 * c.md1;
  w.cw = 0.5 / (k.we * c.md1);
  w.c38 = 3.0 / (8.0 * k.cv_r);
  w.tq = 0.5 * c.dxn * k.re * k.pr * w.c38 * c.q;
  w.C = 6.0 * c.cosang * (2.0 * sqrt(2.0) / (3.0 * sqrt(k.we)) * 9.691686257306483) /
        (3.97 * 3.97 * 3.97);
  return w;
}

__host__ __device__ __forceinline__ double wall_root_f(const WallRootFn& w, double x) {
  const double gx = (x - w.md2) * w.a2;
  const double Tav = w.c38 * (w.base - w.cw * (gx * gx + w.gy2)) + w.tq;
  const double s = sqrt(1.0 - Tav);
  const double md_av = 0.5 * (w.md1 + x);
  return w.a1 * (x - w.md1) + w.C * (md_av - (1.0 + 2.06 * s)) * (md_av - (1.0 - 1.91 * s));
}

__host__ __device__ __forceinline__ bool same_sign(double a, double b) {
  return copysign(1.0, a) * copysign(1.0, b) > 0;  // :1962-1972
}
__host__ __device__ __forceinline__ bool validated(double a, double b) { return fabs(a - b) < 1e-10; }

// :1846-1941 then ridders_method_module.f:112-216.  Returns the root;
// *status gets 1 (no bracket), 2 (not bracketed), 3 (no convergence) or
// 4 (bracketing error).
//
// The sequence of trial points and tests is the reference's; only the order
// of evaluation is changed for latency (one thread per wall column, so the
// chain of dependent root-function calls is the kernel's duration): the
// bracket ends, the guess and the first scan pair are evaluated together,
// before the tests that use them, and Ridders' method starts from the
// function values of its bracket ends already computed (the reference
// evaluates them again; the function is deterministic, so the values and
// the result are the same).
__host__ __device__ inline double wall_root(const WallRoot& c, double T_guess, double md_guess,
                                     const DimConst& k, unsigned int* status) {
  const WallRootFn w = wall_root_fn(c, k);
  double xl = md_vap(T_guess), xh = md_liq(T_guess);
  const double dmd_l = md_guess / 100.0, dmd_r = (3.0 - md_guess) / 100.0;
  const double a1 = md_guess - 1 * dmd_l, b1 = md_guess + 1 * dmd_r;
  double fl = wall_root_f(w, xl), fh = wall_root_f(w, xh);
  const double fmd = wall_root_f(w, md_guess);
  const double fa1 = wall_root_f(w, a1), fb1 = wall_root_f(w, b1);
  if (same_sign(fl, fh)) {
    bool found = false;
    for (int j = 1; j <= 99 && !found; j++) {
      const double a = md_guess - j * dmd_l, b = md_guess + j * dmd_r;
      const double fa = j == 1 ? fa1 : wall_root_f(w, a);
      if (!same_sign(fa, fmd)) {
        xl = a;
        xh = md_guess;
        fl = fa;
        fh = fmd;
        found = true;
        break;
      }
      const double fb = j == 1 ? fb1 : wall_root_f(w, b);
      if (!same_sign(fb, fmd)) {
        xl = md_guess;
        xh = b;
        fl = fmd;
        fh = fb;
        found = true;
      }
    }
    if (!found) {
      *status |= 1u;
      return NAN;
    }
  }
  // Ridders' method, from the bracket [xl, xh] and its values fl, fh
  const double xacc = 1e-12;
  const double UNUSED = (double)(-1.11e30f);
  double x = UNUSED;
  if ((fl > 0.0 && fh < 0.0) || (fl < 0.0 && fh > 0.0)) {
    const double x1 = xl;
    (void)x1;
    for (int j = 1; j <= 60; j++) {
      const double xm = 0.5 * (xl + xh);
      const double fm = wall_root_f(w, xm);
      const double s = sqrt(fm * fm - fl * fh);
      if (validated(s, 0.0)) return x;
      const double xnew = xm + (xm - xl) * (copysign(1.0, fl - fh) * fm / s);
      if (fabs(xnew - x) <= xacc) return x;
      x = xnew;
      const double fnew = wall_root_f(w, x);
      if (validated(fnew, 0.0)) return x;
      if (!validated(copysign(fm, fnew), fm)) {
        xl = xm;
        fl = fm;
        xh = x;
        fh = fnew;
      } else if (!validated(copysign(fl, fnew), fl)) {
        xh = x;
        fh = fnew;
      } else if (!validated(copysign(fh, fnew), fh)) {
        xl = x;
        fl = fnew;
      } else {
        *status |= 8u;
        return x;
      }
      if (fabs(xh - xl) <= xacc) return x;
    }
    *status |= 4u;
    return x;
  }
  if (validated(fl, 0.0)) return xl;
  if (validated(fh, 0.0)) return xh;
  *status |= 2u;
  return x;
}

__host__ __device__ __forceinline__ double ld(const double* p, const Field& f, int v, int x, int y) {
  return NBC_LDG(p + (size_t)v * f.plane + (size_t)y * f.pitch + x);
}

}  // namespace

// Work items of the node pass, in order: W mirror cells, E mirror cells,
// N mirror cells (each only where that side is a mirror), S cells (wall
// columns or mirror cells), then the corner cells that have node work.
// Wall columns span the interior columns plus, on an open side, its two
// ghost columns (the wall corner sections of wall_S_open /
// half_wall_S_open, bc_operators_wall_xy_class.f:340-360).  Corner work:
// mirror corners of reflection_xy (4) and wall_S_reflection (N only: the S
// ones are written with their wall columns), and the reflection_x NW
// corner of half_wall_S_open, which mirrors the open N ghost rows.
struct NodeLayout {
  int n_w, n_e, n_n, n_s;
  int x0, x1;        // wall columns [x0, x1)
  int corners;       // bit c: corner c (0 SW, 1 SE, 2 NW, 3 NE) has node work
};

__host__ __device__ __forceinline__ NodeLayout node_layout(const NodeBcArgs& a) {
  const int ex = a.f.nx - 2 * BC, ey = a.f.ny - 2 * BC;
  NodeLayout L;
  L.n_w = a.open_w ? 0 : BC * ey;
  L.n_e = a.open_e ? 0 : BC * ey;
  L.n_n = a.open_n ? 0 : BC * ex;
  L.x0 = a.open_w ? 0 : BC;
  L.x1 = a.open_e ? a.f.nx : a.f.nx - BC;
  L.n_s = a.south_wall ? L.x1 - L.x0 : BC * ex;
  L.corners = 0;
  if (!a.south_wall) L.corners |= 3;
  if (!a.open_w) L.corners |= 4;
  if (!a.open_e) L.corners |= 8;
  return L;
}

__host__ __device__ inline int node_bc_count(const NodeBcArgs& a) {
  const NodeLayout L = node_layout(a);
  const int nc = (L.corners & 1) + (L.corners >> 1 & 1) + (L.corners >> 2 & 1) + (L.corners >> 3 & 1);
  return L.n_w + L.n_e + L.n_n + L.n_s + nc * BC * BC;
}

// Ghost work item m (NodeLayout order)
__host__ __device__ inline void node_bc_cell(const NodeBcArgs& a, int m) {
  const Field f = a.f;
  const int nx = f.nx, ny = f.ny;
  const int ex = nx - 2 * BC, ey = ny - 2 * BC;
  const NodeLayout L = node_layout(a);
  if (m < 0 || m >= node_bc_count(a)) return;
  const double pre_x[4] = {1.0, -1.0, 1.0, 1.0};
  const double pre_y[4] = {1.0, 1.0, -1.0, 1.0};
  double* u = a.u;
  if (m < L.n_w + L.n_e) {  // reflection_x, bc_operators_reflection_x_class.f:212-234
    const bool east = m >= L.n_w;
    const int r = east ? m - L.n_w : m;
    const int y = BC + r % ey;
    const int col = r / ey;
    const int x = east ? nx - BC + col : col;
    const int sx = mirror_lo_hi(x, nx);
    for (int v = 0; v < 4; v++)
      NBC_ST(&u[(size_t)v * f.plane + (size_t)y * f.pitch + x], pre_x[v] * ld(u, f, v, sx, y));
    return;
  }
  m -= L.n_w + L.n_e;
  if (m < L.n_n) {  // reflection_y, bc_operators_reflection_y_class.f:211-221
    const int x = BC + m % ex;
    const int y = ny - BC + m / ex;
    const int sy = mirror_lo_hi(y, ny);
    for (int v = 0; v < 4; v++)
      NBC_ST(&u[(size_t)v * f.plane + (size_t)y * f.pitch + x], pre_y[v] * ld(u, f, v, x, sy));
    return;
  }
  m -= L.n_n;
  if (m < L.n_s) {
    if (!a.south_wall) {  // reflection_y, :223-233
      const int x = BC + m % ex;
      const int y = m / ex;
      const int sy = mirror_lo_hi(y, ny);
      for (int v = 0; v < 4; v++)
        NBC_ST(&u[(size_t)v * f.plane + (size_t)y * f.pitch + x], pre_y[v] * ld(u, f, v, x, sy));
      return;
    }
    // wall ghost column x: ghost rows 1 (first) and 0 (second),
    // interior rows 2 (first) and 3 (second)
    const int x = L.x0 + m;
    const DimConst& k = a.k;
    // outer columns of wall corners next to an open side: one-sided
    // tangential gradients (gradient_x_x_oneside_L0/R0 and GT_L0/GT_R0,
    // bc_operators_wall_xy_class.f:340-360)
    const int gt = x == 0 ? WG_L0 : (x == nx - 1 ? WG_R0 : WG_CENTRED);
    // temperature guess from u^n at the first interior node
    // (bc_operators_wall_xy_class.f:898-930, temperature_eff
    // dim2d_prim_module.f:652-691)
    double Tg;
    {
      const double r = ld(a.utmp, f, 0, x, 2);
      const double mx = ld(a.utmp, f, 1, x, 2), my = ld(a.utmp, f, 2, x, 2);
      const double E = ld(a.utmp, f, 3, x, 2);
      double gx;
      if (gt == WG_L0) gx = 1.0 / a.dx * (-ld(a.utmp, f, 0, x, 2) + ld(a.utmp, f, 0, x + 1, 2));
      else if (gt == WG_R0) gx = 1.0 / a.dx * (-ld(a.utmp, f, 0, x - 1, 2) + ld(a.utmp, f, 0, x, 2));
      else gx = 0.5 / a.dx * (-ld(a.utmp, f, 0, x - 1, 2) + ld(a.utmp, f, 0, x + 1, 2));
      const double gy = 0.5 / a.dy * (-ld(a.utmp, f, 0, x, 1) + ld(a.utmp, f, 0, x, 3));
      const double vx = mx / r, vy = my / r;
      const double teff = 1.0 / r * (E - 0.5 * r * (vx * vx + vy * vy) -
                                     0.5 / k.we * (gx * gx + gy * gy) + 3.0 * (r * r));
      Tg = 3.0 / (8.0 * k.cv_r) * teff;
    }
    const double md_guess = ld(a.utmp, f, 0, x, 1);
    // compute_wall_S_ghost_cell, wall_xy_equilibrium_module.f:948-1040
    const double r1 = ld(u, f, 0, x, 2), r2 = ld(u, f, 0, x, 3);
    const double mx1 = ld(u, f, 1, x, 2), my1 = ld(u, f, 2, x, 2);
    WallRoot c;
    c.md1 = r1;
    c.md2 = r2;
    // md_y: neighbours of the first interior node.  A mirror W/E ghost is
    // read at its source (the mirror side comes before S in the presets'
    // order and is written by this same launch); an open side's ghost
    // column holds the stage output.  The one-sided types read one side.
    c.my0 = c.my1 = 0.0;
    if (gt != WG_L0)
      c.my0 = x - 1 < BC && !a.open_w ? ld(u, f, 0, mirror_lo_hi(x - 1, nx), 2)
                                      : ld(u, f, 0, x - 1, 2);
    if (gt != WG_R0)
      c.my1 = x + 1 >= nx - BC && !a.open_e ? ld(u, f, 0, mirror_lo_hi(x + 1, nx), 2)
                                            : ld(u, f, 0, x + 1, 2);
    c.gt = gt;
    c.vx = -my1 / r1;
    c.vy = mx1 / r1;
    c.Ed = ld(u, f, 3, x, 2);
    c.dxn = a.dy;
    c.dyt = a.dx;
    c.q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    c.cosang = a.wall.cos_angle;
    unsigned int st = 0;
    const double rg = wall_root(c, Tg, md_guess, k, &st);
    if (st && a.status) {
#ifdef __CUDA_ARCH__
      atomicOr(a.status, st);
#else
      *a.status |= st;
#endif
    }
    const double rg2 = r2 + 3.0 * (-r1 + rg);      // :1439-1465 (high-order extrapolation)
    const double mxg = -1.0 * mx1 / r1 * rg;        // sign_trans
    const double myg = 1.0 * my1 / r1 * rg;         // sign_normal
    NBC_ST(&u[(size_t)1 * f.pitch + x], rg);
    NBC_ST(&u[(size_t)0 * f.pitch + x], rg2);
    NBC_ST(&u[f.plane + (size_t)1 * f.pitch + x], mxg);
    NBC_ST(&u[2 * f.plane + (size_t)1 * f.pitch + x], myg);
    // south corners of a mirror side (reflection_x of these ghost cells,
    // bc_operators_reflection_x_class.f:236-286; after S in the order)
    int cx = -1;
    if (x < 2 * BC && !a.open_w) cx = 2 * BC - 1 - x;
    else if (x >= nx - 2 * BC && !a.open_e) cx = 2 * nx - 2 * BC - 1 - x;
    if (cx >= 0) {
      NBC_ST(&u[(size_t)1 * f.pitch + cx], pre_x[0] * rg);
      NBC_ST(&u[(size_t)0 * f.pitch + cx], pre_x[0] * rg2);
      NBC_ST(&u[f.plane + (size_t)1 * f.pitch + cx], pre_x[1] * mxg);
      NBC_ST(&u[2 * f.plane + (size_t)1 * f.pitch + cx], pre_x[2] * myg);
    }
    return;
  }
  m -= L.n_s;
  {
    const int nc = BC * BC;
    int k = m / nc;  // k-th corner with node work
    const int r = m % nc;
    int c = 0;
    for (; c < 4; c++)
      if (L.corners >> c & 1) {
        if (k == 0) break;
        k--;
      }
    if (c == 4) return;
    const bool east = c & 1, north = c >> 1;
    const int x = (east ? nx - BC : 0) + r % BC;
    const int y = (north ? ny - BC : 0) + r / BC;
    const int sx = mirror_lo_hi(x, nx);
    if (north && a.open_n) {
      // reflection_x of the open N ghost rows (half_wall_S_open's NW corner,
      // last in its order): pre_x * u(mirror x, y)
      for (int v = 0; v < 4; v++)
        NBC_ST(&u[(size_t)v * f.plane + (size_t)y * f.pitch + x], pre_x[v] * ld(u, f, v, sx, y));
      return;
    }
    // mirror corners from the interior: pre_x * pre_y * u(mirror x, mirror y)
    const int sy = mirror_lo_hi(y, ny);
    for (int v = 0; v < 4; v++)
      NBC_ST(&u[(size_t)v * f.plane + (size_t)y * f.pitch + x], pre_x[v] * pre_y[v] * ld(u, f, v, sx, sy));
  }
}

}  // namespace dim2d
