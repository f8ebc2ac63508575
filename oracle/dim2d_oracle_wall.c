/*
 * dim2d_oracle_wall.c -- wall (contact-angle equilibrium) boundary.
 * TEST INFRASTRUCTURE ONLY.
 *
 * src/boundary_conditions/wall_xy/bc_operators_wall_xy_class.f:174-930
 * src/boundary_conditions/wall_xy/wall_xy_equilibrium_module.f:249-2461
 * src/boundary_conditions/wall_xy/ridders_method_module.f:112-216
 * src/physical_models/dim2d/dim2d_state_eq_module.f:56-227
 *
 * Deviations, all stated in the reference terms:
 *  - dwallInternalEnergy_dmd (wall_xy_equilibrium_module.f:2238-2270) tests
 *    an uninitialised local `angle` against 90 degrees before setting it;
 *    this restatement always takes the cosine branch (at 90 degrees the
 *    value is ~1e-17 instead of 0).
 *  - the wall surface is uniform (wall_surface_type = uniform_surface) and
 *    the heat source has no stop time and no extra source.
 *  - where the reference stops the program (root not bracketed, Ridders
 *    not converged) the oracle records a status (orc_status) and returns.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "dim2d_oracle_internal.h"

int orc_status_flag = 0;
int orc_status(void) { return orc_status_flag; }
void orc_clear_status(void) { orc_status_flag = 0; }

/* parameters_constant.f: sd operator types used to select gradients */
enum { GT_INTERIOR = 0, GT_L0 = 1, GT_L1 = 2, GT_R1 = 3, GT_R0 = 4 };

/* ---- dim2d_state_eq_module.f (dim2d_lowTemperature = .false.) ---------- */
/* :196-227 */
double orc_md_vapor(double T) { return 1.0 - 1.91 * sqrt(1.0 - T); }
/* :145-176 */
double orc_md_liquid(double T) { return 1.0 + 2.06 * sqrt(1.0 - T); }
/* :56-71 */
static double surface_tension(double T) {
  double s = sqrt(1.0 - T);
  return 2.0 * sqrt(2.0) / (3.0 * sqrt(P.we)) * (9.691686257306483 * (s * s * s));
}

/* ---- wall_xy_equilibrium_module.f --------------------------------------- */
/* :1645-1707 (no stop time) */
static double get_heat_flux(double t, double x, double y) {
  (void)t; (void)y;
  switch (P.wall_heat_source_choice) {
    case 0: return 0.0;                      /* no_heat_source */
    case 1: return P.wall_maximum_heat_flux; /* constant_heat_source */
    default: {                               /* gaussian_heat_source */
      double z = (x - P.wall_heat_source_center) / P.wall_heat_source_variance;
      return P.wall_maximum_heat_flux * exp(-0.5 * (z * z));
    }
  }
}
/* :1552-1569 */
double orc_wall_heat_flux(double t, double x, double y) { return get_heat_flux(t, x, y); }
/* :1486-1528 (uniform surface) */
static double get_wall_micro_contact_angle(double x, double y) {
  (void)x; (void)y;
  return P.wall_micro_contact_angle;
}
/* :1439-1465 (wall_md_ghost_cell2_choice = wall_dmddx_high_order) */
static double get_wall_md_extra_ghost_cell(double m1, double m2, double m3) {
  return m1 + 3.0 * (-m2 + m3);
}
/* :2238-2270 (cosine branch, see header) */
double orc_dwall_internal_energy_dmd(double md, double T, double micro_angle) {
  double md_vap = orc_md_vapor(T);
  double md_liq = orc_md_liquid(T);
  double st = surface_tension(T);
  double angle = micro_angle * acos(-1.0) / 180.0;
  double d = md_liq - md_vap;
  return 6.0 * (md - md_liq) * (md - md_vap) / (d * d * d) * st * cos(angle);
}
/* :2295-2315 */
double orc_temperature_average(double T0, double delta_x, double q) {
  return T0 + 0.5 * delta_x * P.re * P.pr * 3.0 / (8.0 * P.cv_r) * q;
}
/* :2337-2351 */
static double md_average(double a, double b) { return 0.5 * (a + b); }
/* :2382-2407 */
double orc_wall_temperature(double md, double g2, double vx, double vy, double Ed) {
  return 3.0 / (8.0 * P.cv_r) *
         (Ed / md - 0.5 * (vx * vx + vy * vy) - 0.5 / P.we * g2 / md + 3.0 * md);
}
/* :2433-2461 */
double orc_dmddx(double delta, const double tab[3], int grad_type) {
  switch (grad_type) {
    case GT_L0: return (tab[2] - tab[1]) / delta;
    case GT_R0: return (tab[1] - tab[0]) / delta;
    default: return (tab[2] - tab[0]) / (2.0 * delta);
  }
}
/* :2151-2212 */
double orc_wall_equilibrium_root_fct(double md, const double md_x[2], const double md_y[2],
                                     double vx, double vy, double Ed, double delta_x,
                                     double delta_y, double micro_angle, double q,
                                     int grad_type_x, int grad_type_y) {
  double dmddx_half = (-md + md_x[1]) / (delta_x);
  double md_av = md_average(md, md_x[1]);
  double tx[3] = {md_x[0], md, md_x[1]};
  double ty[3] = {md_y[0], md, md_y[1]};
  double gx = orc_dmddx(delta_x, tx, grad_type_x);
  double gy = orc_dmddx(delta_y, ty, grad_type_y);
  double g2 = gx * gx + gy * gy;
  double T1 = orc_wall_temperature(md, g2, vx, vy, Ed);
  double Tav = orc_temperature_average(T1, delta_x, q);
  return 1.0 / P.we * dmddx_half + orc_dwall_internal_energy_dmd(md_av, Tav, micro_angle);
}

/* wall_x_root_fct (:2016-2103): f(x) = root_fct(md_x(2), [md_x(1), x], ...) */
typedef struct {
  double md_x[2], md_y[2], vx, vy, Ed, delta_x, delta_y, angle, q;
  int gtx, gty;
} root_ctx;
static double root_f(const root_ctx *c, double x) {
  double mx[2] = {c->md_x[0], x};
  return orc_wall_equilibrium_root_fct(c->md_x[1], mx, c->md_y, c->vx, c->vy, c->Ed, c->delta_x,
                                       c->delta_y, c->angle, c->q, c->gtx, c->gty);
}

/* check_data_module.f:28-46 */
static int is_validated(double a, double b) { return fabs(a - b) < 1e-10; }
/* :1962-1972 */
static int have_same_sign(double a, double b) {
  return copysign(1.0, a) * copysign(1.0, b) > 0;
}

/* :1846-1941; returns 0 on success, 1 when no bracket is found */
static int root_brackets(const root_ctx *c, double T_guess, double md_guess, double br[2]) {
  const int MAXIT = 99;
  double xl = orc_md_vapor(T_guess);
  double xh = orc_md_liquid(T_guess);
  double fl = root_f(c, xl);
  double fh = root_f(c, xh);
  if (have_same_sign(fl, fh)) {
    double dmd_l = (md_guess) / (double)(float)(MAXIT + 1);
    double dmd_r = (3.0 - md_guess) / (double)(float)(MAXIT + 1);
    double fmd = root_f(c, md_guess);
    for (int j = 1; j <= MAXIT; j++) {
      xl = md_guess - j * dmd_l;
      xh = md_guess + j * dmd_r;
      fl = root_f(c, xl);
      fh = root_f(c, xh);
      if (!have_same_sign(fl, fmd)) {
        br[0] = xl;
        br[1] = md_guess;
        return 0;
      } else if (!have_same_sign(fh, fmd)) {
        br[0] = md_guess;
        br[1] = xh;
        return 0;
      }
    }
    return 1;
  }
  br[0] = xl;
  br[1] = xh;
  return 0;
}

/* ridders_method_module.f:112-216; status 0 ok, 2 not bracketed, 3 no
 * convergence, 4 bracketing error */
static double ridders(const root_ctx *c, double x1, double x2, double xacc, int *status) {
  const int MAXIT = 60;
  const double UNUSED = (double)(float)-1.11e30;
  double fl = root_f(c, x1), fh = root_f(c, x2);
  double x = UNUSED;
  *status = 0;
  if ((fl > 0.0 && fh < 0.0) || (fl < 0.0 && fh > 0.0)) {
    double xl = x1, xh = x2;
    for (int j = 1; j <= MAXIT; j++) {
      double xm = 0.5 * (xl + xh);
      double fm = root_f(c, xm);
      double s = sqrt(fm * fm - fl * fh);
      if (is_validated(s, 0.0)) return x;
      double xnew = xm + (xm - xl) * (copysign(1.0, fl - fh) * fm / s);
      if (fabs(xnew - x) <= xacc) return x;
      x = xnew;
      double fnew = root_f(c, x);
      if (is_validated(fnew, 0.0)) return x;
      if (!is_validated(copysign(fm, fnew), fm)) {
        xl = xm;
        fl = fm;
        xh = x;
        fh = fnew;
      } else if (!is_validated(copysign(fl, fnew), fl)) {
        xh = x;
        fh = fnew;
      } else if (!is_validated(copysign(fh, fnew), fh)) {
        xl = x;
        fl = fnew;
      } else {
        *status = 4;
        return x;
      }
      if (fabs(xh - xl) <= xacc) return x;
    }
    *status = 3;
    return x;
  } else if (is_validated(fl, 0.0)) {
    return x1;
  } else if (is_validated(fh, 0.0)) {
    return x2;
  }
  *status = 2;
  return x;
}

/* :1747-1821 */
static double get_wall_x_md_ghost_cell(double T_guess, double md_guess, const double md_x[2],
                                       const double md_y[2], double vx, double vy, double Ed,
                                       double delta_x, double delta_y, double angle, double q,
                                       int gtx, int gty) {
  root_ctx c = {{md_x[0], md_x[1]}, {md_y[0], md_y[1]}, vx, vy, Ed, delta_x, delta_y, angle,
                q, gtx, gty};
  double br[2];
  if (root_brackets(&c, T_guess, md_guess, br)) {
    orc_status_flag = 1;
    return NAN;
  }
  int st = 0;
  double md = ridders(&c, br[0], br[1], 1.0 * 1e-12, &st);
  if (st) orc_status_flag = st;
  return md;
}

/* bc_operators_wall_xy_class.f:898-930 */
static void wall_xy_guess(const ov *tmp, int ti, int tj, int mi, int mj, double dx, double dy,
                          gradient_proc gx, gradient_proc gy, double *T_guess,
                          double *md_guess) {
  *T_guess = 3.0 / (8.0 * P.cv_r) * temperature_eff(tmp, ti, tj, dx, dy, gx, gy);
  *md_guess = Q(tmp, mi, mj, 1);
}

#define NO(i, j, k) TD(nodes, nx, ny, i, j, k)

/* :948-1040, 1080-1171, 1211-1304, 1344-1436.  side: 'S','N','W','E' */
static void compute_wall_ghost_cell(const orc_cfg *cf, char side, int i, int j, double t,
                                    const double *x_map, const double *y_map, double *nodes,
                                    double T_guess, double md_guess, int grad_type) {
  const int nx = cf->nx, ny = cf->ny;
  const double dbg = orc_debug_real();
  double md_x[2], md_y[2], vx, vy, Ed, delta_x, delta_y;
  int ii = i, jj = j;  /* first interior node */
  int di = 0, dj = 0;  /* step from the ghost towards the interior */
  switch (side) {
    case 'S': dj = 1; break;
    case 'N': dj = -1; break;
    case 'W': di = 1; break;
    default: di = -1; break;
  }
  ii = i + di;
  jj = j + dj;
  md_x[0] = NO(i + 2 * di, j + 2 * dj, 1);
  md_x[1] = NO(ii, jj, 1);
  if (side == 'S' || side == 'N') {
    switch (grad_type) {
      case GT_L0: md_y[0] = dbg; md_y[1] = NO(i + 1, jj, 1); break;
      case GT_R0: md_y[0] = NO(i - 1, jj, 1); md_y[1] = dbg; break;
      default: md_y[0] = NO(i - 1, jj, 1); md_y[1] = NO(i + 1, jj, 1);
    }
    vx = (side == 'S' ? -1.0 : 1.0) * NO(ii, jj, 3) / NO(ii, jj, 1);
    vy = NO(ii, jj, 2) / NO(ii, jj, 1);
    delta_x = y_map[1] - y_map[0];
    delta_y = x_map[1] - x_map[0];
  } else {
    switch (grad_type) {
      case GT_L0: md_y[0] = dbg; md_y[1] = NO(ii, j + 1, 1); break;
      case GT_R0: md_y[0] = NO(ii, j - 1, 1); md_y[1] = dbg; break;
      default: md_y[0] = NO(ii, j - 1, 1); md_y[1] = NO(ii, j + 1, 1);
    }
    vx = (side == 'W' ? -1.0 : 1.0) * NO(ii, jj, 2) / NO(ii, jj, 1);
    vy = NO(ii, jj, 3) / NO(ii, jj, 1);
    delta_x = x_map[1] - x_map[0];
    delta_y = y_map[1] - y_map[0];
  }
  Ed = NO(ii, jj, 4);
  double angle = get_wall_micro_contact_angle(x_map[i - 1], y_map[j - 1]);
  double q = get_heat_flux(t, x_map[i - 1], y_map[j - 1]);
  NO(i, j, 1) = get_wall_x_md_ghost_cell(T_guess, md_guess, md_x, md_y, vx, vy, Ed, delta_x,
                                         delta_y, angle, q, GT_INTERIOR, grad_type);
  NO(i - di, j - dj, 1) =
      get_wall_md_extra_ghost_cell(NO(i + 2 * di, j + 2 * dj, 1), NO(ii, jj, 1), NO(i, j, 1));
  const double sign_normal = 1.0, sign_trans = -1.0;
  if (side == 'S' || side == 'N') {
    NO(i, j, 2) = sign_trans * NO(ii, jj, 2) / NO(ii, jj, 1) * NO(i, j, 1);
    NO(i, j, 3) = sign_normal * NO(ii, jj, 3) / NO(ii, jj, 1) * NO(i, j, 1);
  } else {
    NO(i, j, 2) = sign_normal * NO(ii, jj, 2) / NO(ii, jj, 1) * NO(i, j, 1);
    NO(i, j, 3) = sign_trans * NO(ii, jj, 3) / NO(ii, jj, 1) * NO(i, j, 1);
  }
}

/* bc_operators_wall_xy_class.f:232-605 */
void orc_wall_apply_on_nodes(const orc_cfg *c, int section, double t, const double *x_map,
                             const double *y_map, const double *nodes_tmp, double *nodes) {
  const int nx = c->nx, ny = c->ny;
  ov tmp = {nx, ny, nodes_tmp};
  const double dx = x_map[1] - x_map[0], dy = y_map[1] - y_map[0];
  int sec[4];
  orc_section(c, section, sec);
  double Tg, mg;
  int i, j;
  switch (section) {
    case ORC_N_EDGE:
      j = sec[2];
      for (i = sec[1]; i <= sec[3]; i++) {
        wall_xy_guess(&tmp, i, j - 1, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                      &mg);
        compute_wall_ghost_cell(c, 'N', i, j, t, x_map, y_map, nodes, Tg, mg, GT_INTERIOR);
      }
      break;
    case ORC_S_EDGE:
      j = sec[2] + BC_SIZE - 1;
      for (i = sec[1]; i <= sec[3]; i++) {
        wall_xy_guess(&tmp, i, j + 1, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                      &mg);
        compute_wall_ghost_cell(c, 'S', i, j, t, x_map, y_map, nodes, Tg, mg, GT_INTERIOR);
      }
      break;
    case ORC_E_EDGE:
      i = sec[1];
      for (j = sec[2]; j <= sec[3]; j++) {
        wall_xy_guess(&tmp, i - 1, j, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                      &mg);
        compute_wall_ghost_cell(c, 'E', i, j, t, x_map, y_map, nodes, Tg, mg, GT_INTERIOR);
      }
      break;
    case ORC_W_EDGE:
      i = sec[1] + BC_SIZE - 1;
      for (j = sec[2]; j <= sec[3]; j++) {
        wall_xy_guess(&tmp, i + 1, j, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                      &mg);
        compute_wall_ghost_cell(c, 'W', i, j, t, x_map, y_map, nodes, Tg, mg, GT_INTERIOR);
      }
      break;
    case ORC_SW_CORNER:
      j = sec[2] + BC_SIZE - 1;
      i = sec[1];
      wall_xy_guess(&tmp, i, j + 1, i, j, dx, dy, gradient_x_x_oneside_L0, gradient_y_interior,
                    &Tg, &mg);
      compute_wall_ghost_cell(c, 'S', i, j, t, x_map, y_map, nodes, Tg, mg, GT_L0);
      i = sec[1] + 1;
      wall_xy_guess(&tmp, i, j + 1, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                    &mg);
      compute_wall_ghost_cell(c, 'S', i, j, t, x_map, y_map, nodes, Tg, mg, GT_L1);
      break;
    case ORC_SE_CORNER:
      j = sec[2] + BC_SIZE - 1;
      i = sec[1];
      wall_xy_guess(&tmp, i, j + 1, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                    &mg);
      compute_wall_ghost_cell(c, 'S', i, j, t, x_map, y_map, nodes, Tg, mg, GT_R1);
      i = sec[1] + 1;
      wall_xy_guess(&tmp, i, j + 1, i, j, dx, dy, gradient_x_x_oneside_R0, gradient_y_interior,
                    &Tg, &mg);
      compute_wall_ghost_cell(c, 'S', i, j, t, x_map, y_map, nodes, Tg, mg, GT_R0);
      break;
    case ORC_NW_CORNER:
      j = sec[2];
      i = sec[1];
      wall_xy_guess(&tmp, i, j - 1, i, j, dx, dy, gradient_x_x_oneside_L0, gradient_y_interior,
                    &Tg, &mg);
      compute_wall_ghost_cell(c, 'N', i, j, t, x_map, y_map, nodes, Tg, mg, GT_L0);
      i = sec[1] + 1;
      wall_xy_guess(&tmp, i, j - 1, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                    &mg);
      compute_wall_ghost_cell(c, 'N', i, j, t, x_map, y_map, nodes, Tg, mg, GT_L1);
      break;
    default: /* NE */
      j = sec[2];
      i = sec[1];
      wall_xy_guess(&tmp, i, j - 1, i, j, dx, dy, gradient_x_interior, gradient_y_interior, &Tg,
                    &mg);
      compute_wall_ghost_cell(c, 'N', i, j, t, x_map, y_map, nodes, Tg, mg, GT_R1);
      i = sec[1] + 1;
      wall_xy_guess(&tmp, i, j - 1, i, j, dx, dy, gradient_x_x_oneside_R0, gradient_y_interior,
                    &Tg, &mg);
      compute_wall_ghost_cell(c, 'N', i, j, t, x_map, y_map, nodes, Tg, mg, GT_R0);
  }
}

/* :445-506 (side_right = East) */
static double wall_flux_x_inviscid_momentum_x(double t, const double *x_map, const double *y_map,
                                              const ov *n, double dx, double dy, int i, int j,
                                              int side_right, gradient_proc gy) {
  double Tl;
  if (!side_right)
    Tl = 3.0 / (8.0 * P.cv_r) * temperature_eff(n, i, j, dx, dy, gradient_x_interior, gy);
  else
    Tl = 3.0 / (8.0 * P.cv_r) * temperature_eff(n, i - 1, j, dx, dy, gradient_x_interior, gy);
  double Th = Tl + dx * 3.0 / (8.0 * P.cv_r) * P.re * P.pr *
                       get_heat_flux(t, x_map[i - 1], y_map[j - 1]);
  double T_half = 0.5 * (Tl + Th);
  double md_half = 0.5 * (Q(n, i - 1, j, 1) + Q(n, i, j, 1));
  return vdw_pressure(T_half, md_half);
}
/* :794-854 (side_right = North) */
static double wall_flux_y_inviscid_momentum_y(double t, const double *x_map, const double *y_map,
                                              const ov *n, double dx, double dy, int i, int j,
                                              int side_right, gradient_proc gx) {
  double Tl;
  if (!side_right)
    Tl = 3.0 / (8.0 * P.cv_r) * temperature_eff(n, i, j, dx, dy, gx, gradient_y_interior);
  else
    Tl = 3.0 / (8.0 * P.cv_r) * temperature_eff(n, i, j - 1, dx, dy, gx, gradient_y_interior);
  double Th = Tl + dy * P.re * P.pr * (3.0 / (8.0 * P.cv_r)) *
                       get_heat_flux(t, x_map[i - 1], y_map[j - 1]);
  double T_half = 0.5 * (Tl + Th);
  double md_half = 0.5 * (Q(n, i, j - 1, 1) + Q(n, i, j, 1));
  return vdw_pressure(T_half, md_half);
}

/* :249-306 */
void orc_compute_wall_flux_x(const ov *n, const sd_ops *s, int i, int j, double t,
                             const double *x_map, const double *y_map, int side_right,
                             gradient_proc gy, double f[4]) {
  const double dx = x_map[1] - x_map[0], dy = y_map[1] - y_map[0];
  double a = s->dfdx(n, i, j, mass_density, dx), b = s->dfdy(n, i, j, mass_density, dy);
  /* :540-562 */
  double cap_x = s->f(n, i, j, mass_density) *
                     (s->d2fdx2(n, i, j, mass_density, dx) + s->d2fdy2(n, i, j, mass_density, dy)) +
                 0.5 * (-(a * a) + (b * b));
  f[0] = 0.0;
  f[1] = wall_flux_x_inviscid_momentum_x(t, x_map, y_map, n, dx, dy, i, j, side_right, gy) -
         1.0 / P.we * cap_x;
  /* :596-610 and :644-661 */
  f[2] = -1.0 / P.re * s->dfdx(n, i, j, velocity_y, dx) -
         1.0 / P.we * (-s->dfdx(n, i, j, mass_density, dx) * s->dfdy(n, i, j, mass_density, dy));
  f[3] = get_heat_flux(t, x_map[i - 1], y_map[j - 1]);
  if (side_right) f[3] = -f[3];
}
/* :342-402 */
void orc_compute_wall_flux_y(const ov *n, const sd_ops *s, int i, int j, double t,
                             const double *x_map, const double *y_map, int side_right,
                             gradient_proc gx, double f[4]) {
  const double dx = x_map[1] - x_map[0], dy = y_map[1] - y_map[0];
  double a = s->dgdx(n, i, j, mass_density, dx), b = s->dgdy(n, i, j, mass_density, dy);
  f[0] = 0.0;
  /* :695-709 and :743-760 */
  f[1] = -1.0 / P.re * s->dgdy(n, i, j, velocity_x, dy) -
         1.0 / P.we * (-s->dgdx(n, i, j, mass_density, dx) * s->dgdy(n, i, j, mass_density, dy));
  /* :888-908 */
  double cap_y = s->g(n, i, j, mass_density) *
                     (s->d2gdx2(n, i, j, mass_density, dx) + s->d2gdy2(n, i, j, mass_density, dy)) +
                 0.5 * ((a * a) - (b * b));
  f[2] = wall_flux_y_inviscid_momentum_y(t, x_map, y_map, n, dx, dy, i, j, side_right, gx) -
         1.0 / P.we * cap_y;
  f[3] = get_heat_flux(t, x_map[i - 1], y_map[j - 1]);
  if (side_right) f[3] = -f[3];
}

/* bc_operators_wall_xy_class.f:702-854 */
void orc_wall_apply_on_fluxes(const orc_cfg *c, int section, double t, const double *x_map,
                              const double *y_map, const ov *n, double dx, double dy,
                              double *flux_x, double *flux_y) {
  const int nx = c->nx, ny = c->ny;
  const sd_ops *s = orc_sd_set(0);
  int sec[4];
  orc_section(c, section, sec);
  double f[4];
  int i, j;
  (void)dx; (void)dy;
#define SETY(ii, jj) for (int k = 0; k < 4; k++) FY(flux_y, nx, ny, ii, jj, k + 1) = f[k]
#define SETX(ii, jj) for (int k = 0; k < 4; k++) FX(flux_x, nx, ny, ii, jj, k + 1) = f[k]
  switch (section) {
    case ORC_N_EDGE:
      j = sec[2];
      for (i = sec[1]; i <= sec[3]; i++) {
        orc_compute_wall_flux_y(n, s, i, j, t, x_map, y_map, 1, gradient_x_interior, f);
        SETY(i, j);
      }
      break;
    case ORC_S_EDGE:
      j = sec[2] + BC_SIZE;
      for (i = sec[1]; i <= sec[3]; i++) {
        orc_compute_wall_flux_y(n, s, i, j, t, x_map, y_map, 0, gradient_x_interior, f);
        SETY(i, j);
      }
      break;
    case ORC_E_EDGE:
      i = sec[1];
      for (j = sec[2]; j <= sec[3]; j++) {
        orc_compute_wall_flux_x(n, s, i, j, t, x_map, y_map, 1, gradient_y_interior, f);
        SETX(i, j);
      }
      break;
    case ORC_W_EDGE:
      i = sec[1] + BC_SIZE;
      for (j = sec[2]; j <= sec[3]; j++) {
        orc_compute_wall_flux_x(n, s, i, j, t, x_map, y_map, 0, gradient_y_interior, f);
        SETX(i, j);
      }
      break;
    case ORC_SW_CORNER:
      j = sec[2] + BC_SIZE;
      i = sec[1];
      orc_compute_wall_flux_y(n, orc_sd_set(1), i, j, t, x_map, y_map, 0, gradient_x_x_oneside_L0, f);
      SETY(i, j);
      i = sec[1] + 1;
      orc_compute_wall_flux_y(n, orc_sd_set(2), i, j, t, x_map, y_map, 0, gradient_x_interior, f);
      SETY(i, j);
      break;
    case ORC_SE_CORNER:
      j = sec[2] + BC_SIZE;
      i = sec[1];
      orc_compute_wall_flux_y(n, orc_sd_set(3), i, j, t, x_map, y_map, 0, gradient_x_interior, f);
      SETY(i, j);
      i = sec[1] + 1;
      orc_compute_wall_flux_y(n, orc_sd_set(4), i, j, t, x_map, y_map, 0, gradient_x_x_oneside_R0, f);
      SETY(i, j);
      break;
    case ORC_NW_CORNER:
      j = sec[2];
      i = sec[1];
      orc_compute_wall_flux_y(n, orc_sd_set(1), i, j, t, x_map, y_map, 1, gradient_x_x_oneside_L0, f);
      SETY(i, j);
      i = sec[1] + 1;
      orc_compute_wall_flux_y(n, orc_sd_set(2), i, j, t, x_map, y_map, 1, gradient_x_interior, f);
      SETY(i, j);
      break;
    default: /* NE */
      j = sec[2];
      i = sec[1];
      orc_compute_wall_flux_y(n, orc_sd_set(3), i, j, t, x_map, y_map, 1, gradient_x_interior, f);
      SETY(i, j);
      i = sec[1] + 1;
      orc_compute_wall_flux_y(n, orc_sd_set(4), i, j, t, x_map, y_map, 1, gradient_x_x_oneside_R0, f);
      SETY(i, j);
  }
#undef SETX
#undef SETY
}

/* capillarity parts of the wall x-flux at face (i,j): which 0 =
 * flux_x_capillarity_momentum_x (:540-562), 1 = flux_x_capillarity_momentum_y
 * (:644-661) */
double orc_wall_capillarity_x(const double *nodes, int nx, int ny, int i, int j, double dx,
                              double dy, int which) {
  ov n = {nx, ny, nodes};
  const sd_ops *s = orc_sd_set(0);
  if (which == 0) {
    double a = s->dfdx(&n, i, j, mass_density, dx), b = s->dfdy(&n, i, j, mass_density, dy);
    return s->f(&n, i, j, mass_density) *
               (s->d2fdx2(&n, i, j, mass_density, dx) + s->d2fdy2(&n, i, j, mass_density, dy)) +
           0.5 * (-(a * a) + (b * b));
  }
  return -s->dfdx(&n, i, j, mass_density, dx) * s->dfdy(&n, i, j, mass_density, dy);
}

/* unit entry point for the known-answer test of wall_xy_equilibrium_module */
void orc_wall_flux_x_at(const double *nodes, int nx, int ny, int i, int j, double t,
                        const double *x_map, const double *y_map, int side_right, double f[4]) {
  ov n = {nx, ny, nodes};
  orc_compute_wall_flux_x(&n, orc_sd_set(0), i, j, t, x_map, y_map, side_right,
                          gradient_y_interior, f);
}
