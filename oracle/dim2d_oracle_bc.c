/*
 * dim2d_oracle_bc.c -- generic boundary-condition dispatcher of the
 * reference (bc_operators_gen_class.f) and the open (Hedstrom) boundary.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dim2d_oracle_internal.h"

/* operator-set ids of orc_sd_set() */
enum { SD_INT = 0, SD_X_L0 = 1, SD_X_L1 = 2, SD_X_R1 = 3, SD_X_R0 = 4,
       SD_Y_L0 = 5, SD_Y_L1 = 6, SD_Y_R1 = 7, SD_Y_R0 = 8 };

static int side_of_section(int section) {
  switch (section) {
    case ORC_N_EDGE: return ORC_N;
    case ORC_S_EDGE: return ORC_S;
    case ORC_E_EDGE: return ORC_E;
    case ORC_W_EDGE: return ORC_W;
    case ORC_NE_CORNER: return ORC_NE;
    case ORC_NW_CORNER: return ORC_NW;
    case ORC_SE_CORNER: return ORC_SE;
    case ORC_SW_CORNER: return ORC_SW;
  }
  return -1;
}

/* ------------------------------------------------------------------ */
/* characteristic algebra: src/physical_models/dim2d/ns_vdw2d_prim_module.f */
/* ------------------------------------------------------------------ */
/* :249-320  jac(row,col) */
static void jacobian_cons_to_prim(double md, double ux, double uy, double Pr, double J[4][4]) {
  double dEdrho = 0.5 * (ux * ux + uy * uy) - 6.0 * md -
                  1.0 / 3.0 * P.cv_r * (Pr + 9.0 * (md - 2.0) * md);
  memset(J, 0, 16 * sizeof(double));
  J[0][0] = 1.0;
  J[0][1] = ux;
  J[1][1] = md;
  J[0][2] = uy;
  J[2][2] = md;
  J[0][3] = dEdrho;
  J[1][3] = md * ux;
  J[2][3] = md * uy;
  J[3][3] = P.cv_r * (1.0 - md / 3.0);
}
/* :574-635 (x) and :744-805 (y)  eig(row,col) */
static void left_eigenvectors(int dir_y, double md, double c, double L[4][4]) {
  double q_c = 0.5 * md * c;
  memset(L, 0, 16 * sizeof(double));
  if (!dir_y) {
    L[2][0] = 1.0;
    L[0][1] = 1.0;
    L[3][1] = -1.0 / (c * c);
    L[1][2] = -q_c;
    L[3][2] = 0.5;
    L[1][3] = q_c;
    L[3][3] = 0.5;
  } else {
    L[1][0] = 1.0;
    L[0][1] = 1.0;
    L[3][1] = -1.0 / (c * c);
    L[2][2] = -q_c;
    L[3][2] = 0.5;
    L[2][3] = q_c;
    L[3][3] = 0.5;
  }
}
/* :657-722 (x) and :827-893 (y) */
static void right_eigenvectors(int dir_y, double md, double c, double R[4][4]) {
  double inv_c = 1.0 / (c * c);
  double inv_q_c = 1.0 / (md * c);
  memset(R, 0, 16 * sizeof(double));
  if (!dir_y) {
    R[1][0] = 1.0;
    R[2][0] = inv_c;
    R[3][0] = inv_c;
    R[2][1] = -inv_q_c;
    R[3][1] = inv_q_c;
    R[0][2] = 1.0;
    R[2][3] = 1.0;
    R[3][3] = 1.0;
  } else {
    R[1][0] = 1.0;
    R[2][0] = inv_c;
    R[3][0] = inv_c;
    R[0][1] = 1.0;
    R[2][2] = -inv_q_c;
    R[3][2] = inv_q_c;
    R[2][3] = 1.0;
    R[3][3] = 1.0;
  }
}

/* pmodel_eq_class.f:2142-2195 (obc_eigenqties_bc) */
static void prim_obc_eigenqties(const double q[4], double prim[5]) {
  prim[0] = q[0];
  prim[1] = q[1] / q[0];
  prim[2] = q[2] / q[0];
  prim[3] = orc_classical_pressure_local(q);
  prim[4] = orc_speed_of_sound(q);
}

/* openbc_operators_module.f:97-136 and hedstrom_xy_module.f:561-576 */
static int incoming_wave(double ev, int side_right) { return side_right ? ev <= 0 : ev >= 0; }

/* hedstrom_xy_module.f:445-558 */
static void timedev_with_openbc(const ov *n, int i, int j, int dir_y, gradient_proc grad,
                                double dn, int side_right, const double *obc_prim,
                                double td[4]) {
  double q[4] = {Q(n, i, j, 1), Q(n, i, j, 2), Q(n, i, j, 3), Q(n, i, j, 4)};
  double prim[5];
  if (obc_prim) memcpy(prim, obc_prim, sizeof prim);
  else prim_obc_eigenqties(q, prim);
  double ev[4], L[4][4], R[4][4], J[4][4];
  double un = dir_y ? prim[2] : prim[1];
  ev[0] = un;  /* ns_vdw2d_prim_module.f:504-552 */
  ev[1] = un;
  ev[2] = un - prim[4];
  ev[3] = un + prim[4];
  left_eigenvectors(dir_y, prim[0], prim[4], L);
  right_eigenvectors(dir_y, prim[0], prim[4], R);
  /* pmodel_eq_class.f:3113-3153 */
  double gp[4] = {grad(n, i, j, mass_density, dn), grad(n, i, j, velocity_x, dn),
                  grad(n, i, j, velocity_y, dn), grad(n, i, j, classical_pressure, dn)};
  double amp[4];
  for (int k = 0; k < 4; k++) {
    if (incoming_wave(ev[k], side_right)) {
      amp[k] = 0.0;
    } else {
      double dot = 0.0;
      for (int m = 0; m < 4; m++) dot += L[m][k] * gp[m];
      amp[k] = -ev[k] * dot;
    }
  }
  double tp[4];
  for (int c = 0; c < 4; c++) {
    double s = 0.0;
    for (int k = 0; k < 4; k++) s += amp[k] * R[k][c];
    tp[c] = s;
  }
  jacobian_cons_to_prim(prim[0], prim[1], prim[2], prim[3], J);
  for (int c = 0; c < 4; c++) {
    double s = 0.0;
    for (int m = 0; m < 4; m++) s += tp[m] * J[m][c];
    td[c] = s;
  }
}

void orc_timedev_with_openbc(const double *nodes, int nx, int ny, int i, int j, int dir_y,
                             int oneside_right, double dn, int side_right,
                             const double *obc_prim, double td[4]) {
  ov n = {nx, ny, nodes};
  gradient_proc g;
  if (!dir_y) g = oneside_right ? gradient_x_x_oneside_R0 : gradient_x_x_oneside_L0;
  else g = oneside_right ? gradient_y_y_oneside_R0 : gradient_y_y_oneside_L0;
  timedev_with_openbc(&n, i, j, dir_y, g, dn, side_right, obc_prim, td);
}

/* openbc_operators_module.f:354-372 */
static void add_body_forces(const double q[4], double body[4]) {
  for (int k = 0; k < 4; k++) body[k] = compute_body_forces(q, k + 1);
}

/* pmodel_eq_class.f:1389-1473 / 1506-1595 with the flux strategy
 * obc_edge_flux_capillarity (parameters_input.f:662) */
static void flux_x_oneside(const ov *n, double dx, double dy, int i, int j, const sd_ops *s,
                           double f[4]) {
  f[0] = flux_x_mass_density(n, s, i, j);
  f[1] = flux_x_momentum_x(n, s, i, j, dx, dy);
  f[2] = flux_x_momentum_y(n, s, i, j, dx, dy);
  f[3] = flux_x_total_energy(n, s, i, j, dx, dy);
}
static void flux_y_oneside(const ov *n, double dx, double dy, int i, int j, const sd_ops *s,
                           double f[4]) {
  f[0] = flux_y_mass_density(n, s, i, j);
  f[1] = flux_y_momentum_x(n, s, i, j, dx, dy);
  f[2] = flux_y_momentum_y(n, s, i, j, dx, dy);
  f[3] = flux_y_total_energy(n, s, i, j, dx, dy);
}

static int is_flux_type(int t) { return t == ORC_BC_FLUXES || t == ORC_BC_FLUX_AND_NODE; }

/* bc_operators_openbc_class.f:437-551 (fixed domain, no bf_alignment) */
static void check_x_flux_interactions(const orc_cfg *c, int *i_min, int *i_max, int right) {
  if (!right) {
    if (is_flux_type(c->bc_type[ORC_SW])) *i_min += 1;
    if (is_flux_type(c->bc_type[ORC_SE])) *i_max -= 1;
  } else {
    if (is_flux_type(c->bc_type[ORC_NW])) *i_min += 1;
    if (is_flux_type(c->bc_type[ORC_NE])) *i_max -= 1;
  }
}
static void check_y_flux_interactions(const orc_cfg *c, int *j_min, int *j_max, int right) {
  if (!right) {
    if (is_flux_type(c->bc_type[ORC_SW])) *j_min += 1;
    if (is_flux_type(c->bc_type[ORC_NW])) *j_max -= 1;
  } else {
    if (is_flux_type(c->bc_type[ORC_SE])) *j_min += 1;
    if (is_flux_type(c->bc_type[ORC_NE])) *j_max -= 1;
  }
}

/* bc_operators_openbc_normal_class.f:563-713 (edges of a fixed domain:
 * only the i_mid range, the grid-point-combining branches need a buffer
 * layer) */
static void fluxes_x_for_bc_y_edge(const ov *n, double dx, double dy, const sd_ops *s1,
                                   const sd_ops *s2, int i_min, int i_max, int j,
                                   double *flux_x) {
  const int nx = n->nx, ny = n->ny;
  const int i_lim_min = BC_SIZE, i_lim_max = nx - BC_SIZE + 2;
  const int i_mid_min = i_min > i_lim_min + 1 ? i_min : i_lim_min + 1;
  const int i_mid_max = i_max < i_lim_max - 1 ? i_max : i_lim_max - 1;
  double f[4];
  for (int i = i_mid_min; i <= i_mid_max; i++) {
    flux_x_oneside(n, dx, dy, i, j, s1, f);
    for (int k = 0; k < 4; k++) FX(flux_x, nx, ny, i, j, k + 1) = f[k];
  }
  for (int i = i_mid_min; i <= i_mid_max; i++) {
    flux_x_oneside(n, dx, dy, i, j + 1, s2, f);
    for (int k = 0; k < 4; k++) FX(flux_x, nx, ny, i, j + 1, k + 1) = f[k];
  }
}
/* bc_operators_openbc_normal_class.f:344-511 */
static void fluxes_y_for_bc_x_edge(const ov *n, double dx, double dy, const sd_ops *s1,
                                   const sd_ops *s2, int i, int j_min, int j_max,
                                   double *flux_y) {
  const int nx = n->nx, ny = n->ny;
  const int j_lim_min = BC_SIZE, j_lim_max = ny - BC_SIZE + 2;
  const int j_mid_min = j_min > j_lim_min + 1 ? j_min : j_lim_min + 1;
  const int j_mid_max = j_max < j_lim_max - 1 ? j_max : j_lim_max - 1;
  double f[4];
  for (int j = j_mid_min; j <= j_mid_max; j++) {
    flux_y_oneside(n, dx, dy, i, j, s1, f);
    for (int k = 0; k < 4; k++) FY(flux_y, nx, ny, i, j, k + 1) = f[k];
    flux_y_oneside(n, dx, dy, i + 1, j, s2, f);
    for (int k = 0; k < 4; k++) FY(flux_y, nx, ny, i + 1, j, k + 1) = f[k];
  }
}

/* hedstrom_xy_module.f:262-305 */
static void timedev_y_edge_local(const ov *n, int i, int j, const double *flux_x, double dx,
                                 double dy, int right, double td[4]) {
  const int nx = n->nx, ny = n->ny;
  double ob[4], body[4];
  double q[4] = {Q(n, i, j, 1), Q(n, i, j, 2), Q(n, i, j, 3), Q(n, i, j, 4)};
  timedev_with_openbc(n, i, j, 1, right ? gradient_y_y_oneside_R0 : gradient_y_y_oneside_L0, dy,
                      right, NULL, ob);
  add_body_forces(q, body);
  for (int k = 0; k < 4; k++)
    td[k] = 1.0 / dx * (FX(flux_x, nx, ny, i, j, k + 1) - FX(flux_x, nx, ny, i + 1, j, k + 1)) +
            ob[k] + body[k];
}
/* hedstrom_xy_module.f:175-218 */
static void timedev_x_edge_local(const ov *n, int i, int j, const double *flux_y, double dx,
                                 double dy, int right, double td[4]) {
  const int nx = n->nx, ny = n->ny;
  double ob[4], body[4];
  double q[4] = {Q(n, i, j, 1), Q(n, i, j, 2), Q(n, i, j, 3), Q(n, i, j, 4)};
  timedev_with_openbc(n, i, j, 0, right ? gradient_x_x_oneside_R0 : gradient_x_x_oneside_L0, dx,
                      right, NULL, ob);
  add_body_forces(q, body);
  for (int k = 0; k < 4; k++)
    td[k] = ob[k] +
            1.0 / dy * (FY(flux_y, nx, ny, i, j, k + 1) - FY(flux_y, nx, ny, i, j + 1, k + 1)) +
            body[k];
}
/* hedstrom_xy_module.f:349-400 */
static void timedev_corner_local(const ov *n, int i, int j, double dx, double dy, int right_x,
                                 int right_y, double td[4]) {
  double ox[4], oy[4], body[4];
  double q[4] = {Q(n, i, j, 1), Q(n, i, j, 2), Q(n, i, j, 3), Q(n, i, j, 4)};
  timedev_with_openbc(n, i, j, 0, right_x ? gradient_x_x_oneside_R0 : gradient_x_x_oneside_L0,
                      dx, right_x, NULL, ox);
  timedev_with_openbc(n, i, j, 1, right_y ? gradient_y_y_oneside_R0 : gradient_y_y_oneside_L0,
                      dy, right_y, NULL, oy);
  add_body_forces(q, body);
  for (int k = 0; k < 4; k++) td[k] = ox[k] + oy[k] + body[k];
}

/* bc_operators_hedstrom_xy_class.f:182-496 (apply_bc_on_timedev_2ndorder) */
static void hedstrom_apply_on_timedev(const orc_cfg *c, int section, const ov *n, double dx,
                                      double dy, double *flux_x, double *flux_y,
                                      double *time_dev) {
  const int nx = c->nx, ny = c->ny;
  double td[4];
  int i, j, i_min, i_max, j_min, j_max;
  switch (section) {
    case ORC_N_EDGE:
      j = ny - BC_SIZE + 1;
      i_min = BC_SIZE + 1;
      i_max = nx - BC_SIZE + 1;
      check_x_flux_interactions(c, &i_min, &i_max, 1);
      fluxes_x_for_bc_y_edge(n, dx, dy, orc_sd_set(SD_Y_R1), orc_sd_set(SD_Y_R0), i_min, i_max,
                             j, flux_x);
      for (j = ny - BC_SIZE + 1; j <= ny; j++)
        for (i = BC_SIZE + 1; i <= nx - BC_SIZE; i++) {
          timedev_y_edge_local(n, i, j, flux_x, dx, dy, 1, td);
          for (int k = 0; k < 4; k++) TD(time_dev, nx, ny, i, j, k + 1) = td[k];
        }
      break;
    case ORC_S_EDGE:
      j = 1;
      i_min = BC_SIZE + 1;
      i_max = nx - BC_SIZE + 1;
      check_x_flux_interactions(c, &i_min, &i_max, 0);
      fluxes_x_for_bc_y_edge(n, dx, dy, orc_sd_set(SD_Y_L0), orc_sd_set(SD_Y_L1), i_min, i_max,
                             j, flux_x);
      for (j = 1; j <= BC_SIZE; j++)
        for (i = BC_SIZE + 1; i <= nx - BC_SIZE; i++) {
          timedev_y_edge_local(n, i, j, flux_x, dx, dy, 0, td);
          for (int k = 0; k < 4; k++) TD(time_dev, nx, ny, i, j, k + 1) = td[k];
        }
      break;
    case ORC_E_EDGE:
      i = nx - BC_SIZE + 1;
      j_min = BC_SIZE + 1;
      j_max = ny - BC_SIZE + 1;
      check_y_flux_interactions(c, &j_min, &j_max, 1);
      fluxes_y_for_bc_x_edge(n, dx, dy, orc_sd_set(SD_X_R1), orc_sd_set(SD_X_R0), i, j_min, j_max,
                             flux_y);
      for (j = BC_SIZE + 1; j <= ny - BC_SIZE; j++)
        for (i = nx - BC_SIZE + 1; i <= nx; i++) {
          timedev_x_edge_local(n, i, j, flux_y, dx, dy, 1, td);
          for (int k = 0; k < 4; k++) TD(time_dev, nx, ny, i, j, k + 1) = td[k];
        }
      break;
    case ORC_W_EDGE:
      i = 1;
      j_min = BC_SIZE + 1;
      j_max = ny - BC_SIZE + 1;
      check_y_flux_interactions(c, &j_min, &j_max, 0);
      fluxes_y_for_bc_x_edge(n, dx, dy, orc_sd_set(SD_X_L0), orc_sd_set(SD_X_L1), i, j_min, j_max,
                             flux_y);
      for (j = BC_SIZE + 1; j <= ny - BC_SIZE; j++)
        for (i = 1; i <= BC_SIZE; i++) {
          timedev_x_edge_local(n, i, j, flux_y, dx, dy, 0, td);
          for (int k = 0; k < 4; k++) TD(time_dev, nx, ny, i, j, k + 1) = td[k];
        }
      break;
    default: {
      int x0 = (section == ORC_SE_CORNER || section == ORC_NE_CORNER) ? nx - BC_SIZE + 1 : 1;
      int y0 = (section == ORC_NW_CORNER || section == ORC_NE_CORNER) ? ny - BC_SIZE + 1 : 1;
      int rx = x0 != 1, ry = y0 != 1;
      for (j = y0; j <= y0 + BC_SIZE - 1; j++)
        for (i = x0; i <= x0 + BC_SIZE - 1; i++) {
          timedev_corner_local(n, i, j, dx, dy, rx, ry, td);
          for (int k = 0; k < 4; k++) TD(time_dev, nx, ny, i, j, k + 1) = td[k];
        }
    }
  }
}

/* ------------------------------------------------------------------ */
/* dispatcher: src/boundary_conditions/bc_operators_gen_class.f         */
/* ------------------------------------------------------------------ */

/* :238-407: walk bc_order1..8 and apply the node-type operators */
void orc_bc_gen_apply_on_nodes(const orc_cfg *c, double t, const double *x_map,
                               const double *y_map, const double *nodes_tmp, double *nodes) {
  for (int k = 0; k < 8; k++) {
    int s = side_of_section(c->bc_order[k]);
    if (s < 0) continue;
    int type = c->bc_type[s];
    if (type != ORC_BC_NODES && type != ORC_BC_FLUX_AND_NODE) continue;
    switch (c->bc_choice[s]) {
      case ORC_REFLECTION_X:
      case ORC_REFLECTION_Y:
        orc_reflection_apply_on_nodes(c, c->bc_order[k], c->bc_choice[s], nodes);
        break;
      case ORC_WALL:
        orc_wall_apply_on_nodes(c, c->bc_order[k], t, x_map, y_map, nodes_tmp, nodes);
        break;
      default:
        fprintf(stderr, "oracle: bc_choice %d has no node operator\n", c->bc_choice[s]);
        abort();
    }
  }
}

/* :509-601: SW, S, SE, W, E, NW, N, NE */
void orc_bc_apply_on_fluxes(const orc_cfg *c, double t, const double *x_map, const double *y_map,
                            const ov *n, double dx, double dy, double *flux_x, double *flux_y) {
  static const int order[8] = {ORC_SW_CORNER, ORC_S_EDGE, ORC_SE_CORNER, ORC_W_EDGE,
                               ORC_E_EDGE, ORC_NW_CORNER, ORC_N_EDGE, ORC_NE_CORNER};
  for (int k = 0; k < 8; k++) {
    int s = side_of_section(order[k]);
    if (!is_flux_type(c->bc_type[s])) continue;
    if (c->bc_choice[s] != ORC_WALL) {
      fprintf(stderr, "oracle: bc_choice %d has no flux operator\n", c->bc_choice[s]);
      abort();
    }
    orc_wall_apply_on_fluxes(c, order[k], t, x_map, y_map, n, dx, dy, flux_x, flux_y);
  }
}

/* :880-978: SW, S, SE, W, E, NW, N, NE */
void orc_bc_apply_on_timedev(const orc_cfg *c, double t, const double *x_map,
                             const double *y_map, const ov *n, double dx, double dy,
                             double *flux_x, double *flux_y, double *time_dev) {
  static const int order[8] = {ORC_SW_CORNER, ORC_S_EDGE, ORC_SE_CORNER, ORC_W_EDGE,
                               ORC_E_EDGE, ORC_NW_CORNER, ORC_N_EDGE, ORC_NE_CORNER};
  (void)t; (void)x_map; (void)y_map;
  for (int k = 0; k < 8; k++) {
    int s = side_of_section(order[k]);
    if (c->bc_type[s] != ORC_BC_TIMEDEV) continue;
    if (c->bc_choice[s] != ORC_HEDSTROM) {
      fprintf(stderr, "oracle: bc_choice %d has no time-derivative operator\n", c->bc_choice[s]);
      abort();
    }
    hedstrom_apply_on_timedev(c, order[k], n, dx, dy, flux_x, flux_y, time_dev);
  }
}
