/*
 * dim2d_oracle.c -- line-faithful CPU restatement of the reference's DIM
 * time-derivative hot path.  TEST INFRASTRUCTURE ONLY (the checker): the
 * product never links or calls this file.
 *
 * Every function cites the reference file:line it restates (paths relative
 * to the reference project root).  Expression structure follows the Fortran
 * (left-to-right evaluation, x**2 as x*x, same parenthesisation); build with
 * -ffp-contract=off so no FMA contraction changes the rounding order.
 *
 * Parity status: pinned by the reference's own known-answer tests
 * (Mattsson operators, DIM face fluxes, periodic ghost cells); see
 * tests/test_oracle_golden.py.
 */
#include "dim2d_oracle.h"
#include "dim2d_oracle_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* parameters: src/physical_models/dim2d/dim2d_parameters.f:179-199     */
/* (the reference's "for tests" constant set is the default here)      */
/* ------------------------------------------------------------------ */
orc_params P = {
  /* re */ 5.0, /* we */ 10.0, /* pr */ 20.0, /* cv_r */ 2.5,
  /* viscous_r */ -1.5,
  /* gravity_ac */ 0, /* gravity */ 0.0,
  /* wall_micro_contact_angle */ 90.0, /* wall_heat_source_choice */ 0,
  /* wall_maximum_heat_flux */ 0.0, /* center */ 0.0, /* variance */ 1.0,
  /* obc_eigenqties_strategy */ 0, /* obc_edge_flux_strategy */ 0,
  /* T0 */ 0.95, /* flow_velocity */ 0.0
};

void orc_set_params(const orc_params *p) { P = *p; }
void orc_get_params(orc_params *p) { *p = P; }
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* NF90_FILL_DOUBLE, used as debug_real (parameters_input.f:880-892) */
double orc_debug_real(void) { return 9.9692099683868690e+36; }

/* ------------------------------------------------------------------ */
/* primitive variables: src/physical_models/dim2d/dim2d_prim_module.f  */
/* ------------------------------------------------------------------ */
/* :99-110 */
double mass_density(const ov *n, int i, int j) { return Q(n, i, j, 1); }
/* :135-146 */
double momentum_x(const ov *n, int i, int j) { return Q(n, i, j, 2); }
/* :171-182 */
double momentum_y(const ov *n, int i, int j) { return Q(n, i, j, 3); }
/* :206-217 */
double total_energy(const ov *n, int i, int j) { return Q(n, i, j, 4); }
/* :242-253 */
double velocity_x(const ov *n, int i, int j) { return Q(n, i, j, 2) / Q(n, i, j, 1); }
/* :278-289 */
double velocity_y(const ov *n, int i, int j) { return Q(n, i, j, 3) / Q(n, i, j, 1); }

/* :425-453 */
double orc_classical_pressure_local(const double q[4]) {
  return 3.0 / ((3.0 - q[0]) * P.cv_r) *
             (q[3] - 0.5 * q[0] * ((q[1] / q[0]) * (q[1] / q[0]) +
                                   (q[2] / q[0]) * (q[2] / q[0])) +
              3.0 * (q[0] * q[0])) -
         3.0 * (q[0] * q[0]);
}
/* :392-403 */
double classical_pressure(const ov *n, int i, int j) {
  double q[4] = {Q(n, i, j, 1), Q(n, i, j, 2), Q(n, i, j, 3), Q(n, i, j, 4)};
  return orc_classical_pressure_local(q);
}
/* :476-488 */
double vdw_pressure(double temperature, double md) {
  return 8.0 * md * temperature / (3.0 - md) - 3.0 * (md * md);
}
/* :515-544 */
double classical_temperature_eff(const ov *n, int i, int j) {
  double r = Q(n, i, j, 1), ux = Q(n, i, j, 2) / r, uy = Q(n, i, j, 3) / r;
  return 1.0 / r * (Q(n, i, j, 4) - 0.5 * r * (ux * ux + uy * uy) + 3.0 * (r * r));
}
/* :582-613 */
double capillarity_temperature_eff(const ov *n, int i, int j, double dx, double dy,
                                   gradient_proc gx, gradient_proc gy) {
  double a = gx(n, i, j, mass_density, dx);
  double b = gy(n, i, j, mass_density, dy);
  return 0.5 / Q(n, i, j, 1) * (a * a + b * b);
}
/* :652-691 */
double temperature_eff(const ov *n, int i, int j, double dx, double dy,
                       gradient_proc gx, gradient_proc gy) {
  double r = Q(n, i, j, 1), ux = Q(n, i, j, 2) / r, uy = Q(n, i, j, 3) / r;
  double a = gx(n, i, j, mass_density, dx);
  double b = gy(n, i, j, mass_density, dy);
  return 1.0 / r * (Q(n, i, j, 4) - 0.5 * r * (ux * ux + uy * uy) -
                    0.5 / P.we * (a * a + b * b) + 3.0 * (r * r));
}
/* :718-750 */
double classical_pressure_xwork(const ov *n, int i, int j) {
  return classical_pressure(n, i, j) * Q(n, i, j, 2) / Q(n, i, j, 1);
}
/* :777-807 */
double classical_pressure_ywork(const ov *n, int i, int j) {
  return classical_pressure(n, i, j) * Q(n, i, j, 3) / Q(n, i, j, 1);
}
/* :832-843 */
double qx_transport_x(const ov *n, int i, int j) {
  return Q(n, i, j, 2) * Q(n, i, j, 2) / Q(n, i, j, 1);
}
/* :868-881 */
double qy_transport_x(const ov *n, int i, int j) {
  return Q(n, i, j, 3) * Q(n, i, j, 2) / Q(n, i, j, 1);
}
/* :906-919 */
double qx_transport_y(const ov *n, int i, int j) {
  return Q(n, i, j, 2) * Q(n, i, j, 3) / Q(n, i, j, 1);
}
/* :944-955 */
double qy_transport_y(const ov *n, int i, int j) {
  return Q(n, i, j, 3) * Q(n, i, j, 3) / Q(n, i, j, 1);
}
/* :980-993 */
double energy_transport_x(const ov *n, int i, int j) {
  return Q(n, i, j, 4) * Q(n, i, j, 2) / Q(n, i, j, 1);
}
/* :1018-1031 */
double energy_transport_y(const ov *n, int i, int j) {
  return Q(n, i, j, 4) * Q(n, i, j, 3) / Q(n, i, j, 1);
}
/* :1056-1071 */
double capillarity_pressure(const ov *n, int i, int j) {
  return 1.0 / (3.0 - Q(n, i, j, 1));
}
/* :1096-1113 */
double capillarity_pressure_xwork(const ov *n, int i, int j) {
  return Q(n, i, j, 2) / (Q(n, i, j, 1) * (3.0 - Q(n, i, j, 1)));
}
/* :1138-1155 */
double capillarity_pressure_ywork(const ov *n, int i, int j) {
  return Q(n, i, j, 3) / (Q(n, i, j, 1) * (3.0 - Q(n, i, j, 1)));
}
/* :1179-1215 */
double orc_speed_of_sound(const double q[4]) {
  double Pr = orc_classical_pressure_local(q);
  double e = Pr + (q[0] * q[0]) * (-3.0 + 2.0 * q[0]);
  double b = sqrt((Pr + 3.0 * (q[0] * q[0])) / (P.cv_r * e));
  double a = 1.0 / sqrt(1.0 + b * b);
  double d = sqrt(q[0] * q[0] * q[0]) * sqrt((3.0 - q[0]) / e);
  return sqrt(3.0) * q[0] / (a * d);
}

/* ------------------------------------------------------------------ */
/* centred / one-sided gradients:                                      */
/* src/sd_operators/mattsson_operators/sd_operators_fd_module.f        */
/* ------------------------------------------------------------------ */
/* :71-96 */
double gradient_x_interior(const ov *n, int i, int j, primary_proc p, double dn) {
  return 0.5 / dn * (-p(n, i - 1, j) + p(n, i + 1, j));
}
/* :128-153 */
double gradient_y_interior(const ov *n, int i, int j, primary_proc p, double dn) {
  return 0.5 / dn * (-p(n, i, j - 1) + p(n, i, j + 1));
}
/* :182-207 */
double gradient_x_x_oneside_L0(const ov *n, int i, int j, primary_proc p, double dn) {
  return 1.0 / dn * (-p(n, i, j) + p(n, i + 1, j));
}
/* :275-300 */
double gradient_x_x_oneside_R0(const ov *n, int i, int j, primary_proc p, double dn) {
  return 1.0 / dn * (-p(n, i - 1, j) + p(n, i, j));
}
/* :332-357 */
double gradient_y_y_oneside_L0(const ov *n, int i, int j, primary_proc p, double dn) {
  return 1.0 / dn * (-p(n, i, j) + p(n, i, j + 1));
}
/* :425-450 */
double gradient_y_y_oneside_R0(const ov *n, int i, int j, primary_proc p, double dn) {
  return 1.0 / dn * (-p(n, i, j - 1) + p(n, i, j));
}

/* ------------------------------------------------------------------ */
/* Mattsson interior operators:                                        */
/* src/sd_operators/mattsson_operators/sd_operators_class.f            */
/* ------------------------------------------------------------------ */
/* :160-183 */
static double f_mt(const ov *n, int i, int j, primary_proc p) {
  return 0.5 * (+p(n, i - 1, j) + p(n, i, j));
}
/* :214-236 */
static double dfdx_mt(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / dx * (-p(n, i - 1, j) + p(n, i, j));
}
/* :274-298 */
static double dfdx_nl_mt(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx * (-p(n, i - 1, j, dx, dy, gradient_x_interior, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_interior));
}
/* :359-388 */
static double dfdy_mt(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / (2.0 * dy) *
         (-0.5 * p(n, i - 1, j - 1) - 0.5 * p(n, i, j - 1) + 0.5 * p(n, i - 1, j + 1) +
          0.5 * p(n, i, j + 1));
}
/* :421-451 */
static double d2fdx2_mt(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.5 / (dx * dx) * (+p(n, i - 2, j) - p(n, i - 1, j) - p(n, i, j) + p(n, i + 1, j));
}
/* :485-525 */
static double d2fdy2_mt(const ov *n, int i, int j, primary_proc p, double dy) {
  return (1.0 / (dy * dy)) *
         (+0.5 * p(n, i - 1, j - 1) + 0.5 * p(n, i, j - 1) -
          2.0 * (+0.5 * p(n, i - 1, j) + 0.5 * p(n, i, j)) + 0.5 * p(n, i - 1, j + 1) +
          0.5 * p(n, i, j + 1));
}
/* :562-592 */
static double d2fdxdy_mt(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (p(n, i - 1, j - 1) - p(n, i, j - 1) - p(n, i - 1, j + 1) + p(n, i, j + 1)) * 0.5 /
         (dy * dx);
}
/* :622-648 */
static double g_mt(const ov *n, int i, int j, primary_proc p) {
  return 0.5 * (+p(n, i, j - 1) + p(n, i, j));
}
/* :681-712 */
static double dgdx_mt(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.25 / dx *
         (-p(n, i - 1, j - 1) - p(n, i - 1, j) + p(n, i + 1, j - 1) + p(n, i + 1, j));
}
/* :744-771 */
static double dgdy_mt(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / dy * (-p(n, i, j - 1) + p(n, i, j));
}
/* :806-834 */
static double dgdy_nl_mt(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy * (-p(n, i, j - 1, dx, dy, gradient_x_interior, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_interior));
}
/* :868-907 */
static double d2gdx2_mt(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.5 / (dx * dx) *
         (+p(n, i - 1, j - 1) + p(n, i - 1, j) - 2.0 * (+p(n, i, j - 1) + p(n, i, j)) +
          p(n, i + 1, j - 1) + p(n, i + 1, j));
}
/* :940-970 */
static double d2gdy2_mt(const ov *n, int i, int j, primary_proc p, double dy) {
  return 0.5 / (dy * dy) * (+p(n, i, j - 2) - p(n, i, j - 1) - p(n, i, j) + p(n, i, j + 1));
}
/* :1007-1039 */
static double d2gdxdy_mt(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (p(n, i - 1, j - 1) - p(n, i - 1, j) - p(n, i + 1, j - 1) + p(n, i + 1, j)) * 0.5 /
         (dx * dy);
}

const sd_ops SD_INTERIOR = {
  f_mt, dfdx_mt, dfdy_mt, d2fdx2_mt, d2fdy2_mt, d2fdxdy_mt, dfdx_nl_mt,
  g_mt, dgdx_mt, dgdy_mt, d2gdx2_mt, d2gdy2_mt, d2gdxdy_mt, dgdy_nl_mt,
  gradient_x_interior, gradient_y_interior
};

/* ------------------------------------------------------------------ */
/* DIM flux formulas: src/physical_models/dim2d/dim2d_fluxes_module.f  */
/* ------------------------------------------------------------------ */
/* :103-117 */
double flux_x_mass_density(const ov *n, const sd_ops *s, int i, int j) {
  return s->f(n, i, j, momentum_x);
}
/* :145-159 */
double flux_y_mass_density(const ov *n, const sd_ops *s, int i, int j) {
  return s->g(n, i, j, momentum_y);
}
/* :570-586 */
double flux_x_inviscid_momentum_x(const ov *n, const sd_ops *s, int i, int j) {
  return s->f(n, i, j, qx_transport_x) + s->f(n, i, j, classical_pressure);
}
/* :621-639 */
double flux_x_viscid_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return (2.0 + P.viscous_r) * s->dfdx(n, i, j, velocity_x, dx) +
         P.viscous_r * s->dfdy(n, i, j, velocity_y, dy);
}
/* :674-704 */
double flux_x_capillarity_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx,
                                     double dy) {
  double a = s->dfdx(n, i, j, mass_density, dx);
  double b = s->dfdy(n, i, j, mass_density, dy);
  return 1.5 / P.cv_r * s->f(n, i, j, capillarity_pressure) * (a * a + b * b) +
         s->f(n, i, j, mass_density) *
             (s->d2fdx2(n, i, j, mass_density, dx) + s->d2fdy2(n, i, j, mass_density, dy)) +
         0.5 * (-(a * a) + (b * b));
}
/* :755-769 */
double flux_y_inviscid_momentum_x(const ov *n, const sd_ops *s, int i, int j) {
  return s->g(n, i, j, qx_transport_y);
}
/* :804-821 */
double flux_y_viscid_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return s->dgdy(n, i, j, velocity_x, dy) + s->dgdx(n, i, j, velocity_y, dx);
}
/* :856-873 */
double flux_y_capillarity_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx,
                                     double dy) {
  return -s->dgdx(n, i, j, mass_density, dx) * s->dgdy(n, i, j, mass_density, dy);
}
/* :902-916 */
double flux_x_inviscid_momentum_y(const ov *n, const sd_ops *s, int i, int j) {
  return s->f(n, i, j, qy_transport_x);
}
/* :951-968 */
double flux_x_viscid_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return s->dfdy(n, i, j, velocity_x, dy) + s->dfdx(n, i, j, velocity_y, dx);
}
/* :1003-1020 */
double flux_x_capillarity_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx,
                                     double dy) {
  return -s->dfdx(n, i, j, mass_density, dx) * s->dfdy(n, i, j, mass_density, dy);
}
/* :1049-1064 */
double flux_y_inviscid_momentum_y(const ov *n, const sd_ops *s, int i, int j) {
  return s->g(n, i, j, qy_transport_y) + s->g(n, i, j, classical_pressure);
}
/* :1099-1116 */
double flux_y_viscid_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return P.viscous_r * s->dgdx(n, i, j, velocity_x, dx) +
         (2 + P.viscous_r) * s->dgdy(n, i, j, velocity_y, dy);
}
/* :1151-1179 */
double flux_y_capillarity_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx,
                                     double dy) {
  double a = s->dgdx(n, i, j, mass_density, dx);
  double b = s->dgdy(n, i, j, mass_density, dy);
  return 1.5 / P.cv_r * s->g(n, i, j, capillarity_pressure) * (a * a + b * b) +
         s->g(n, i, j, mass_density) *
             (s->d2gdx2(n, i, j, mass_density, dx) + s->d2gdy2(n, i, j, mass_density, dy)) +
         0.5 * ((a * a) - (b * b));
}
/* :1207-1222 */
double flux_x_inviscid_total_energy(const ov *n, const sd_ops *s, int i, int j) {
  return s->f(n, i, j, energy_transport_x) + s->f(n, i, j, classical_pressure_xwork);
}
/* :1256-1300 */
double flux_x_viscid_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx,
                                  double dy) {
  double ux = s->f(n, i, j, velocity_x);
  double uy = s->f(n, i, j, velocity_y);
  return ux * ((2 + P.viscous_r) * s->dfdx(n, i, j, velocity_x, dx) +
               P.viscous_r * s->dfdy(n, i, j, velocity_y, dy)) +
         uy * (s->dfdy(n, i, j, velocity_x, dy) + s->dfdx(n, i, j, velocity_y, dx)) +
         1.0 / P.pr * s->dfdx(n, i, j, classical_temperature_eff, dx);
}
/* :1334-1415 */
double flux_x_capillarity_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx,
                                       double dy) {
  double ux = s->f(n, i, j, velocity_x);
  double uy = s->f(n, i, j, velocity_y);
  double duxdx = s->dfdx(n, i, j, velocity_x, dx);
  double duydy = s->dfdy(n, i, j, velocity_y, dy);
  double drhodx = s->dfdx(n, i, j, mass_density, dx);
  double drhody = s->dfdy(n, i, j, mass_density, dy);
  return 1.5 / P.cv_r * s->f(n, i, j, capillarity_pressure_xwork) *
             ((drhodx * drhodx) + (drhody * drhody)) +
         s->f(n, i, j, momentum_x) *
             (s->d2fdx2(n, i, j, mass_density, dx) + s->d2fdy2(n, i, j, mass_density, dy)) +
         0.5 * ux * (-(drhodx * drhodx) + (drhody * drhody)) - drhodx * drhody * uy -
         s->f(n, i, j, mass_density) * drhodx * (duxdx + duydy) -
         1.0 / (P.re * P.pr) * s->dfdx_nl(n, i, j, capillarity_temperature_eff, dx, dy);
}
/* :1443-1458 */
double flux_y_inviscid_total_energy(const ov *n, const sd_ops *s, int i, int j) {
  return s->g(n, i, j, energy_transport_y) + s->g(n, i, j, classical_pressure_ywork);
}
/* :1492-1537 */
double flux_y_viscid_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx,
                                  double dy) {
  double ux = s->g(n, i, j, velocity_x);
  double uy = s->g(n, i, j, velocity_y);
  double duxdx = s->dgdx(n, i, j, velocity_x, dx);
  double duydy = s->dgdy(n, i, j, velocity_y, dy);
  return ux * (s->dgdy(n, i, j, velocity_x, dy) + s->dgdx(n, i, j, velocity_y, dx)) +
         uy * (P.viscous_r * duxdx + (2.0 + P.viscous_r) * duydy) +
         1.0 / P.pr * s->dgdy(n, i, j, classical_temperature_eff, dy);
}
/* :1571-1649 */
double flux_y_capillarity_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx,
                                       double dy) {
  double ux = s->g(n, i, j, velocity_x);
  double uy = s->g(n, i, j, velocity_y);
  double duxdx = s->dgdx(n, i, j, velocity_x, dx);
  double duydy = s->dgdy(n, i, j, velocity_y, dy);
  double drhodx = s->dgdx(n, i, j, mass_density, dx);
  double drhody = s->dgdy(n, i, j, mass_density, dy);
  double a = s->dgdx(n, i, j, mass_density, dx);
  double b = s->dgdy(n, i, j, mass_density, dy);
  return 1.5 / P.cv_r * s->g(n, i, j, capillarity_pressure_ywork) * ((a * a) + (b * b)) +
         s->g(n, i, j, momentum_y) *
             (s->d2gdx2(n, i, j, mass_density, dx) + s->d2gdy2(n, i, j, mass_density, dy)) +
         0.5 * uy * ((drhodx * drhodx) - (drhody * drhody)) - drhodx * drhody * ux -
         s->g(n, i, j, mass_density) * drhody * (duxdx + duydy) -
         1.0 / (P.re * P.pr) * s->dgdy_nl(n, i, j, capillarity_temperature_eff, dx, dy);
}
/* :193-222 */
double flux_x_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return flux_x_inviscid_momentum_x(n, s, i, j) -
         1.0 / P.re * flux_x_viscid_momentum_x(n, s, i, j, dx, dy) -
         1.0 / P.we * flux_x_capillarity_momentum_x(n, s, i, j, dx, dy);
}
/* :256-285 */
double flux_y_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return flux_y_inviscid_momentum_x(n, s, i, j) -
         1.0 / P.re * flux_y_viscid_momentum_x(n, s, i, j, dx, dy) -
         1.0 / P.we * flux_y_capillarity_momentum_x(n, s, i, j, dx, dy);
}
/* :319-348 */
double flux_x_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return flux_x_inviscid_momentum_y(n, s, i, j) -
         1.0 / P.re * flux_x_viscid_momentum_y(n, s, i, j, dx, dy) -
         1.0 / P.we * flux_x_capillarity_momentum_y(n, s, i, j, dx, dy);
}
/* :382-411 */
double flux_y_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return flux_y_inviscid_momentum_y(n, s, i, j) -
         1.0 / P.re * flux_y_viscid_momentum_y(n, s, i, j, dx, dy) -
         1.0 / P.we * flux_y_capillarity_momentum_y(n, s, i, j, dx, dy);
}
/* :445-477 */
double flux_x_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return flux_x_inviscid_total_energy(n, s, i, j) -
         1.0 / P.re * flux_x_viscid_total_energy(n, s, i, j, dx, dy) -
         1.0 / P.we * flux_x_capillarity_total_energy(n, s, i, j, dx, dy);
}
/* :511-541 */
double flux_y_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx, double dy) {
  return flux_y_inviscid_total_energy(n, s, i, j) -
         1.0 / P.re * flux_y_viscid_total_energy(n, s, i, j, dx, dy) -
         1.0 / P.we * flux_y_capillarity_total_energy(n, s, i, j, dx, dy);
}

/* ------------------------------------------------------------------ */
/* unit-level entry points for the golden tests                        */
/* ------------------------------------------------------------------ */
/* secondary procedure of the operator test,
 * test_augeanstables/test_mattsson_operators.f:1219-1238 */
static double gradient_av(const ov *n, int i, int j, double dx, double dy, gradient_proc gx,
                          gradient_proc gy) {
  return gx(n, i, j, mass_density, dx) + gy(n, i, j, mass_density, dy);
}

double orc_sd_operator(int set, int op, const double *nodes, int nx, int ny, int i, int j,
                       double dx, double dy) {
  ov n = {nx, ny, nodes};
  const sd_ops *s = orc_sd_set(set);
  if (!s) return NAN;
  switch (op) {
    case 0: return s->f(&n, i, j, mass_density);
    case 1: return s->dfdx(&n, i, j, mass_density, dx);
    case 2: return s->dfdy(&n, i, j, mass_density, dy);
    case 3: return s->d2fdx2(&n, i, j, mass_density, dx);
    case 4: return s->d2fdy2(&n, i, j, mass_density, dy);
    case 5: return s->d2fdxdy(&n, i, j, mass_density, dx, dy);
    case 6: return s->gx(&n, i, j, mass_density, dx);
    case 7: return s->g(&n, i, j, mass_density);
    case 8: return s->dgdx(&n, i, j, mass_density, dx);
    case 9: return s->dgdy(&n, i, j, mass_density, dy);
    case 10: return s->d2gdx2(&n, i, j, mass_density, dx);
    case 11: return s->d2gdy2(&n, i, j, mass_density, dy);
    case 12: return s->d2gdxdy(&n, i, j, mass_density, dx, dy);
    case 13: return s->gy(&n, i, j, mass_density, dy);
    case 14: return s->dfdx_nl(&n, i, j, gradient_av, dx, dy);
    case 15: return s->dgdy_nl(&n, i, j, gradient_av, dx, dy);
  }
  return NAN;
}

double orc_flux_function(int which, const double *nodes, int nx, int ny, int i, int j,
                         double dx, double dy) {
  ov n = {nx, ny, nodes};
  const sd_ops *s = &SD_INTERIOR;
  switch (which) {
    case 1: return flux_x_mass_density(&n, s, i, j);
    case 2: return flux_y_mass_density(&n, s, i, j);
    case 3: return flux_x_inviscid_momentum_x(&n, s, i, j);
    case 4: return flux_x_viscid_momentum_x(&n, s, i, j, dx, dy);
    case 5: return flux_x_capillarity_momentum_x(&n, s, i, j, dx, dy);
    case 6: return flux_x_momentum_x(&n, s, i, j, dx, dy);
    case 7: return flux_y_inviscid_momentum_x(&n, s, i, j);
    case 8: return flux_y_viscid_momentum_x(&n, s, i, j, dx, dy);
    case 9: return flux_y_capillarity_momentum_x(&n, s, i, j, dx, dy);
    case 10: return flux_y_momentum_x(&n, s, i, j, dx, dy);
    case 11: return flux_x_inviscid_momentum_y(&n, s, i, j);
    case 12: return flux_x_viscid_momentum_y(&n, s, i, j, dx, dy);
    case 13: return flux_x_capillarity_momentum_y(&n, s, i, j, dx, dy);
    case 14: return flux_x_momentum_y(&n, s, i, j, dx, dy);
    case 15: return flux_y_inviscid_momentum_y(&n, s, i, j);
    case 16: return flux_y_viscid_momentum_y(&n, s, i, j, dx, dy);
    case 17: return flux_y_capillarity_momentum_y(&n, s, i, j, dx, dy);
    case 18: return flux_y_momentum_y(&n, s, i, j, dx, dy);
    case 19: return flux_x_inviscid_total_energy(&n, s, i, j);
    case 20: return flux_x_viscid_total_energy(&n, s, i, j, dx, dy);
    case 21: return flux_x_capillarity_total_energy(&n, s, i, j, dx, dy);
    case 22: return flux_x_total_energy(&n, s, i, j, dx, dy);
    case 23: return flux_y_inviscid_total_energy(&n, s, i, j);
    case 24: return flux_y_viscid_total_energy(&n, s, i, j, dx, dy);
    case 25: return flux_y_capillarity_total_energy(&n, s, i, j, dx, dy);
    case 26: return flux_y_total_energy(&n, s, i, j, dx, dy);
  }
  return NAN;
}

/* ------------------------------------------------------------------ */
/* pmodel_eq: src/physical_models/dim2d/pmodel_eq_class.f              */
/* ------------------------------------------------------------------ */
/* :1073-1114  flux_x(nx+1,ny,ne) */
void compute_flux_x(const ov *n, double dx, double dy, double *flux_x) {
  const int nx = n->nx, ny = n->ny;
  const sd_ops *s = &SD_INTERIOR;
#pragma omp parallel for schedule(static)
  for (int j = 1 + BC_SIZE; j <= ny - BC_SIZE; j++) {
    for (int i = 1 + BC_SIZE; i <= nx + 1 - BC_SIZE; i++) {
      FX(flux_x, nx, ny, i, j, 1) = flux_x_mass_density(n, s, i, j);
      FX(flux_x, nx, ny, i, j, 2) = flux_x_momentum_x(n, s, i, j, dx, dy);
      FX(flux_x, nx, ny, i, j, 3) = flux_x_momentum_y(n, s, i, j, dx, dy);
      FX(flux_x, nx, ny, i, j, 4) = flux_x_total_energy(n, s, i, j, dx, dy);
    }
  }
}
/* :1140-1180  flux_y(nx,ny+1,ne) */
void compute_flux_y(const ov *n, double dx, double dy, double *flux_y) {
  const int nx = n->nx, ny = n->ny;
  const sd_ops *s = &SD_INTERIOR;
#pragma omp parallel for schedule(static)
  for (int j = 1 + BC_SIZE; j <= ny + 1 - BC_SIZE; j++) {
    for (int i = 1 + BC_SIZE; i <= nx - BC_SIZE; i++) {
      FY(flux_y, nx, ny, i, j, 1) = flux_y_mass_density(n, s, i, j);
      FY(flux_y, nx, ny, i, j, 2) = flux_y_momentum_x(n, s, i, j, dx, dy);
      FY(flux_y, nx, ny, i, j, 3) = flux_y_momentum_y(n, s, i, j, dx, dy);
      FY(flux_y, nx, ny, i, j, 4) = flux_y_total_energy(n, s, i, j, dx, dy);
    }
  }
}
/* :1840-1918 (conservative form, prim = .false.) */
double compute_body_forces(const double q[4], int k) {
  if (!P.gravity_ac) return 0.0;
  switch (k) {
    case 3: return -q[0] * P.gravity;
    case 4: return -q[2] * P.gravity;
    default: return 0.0;
  }
}

/* ------------------------------------------------------------------ */
/* td_operators: src/td_operators/finitevolume/td_operators_class.f    */
/* ------------------------------------------------------------------ */
static int any_type(const orc_cfg *c, int type) {
  if (c->periodic) return type == ORC_BC_NODES;
  for (int k = 0; k < 8; k++)
    if (c->bc_type[k] == type) return 1;
  return 0;
}
static int shall_bc_on_fluxes(const orc_cfg *c) {
  return any_type(c, ORC_BC_FLUXES) || any_type(c, ORC_BC_FLUX_AND_NODE);
}
static int shall_bc_on_timedev(const orc_cfg *c) { return any_type(c, ORC_BC_TIMEDEV); }

/* :119-235 */
void orc_compute_time_dev(const orc_cfg *c, double t, const double *nodes, const double *x_map,
                          const double *y_map, double *time_dev) {
  const int nx = c->nx, ny = c->ny;
  ov n = {nx, ny, nodes};
  size_t npl = (size_t)nx * ny;
  /* :150-154 */
  for (size_t m = 0; m < npl * NE; m++) time_dev[m] = orc_debug_real();
  /* :157-158 */
  double dx = x_map[1] - x_map[0];
  double dy = y_map[1] - y_map[0];
  double *flux_x = (double *)calloc((size_t)(nx + 1) * ny * NE, sizeof(double));
  double *flux_y = (double *)calloc((size_t)nx * (ny + 1) * NE, sizeof(double));
  /* :163-166 */
  compute_flux_x(&n, dx, dy, flux_x);
  compute_flux_y(&n, dx, dy, flux_y);
  /* :171-177 */
  if (!c->periodic && shall_bc_on_fluxes(c))
    orc_bc_apply_on_fluxes(c, t, x_map, y_map, &n, dx, dy, flux_x, flux_y);
  /* :181-194 */
  for (int k = 1; k <= NE; k++) {
#pragma omp parallel for schedule(static)
    for (int j = 1 + BC_SIZE; j <= ny - BC_SIZE; j++) {
      for (int i = 1 + BC_SIZE; i <= nx - BC_SIZE; i++) {
        double q[4] = {Q(&n, i, j, 1), Q(&n, i, j, 2), Q(&n, i, j, 3), Q(&n, i, j, 4)};
        TD(time_dev, nx, ny, i, j, k) =
            (FX(flux_x, nx, ny, i, j, k) / dx - FX(flux_x, nx, ny, i + 1, j, k) / dx) +
            (FY(flux_y, nx, ny, i, j, k) / dy - FY(flux_y, nx, ny, i, j + 1, k) / dy) +
            compute_body_forces(q, k);
      }
    }
  }
  /* :199-233 */
  if (!c->periodic && shall_bc_on_timedev(c))
    orc_bc_apply_on_timedev(c, t, x_map, y_map, &n, dx, dy, flux_x, flux_y, time_dev);
  free(flux_x);
  free(flux_y);
}

/* ------------------------------------------------------------------ */
/* periodic_xy legacy class:                                           */
/* src/boundary_conditions/periodic_xy/bc_operators_class.f:116-199    */
/* ------------------------------------------------------------------ */
static void periodic_apply_bc_on_nodes(int nx, int ny, double *nodes) {
  const int period_x = nx - 2 * BC_SIZE, period_y = ny - 2 * BC_SIZE;
  for (int k = 1; k <= NE; k++)
    for (int j = 1 + BC_SIZE; j <= ny - BC_SIZE; j++)
      for (int i = 1; i <= BC_SIZE; i++) {
        TD(nodes, nx, ny, i, j, k) = TD(nodes, nx, ny, i + period_x, j, k);
        TD(nodes, nx, ny, i + period_x + BC_SIZE, j, k) = TD(nodes, nx, ny, i + BC_SIZE, j, k);
      }
  for (int k = 1; k <= NE; k++)
    for (int j = 1; j <= BC_SIZE; j++)
      for (int i = 1; i <= nx; i++) {
        TD(nodes, nx, ny, i, j, k) = TD(nodes, nx, ny, i, j + period_y, k);
        TD(nodes, nx, ny, i, j + period_y + BC_SIZE, k) = TD(nodes, nx, ny, i, j + BC_SIZE, k);
      }
}

/* field_abstract_class.f:447-463 and bc_operators_gen_class.f:238-407 */
void orc_apply_bc_on_nodes(const orc_cfg *c, double t, const double *x_map, const double *y_map,
                           const double *nodes_tmp, double *nodes) {
  if (c->periodic) {
    periodic_apply_bc_on_nodes(c->nx, c->ny, nodes);
    return;
  }
  orc_bc_gen_apply_on_nodes(c, t, x_map, y_map, nodes_tmp, nodes);
}

/* ------------------------------------------------------------------ */
/* RK3-TVD: src/td_integrator/rungekutta3rdtvd/rk3tvd_steps_module.f   */
/* ------------------------------------------------------------------ */
/* :52-100 (borders ignored: all points including ghosts) */
static void compute_1st_step(int nx, int ny, double *nodes, double dt, double *nodes_tmp,
                             const double *time_dev) {
  size_t m, npl = (size_t)nx * ny * NE;
  for (m = 0; m < npl; m++) {
    nodes_tmp[m] = nodes[m];
    nodes[m] = nodes[m] + dt * time_dev[m];
  }
}
/* :205-269 */
static void compute_2nd_step(int nx, int ny, double *nodes, double dt, const double *nodes_tmp,
                             const double *time_dev, const int xb[2], const int yb[2]) {
  const double b2 = 0.75;
  for (int k = 1; k <= NE; k++)
    for (int j = yb[0]; j <= yb[1]; j++)
      for (int i = xb[0]; i <= xb[1]; i++)
        TD(nodes, nx, ny, i, j, k) =
            b2 * TD(nodes_tmp, nx, ny, i, j, k) +
            (1.0 - b2) * (TD(nodes, nx, ny, i, j, k) + dt * TD(time_dev, nx, ny, i, j, k));
}
/* :424-490 */
static void compute_3rd_step(int nx, int ny, double *nodes, double dt, const double *nodes_tmp,
                             const double *time_dev, const int xb[2], const int yb[2]) {
  const double b3 = 1.0 / 3.0;
  for (int k = 1; k <= NE; k++)
    for (int j = yb[0]; j <= yb[1]; j++)
      for (int i = xb[0]; i <= xb[1]; i++)
        TD(nodes, nx, ny, i, j, k) =
            b3 * TD(nodes_tmp, nx, ny, i, j, k) +
            (1.0 - b3) * (TD(nodes, nx, ny, i, j, k) + dt * TD(time_dev, nx, ny, i, j, k));
}

/* field_abstract_class.f:244-270 */
static void ini_for_time_int(const orc_cfg *c, int xb[2], int yb[2]) {
  xb[0] = BC_SIZE + 1;
  xb[1] = c->nx - BC_SIZE;
  yb[0] = BC_SIZE + 1;
  yb[1] = c->ny - BC_SIZE;
  if (c->periodic) return;
  if (c->bc_type[ORC_W] == ORC_BC_TIMEDEV) xb[0] -= BC_SIZE;
  if (c->bc_type[ORC_E] == ORC_BC_TIMEDEV) xb[1] += BC_SIZE;
  if (c->bc_type[ORC_S] == ORC_BC_TIMEDEV) yb[0] -= BC_SIZE;
  if (c->bc_type[ORC_N] == ORC_BC_TIMEDEV) yb[1] += BC_SIZE;
}

/* td_integrator_class.f:103-161, field_class.f:61-72 */
int orc_integrate(const orc_cfg *c, double *nodes, const double *x_map, const double *y_map,
                  double *t, double dt, int nsteps) {
  const int nx = c->nx, ny = c->ny;
  size_t sz = (size_t)nx * ny * NE;
  double *nodes_tmp = (double *)malloc(sz * sizeof(double));
  double *time_dev = (double *)malloc(sz * sizeof(double));
  int xb[2], yb[2];
  ini_for_time_int(c, xb, yb);
  for (int s = 0; s < nsteps; s++) {
    orc_compute_time_dev(c, *t, nodes, x_map, y_map, time_dev);
    compute_1st_step(nx, ny, nodes, dt, nodes_tmp, time_dev);
    orc_apply_bc_on_nodes(c, *t, x_map, y_map, nodes_tmp, nodes);

    orc_compute_time_dev(c, *t, nodes, x_map, y_map, time_dev);
    compute_2nd_step(nx, ny, nodes, dt, nodes_tmp, time_dev, xb, yb);
    orc_apply_bc_on_nodes(c, *t, x_map, y_map, nodes_tmp, nodes);

    orc_compute_time_dev(c, *t, nodes, x_map, y_map, time_dev);
    compute_3rd_step(nx, ny, nodes, dt, nodes_tmp, time_dev, xb, yb);
    orc_apply_bc_on_nodes(c, *t, x_map, y_map, nodes_tmp, nodes);

    *t = *t + dt;
    if (orc_status()) break; /* the reference stops the program here */
  }
  free(nodes_tmp);
  free(time_dev);
  return orc_status();
}

/* field_abstract_class.f:286-315 */
void orc_ini_coordinates(int nx, int ny, double x_min, double x_max, double y_min, double y_max,
                         double *x_map, double *y_map) {
  double dx = (x_max - x_min) / (nx - 1 - 2 * BC_SIZE);
  double dy = (y_max - y_min) / (ny - 1 - 2 * BC_SIZE);
  for (int i = 1; i <= nx; i++) x_map[i - 1] = x_min + (i - 1 - BC_SIZE) * dx;
  for (int j = 1; j <= ny; j++) y_map[j - 1] = y_min + (j - 1 - BC_SIZE) * dy;
}
