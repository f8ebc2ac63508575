/*
 * Internal declarations shared by the oracle's translation units.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef DIM2D_ORACLE_INTERNAL_H
#define DIM2D_ORACLE_INTERNAL_H

#include <stddef.h>
#include "dim2d_oracle.h"

#define NE 4
#define BC_SIZE 2 /* parameters_input.f:81 */

/* read-only view of nodes(nx,ny,ne), 1-based accessors */
typedef struct {
  int nx, ny;
  const double *q;
} ov;

#define Q(n, i, j, k) ((n)->q[((size_t)((k)-1) * (n)->ny + (size_t)((j)-1)) * (n)->nx + (size_t)((i)-1)])
#define TD(a, nx, ny, i, j, k) ((a)[((size_t)((k)-1) * (ny) + (size_t)((j)-1)) * (nx) + (size_t)((i)-1)])
#define FX(a, nx, ny, i, j, k) ((a)[((size_t)((k)-1) * (ny) + (size_t)((j)-1)) * ((nx) + 1) + (size_t)((i)-1)])
#define FY(a, nx, ny, i, j, k) ((a)[((size_t)((k)-1) * ((ny) + 1) + (size_t)((j)-1)) * (nx) + (size_t)((i)-1)])

/* interface_primary.f: get_primary_var / gradient_proc / get_secondary_var */
typedef double (*primary_proc)(const ov *n, int i, int j);
typedef double (*gradient_proc)(const ov *n, int i, int j, primary_proc p, double dn);
typedef double (*secondary_proc)(const ov *n, int i, int j, double dx, double dy,
                                 gradient_proc gx, gradient_proc gy);

/* one Mattsson operator set (sd_operators_abstract_class.f) */
typedef struct {
  double (*f)(const ov *, int, int, primary_proc);
  double (*dfdx)(const ov *, int, int, primary_proc, double);
  double (*dfdy)(const ov *, int, int, primary_proc, double);
  double (*d2fdx2)(const ov *, int, int, primary_proc, double);
  double (*d2fdy2)(const ov *, int, int, primary_proc, double);
  double (*d2fdxdy)(const ov *, int, int, primary_proc, double, double);
  double (*dfdx_nl)(const ov *, int, int, secondary_proc, double, double);
  double (*g)(const ov *, int, int, primary_proc);
  double (*dgdx)(const ov *, int, int, primary_proc, double);
  double (*dgdy)(const ov *, int, int, primary_proc, double);
  double (*d2gdx2)(const ov *, int, int, primary_proc, double);
  double (*d2gdy2)(const ov *, int, int, primary_proc, double);
  double (*d2gdxdy)(const ov *, int, int, primary_proc, double, double);
  double (*dgdy_nl)(const ov *, int, int, secondary_proc, double, double);
  gradient_proc gx, gy; /* gradient procedures the set's *_nl operators use */
} sd_ops;

extern orc_params P;
extern const sd_ops SD_INTERIOR;
const sd_ops *orc_sd_set(int set);

/* primitives (dim2d_prim_module.f) */
double mass_density(const ov *n, int i, int j);
double momentum_x(const ov *n, int i, int j);
double momentum_y(const ov *n, int i, int j);
double total_energy(const ov *n, int i, int j);
double velocity_x(const ov *n, int i, int j);
double velocity_y(const ov *n, int i, int j);
double classical_pressure(const ov *n, int i, int j);
double vdw_pressure(double temperature, double md);
double classical_temperature_eff(const ov *n, int i, int j);
double capillarity_temperature_eff(const ov *n, int i, int j, double dx, double dy,
                                   gradient_proc gx, gradient_proc gy);
double temperature_eff(const ov *n, int i, int j, double dx, double dy, gradient_proc gx,
                       gradient_proc gy);
double classical_pressure_xwork(const ov *n, int i, int j);
double classical_pressure_ywork(const ov *n, int i, int j);
double qx_transport_x(const ov *n, int i, int j);
double qy_transport_x(const ov *n, int i, int j);
double qx_transport_y(const ov *n, int i, int j);
double qy_transport_y(const ov *n, int i, int j);
double energy_transport_x(const ov *n, int i, int j);
double energy_transport_y(const ov *n, int i, int j);
double capillarity_pressure(const ov *n, int i, int j);
double capillarity_pressure_xwork(const ov *n, int i, int j);
double capillarity_pressure_ywork(const ov *n, int i, int j);

/* gradients (sd_operators_fd_module.f) */
double gradient_x_interior(const ov *n, int i, int j, primary_proc p, double dn);
double gradient_y_interior(const ov *n, int i, int j, primary_proc p, double dn);
double gradient_x_x_oneside_L0(const ov *n, int i, int j, primary_proc p, double dn);
double gradient_x_x_oneside_R0(const ov *n, int i, int j, primary_proc p, double dn);
double gradient_y_y_oneside_L0(const ov *n, int i, int j, primary_proc p, double dn);
double gradient_y_y_oneside_R0(const ov *n, int i, int j, primary_proc p, double dn);

/* flux formulas (dim2d_fluxes_module.f) */
double flux_x_mass_density(const ov *n, const sd_ops *s, int i, int j);
double flux_y_mass_density(const ov *n, const sd_ops *s, int i, int j);
double flux_x_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_y_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_x_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_y_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_x_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_y_total_energy(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_x_inviscid_momentum_x(const ov *n, const sd_ops *s, int i, int j);
double flux_x_viscid_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_x_capillarity_momentum_x(const ov *n, const sd_ops *s, int i, int j, double dx,
                                     double dy);
double flux_y_inviscid_momentum_y(const ov *n, const sd_ops *s, int i, int j);
double flux_y_viscid_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx, double dy);
double flux_y_capillarity_momentum_y(const ov *n, const sd_ops *s, int i, int j, double dx,
                                     double dy);

/* pmodel_eq_class.f */
void compute_flux_x(const ov *n, double dx, double dy, double *flux_x);
void compute_flux_y(const ov *n, double dx, double dy, double *flux_y);
double compute_body_forces(const double q[4], int k);

/* boundary conditions (dim2d_oracle_bc.c) */
void orc_bc_gen_apply_on_nodes(const orc_cfg *c, double t, const double *x_map,
                               const double *y_map, const double *nodes_tmp, double *nodes);
void orc_bc_apply_on_fluxes(const orc_cfg *c, double t, const double *x_map, const double *y_map,
                            const ov *n, double dx, double dy, double *flux_x, double *flux_y);
void orc_bc_apply_on_timedev(const orc_cfg *c, double t, const double *x_map,
                             const double *y_map, const ov *n, double dx, double dy,
                             double *flux_x, double *flux_y, double *time_dev);
/* section bounds [type, i_min, j_min, i_max/j_max] (bc_operators_gen_class.f:95-102) */
void orc_section(const orc_cfg *c, int section, int sec[4]);
void orc_reflection_apply_on_nodes(const orc_cfg *c, int section, int choice, double *nodes);
void orc_wall_apply_on_nodes(const orc_cfg *c, int section, double t, const double *x_map,
                             const double *y_map, const double *nodes_tmp, double *nodes);
void orc_wall_apply_on_fluxes(const orc_cfg *c, int section, double t, const double *x_map,
                              const double *y_map, const ov *n, double dx, double dy,
                              double *flux_x, double *flux_y);

#endif
