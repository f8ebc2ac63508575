/*
 * dim2d_oracle_bc.c -- generic boundary-condition dispatcher of the
 * reference (bc_operators_gen_class.f) and the operator-set registry.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "dim2d_oracle_internal.h"

/* bc_operators_gen_class.f:238-407: walk bc_order1..8 and apply the
 * node-type operators of each section */
void orc_bc_gen_apply_on_nodes(const orc_cfg *c, double t, const double *x_map,
                               const double *y_map, const double *nodes_tmp, double *nodes) {
  (void)c; (void)t; (void)x_map; (void)y_map; (void)nodes_tmp; (void)nodes;
  fprintf(stderr, "oracle: generic node boundary conditions not available\n");
  abort();
}

/* bc_operators_gen_class.f:509-601 */
void orc_bc_apply_on_fluxes(const orc_cfg *c, double t, const double *x_map, const double *y_map,
                            const ov *n, double dx, double dy, double *flux_x, double *flux_y) {
  (void)c; (void)t; (void)x_map; (void)y_map; (void)n; (void)dx; (void)dy; (void)flux_x;
  (void)flux_y;
  fprintf(stderr, "oracle: flux boundary conditions not available\n");
  abort();
}

/* bc_operators_gen_class.f:880-978 */
void orc_bc_apply_on_timedev(const orc_cfg *c, double t, const double *x_map,
                             const double *y_map, const ov *n, double dx, double dy,
                             const double *flux_x, const double *flux_y, double *time_dev) {
  (void)c; (void)t; (void)x_map; (void)y_map; (void)n; (void)dx; (void)dy; (void)flux_x;
  (void)flux_y; (void)time_dev;
  fprintf(stderr, "oracle: time-derivative boundary conditions not available\n");
  abort();
}
