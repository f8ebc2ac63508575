/*
 * dim2d_oracle_wall.c -- wall (contact-angle equilibrium) boundary.
 * TEST INFRASTRUCTURE ONLY.
 */
#include <stdio.h>
#include <stdlib.h>

#include "dim2d_oracle_internal.h"

void orc_wall_apply_on_nodes(const orc_cfg *c, int section, double t, const double *x_map,
                             const double *y_map, const double *nodes_tmp, double *nodes) {
  (void)c; (void)section; (void)t; (void)x_map; (void)y_map; (void)nodes_tmp; (void)nodes;
  fprintf(stderr, "oracle: wall boundary not restated yet\n");
  abort();
}

void orc_wall_apply_on_fluxes(const orc_cfg *c, int section, double t, const double *x_map,
                              const double *y_map, const ov *n, double dx, double dy,
                              double *flux_x, double *flux_y) {
  (void)c; (void)section; (void)t; (void)x_map; (void)y_map; (void)n; (void)dx; (void)dy;
  (void)flux_x; (void)flux_y;
  fprintf(stderr, "oracle: wall boundary not restated yet\n");
  abort();
}
