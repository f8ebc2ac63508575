/*
 * dim2d_oracle_masked.c -- the masked ("_nopt") interior operators that
 * buffer layers run on their own grids, identified point by point by
 * grdpts_id (parameters_bf_layer.f:41-44: no_pt 0, interior_pt 1,
 * bc_interior_pt 2, bc_pt 3).  TEST INFRASTRUCTURE ONLY.
 *
 * Restated here: the interior part of compute_time_dev_nopt
 * (td_operators_class.f:293-417 with pmodel_eq_class.f:1215-1360:
 * fluxes where grdpts_id is interior_pt or bc_interior_pt, the time
 * derivative where it is interior_pt) and the masked RK3 stages
 * (rk3tvd_steps_module.f:130-614).  The boundary sections of a layer
 * (apply_bc_on_fluxes_nopt / apply_bc_on_timedev_nopt) are not restated.
 * Arrays: nodes(nx,ny,4), grdpts_id(nx,ny), borders 1-based inclusive.
 */
#include <math.h>
#include <stdlib.h>

#include "dim2d_oracle_internal.h"

enum { NO_PT = 0, INTERIOR_PT = 1, BC_INTERIOR_PT = 2 };
#define GID(g, nx, i, j) ((g)[(size_t)((j)-1) * (nx) + (size_t)((i)-1)])

/* time_dev(i,j,:) at the interior_pt points inside the borders; other
 * points of time_dev are left as they are.  Faces the layer does not
 * compute (a neighbour that is neither interior_pt nor bc_interior_pt)
 * stay NaN, so a point that would read one shows it. */
void orc_compute_time_dev_masked(int nx, int ny, const double *nodes, const int *grdpts_id,
                                 double dx, double dy, const int xb[2], const int yb[2],
                                 double *time_dev) {
  ov n = {nx, ny, nodes};
  const sd_ops *s = &SD_INTERIOR;
  double *flux_x = (double *)malloc((size_t)(nx + 1) * ny * NE * sizeof(double));
  double *flux_y = (double *)malloc((size_t)nx * (ny + 1) * NE * sizeof(double));
  for (size_t m = 0; m < (size_t)(nx + 1) * ny * NE; m++) flux_x[m] = NAN;
  for (size_t m = 0; m < (size_t)nx * (ny + 1) * NE; m++) flux_y[m] = NAN;
  /* pmodel_eq_class.f:1215-1269 */
  for (int j = BC_SIZE + 1; j <= ny - BC_SIZE; j++)
    for (int i = BC_SIZE + 1; i <= nx - BC_SIZE + 1; i++) {
      const int g = GID(grdpts_id, nx, i, j);
      if (g != INTERIOR_PT && g != BC_INTERIOR_PT) continue;
      FX(flux_x, nx, ny, i, j, 1) = flux_x_mass_density(&n, s, i, j);
      FX(flux_x, nx, ny, i, j, 2) = flux_x_momentum_x(&n, s, i, j, dx, dy);
      FX(flux_x, nx, ny, i, j, 3) = flux_x_momentum_y(&n, s, i, j, dx, dy);
      FX(flux_x, nx, ny, i, j, 4) = flux_x_total_energy(&n, s, i, j, dx, dy);
    }
  /* :1304-1360 */
  for (int j = BC_SIZE + 1; j <= ny - BC_SIZE + 1; j++)
    for (int i = BC_SIZE + 1; i <= nx - BC_SIZE; i++) {
      const int g = GID(grdpts_id, nx, i, j);
      if (g != INTERIOR_PT && g != BC_INTERIOR_PT) continue;
      FY(flux_y, nx, ny, i, j, 1) = flux_y_mass_density(&n, s, i, j);
      FY(flux_y, nx, ny, i, j, 2) = flux_y_momentum_x(&n, s, i, j, dx, dy);
      FY(flux_y, nx, ny, i, j, 3) = flux_y_momentum_y(&n, s, i, j, dx, dy);
      FY(flux_y, nx, ny, i, j, 4) = flux_y_total_energy(&n, s, i, j, dx, dy);
    }
  /* td_operators_class.f:373-394 */
  for (int k = 1; k <= NE; k++)
    for (int j = yb[0]; j <= yb[1]; j++)
      for (int i = xb[0]; i <= xb[1]; i++) {
        if (GID(grdpts_id, nx, i, j) != INTERIOR_PT) continue;
        double q[4] = {Q(&n, i, j, 1), Q(&n, i, j, 2), Q(&n, i, j, 3), Q(&n, i, j, 4)};
        TD(time_dev, nx, ny, i, j, k) =
            (FX(flux_x, nx, ny, i, j, k) / dx - FX(flux_x, nx, ny, i + 1, j, k) / dx) +
            (FY(flux_y, nx, ny, i, j, k) / dy - FY(flux_y, nx, ny, i, j + 1, k) / dy) +
            compute_body_forces(q, k);
      }
  free(flux_x);
  free(flux_y);
}

/* compute_1st/2nd/3rd_step_nopt, rk3tvd_steps_module.f:130-177, 300-394,
 * 520-614: stage 1 over every point that is not no_pt (borders unused),
 * stages 2 and 3 over those inside the borders, with the coefficient pairs
 * (0.75, 0.25) and (1/3, 2/3) written out as the reference does */
void orc_rk_stage_masked(int stage, int nx, int ny, double *nodes, double *nodes_tmp,
                         const double *time_dev, const int *grdpts_id, double dt,
                         const int xb[2], const int yb[2]) {
  if (stage == 1) {
    for (int k = 1; k <= NE; k++)
      for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++)
          if (GID(grdpts_id, nx, i, j) != NO_PT) {
            TD(nodes_tmp, nx, ny, i, j, k) = TD(nodes, nx, ny, i, j, k);
            TD(nodes, nx, ny, i, j, k) =
                TD(nodes, nx, ny, i, j, k) + dt * TD(time_dev, nx, ny, i, j, k);
          }
    return;
  }
  const double b = stage == 2 ? 0.75 : 1.0 / 3.0;
  const double b_m = stage == 2 ? 0.25 : 2.0 / 3.0;
  for (int k = 1; k <= NE; k++)
    for (int j = yb[0]; j <= yb[1]; j++)
      for (int i = xb[0]; i <= xb[1]; i++)
        if (GID(grdpts_id, nx, i, j) != NO_PT)
          TD(nodes, nx, ny, i, j, k) =
              b * TD(nodes_tmp, nx, ny, i, j, k) +
              b_m * (TD(nodes, nx, ny, i, j, k) + dt * TD(time_dev, nx, ny, i, j, k));
}
