/*
 * dim2d_oracle_reflect.c -- reflection node operators.
 * TEST INFRASTRUCTURE ONLY.
 *
 * src/boundary_conditions/reflection_xy/bc_operators_reflection_x_class.f:178-296
 * src/boundary_conditions/reflection_xy/bc_operators_reflection_y_class.f:178-289
 * prefactors: reflection_xy_module.f:50-110 with the DIM variable types
 * (scalar, vector_x, vector_y, scalar), pmodel_eq_class.f:613-624.
 */
#include <math.h>

#include "dim2d_oracle_internal.h"

/* the generic sections, bc_operators_gen_class.f:95-102 */
void orc_section(const orc_cfg *c, int section, int sec[4]) {
  const int nx = c->nx, ny = c->ny;
  switch (section) {
    case ORC_SW_CORNER: sec[0] = section; sec[1] = 1; sec[2] = 1; sec[3] = 0; break;
    case ORC_S_EDGE: sec[0] = section; sec[1] = BC_SIZE + 1; sec[2] = 1; sec[3] = nx - BC_SIZE; break;
    case ORC_SE_CORNER: sec[0] = section; sec[1] = nx - BC_SIZE + 1; sec[2] = 1; sec[3] = 0; break;
    case ORC_W_EDGE: sec[0] = section; sec[1] = 1; sec[2] = BC_SIZE + 1; sec[3] = ny - BC_SIZE; break;
    case ORC_E_EDGE: sec[0] = section; sec[1] = nx - BC_SIZE + 1; sec[2] = BC_SIZE + 1; sec[3] = ny - BC_SIZE; break;
    case ORC_NW_CORNER: sec[0] = section; sec[1] = 1; sec[2] = ny - BC_SIZE + 1; sec[3] = 0; break;
    case ORC_N_EDGE: sec[0] = section; sec[1] = BC_SIZE + 1; sec[2] = ny - BC_SIZE + 1; sec[3] = nx - BC_SIZE; break;
    default: sec[0] = section; sec[1] = nx - BC_SIZE + 1; sec[2] = ny - BC_SIZE + 1; sec[3] = 0; break;
  }
}

/* check_data_module.f:28-46 with debug_real */
static int is_debug(double v) { return fabs(v - orc_debug_real()) < 1e-10; }

void orc_reflection_apply_on_nodes(const orc_cfg *c, int section, int choice, double *nodes) {
  const int nx = c->nx, ny = c->ny;
  int sec[4];
  orc_section(c, section, sec);
  if (choice == ORC_REFLECTION_X) {
    const int pre[4] = {1, -1, 1, 1};
    const int refl_E = 2 * sec[1] - 1;
    const int refl_W = 2 * sec[1] + 2 * BC_SIZE - 1;
    for (int k = 1; k <= NE; k++) {
      if (section == ORC_E_EDGE || section == ORC_W_EDGE) {
        const int r = section == ORC_E_EDGE ? refl_E : refl_W;
        for (int j = sec[2]; j <= sec[3]; j++)
          for (int i = sec[1]; i <= sec[1] + BC_SIZE - 1; i++)
            TD(nodes, nx, ny, i, j, k) = pre[k - 1] * TD(nodes, nx, ny, r - i, j, k);
      } else {
        const int r = (section == ORC_SW_CORNER || section == ORC_NW_CORNER) ? refl_W : refl_E;
        for (int j = sec[2]; j <= sec[2] + BC_SIZE - 1; j++)
          for (int i = sec[1]; i <= sec[1] + BC_SIZE - 1; i++) {
            double src = TD(nodes, nx, ny, r - i, j, k);
            TD(nodes, nx, ny, i, j, k) = is_debug(src) ? orc_debug_real() : pre[k - 1] * src;
          }
      }
    }
  } else {
    const int pre[4] = {1, 1, -1, 1};
    const int refl_N = 2 * sec[2] - 1;
    const int refl_S = 2 * sec[2] + 2 * BC_SIZE - 1;
    for (int k = 1; k <= NE; k++) {
      if (section == ORC_N_EDGE || section == ORC_S_EDGE) {
        const int r = section == ORC_N_EDGE ? refl_N : refl_S;
        for (int j = sec[2]; j <= sec[2] + BC_SIZE - 1; j++)
          for (int i = sec[1]; i <= sec[3]; i++)
            TD(nodes, nx, ny, i, j, k) = pre[k - 1] * TD(nodes, nx, ny, i, r - j, k);
      } else {
        const int r = (section == ORC_SW_CORNER || section == ORC_SE_CORNER) ? refl_S : refl_N;
        for (int j = sec[2]; j <= sec[2] + BC_SIZE - 1; j++)
          for (int i = sec[1]; i <= sec[1] + BC_SIZE - 1; i++) {
            double src = TD(nodes, nx, ny, i, r - j, k);
            TD(nodes, nx, ny, i, j, k) = is_debug(src) ? orc_debug_real() : pre[k - 1] * src;
          }
      }
    }
  }
}
