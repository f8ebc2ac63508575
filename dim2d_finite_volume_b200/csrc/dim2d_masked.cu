// dim2d_masked.cu -- the masked ("_nopt") interior operators of buffer-layer
// grids on sm_100a.
//
// A buffer layer of the reference (src/boundary_conditions/open_bc/
// buffer_layer) carries its own nodes(nx,ny,4) and a map grdpts_id(nx,ny)
// marking each point no_pt (0), interior_pt (1), bc_interior_pt (2) or bc_pt
// (3) (parameters_bf_layer.f:41-44).  These kernels are the area-sized part
// of stepping such a grid:
//   * time derivative at the interior_pt points inside the borders
//     (td_operators_class.f:293-417): the warp-strip kernel (k_strip,
//     dim2d_strip.cu) where nx is even and the nodes 16-byte aligned, else
//     the interior tile kernel (k_interior, dim2d_interior.cu), over the
//     border box, in their masked mode -- primitives
//     once per node, each face flux once with the interior Mattsson operators
//     and the DIM flux formulas (every face of an interior_pt point lies
//     between interior_pt / bc_interior_pt points, where the reference
//     computes its fluxes, pmodel_eq_class.f:1215-1360), divergence and body
//     forces, written where grdpts_id is interior_pt;
//   * the masked RK3 stages (rk3tvd_steps_module.f:130-614): stage 1 over
//     every point that is not no_pt, stages 2 and 3 over those inside the
//     borders, with the reference's coefficient pairs (0.75, 0.25) and
//     (1/3, 2/3).
// The layer's boundary sections (bc_pt / bc_interior_pt points) stay with
// the host-driven layer code.  Arrays live on the device, owned by the
// caller; nothing is allocated.
#include <algorithm>

#include "dim2d_internal.h"

namespace dim2d {
namespace {

// One thread per point of a row; blocks stride over the rows.  The state
// loads are issued together with the grdpts_id load (every array covers the
// whole grid, so the loads of no_pt points stay in bounds) and only the
// stores wait for the map: one memory latency per point instead of two.
__global__ void __launch_bounds__(256) k_rk_stage_masked(int stage, double* __restrict__ u,
                                                         double* __restrict__ utmp,
                                                         const double* __restrict__ td,
                                                         const int* __restrict__ gid, Field f,
                                                         double dt, int x0, int x1, int y0,
                                                         int y1) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= f.nx) return;
  const bool in_x = x >= x0 && x <= x1;
  const double b = stage == 2 ? 0.75 : 1.0 / 3.0;
  const double b_m = stage == 2 ? 0.25 : 2.0 / 3.0;
  for (int y = blockIdx.y; y < f.ny; y += gridDim.y) {
    const size_t m = (size_t)y * f.pitch + x;
    if (stage != 1 && !(in_x && y >= y0 && y <= y1)) continue;  // outside the borders
    const int g = __ldg(gid + m);
    double q[4], l[4], q0[4];
#pragma unroll
    for (int v = 0; v < 4; v++) {
      q[v] = u[m + v * f.plane];
      l[v] = __ldg(td + m + v * f.plane);
      q0[v] = stage == 1 ? 0.0 : utmp[m + v * f.plane];
    }
    if (g == 0) continue;  // no_pt
    if (stage == 1) {
#pragma unroll
      for (int v = 0; v < 4; v++) {
        utmp[m + v * f.plane] = q[v];
        u[m + v * f.plane] = q[v] + dt * l[v];
      }
    } else {
#pragma unroll
      for (int v = 0; v < 4; v++) u[m + v * f.plane] = b * q0[v] + b_m * (q[v] + dt * l[v]);
    }
  }
}

int check_grid(const char* what, int nx, int ny, const int xb[2], const int yb[2]) {
  if (nx < 2 * BC + 2 || ny < 2 * BC + 2 || nx > 65536 || ny > 65536)
    return set_error(DIM2D_ERR_ARG, "%s: nx, ny must be in [%d, 65536] (got %d x %d)", what,
                     2 * BC + 2, nx, ny);
  if (!xb || !yb || xb[0] < 1 || xb[1] > nx || yb[0] < 1 || yb[1] > ny)
    return set_error(DIM2D_ERR_ARG, "%s: borders outside the grid", what);
  return DIM2D_OK;
}

}  // namespace
}  // namespace dim2d

using namespace dim2d;

extern "C" {

int dim2d_time_dev_masked(const dim2d_params* p, int nx, int ny, const double* nodes,
                          const int* grdpts_id, double dx, double dy, const int x_borders[2],
                          const int y_borders[2], double* time_dev, void* stream) {
  if (!p || !nodes || !grdpts_id || !time_dev)
    return set_error(DIM2D_ERR_ARG, "time_dev_masked: null argument");
  int rc = check_grid("time_dev_masked", nx, ny, x_borders, y_borders);
  if (rc) return rc;
  if (!(dx > 0) || !(dy > 0)) return set_error(DIM2D_ERR_ARG, "time_dev_masked: bad dx/dy");
  StageArgs a{};
  a.f.nx = nx;
  a.f.ny = ny;
  a.f.pitch = nx;
  a.f.plane = (size_t)nx * ny;
  // the faces of a point at least BC points inside the grid stay inside it
  a.box_x0 = std::max(x_borders[0] - 1, BC);
  a.box_x1 = std::min(x_borders[1] - 1, nx - 1 - BC);
  a.box_y0 = std::max(y_borders[0] - 1, BC);
  a.box_y1 = std::min(y_borders[1] - 1, ny - 1 - BC);
  if (a.box_x0 > a.box_x1 || a.box_y0 > a.box_y1) return DIM2D_OK;
  a.uin = nodes;
  a.uout = time_dev;
  a.mask = grdpts_id;
  a.dx = dx;
  a.dy = dy;
  a.rdx = 1.0 / dx;
  a.rdy = 1.0 / dy;
  a.k = make_const(*p);
  const cudaError_t e = launch_time_dev_masked(a, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_error(e, "time_dev_masked");
  return DIM2D_OK;
}

int dim2d_rk_stage_masked(int stage, int nx, int ny, double* nodes, double* nodes_tmp,
                          const double* time_dev, const int* grdpts_id, double dt,
                          const int x_borders[2], const int y_borders[2], void* stream) {
  if (!nodes || !nodes_tmp || !time_dev || !grdpts_id)
    return set_error(DIM2D_ERR_ARG, "rk_stage_masked: null argument");
  if (stage < 1 || stage > 3) return set_error(DIM2D_ERR_ARG, "rk_stage_masked: stage %d", stage);
  int rc = check_grid("rk_stage_masked", nx, ny, x_borders, y_borders);
  if (rc) return rc;
  Field f;
  f.nx = nx;
  f.ny = ny;
  f.pitch = nx;
  f.plane = (size_t)nx * ny;
  const dim3 grid((nx + 255) / 256, std::min(ny, 65535));
  k_rk_stage_masked<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      stage, nodes, nodes_tmp, time_dev, grdpts_id, f, dt, x_borders[0] - 1, x_borders[1] - 1,
      y_borders[0] - 1, y_borders[1] - 1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "rk_stage_masked");
  return DIM2D_OK;
}

}  // extern "C"
