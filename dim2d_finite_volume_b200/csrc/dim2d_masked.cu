// dim2d_masked.cu -- the masked ("_nopt") interior operators of buffer-layer
// grids on sm_100a.
//
// A buffer layer of the reference (src/boundary_conditions/open_bc/
// buffer_layer) carries its own nodes(nx,ny,4) and a map grdpts_id(nx,ny)
// marking each point no_pt (0), interior_pt (1), bc_interior_pt (2) or bc_pt
// (3) (parameters_bf_layer.f:41-44).  These kernels are the area-sized part
// of stepping such a grid:
//   * time derivative at the interior_pt points inside the borders
//     (td_operators_class.f:293-417): the four faces of the point with the
//     interior Mattsson operators and the DIM flux formulas (every face of an
//     interior_pt point lies between interior_pt / bc_interior_pt points,
//     where the reference computes its fluxes, pmodel_eq_class.f:1215-1360),
//     divergence and body forces;
//   * the masked RK3 stages (rk3tvd_steps_module.f:130-614): stage 1 over
//     every point that is not no_pt, stages 2 and 3 over those inside the
//     borders, with the reference's coefficient pairs (0.75, 0.25) and
//     (1/3, 2/3).
// The layer's boundary sections (bc_pt / bc_interior_pt points) stay with
// the host-driven layer code.  Arrays live on the device, owned by the
// caller; nothing is allocated.
#include <cstring>

#include "dim2d_internal.h"
#include "dim2d_open.cuh"

namespace dim2d {
namespace {

constexpr int INTERIOR_PT = 1;

__global__ void __launch_bounds__(128) k_time_dev_masked(const double* __restrict__ u,
                                                         const int* __restrict__ gid, Field f,
                                                         double rdx, double rdy, DimConst k,
                                                         int x0, int x1, int y0, int y1,
                                                         double* __restrict__ td) {
  const int w = x1 - x0 + 1;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (long long)w * (y1 - y0 + 1)) return;
  const int x = x0 + (int)(m % w), y = y0 + (int)(m / w);
  const size_t o = (size_t)y * f.pitch + x;
  if (gid[o] != INTERIOR_PT) return;
  double Fl[4], Fr[4], Gb[4], Gt[4];
  frame_face_flux(Frame{u, f, x, y, false}, T_INT, rdx, rdy, k, Fl);
  frame_face_flux(Frame{u, f, x + 1, y, false}, T_INT, rdx, rdy, k, Fr);
  frame_face_flux(Frame{u, f, x, y, true}, T_INT, rdy, rdx, k, Gb);
  frame_face_flux(Frame{u, f, x, y + 1, true}, T_INT, rdy, rdx, k, Gt);
  // y-face frames order their fluxes (mass, momentum_y, momentum_x, energy)
  double L[4];
  L[0] = (Fl[0] - Fr[0]) * rdx + (Gb[0] - Gt[0]) * rdy;
  L[1] = (Fl[1] - Fr[1]) * rdx + (Gb[2] - Gt[2]) * rdy;
  L[2] = (Fl[2] - Fr[2]) * rdx + (Gb[1] - Gt[1]) * rdy;
  L[3] = (Fl[3] - Fr[3]) * rdx + (Gb[3] - Gt[3]) * rdy;
  if (k.gravity_ac) {  // pmodel_eq_class.f:1889-1904
    L[2] += -u[o] * k.gravity;
    L[3] += -u[o + 2 * f.plane] * k.gravity;
  }
#pragma unroll
  for (int v = 0; v < 4; v++) td[o + v * f.plane] = L[v];
}

__global__ void __launch_bounds__(256) k_rk_stage_masked(int stage, double* __restrict__ u,
                                                         double* __restrict__ utmp,
                                                         const double* __restrict__ td,
                                                         const int* __restrict__ gid, Field f,
                                                         double dt, int x0, int x1, int y0,
                                                         int y1) {
  const size_t cells = f.plane;
  for (size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x; m < cells;
       m += (size_t)gridDim.x * blockDim.x) {
    if (gid[m] == 0) continue;  // no_pt
    const int x = (int)(m % f.pitch), y = (int)(m / f.pitch);
    if (stage == 1) {
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const size_t o = m + v * f.plane;
        utmp[o] = u[o];
        u[o] = u[o] + dt * td[o];
      }
    } else if (x >= x0 && x <= x1 && y >= y0 && y <= y1) {
      const double b = stage == 2 ? 0.75 : 1.0 / 3.0;
      const double b_m = stage == 2 ? 0.25 : 2.0 / 3.0;
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const size_t o = m + v * f.plane;
        u[o] = b * utmp[o] + b_m * (u[o] + dt * td[o]);
      }
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
  Field f;
  f.nx = nx;
  f.ny = ny;
  f.pitch = nx;
  f.plane = (size_t)nx * ny;
  // the faces of a point at least BC points inside the grid stay inside it
  const int x0 = std::max(x_borders[0] - 1, BC), x1 = std::min(x_borders[1] - 1, nx - 1 - BC);
  const int y0 = std::max(y_borders[0] - 1, BC), y1 = std::min(y_borders[1] - 1, ny - 1 - BC);
  if (x0 > x1 || y0 > y1) return DIM2D_OK;
  const long long cells = (long long)(x1 - x0 + 1) * (y1 - y0 + 1);
  k_time_dev_masked<<<(unsigned)((cells + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      nodes, grdpts_id, f, 1.0 / dx, 1.0 / dy, make_const(*p), x0, x1, y0, y1, time_dev);
  const cudaError_t e = cudaGetLastError();
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
  const long long blocks = std::min<long long>((f.plane + 255) / 256, 148 * 8);
  k_rk_stage_masked<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      stage, nodes, nodes_tmp, time_dev, grdpts_id, f, dt, x_borders[0] - 1, x_borders[1] - 1,
      y_borders[0] - 1, y_borders[1] - 1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "rk_stage_masked");
  return DIM2D_OK;
}

}  // extern "C"
