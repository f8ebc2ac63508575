// dim2d_kernels.cuh -- launch interface of the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include "dim2d_physics.cuh"

namespace dim2d {

constexpr int BC = 2;  // bc_size, parameters_input.f:81

// Device view of one field: 4 planes of ny rows, `pitch` doubles per row
// (pitch >= nx, even, so every row starts on a 16-byte boundary).
struct Field {
  int nx, ny, pitch;
  size_t plane;  // ny * pitch
};

// Boundary layout of a field, resolved on the host from bc_choice/bc_type.
enum SideKind : int { SIDE_PERIODIC = 0, SIDE_WALL = 1, SIDE_OPEN = 2, SIDE_REFLECT = 3 };

struct StageArgs {
  const double* __restrict__ uin;  // state the stencil reads
  const double* __restrict__ u0;   // u^n (stages 2 and 3)
  double* __restrict__ uout;       // stage output
  Field f;
  double dx, dy, rdx, rdy;         // grid step and inverses
  double dt;
  double b;                        // stage weight: out = b*u0 + (1-b)*(uin + dt*L)
  int stage;                       // 1, 2, 3
  int periodic;                    // write periodic ghost images of edge cells
  int wall_w, wall_e, wall_s, wall_n;  // wall flux override on that side
  DimConst k;
};

// Tile of the fused interior kernel: TX x TY interior cells per CTA.
constexpr int TILE_X = 32;
constexpr int TILE_Y = 8;
size_t interior_smem_bytes();

cudaError_t launch_interior_stage(const StageArgs& a, cudaStream_t s);
cudaError_t launch_time_dev(const double* uin, double* td, const Field& f, double rdx, double rdy,
                            const DimConst& k, cudaStream_t s);
// open (Hedstrom) ghost cells of a field open on all sides; mode 0 writes
// L(u) into a.uout, mode 1 the RK stage update
cudaError_t launch_open_ghosts(const StageArgs& a, int mode, cudaStream_t s);
cudaError_t launch_fill(double* p, double v, size_t n, cudaStream_t s);
cudaError_t launch_periodic_ghosts(double* u, const Field& f, cudaStream_t s);
cudaError_t launch_cfl_max(const double* u, const Field& f, const DimConst& k, double* out,
                           cudaStream_t s);

}  // namespace dim2d
