// dim2d_open.cu -- stand-alone kernel of the open-boundary ghost cells
// (device code in dim2d_open.cuh).
#include "dim2d_open.cuh"

namespace dim2d {

namespace {

template <int MODE>
__global__ void __launch_bounds__(128) k_open_ghosts(StageArgs a) {
  open_ghost_cell(a, blockIdx.x * blockDim.x + threadIdx.x, MODE);
}

}  // namespace

cudaError_t launch_open_ghosts(const StageArgs& a, int mode, cudaStream_t s) {
  const int total = open_ghost_count(a.f, a.open);
  if (total == 0) return cudaSuccess;
  const int blocks = (total + 127) / 128;
  if (mode == 0) k_open_ghosts<0><<<blocks, 128, 0, s>>>(a);
  else k_open_ghosts<1><<<blocks, 128, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace dim2d
