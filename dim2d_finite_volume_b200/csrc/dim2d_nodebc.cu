// dim2d_nodebc.cu -- launches of the node boundary pass (one field, or
// every domain of a batch); the per-cell work is node_bc_cell() in
// dim2d_nodebc.cuh.
#include "dim2d_nodebc.cuh"

namespace dim2d {

namespace {
// the stage launch that follows may start at once (programmatic dependent
// launch); its warps that read this pass's ghost cells wait for its end
__device__ __forceinline__ void allow_dependents() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

__global__ void __launch_bounds__(128) k_node_bc(NodeBcArgs a) {
  allow_dependents();
  node_bc_cell(a, blockIdx.x * blockDim.x + threadIdx.x);
}

// node boundary arguments of domain i of a batched launch
__host__ __device__ __forceinline__ NodeBcArgs batch_node_args(const NodeBcBatchArgs& P, int i) {
  const NodeBcDomain& d = P.d[i];
  NodeBcArgs a;
  a.utmp = d.utmp;
  a.u = d.u;
  a.f = d.f;
  a.dx = d.dx;
  a.dy = d.dy;
  a.rdx = d.rdx;
  a.rdy = d.rdy;
  a.t = 0.0;
  a.xmap0 = d.xmap0;
  a.ymap0 = d.ymap0;
  a.south_wall = d.south_wall;
  a.corners_y = d.corners_y;
  a.open_w = d.open_w;
  a.open_e = d.open_e;
  a.open_n = d.open_n;
  a.status = d.status;
  a.wall = P.wall;
  a.k = P.k;
  return a;
}

// node boundary pass of every domain of a batch: CTAs [cta0_i, cta0_i+1)
// belong to domain i
__global__ void __launch_bounds__(128) k_node_bc_batch(const __grid_constant__ NodeBcBatchArgs P) {
  allow_dependents();
  const int b = blockIdx.x;
  int lo = 0, hi = P.ndom - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P.d[mid].cta0 <= b) lo = mid;
    else hi = mid - 1;
  }
  node_bc_cell(batch_node_args(P, lo), (b - P.d[lo].cta0) * 128 + threadIdx.x);
}
}  // namespace

cudaError_t launch_node_bc(const NodeBcArgs& a, cudaStream_t s) {
  const int n = node_bc_count(a);
  k_node_bc<<<(n + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_node_bc_batch(NodeBcBatchArgs& P, cudaStream_t s) {
  if (P.ndom <= 0) return cudaSuccess;
  if (P.ndom > BATCH_MAX) return cudaErrorInvalidValue;
  long long ctas = 0;
  for (int i = 0; i < P.ndom; i++) {
    P.d[i].cta0 = (int)ctas;
    ctas += (node_bc_count(batch_node_args(P, i)) + 127) / 128;
  }
  if (ctas > 0x7fffffffLL) return cudaErrorInvalidValue;
  void* args[] = {&P};
  return cudaLaunchKernel((const void*)k_node_bc_batch, dim3((unsigned)ctas), dim3(128), args, 0, s);
}

}  // namespace dim2d
