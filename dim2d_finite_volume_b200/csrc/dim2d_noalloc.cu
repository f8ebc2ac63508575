// dim2d_noalloc.cu -- dim2d_step_noalloc: the RK3 time step without any
// device allocation.
//
// dim2d_step keeps its two RK3 stage copies in buffers that dim2d_create
// obtains with cudaMalloc.  Some callers cannot allocate device memory:
// hosts that hand every byte of HBM out from their own pool or arena (a
// serving loop that pre-sizes memory for admitted requests, a Fortran
// code whose arrays live in CUDA-Fortran or OpenACC managed storage), and
// time-stepping loops that must not allocate because cudaMalloc
// synchronises the device.  For them this entry point takes the field as
// a device pointer and runs the same stage kernels with the stage copies
// placed in one file-scope __device__ array of fixed size.
//
// Limits and sharing rules (also stated in include/dim2d.h):
//   * at most DIM2D_NOALLOC_MAX_CELLS = nx*ny cells (ghosts included);
//     the array holds 2 x 4 x that many doubles (16 MiB) on every GPU
//     that loads the library, until the process exits;
//   * every call on a device uses the same array, which keeps the last
//     call's contents: each call clears the part it uses before stepping,
//     and calls that overlap on the GPU (different streams, or host
//     threads not ordered by the caller) race on it;
//   * the first call in a CUDA context, with that context current, looks
//     up the array's device address (cudaGetSymbolAddress) and keeps it
//     for that context; make that first call before any stream capture.
//     The cache is keyed by the context's unique id, so a new context on
//     the same device (after cudaDeviceReset, or one made current with
//     cuCtxSetCurrent) gets its own lookup;
//   * boundary configurations: periodic_xy and hedstrom_xy only (the ones
//     without a node boundary pass: no wall status word is needed);
//   * after a non-zero return the contents of `nodes` are undefined.
#include <cuda.h>

#include <cmath>
#include <mutex>

#include "dim2d_internal.h"

using namespace dim2d;

namespace {

constexpr size_t kMaxCells = DIM2D_NOALLOC_MAX_CELLS;
constexpr size_t kScratchDoubles = 2 * 4 * kMaxCells;
constexpr int kMaxContexts = 64;

// Two stage copies of the field; only device code and the looked-up
// address below may touch it (in host code the name is a host-side
// stand-in, not a device address).
__device__ __align__(256) double g_stage_scratch[kScratchDoubles];

// Unique id of the current CUDA context, through the driver entry point
// (no link-time dependency on libcuda): cuCtxGetCurrent + cuCtxGetId.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// 0 and *id set when a context is current; 1 when none is; else an error
int current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    fn = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(fn);
  });
  if (!get_current || !get_id)
    return set_error(DIM2D_ERR_CUDA, "step_noalloc: driver entry points cuCtxGetCurrent / "
                                     "cuCtxGetId not available");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS)
    return set_error(DIM2D_ERR_CUDA, "step_noalloc: cuCtxGetCurrent failed");
  if (!ctx) return 1;
  if (get_id(ctx, id) != CUDA_SUCCESS)
    return set_error(DIM2D_ERR_CUDA, "step_noalloc: cuCtxGetId failed");
  return 0;
}

std::mutex g_scratch_mu;
struct ScratchEntry {
  unsigned long long ctx_id;
  double* addr;
};
ScratchEntry g_scratch[kMaxContexts] = {};
int g_scratch_n = 0;

int lookup_symbol(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_stage_scratch);
  if (e != cudaSuccess || !p)
    return cuda_error(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                      "step_noalloc: cudaGetSymbolAddress");
  *out = static_cast<double*>(p);
  return DIM2D_OK;
}

int scratch_address(double** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  double* addr = nullptr;
  if (rc == 1) {
    // no context yet: the runtime's first call binds the current device's
    // primary context, then that context is the key
    rc = lookup_symbol(&addr);
    if (rc) return rc;
    rc = current_context_id(&id);
    if (rc == 1) return set_error(DIM2D_ERR_CUDA, "step_noalloc: no current CUDA context");
  }
  if (rc) return rc;
  for (int i = 0; i < g_scratch_n; i++)
    if (g_scratch[i].ctx_id == id) {
      *out = g_scratch[i].addr;
      return DIM2D_OK;
    }
  if (!addr) {
    rc = lookup_symbol(&addr);
    if (rc) return rc;
  }
  // a full table reuses a slot (the context that held it gets looked up
  // again if it is still alive)
  const int slot = g_scratch_n < kMaxContexts ? g_scratch_n++ : (int)(id % kMaxContexts);
  g_scratch[slot] = ScratchEntry{id, addr};
  *out = addr;
  return DIM2D_OK;
}

}  // namespace

extern "C" int dim2d_step_noalloc(const dim2d_params* p, int nx, int ny, const int bc_choice[8],
                                  const int bc_type[8], const int bc_order[8], double* nodes,
                                  const double* x_map, const double* y_map, double dt,
                                  int nsteps, void* stream) {
  if (!p || !bc_choice || !bc_type || !bc_order || !nodes || !x_map || !y_map)
    return set_error(DIM2D_ERR_ARG, "step_noalloc: null argument");
  if (nx < 8 || ny < 8)
    return set_error(DIM2D_ERR_ARG, "step_noalloc: nx, ny must be >= 8 (got %d x %d)", nx, ny);
  if ((size_t)nx * (size_t)ny > kMaxCells)
    return set_error(DIM2D_ERR_ARG,
                     "step_noalloc: nx*ny = %zu exceeds the fixed scratch limit of %zu cells "
                     "(DIM2D_NOALLOC_MAX_CELLS); use dim2d_create/dim2d_step for larger fields",
                     (size_t)nx * (size_t)ny, kMaxCells);
  if (nsteps < 0 || !std::isfinite(dt)) return set_error(DIM2D_ERR_ARG, "step_noalloc: bad dt/nsteps");
  if (!(p->re > 0) || !(p->we > 0) || !(p->pr > 0) || !(p->cv_r > 0))
    return set_error(DIM2D_ERR_ARG, "step_noalloc: re, we, pr, cv_r must be positive");
  int side_kind[8], periodic = 0;
  int rc = resolve_sides(bc_choice, bc_type, side_kind, &periodic);
  if (rc) return rc;
  const int open = all_open(bc_choice, bc_type);
  if (!periodic && !open)
    return set_error(DIM2D_ERR_UNSUPPORTED,
                     "step_noalloc: configuration not provided (periodic_xy and hedstrom_xy are)");
  const double dx = x_map[1] - x_map[0], dy = y_map[1] - y_map[0];
  if (!(dx > 0) || !(dy > 0)) return set_error(DIM2D_ERR_ARG, "step_noalloc: x_map/y_map not increasing");

  double* scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc) return rc;

  // a handle on the stack that owns nothing: A = the caller's field,
  // B and C = the two halves of the static scratch
  dim2d_handle h;
  h.p = *p;
  h.k = make_const(*p);
  h.precision = DIM2D_FP64;
  h.periodic = periodic;
  h.open_all = open;
  h.open_mask = open ? OPEN_ALL : 0;
  for (int s = 0; s < 8; s++) {
    h.bc_choice[s] = bc_choice[s];
    h.bc_type[s] = bc_type[s];
    h.bc_order[s] = bc_order[s];
    h.side_kind[s] = side_kind[s];
  }
  h.f.nx = nx;
  h.f.ny = ny;
  h.f.pitch = nx;  // the caller's Fortran layout
  h.f.plane = (size_t)nx * ny;
  h.A = nodes;
  h.B = scratch;
  h.C = scratch + 4 * h.f.plane;
  h.dx = dx;
  h.dy = dy;
  h.rdx = 1.0 / dx;
  h.rdy = 1.0 / dy;
  h.uploaded = true;
  h.stream = static_cast<cudaStream_t>(stream);

  // the array keeps the previous call's contents: start from zeros
  cudaError_t e = cudaMemsetAsync(scratch, 0, 2 * 4 * h.f.plane * sizeof(double), h.stream);
  if (e != cudaSuccess) return cuda_error(e, "step_noalloc: clear scratch");
  for (int s = 0; s < nsteps; s++) {
    rc = rk3_step(&h, dt);
    if (rc) return rc;
  }
  // after an odd number of steps the newest state sits in the scratch
  if (h.A != nodes) {
    e = cudaMemcpyAsync(nodes, h.A, 4 * h.f.plane * sizeof(double), cudaMemcpyDeviceToDevice,
                        h.stream);
    if (e != cudaSuccess) return cuda_error(e, "step_noalloc: copy back");
  }
  return DIM2D_OK;
}
