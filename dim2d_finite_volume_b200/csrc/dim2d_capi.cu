// dim2d_capi.cu -- the extern "C" boundary (include/dim2d.h) over the
// sm_100a kernels.  One handle owns one field resident in HBM: three
// pitched FP64 copies (u^n, and the two stage buffers the RK3 scheme
// ping-pongs through) plus x_map / y_map.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "../../include/dim2d.h"
#include "dim2d_kernels.cuh"
#include "dim2d_internal.h"

using namespace dim2d;

namespace {
thread_local std::string g_last_error;
// autotuner cache: (nx, ny, boundary class) -> variant
std::mutex g_tune_mu;
std::map<long long, int> g_tune;
}

namespace dim2d {

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_error(cudaError_t e, const char* where) {
  return set_error(DIM2D_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

DimConst make_const(const dim2d_params& p) {
  DimConst k{};
  k.re = p.re;
  k.we = p.we;
  k.pr = p.pr;
  k.cv_r = p.cv_r;
  k.viscous_r = p.viscous_r;
  k.ire = 1.0 / p.re;
  k.iwe = 1.0 / p.we;
  k.ipr = 1.0 / p.pr;
  k.irepr = 1.0 / (p.re * p.pr);
  k.c15cv = 1.5 / p.cv_r;
  k.c3cv = 3.0 / p.cv_r;
  k.two_mu = 2.0 + p.viscous_r;
  k.c38cv = 3.0 / (8.0 * p.cv_r);
  k.gravity_ac = p.gravity_ac;
  k.gravity = p.gravity;
  return k;
}

int pitch_for(int nx) { return (nx + 15) / 16 * 16; }

// Resolve the reference's per-section bc choices into per-side kinds
// (library_config.py:41-230 maps the presets onto these choices).
int resolve_sides(const int bc_choice[8], const int bc_type[8], int side_kind[8], int* periodic) {
  int nper = 0;
  for (int s = 0; s < 8; s++) {
    const int c = bc_choice[s];
    if (c == DIM2D_PERIODIC_X || c == DIM2D_PERIODIC_Y) {
      side_kind[s] = SIDE_PERIODIC;
      nper++;
    } else if (c == DIM2D_WALL) {
      side_kind[s] = SIDE_WALL;
    } else if (c == DIM2D_HEDSTROM) {
      side_kind[s] = SIDE_OPEN;
    } else if (c == DIM2D_REFLECTION_X || c == DIM2D_REFLECTION_Y) {
      side_kind[s] = SIDE_REFLECT;
    } else {
      return set_error(DIM2D_ERR_ARG, "bc_choice[%d] = %d is not a known choice", s, c);
    }
    if (bc_type[s] < 0 || bc_type[s] > 3)
      return set_error(DIM2D_ERR_ARG, "bc_type[%d] = %d is not a known type", s, bc_type[s]);
  }
  if (nper != 0 && nper != 8)
    return set_error(DIM2D_ERR_UNSUPPORTED,
                     "periodic boundaries must be periodic on all sides (periodic_xy)");
  *periodic = nper == 8;
  return DIM2D_OK;
}

int classify_mirrors(const int bc_choice[8], const int bc_type[8], int* south_wall,
                     int* corners_y) {
  const int N = DIM2D_SIDE_N, S = DIM2D_SIDE_S, E = DIM2D_SIDE_E, W = DIM2D_SIDE_W;
  if (bc_choice[N] != DIM2D_REFLECTION_Y || bc_type[N] != DIM2D_BC_NODES) return 0;
  if (bc_choice[E] != DIM2D_REFLECTION_X || bc_type[E] != DIM2D_BC_NODES) return 0;
  if (bc_choice[W] != DIM2D_REFLECTION_X || bc_type[W] != DIM2D_BC_NODES) return 0;
  int wall = 0;
  if (bc_choice[S] == DIM2D_WALL && bc_type[S] == DIM2D_BC_FLUX_AND_NODE) wall = 1;
  else if (bc_choice[S] != DIM2D_REFLECTION_Y || bc_type[S] != DIM2D_BC_NODES) return 0;
  const int c0 = bc_choice[DIM2D_SIDE_NE];
  if (c0 != DIM2D_REFLECTION_X && c0 != DIM2D_REFLECTION_Y) return 0;
  for (int s = DIM2D_SIDE_NE; s <= DIM2D_SIDE_SW; s++)
    if (bc_choice[s] != c0 || bc_type[s] != DIM2D_BC_NODES) return 0;
  // the wall corners mirror the wall ghost cells along x
  if (wall && c0 != DIM2D_REFLECTION_X) return 0;
  *south_wall = wall;
  *corners_y = c0 == DIM2D_REFLECTION_Y;
  return 1;
}

int classify_open_wall(const int bc_choice[8], const int bc_type[8], const int bc_order[8],
                       int* open_w) {
  auto is = [&](int side, int choice, int type) {
    return bc_choice[side] == choice && bc_type[side] == type;
  };
  auto open = [&](int side) { return is(side, DIM2D_HEDSTROM, DIM2D_BC_TIMEDEV); };
  auto wall = [&](int side) { return is(side, DIM2D_WALL, DIM2D_BC_FLUX_AND_NODE); };
  auto mirror = [&](int side) { return is(side, DIM2D_REFLECTION_X, DIM2D_BC_NODES); };
  if (!open(DIM2D_SIDE_N) || !open(DIM2D_SIDE_E) || !open(DIM2D_SIDE_NE)) return 0;
  if (!wall(DIM2D_SIDE_S) || !wall(DIM2D_SIDE_SE)) return 0;
  int w;
  if (open(DIM2D_SIDE_W) && open(DIM2D_SIDE_NW) && wall(DIM2D_SIDE_SW)) w = 1;
  else if (mirror(DIM2D_SIDE_W) && mirror(DIM2D_SIDE_NW) && mirror(DIM2D_SIDE_SW)) w = 0;
  else return 0;
  if (!w) {
    // half_wall_S_open: the S wall reads the W mirror ghosts, the SW corner
    // mirrors the S wall ghosts (library_config.py:147 orders W, S, SE, SW)
    int pos[9];
    for (int i = 0; i < 9; i++) pos[i] = -1;
    for (int k = 0; k < 8; k++)
      if (bc_order[k] >= 1 && bc_order[k] <= 8) pos[bc_order[k]] = k;
    if (pos[DIM2D_W_EDGE] < 0 || pos[DIM2D_S_EDGE] < 0 || pos[DIM2D_SW_CORNER] < 0 ||
        pos[DIM2D_W_EDGE] > pos[DIM2D_S_EDGE] || pos[DIM2D_SW_CORNER] < pos[DIM2D_S_EDGE])
      return -set_error(DIM2D_ERR_UNSUPPORTED,
                       "create: half_wall_S_open needs the W edge before the S edge and the "
                       "SW corner after it in bc_order");
  }
  *open_w = w;
  return 1;
}

WallConst make_wall(const dim2d_params& p) {
  WallConst w{};
  w.cos_angle = std::cos(p.wall_micro_contact_angle * std::acos(-1.0) / 180.0);
  w.heat_choice = p.wall_heat_source_choice;
  w.qmax = p.wall_maximum_heat_flux;
  w.qcenter = p.wall_heat_source_center;
  w.qvariance = p.wall_heat_source_variance;
  return w;
}

int all_open(const int bc_choice[8], const int bc_type[8]) {
  for (int s = 0; s < 8; s++)
    if (bc_choice[s] != DIM2D_HEDSTROM || bc_type[s] != DIM2D_BC_TIMEDEV) return 0;
  return 1;
}

}  // namespace dim2d

extern "C" {

void dim2d_default_params(dim2d_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->re = 5.0;
  p->we = 10.0;
  p->pr = 20.0;
  p->cv_r = 2.5;
  p->viscous_r = -1.5;
  p->gravity_ac = 0;
  p->gravity = 0.0;
  p->wall_micro_contact_angle = 90.0;
  p->wall_heat_source_choice = 0;
  p->wall_maximum_heat_flux = 0.0;
  p->wall_heat_source_center = 0.0;
  p->wall_heat_source_variance = 1.0;
  p->obc_eigenqties_strategy = 0;
  p->obc_edge_flux_strategy = 0;
  p->T0 = 0.95;
  p->flow_velocity = 0.0;
}

const char* dim2d_last_error(void) { return g_last_error.c_str(); }
const char* dim2d_version(void) { return "dim2d-b200 0.1 (sm_100a)"; }

int dim2d_ini_coordinates(int nx, int ny, double x_min, double x_max, double y_min, double y_max,
                          double* x_map, double* y_map) {
  if (nx < 2 * BC + 2 || ny < 2 * BC + 2 || !x_map || !y_map)
    return set_error(DIM2D_ERR_ARG, "ini_coordinates: bad arguments");
  const double dx = (x_max - x_min) / (nx - 1 - 2 * BC);
  const double dy = (y_max - y_min) / (ny - 1 - 2 * BC);
  for (int i = 1; i <= nx; i++) x_map[i - 1] = x_min + (i - 1 - BC) * dx;
  for (int j = 1; j <= ny; j++) y_map[j - 1] = y_min + (j - 1 - BC) * dy;
  return DIM2D_OK;
}

int dim2d_create(const dim2d_params* p, int nx, int ny, const int bc_choice[8],
                 const int bc_type[8], const int bc_order[8], int precision,
                 dim2d_handle** out) {
  return create_field(p, nx, ny, bc_choice, bc_type, bc_order, precision, nullptr, out);
}

}  // extern "C"

// dim2d_create; with `pool` set, the buffers come from the device's
// stream-ordered pool on that stream (no device-wide synchronisation on
// allocation or release) and the field runs on `pool`
int dim2d::create_field(const dim2d_params* p, int nx, int ny, const int bc_choice[8],
                        const int bc_type[8], const int bc_order[8], int precision,
                        cudaStream_t pool, dim2d_handle** out) {
  if (!p || !bc_choice || !bc_type || !bc_order || !out)
    return set_error(DIM2D_ERR_ARG, "create: null argument");
  *out = nullptr;
  if (nx < 8 || ny < 8)
    return set_error(DIM2D_ERR_ARG, "create: nx, ny must be >= 8 (got %d x %d)", nx, ny);
  if (nx > 65536 || ny > 65536)
    return set_error(DIM2D_ERR_ARG, "create: nx, ny must be <= 65536");
  if (precision != DIM2D_FP64 && precision != DIM2D_MIXED)
    return set_error(DIM2D_ERR_ARG, "create: unknown precision %d", precision);
  if (!(p->re > 0) || !(p->we > 0) || !(p->pr > 0) || !(p->cv_r > 0))
    return set_error(DIM2D_ERR_ARG, "create: re, we, pr, cv_r must be positive");
  int side_kind[8], periodic = 0;
  int rc = resolve_sides(bc_choice, bc_type, side_kind, &periodic);
  if (rc) return rc;
  const int open = all_open(bc_choice, bc_type);
  int south_wall = 0, corners_y = 0;
  const int mirrors = !periodic && !open && classify_mirrors(bc_choice, bc_type, &south_wall,
                                                             &corners_y);
  int open_w = 0;
  int open_wall = 0;
  if (!periodic && !open && !mirrors) {
    open_wall = classify_open_wall(bc_choice, bc_type, bc_order, &open_w);
    if (open_wall < 0) return -open_wall;
    if (open_wall) south_wall = 1;
  }
  if (!periodic && !open && !mirrors && !open_wall)
    return set_error(DIM2D_ERR_UNSUPPORTED,
                     "create: boundary configuration not provided (periodic_xy, hedstrom_xy, "
                     "reflection_xy, wall_S_reflection, wall_S_open and half_wall_S_open are)");
  if (south_wall && p->wall_heat_source_choice != 0 && !(p->wall_heat_source_variance > 0) &&
      p->wall_heat_source_choice == 2)
    return set_error(DIM2D_ERR_ARG, "create: gaussian heat source needs a positive variance");

  dim2d_handle* h = new dim2d_handle();
  h->p = *p;
  h->k = make_const(*p);
  h->precision = precision;
  h->periodic = periodic;
  h->open_all = open;
  h->mirrors = mirrors;
  h->south_wall = south_wall;
  h->corners_y = corners_y;
  if (open) h->open_mask = OPEN_ALL;
  if (mirrors) h->node_sides = NODE_W | NODE_E | NODE_S | NODE_N;
  if (open_wall) {
    h->open_n = h->open_e = 1;
    h->open_w = open_w;
    h->open_mask = OPEN_N | OPEN_E | OPEN_NE | (open_w ? OPEN_W | OPEN_NW : 0);
    h->node_sides = NODE_S | (open_w ? 0 : NODE_W);
  }
  h->wall = make_wall(*p);
  std::memcpy(h->bc_choice, bc_choice, sizeof h->bc_choice);
  std::memcpy(h->bc_type, bc_type, sizeof h->bc_type);
  std::memcpy(h->bc_order, bc_order, sizeof h->bc_order);
  std::memcpy(h->side_kind, side_kind, sizeof h->side_kind);
  h->f.nx = nx;
  h->f.ny = ny;
  h->f.pitch = pitch_for(nx);
  h->f.plane = (size_t)ny * h->f.pitch;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e != cudaSuccess) {
    delete h;
    return cuda_error(e, "create: cudaGetDevice");
  }
  const size_t bytes = 4 * h->f.plane * sizeof(double);
  h->pool = pool;
  auto alloc = [&](double** b, size_t n) {
    return pool ? cudaMallocAsync((void**)b, n, pool) : cudaMalloc(b, n);
  };
  double** bufs[3] = {&h->A, &h->B, &h->C};
  for (double** b : bufs) {
    e = alloc(b, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      dim2d_destroy(h);
      return set_error(DIM2D_ERR_NOMEM, "create: allocation of %zu bytes failed: %s", bytes,
                       cudaGetErrorString(e));
    }
  }
  e = alloc(&h->x_map, nx * sizeof(double));
  if (e == cudaSuccess) e = alloc(&h->y_map, ny * sizeof(double));
  if (e == cudaSuccess) e = alloc(&h->scalar, 4 * sizeof(double));
  if (e == cudaSuccess) h->status = reinterpret_cast<unsigned int*>(h->scalar + 2);
  if (e == cudaSuccess && !pool)
    e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaGetLastError();
    dim2d_destroy(h);
    return set_error(DIM2D_ERR_NOMEM, "create: allocation failed: %s", cudaGetErrorString(e));
  }
  h->stream = pool ? pool : h->own_stream;
  // keep never-written pitch padding and ghost cells defined
  for (double* b : {h->A, h->B, h->C}) cudaMemsetAsync(b, 0, bytes, h->stream);
  cudaMemsetAsync(h->scalar, 0, 4 * sizeof(double), h->stream);
  *out = h;
  return DIM2D_OK;
}

extern "C" {

int dim2d_destroy(dim2d_handle* h) {
  if (!h) return DIM2D_OK;
  if (h->batch) dim2d_batch_remove(h->batch, h);
  if (h->stream && !h->pool) cudaStreamSynchronize(h->stream);
  if (h->copy_stream) {
    cudaStreamSynchronize(h->copy_stream);
    cudaStreamDestroy(h->copy_stream);
    cudaEventDestroy(h->copy_ready);
    cudaEventDestroy(h->copy_done);
  }
  drop_graphs(h);
  if (h->pplan) {
    persist_free(*h->pplan);
    delete h->pplan;
  }
  for (cudaEvent_t ev : h->prof_ev) cudaEventDestroy(ev);
  // pooled buffers are released in stream order, after the queued work
  auto release = [&](void* b) {
    if (!b) return;
    if (h->pool) cudaFreeAsync(b, h->pool);
    else cudaFree(b);
  };
  release(h->A);
  release(h->B);
  release(h->C);
  release(h->x_map);
  release(h->y_map);
  release(h->scalar);
  release(h->td);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return DIM2D_OK;
}

int dim2d_set_stream(dim2d_handle* h, void* stream) {
  if (!h) return set_error(DIM2D_ERR_ARG, "set_stream: null handle");
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return DIM2D_OK;
}

int dim2d_sync(dim2d_handle* h) {
  if (!h) return set_error(DIM2D_ERR_ARG, "sync: null handle");
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess && h->copy_stream) e = cudaStreamSynchronize(h->copy_stream);
  if (e != cudaSuccess) return cuda_error(e, "sync");
  return DIM2D_OK;
}

int dim2d_upload(dim2d_handle* h, const double* nodes, const double* x_map, const double* y_map,
                 double t) {
  if (!h || !nodes || !x_map || !y_map) return set_error(DIM2D_ERR_ARG, "upload: null argument");
  const Field& f = h->f;
  cudaError_t e = wait_copy_if(h, h->A);  // a pending asynchronous copy of A lands first
  if (e == cudaSuccess) e = wait_copy_if(h, h->B);  // ... or of a stage buffer
  if (e == cudaSuccess) e = wait_copy_if(h, h->C);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(h->A, f.pitch * sizeof(double), nodes, f.nx * sizeof(double),
                                    f.nx * sizeof(double), 4 * (size_t)f.ny,
                                    cudaMemcpyHostToDevice, h->stream);
  // Ghost cells that no boundary operator writes (for a south wall: the
  // energy of both ghost rows and the momenta of the outer one) keep the
  // uploaded values in all three buffers, so the state holds them whichever
  // buffer it is in.  (The reference adds dt times an unset time derivative
  // there, compute_1st_step over all nodes, rk3tvd_steps_module.f:52-100,
  // and never reads them.)
  if (e == cudaSuccess) e = launch_copy_frame(h->A, h->B, h->C, f, h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->x_map, x_map, f.nx * sizeof(double), cudaMemcpyHostToDevice,
                        h->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->y_map, y_map, f.ny * sizeof(double), cudaMemcpyHostToDevice,
                        h->stream);
  if (e != cudaSuccess) return cuda_error(e, "upload");
  // td_operators_class.f:157-158
  const double dx = x_map[1] - x_map[0], dy = y_map[1] - y_map[0];
  if (!(dx > 0) || !(dy > 0)) return set_error(DIM2D_ERR_ARG, "upload: x_map/y_map not increasing");
  // captured step graphs hold dx, dy and the map origins as kernel
  // parameters: keep them only while those are unchanged
  if (!h->uploaded || dx != h->dx || dy != h->dy || x_map[0] != h->xmap0 || y_map[0] != h->ymap0) {
    h->graph_dt = -1.0;
    h->pdt = -1.0;  // and the persistent kernel's tables
  }
  h->dx = dx;
  h->dy = dy;
  h->rdx = 1.0 / h->dx;
  h->rdy = 1.0 / h->dy;
  h->xmap0 = x_map[0];
  h->ymap0 = y_map[0];
  h->x_min = x_map[BC];
  h->x_max = x_map[f.nx - 1 - BC];
  h->y_min = y_map[BC];
  h->y_max = y_map[f.ny - 1 - BC];
  h->t = t;
  h->uploaded = true;
  return DIM2D_OK;
}

int dim2d_download(dim2d_handle* h, double* nodes, double* t) {
  if (!h || !nodes) return set_error(DIM2D_ERR_ARG, "download: null argument");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "download: no state uploaded");
  const Field& f = h->f;
  cudaError_t e = cudaMemcpy2DAsync(nodes, f.nx * sizeof(double), h->A, f.pitch * sizeof(double),
                                    f.nx * sizeof(double), 4 * (size_t)f.ny,
                                    cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_error(e, "download");
  if (t) *t = h->t;
  return check_status(h);
}

int dim2d_download_async(dim2d_handle* h, double* nodes, double* t) {
  if (!h || !nodes) return set_error(DIM2D_ERR_ARG, "download_async: null argument");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "download_async: no state");
  if (h->batch) return set_error(DIM2D_ERR_ARG, "download_async: the field is in a batch");
  cudaError_t e = cudaSuccess;
  if (!h->copy_stream) {
    e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->copy_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->copy_done, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_error(e, "download_async");
  }
  // a previous copy of the other buffer may still be pending: order it first
  if (h->copy_pending) e = cudaStreamWaitEvent(h->stream, h->copy_done, 0);
  const Field& f = h->f;
  if (e == cudaSuccess) e = cudaEventRecord(h->copy_ready, h->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->copy_stream, h->copy_ready, 0);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(nodes, f.nx * sizeof(double), h->A, f.pitch * sizeof(double),
                          f.nx * sizeof(double), 4 * (size_t)f.ny, cudaMemcpyDeviceToHost,
                          h->copy_stream);
  if (e == cudaSuccess) e = cudaEventRecord(h->copy_done, h->copy_stream);
  if (e != cudaSuccess) return cuda_error(e, "download_async");
  h->copy_src = h->A;
  h->copy_pending = true;
  if (t) *t = h->t;
  return DIM2D_OK;
}

int dim2d_copy_done(dim2d_handle* h) {
  if (!h) return set_error(DIM2D_ERR_ARG, "copy_done: null handle");
  if (!h->copy_done) return 1;
  const cudaError_t e = cudaEventQuery(h->copy_done);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) {
    cudaGetLastError();
    return 0;
  }
  return -cuda_error(e, "copy_done");
}

int dim2d_host_alloc(size_t bytes, void** p) {
  if (!p) return set_error(DIM2D_ERR_ARG, "host_alloc: null argument");
  *p = nullptr;
  cudaError_t e = cudaMallocHost(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(DIM2D_ERR_NOMEM, "host_alloc: %zu bytes: %s", bytes, cudaGetErrorString(e));
  }
  return DIM2D_OK;
}

int dim2d_host_free(void* p) {
  if (p) cudaFreeHost(p);
  return DIM2D_OK;
}

int dim2d_device_state(dim2d_handle* h, double** nodes, int* pitch) {
  if (!h) return set_error(DIM2D_ERR_ARG, "device_state: null handle");
  if (nodes) *nodes = h->A;
  if (pitch) *pitch = h->f.pitch;
  return DIM2D_OK;
}

long long dim2d_launch_count(const dim2d_handle* h) { return h ? h->launches : 0; }

int dim2d_set_variant(dim2d_handle* h, int variant) {
  if (!h) return set_error(DIM2D_ERR_ARG, "set_variant: null handle");
  if (variant < 0 || variant >= NUM_VARIANTS)
    return set_error(DIM2D_ERR_ARG, "set_variant: variant %d out of range", variant);
  h->variant = variant;
  h->graph_dt = -1.0;  // the captured kernels belong to the previous variant
  return DIM2D_OK;
}

int dim2d_get_variant(const dim2d_handle* h) { return h ? h->variant : -1; }

int dim2d_autotune(dim2d_handle* h, int* chosen, double* times_ms) {
  if (!h) return set_error(DIM2D_ERR_ARG, "autotune: null handle");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "autotune: no state");
  const int cls = h->periodic ? 0
                  : h->open_all ? 1
                  : h->open_mask ? 4 + h->open_w
                  : h->south_wall ? 2 : 3;
  // size, boundary class (bits 0-2) and precision (bit 3): the FP64 and the
  // mixed-precision kernels of one size may prefer different shapes
  const long long key = ((long long)h->f.nx << 32) ^ ((long long)h->f.ny << 4) ^
                        ((long long)(h->precision == DIM2D_MIXED) << 3) ^ cls;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end() && !times_ms) {
      h->variant = it->second;
      if (chosen) *chosen = h->variant;
      return DIM2D_OK;
    }
  }
  cudaError_t e = wait_copy_if(h, h->B);  // the dry steps write B and C
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = 0;
  double best_ms = 1e30;
  const int saved = h->variant;
  for (int v = 0; v < NUM_VARIANTS; v++) {
    h->variant = v;
    // a dry RK3 step: the three stages with their boundary passes, dt = 0,
    // writing only the stage buffers B and C (A, the state, is read only
    // and the buffers are not swapped)
    auto dry_step = [&]() -> cudaError_t {
      if (v == PERSIST_VARIANT)
        return persist_steps(h, 0.0, 1, 0.0) == DIM2D_OK ? cudaSuccess : cudaErrorLaunchFailure;
      const double* in[3] = {h->A, h->B, h->C};
      double* out[3] = {h->B, h->C, h->B};
      for (int st = 1; st <= 3; st++) {
        const StageArgs a = make_stage_args(h, in[st - 1], out[st - 1], 0.0, st);
        cudaError_t r = launch_stage_work(h, a, 1);
        if (r != cudaSuccess) return r;
        if (!h->periodic && !h->open_all && apply_bc_on_nodes(h, h->A, out[st - 1]))
          return cudaErrorLaunchFailure;
      }
      return cudaSuccess;
    };
    e = dry_step();
    if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
    const int reps = 3;
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = dry_step();
    if (e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) break;
    const double per = ms / reps;
    if (times_ms) times_ms[v] = per;
    if (per < best_ms) {
      best_ms = per;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) {
    h->variant = saved;
    return cuda_error(e, "autotune");
  }
  h->variant = best;
  h->graph_dt = -1.0;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = best;
  }
  if (chosen) *chosen = best;
  return DIM2D_OK;
}

int dim2d_profile(dim2d_handle* h, int enable) {
  if (!h) return set_error(DIM2D_ERR_ARG, "profile: null handle");
  h->prof = enable != 0;
  h->prof_used = 0;
  return DIM2D_OK;
}

int dim2d_profile_read(dim2d_handle* h, double* ms, long long* launches) {
  if (!h || !ms || !launches) return set_error(DIM2D_ERR_ARG, "profile_read: null argument");
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_error(e, "profile_read");
  double tot = 0.0;
  for (size_t i = 0; i + 1 < h->prof_used; i += 2) {
    float m = 0.f;
    e = cudaEventElapsedTime(&m, h->prof_ev[i], h->prof_ev[i + 1]);
    if (e != cudaSuccess) return cuda_error(e, "profile_read elapsed");
    tot += m;
  }
  *ms = tot;
  *launches = (long long)(h->prof_used / 2);
  return DIM2D_OK;
}

int dim2d_apply_bc_on_nodes(dim2d_handle* h) {
  if (!h) return set_error(DIM2D_ERR_ARG, "apply_bc_on_nodes: null handle");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "apply_bc_on_nodes: no state");
  cudaError_t e = wait_copy_if(h, h->A);
  if (e != cudaSuccess) return cuda_error(e, "apply_bc_on_nodes");
  return apply_bc_on_nodes(h, h->A, h->A);
}

int dim2d_time_dev(dim2d_handle* h, double* time_dev) {
  if (!h || !time_dev) return set_error(DIM2D_ERR_ARG, "time_dev: null argument");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "time_dev: no state");
  const Field& f = h->f;
  cudaError_t e = cudaSuccess;
  if (!h->td)
    e = h->pool ? cudaMallocAsync((void**)&h->td, 4 * f.plane * sizeof(double), h->pool)
                : cudaMalloc(&h->td, 4 * f.plane * sizeof(double));
  if (e != cudaSuccess) return set_error(DIM2D_ERR_NOMEM, "time_dev: %s", cudaGetErrorString(e));
  // td_operators_class.f:150-154: every cell starts at debug_real
  e = launch_fill(h->td, 9.9692099683868690e+36, 4 * f.plane, h->stream);
  h->launches++;
  // interior cells, and on open fields the ghost cells
  // (bc_operators_hedstrom_xy_class.f:182-496)
  if (e == cudaSuccess) e = launch_stage_work(h, make_stage_args(h, h->A, h->td, 0.0, 0), 0);
  if (e != cudaSuccess) return cuda_error(e, "time_dev");
  e = cudaMemcpy2DAsync(time_dev, f.nx * sizeof(double), h->td, f.pitch * sizeof(double),
                        f.nx * sizeof(double), 4 * (size_t)f.ny, cudaMemcpyDeviceToHost,
                        h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_error(e, "time_dev copy");
  return DIM2D_OK;
}

int dim2d_cfl_dt(dim2d_handle* h, double cfl, double* dt) {
  if (!h || !dt || !(cfl > 0)) return set_error(DIM2D_ERR_ARG, "cfl_dt: bad argument");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "cfl_dt: no state");
  cudaError_t e = launch_cfl_max(h->A, h->f, h->k, h->scalar, h->stream);
  h->launches++;
  double smax = 0.0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&smax, h->scalar, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_error(e, "cfl_dt");
  if (!(smax > 0) || !std::isfinite(smax))
    return set_error(DIM2D_ERR_ARG, "cfl_dt: max(c+|u|) = %g is not a positive finite value", smax);
  *dt = cfl * std::fmin(h->dx, h->dy) / smax;
  return DIM2D_OK;
}

int dim2d_step(dim2d_handle* h, double dt, int nsteps) {
  if (!h) return set_error(DIM2D_ERR_ARG, "step: null handle");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "step: no state uploaded");
  if (nsteps < 0 || !std::isfinite(dt)) return set_error(DIM2D_ERR_ARG, "step: bad dt/nsteps");
  if (h->batch) return set_error(DIM2D_ERR_ARG, "step: the field is advanced by its batch");
  return rk3_steps(h, dt, nsteps);
}

int dim2d_set_graphs(dim2d_handle* h, int enable) {
  if (!h) return set_error(DIM2D_ERR_ARG, "set_graphs: null handle");
  h->use_graphs = enable != 0;
  return DIM2D_OK;
}

}  // extern "C"
