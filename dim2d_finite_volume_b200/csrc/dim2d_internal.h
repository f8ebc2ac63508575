// dim2d_internal.h -- host-side handle and helpers behind include/dim2d.h.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <vector>

#include "../../include/dim2d.h"
#include "dim2d_kernels.cuh"

// Work tables of the persistent kernel for a set of fields of one precision
// (dim2d_persist.cu): per-field descriptors, the per-step item list and the
// per-band strip+ghost item counts in device memory, and the launch
// counters.  The tables hold the fields' buffers as they were when built;
// launches pass the step parity since then.
struct PersistPlan {
  dim2d::PDomain* dom = nullptr;
  dim2d::PItem* items = nullptr;
  int* sg = nullptr;
  unsigned long long* ctr = nullptr;  // [0] next item, band counters, node counters
  unsigned int* ctl = nullptr;        // [0] abort flag, [1] error word
  long long items_per_step = 0;
  int nfields = 0;
  int nbands = 0;
  int rows = 0;   // rows per band / strip item
  int ctas = 0;   // CTAs of the last launch
  bool mixed = false;
  bool valid = false;
  dim2d::DimConst k{};
  dim2d::WallConst wall{};
};

struct dim2d_handle {
  int device = 0;
  dim2d_params p{};
  dim2d::DimConst k{};
  int precision = 0;
  int periodic = 0;
  int open_all = 0;  // hedstrom_xy: every section open, type bc_timedev
  int mirrors = 0;     // reflection_xy or wall_S_reflection (node pass kernel)
  int south_wall = 0;  // wall on S: wall_S_reflection, wall_S_open, half_wall_S_open
  int corners_y = 0;   // corner sections are reflection_y
  // open (Hedstrom) sections: dim2d::OPEN_* mask of the time-integrated ghost
  // sections (all of them for hedstrom_xy) and the open sides of the mixed
  // presets wall_S_open / half_wall_S_open
  int open_mask = 0;
  int open_w = 0, open_e = 0, open_n = 0;
  // dim2d::NODE_* sides whose ghost cells the node pass writes (mirrors, wall)
  int node_sides = 0;
  dim2d::WallConst wall{};
  unsigned int* status = nullptr;  // wall root status word (device)
  double xmap0 = 0, ymap0 = 0;     // x_map(1), y_map(1)
  int variant = 0;                 // stage-kernel variant (dim2d_set_variant)
  struct dim2d_batch* batch = nullptr;  // batch this field belongs to, if any
  // dim2d_download_async: side stream, its events, and the buffer being copied
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
  const double* copy_src = nullptr;
  bool copy_pending = false;
  int bc_choice[8]{}, bc_type[8]{}, bc_order[8]{};
  int side_kind[8]{};
  dim2d::Field f{};
  // A = u^n (the field), B and C = stage buffers
  double* A = nullptr;
  double* B = nullptr;
  double* C = nullptr;
  double* td = nullptr;  // time_dev buffer, allocated on first use
  double* x_map = nullptr;
  double* y_map = nullptr;
  double* scalar = nullptr;  // [0] CFL reduction, [2] wall status word (status),
                             // [3] health word of a served request (health_word)
  double dx = 0, dy = 0, rdx = 0, rdy = 0;
  double x_min = 0, x_max = 0, y_min = 0, y_max = 0;
  double t = 0;
  bool uploaded = false;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t pool = nullptr;  // buffers from the stream-ordered pool on this stream
  long long launches = 0;
  // captured one-step graphs, one per buffer parity (which buffer holds
  // u^n); slot i is valid for graph_dt[i] and graph_A[i].  graph_dt = -1
  // invalidates both (set by anything that changes kernel parameters).
  bool use_graphs = true;
  cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
  double graph_dt = -1.0;
  const double* graph_A[2] = {nullptr, nullptr};
  long long graph_launches[2] = {0, 0};  // kernel launches in one replay
  // stage-kernel variant 6: the persistent kernel, tables built on first
  // use (pplan), steps since then (pparity)
  PersistPlan* pplan = nullptr;
  dim2d::PDomain pdom0{};  // buffers the tables were built with
  double pdt = -1.0;       // dt the tables hold (-1: rebuild)
  // live timing of the interior stage kernel (dim2d_profile)
  bool prof = false;
  std::vector<cudaEvent_t> prof_ev;  // start/stop pairs
  size_t prof_used = 0;
};

namespace dim2d {
int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* where);
DimConst make_const(const dim2d_params& p);
int pitch_for(int nx);
int resolve_sides(const int bc_choice[8], const int bc_type[8], int side_kind[8], int* periodic);
// 1 if all eight sections are hedstrom_choice with type bc_timedev
int all_open(const int bc_choice[8], const int bc_type[8]);
}  // namespace dim2d

// Mirror / south-wall configurations (library_config.py:58-115): returns 1
// and sets the flags when bc_choice/bc_type are reflection_xy or
// wall_S_reflection.
namespace dim2d {
int classify_mirrors(const int bc_choice[8], const int bc_type[8], int* south_wall,
                     int* corners_y);
// wall_S_open or half_wall_S_open (library_config.py:118-150): returns 1
// and sets *open_w (1 for wall_S_open, 0 for half_wall_S_open's mirror W);
// returns minus an error code (set_error) for a section order the kernels
// do not reproduce, 0 for any other configuration
int classify_open_wall(const int bc_choice[8], const int bc_type[8], const int bc_order[8],
                       int* open_w);
WallConst make_wall(const dim2d_params& p);
// dim2d_create; pool != nullptr: stream-ordered allocations on `pool`,
// which also becomes the field's stream
int create_field(const dim2d_params* p, int nx, int ny, const int bc_choice[8],
                 const int bc_type[8], const int bc_order[8], int precision, cudaStream_t pool,
                 dim2d_handle** out);
}  // namespace dim2d

// dim2d_step.cu
dim2d::StageArgs make_stage_args(const dim2d_handle* h, const double* uin, double* uout,
                                 double dt, int st);
int rk3_step(dim2d_handle* h, double dt);
// nsteps RK3 steps; each step replays a captured CUDA graph when graphs are
// enabled and the handle is not profiling
int rk3_steps(dim2d_handle* h, double dt, int nsteps);
// variant 6 (the persistent kernel): nsteps steps as one launch;
// dt_scale 0 = dry step of the autotuner
constexpr int PERSIST_VARIANT = 6;
int persist_steps(dim2d_handle* h, double dt, int nsteps, double dt_scale);
// the complete work of one stage (mode 1) or time derivative (mode 0): the
// stage kernel and, on open fields where the stage kernel does not cover
// them, the ghost-cell kernel; counts launches, profiles the stage kernel
cudaError_t launch_stage_work(dim2d_handle* h, const dim2d::StageArgs& a, int mode);
int apply_bc_on_nodes(dim2d_handle* h, const double* nodes_tmp, double* nodes);
int check_status(dim2d_handle* h);
// device word the serving loop's check sets: bit 0 a non-finite value in the
// field, bit 1 the wall status word set (zero at creation)
inline unsigned int* health_word(dim2d_handle* h) {
  return reinterpret_cast<unsigned int*>(h->scalar + 3);
}
// bracket one launch with profiling events (no-op unless h->prof)
void prof_begin(dim2d_handle* h);
void prof_end(dim2d_handle* h);
void drop_graphs(dim2d_handle* h);
// before work on h->stream writes `target`: wait for a pending
// dim2d_download_async copy whose source it is
cudaError_t wait_copy_if(dim2d_handle* h, const double* target);

// dim2d_persist.cu
void persist_free(PersistPlan& pl);
int persist_build(PersistPlan& pl, const std::vector<dim2d_handle*>& hs,
                  const std::vector<double>& dts, int rows, cudaStream_t s);
// nsteps steps of every field of the plan (dt_scale 0: dry steps that
// write only the stage buffers); step0 = steps taken since the build
cudaError_t persist_launch(PersistPlan& pl, int nsteps, int step0, double dt_scale,
                           unsigned long long wait_ns, long long withhold, cudaStream_t s);
// reads and clears the plan's error word (synchronous): DIM2D_ERR_TIMEOUT
// if a launch stopped at a wait that ran out
int persist_error(PersistPlan& pl);
