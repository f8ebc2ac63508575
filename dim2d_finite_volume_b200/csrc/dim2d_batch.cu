// dim2d_batch.cu -- many fields advanced together (include/dim2d.h,
// dim2d_batch_*).  No counterpart in the reference, which advances one
// field per process (td_integrator_class.f:103-161 per field).
//
// Members are ordinary handles (dim2d_create + dim2d_upload); the batch
// borrows their device buffers.  Members are grouped by boundary kind:
//   G_PERIODIC  periodic_xy            strip kernel writes the ghost images
//   G_OPEN      hedstrom_xy            ghost cells fused into the launch
//   G_WALL      wall_S_reflection,     strip kernel + node boundary pass; the
//               wall_S_open,           open sections' ghost cells fused into
//               half_wall_S_open       the launch
//   G_MIRROR    reflection_xy          strip kernel + node boundary pass
// and by precision (groups 4..7: the same kinds, DIM2D_MIXED fields).
// One RK stage of a group is one batched launch over all its domains (plus
// one batched node pass), so a step is at most 8 x 3 x 2 launches however
// many domains there are.  The groups are independent: a captured step
// graph holds one chain per group as parallel branches, so the kinds
// overlap on the device.  Two graphs are kept, one per buffer parity
// (which of A/B holds u^n), and rebuilt when members, dt or shapes change.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "dim2d_internal.h"
#include "dim2d_nodebc.cuh"
#include "dim2d_open.cuh"

using namespace dim2d;

namespace {
enum Group : int { G_PERIODIC = 0, G_OPEN, G_WALL, G_MIRROR, NKINDS, NGROUPS = 2 * NKINDS };
constexpr int NSHAPES = 5;  // strip shapes, as dim2d_set_variant 1..5

int group_of(const dim2d_handle* h) {
  const int mix = h->precision == DIM2D_MIXED ? NKINDS : 0;
  if (h->periodic) return G_PERIODIC + mix;
  if (h->open_all) return G_OPEN + mix;
  return (h->south_wall ? G_WALL : G_MIRROR) + mix;
}
int kind_of(int g) {
  g %= NKINDS;
  return g == G_OPEN ? BK_OPEN : (g == G_WALL ? BK_WALL : BK_PLAIN);
}
bool has_node_pass(int g) { return g % NKINDS == G_WALL || g % NKINDS == G_MIRROR; }
bool is_mixed(int g) { return g >= NKINDS; }
}  // namespace

struct dim2d_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t side[NGROUPS] = {};
  cudaEvent_t fork = nullptr, join[NGROUPS] = {}, done = nullptr;
  std::vector<dim2d_handle*> m;
  std::vector<double> dt;
  dim2d_params p{};
  int shape[NGROUPS] = {1, 1, 1, 1, 1, 1, 1, 1};
  bool use_graphs = true;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_launches[2] = {0, 0};
  bool graphs_valid = false;
  int parity = 0;
  long long launches = 0;
  // persistent mode (dim2d_batch_set_persistent): one kernel per precision
  // advances all members of that precision by the requested steps
  bool persistent = false;
  PersistPlan plan[2];
  int rows = 16;                      // rows per strip item
  long long pparity = 0;              // steps since the plans were built
  unsigned long long wait_ns = 2000000000ull;
  long long withhold = -1;
};

namespace {

void drop_batch_graphs(dim2d_batch* b) {
  for (int i = 0; i < 2; i++) {
    if (b->graph[i]) cudaGraphExecDestroy(b->graph[i]);
    b->graph[i] = nullptr;
  }
  b->graphs_valid = false;
  b->parity = 0;
}

// Stage `st` of the members of group g (indices idx): batched stage launch,
// then the batched node pass.  in/out per stage: 1: A->B, 2: B->C, 3: C->B,
// u^n = A.  dt_scale 0 gives the dry step of the autotuner.
cudaError_t group_stage(dim2d_batch* b, int g, const std::vector<int>& idx, int st, int shape,
                        double dt_scale, cudaStream_t s) {
  static thread_local BatchStageArgs P;
  static thread_local NodeBcBatchArgs Q;
  for (size_t c0 = 0; c0 < idx.size(); c0 += BATCH_MAX) {
    const int n = (int)std::min<size_t>(BATCH_MAX, idx.size() - c0);
    const dim2d_handle* h0 = b->m[idx[c0]];
    P.k = h0->k;
    P.wall = h0->wall;
    P.stage = st;
    P.b = st == 2 ? 0.75 : (st == 3 ? 1.0 / 3.0 : 0.0);  // rk3tvd_steps_module.f:225,444
    P.ndom = n;
    Q.k = h0->k;
    Q.wall = h0->wall;
    Q.ndom = n;
    for (int j = 0; j < n; j++) {
      const int i = idx[c0 + j];
      dim2d_handle* h = b->m[i];
      const double* in = st == 1 ? h->A : (st == 2 ? h->B : h->C);
      double* out = st == 2 ? h->C : h->B;
      BatchDomain& d = P.d[j];
      d.f = h->f;
      d.uin = in;
      d.u0 = h->A;
      d.uout = out;
      d.dx = h->dx;
      d.dy = h->dy;
      d.rdx = h->rdx;
      d.rdy = h->rdy;
      d.dt = b->dt[i] * dt_scale;
      d.xmap0 = h->xmap0;
      d.periodic = h->periodic;
      d.wall_s = h->south_wall;
      d.open = h->open_mask;
      d.node_sides = st >= 2 && has_node_pass(g) ? h->node_sides : 0;
      NodeBcDomain& q = Q.d[j];
      q.utmp = h->A;
      q.u = out;
      q.f = h->f;
      q.dx = h->dx;
      q.dy = h->dy;
      q.rdx = h->rdx;
      q.rdy = h->rdy;
      q.xmap0 = h->xmap0;
      q.ymap0 = h->ymap0;
      q.south_wall = h->south_wall;
      q.corners_y = h->corners_y;
      q.open_w = h->open_w;
      q.open_e = h->open_e;
      q.open_n = h->open_n;
      q.status = h->status;
    }
    cudaError_t e = launch_strip_batch(P, kind_of(g), shape, is_mixed(g), s);
    b->launches++;
    if (e != cudaSuccess) return e;
    if (has_node_pass(g)) {
      e = launch_node_bc_batch(Q, s);
      b->launches++;
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

std::vector<int> members_of(const dim2d_batch* b, int g) {
  std::vector<int> idx;
  for (size_t i = 0; i < b->m.size(); i++)
    if (group_of(b->m[i]) == g) idx.push_back((int)i);
  return idx;
}

// One step of every group, each group's chain on its own stream forked from
// b->stream (so the chains overlap); joined back into b->stream.
cudaError_t launch_step(dim2d_batch* b, double dt_scale) {
  cudaError_t e = cudaEventRecord(b->fork, b->stream);
  for (int g = 0; g < NGROUPS && e == cudaSuccess; g++) {
    const std::vector<int> idx = members_of(b, g);
    if (idx.empty()) continue;
    e = cudaStreamWaitEvent(b->side[g], b->fork, 0);
    for (int st = 1; st <= 3 && e == cudaSuccess; st++)
      e = group_stage(b, g, idx, st, b->shape[g], dt_scale, b->side[g]);
    if (e == cudaSuccess) e = cudaEventRecord(b->join[g], b->side[g]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[g], 0);
  }
  return e;
}

void swap_members(dim2d_batch* b) {
  for (dim2d_handle* h : b->m) std::swap(h->A, h->B);
}

// capture the step graph of the current buffer parity into slot `slot`
int capture(dim2d_batch* b, int slot) {
  const long long n0 = b->launches;
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DIM2D_ERR_UNSUPPORTED;
  }
  cudaError_t el = launch_step(b, 1.0);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->stream, &g);
  b->graph_launches[slot] = b->launches - n0;
  b->launches = n0;
  cudaGraphExec_t x = nullptr;
  if (el == cudaSuccess && e == cudaSuccess && g) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  if (el != cudaSuccess || e != cudaSuccess || !x) {
    cudaGetLastError();
    return el != cudaSuccess ? cuda_error(el, "batch capture") : DIM2D_ERR_UNSUPPORTED;
  }
  b->graph[slot] = x;
  return DIM2D_OK;
}

int build_graphs(dim2d_batch* b) {
  drop_batch_graphs(b);
  int rc = capture(b, 0);
  if (!rc) {
    swap_members(b);  // host view of the other parity; nothing runs
    rc = capture(b, 1);
    swap_members(b);
  }
  if (rc) {
    drop_batch_graphs(b);
    return rc;
  }
  b->graphs_valid = true;
  b->parity = 0;
  return DIM2D_OK;
}

int find(const dim2d_batch* b, const dim2d_handle* h) {
  for (size_t i = 0; i < b->m.size(); i++)
    if (b->m[i] == h) return (int)i;
  return -1;
}

// later work on each member's own stream (download, ...) waits for the batch
int publish(dim2d_batch* b) {
  if (!b->done) return DIM2D_OK;
  cudaError_t e = cudaEventRecord(b->done, b->stream);
  for (dim2d_handle* h : b->m)
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->stream, b->done, 0);
  return e == cudaSuccess ? DIM2D_OK : cuda_error(e, "batch");
}

void drop_plans(dim2d_batch* b) {
  for (PersistPlan& pl : b->plan) persist_free(pl);
  b->pparity = 0;
}

// tables of the members of precision cls (0 FP64, 1 DIM2D_MIXED)
int build_plan(dim2d_batch* b, int cls, int rows) {
  std::vector<dim2d_handle*> hs;
  std::vector<double> dts;
  for (size_t i = 0; i < b->m.size(); i++)
    if ((b->m[i]->precision == DIM2D_MIXED) == (cls == 1)) {
      hs.push_back(b->m[i]);
      dts.push_back(b->dt[i]);
    }
  return persist_build(b->plan[cls], hs, dts, rows, b->stream);
}

// tables of both precisions for the current members and rows: kept while
// both are valid for b->rows, else both rebuilt (they share the buffer
// parity counted by b->pparity)
int ensure_plans(dim2d_batch* b) {
  bool current = true;
  for (const PersistPlan& pl : b->plan) current = current && pl.valid && pl.rows == b->rows;
  if (current) return DIM2D_OK;
  drop_plans(b);
  for (int cls = 0; cls < 2; cls++) {
    int rc = build_plan(b, cls, b->rows);
    if (rc) {
      drop_plans(b);
      return rc;
    }
  }
  return DIM2D_OK;
}

// nsteps persistent steps of every member: one launch per precision, the
// two precisions on their own streams forked from b->stream
cudaError_t persistent_steps(dim2d_batch* b, int nsteps, double dt_scale) {
  cudaError_t e = cudaEventRecord(b->fork, b->stream);
  for (int cls = 0; cls < 2 && e == cudaSuccess; cls++) {
    if (b->plan[cls].nfields == 0) continue;
    cudaStream_t s = b->side[cls];
    e = cudaStreamWaitEvent(s, b->fork, 0);
    if (e == cudaSuccess)
      e = persist_launch(b->plan[cls], nsteps, (int)(b->pparity & 1), dt_scale, b->wait_ns,
                         b->withhold, s);
    if (e == cudaSuccess) b->launches++;
    if (e == cudaSuccess) e = cudaEventRecord(b->join[cls], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[cls], 0);
  }
  return e;
}

// error words of the persistent launches since the last check (synchronous)
int persistent_errors(dim2d_batch* b) {
  for (PersistPlan& pl : b->plan) {
    int rc = persist_error(pl);
    if (rc) return rc;
  }
  return DIM2D_OK;
}

}  // namespace

extern "C" {

int dim2d_batch_create(dim2d_batch** out) {
  if (!out) return set_error(DIM2D_ERR_ARG, "batch_create: null argument");
  *out = nullptr;
  dim2d_batch* b = new dim2d_batch();
  cudaGetDevice(&b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
  for (int g = 0; g < NGROUPS && e == cudaSuccess; g++) {
    e = cudaStreamCreateWithFlags(&b->side[g], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[g], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    int rc = cuda_error(e, "batch_create");
    dim2d_batch_destroy(b);
    return rc;
  }
  b->stream = b->own_stream;
  *out = b;
  return DIM2D_OK;
}

int dim2d_batch_add(dim2d_batch* b, dim2d_handle* h, double dt) {
  if (!b || !h) return set_error(DIM2D_ERR_ARG, "batch_add: null argument");
  if (!h->uploaded) return set_error(DIM2D_ERR_NOT_READY, "batch_add: field has no state");
  if (h->batch) return set_error(DIM2D_ERR_ARG, "batch_add: field is already in a batch");
  if (!(dt >= 0) || !std::isfinite(dt)) return set_error(DIM2D_ERR_ARG, "batch_add: bad dt");
  if (h->device != b->device)
    return set_error(DIM2D_ERR_ARG, "batch_add: field lives on device %d, batch on %d",
                     h->device, b->device);
  if (!b->m.empty() && std::memcmp(&b->p, &h->p, sizeof(dim2d_params)) != 0)
    return set_error(DIM2D_ERR_UNSUPPORTED,
                     "batch_add: batch members must share the physical constants");
  if (h->f.pitch % 2 != 0) return set_error(DIM2D_ERR_UNSUPPORTED, "batch_add: odd pitch");
  // the batch's work follows what was queued on the field's stream,
  // including an asynchronous download of the field
  cudaError_t e = cudaSuccess;
  if (h->copy_pending) {
    e = cudaStreamWaitEvent(h->stream, h->copy_done, 0);
    h->copy_pending = false;
  }
  if (e == cudaSuccess) e = cudaEventRecord(b->done, h->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->done, 0);
  if (e != cudaSuccess) return cuda_error(e, "batch_add");
  if (b->m.empty()) b->p = h->p;
  b->m.push_back(h);
  b->dt.push_back(dt);
  h->batch = b;
  drop_batch_graphs(b);
  drop_plans(b);
  return DIM2D_OK;
}

int dim2d_batch_remove(dim2d_batch* b, dim2d_handle* h) {
  if (!b || !h) return set_error(DIM2D_ERR_ARG, "batch_remove: null argument");
  const int i = find(b, h);
  if (i < 0) return set_error(DIM2D_ERR_ARG, "batch_remove: field is not in this batch");
  int rc = publish(b);  // the field's own stream waits for the batch's work
  b->m.erase(b->m.begin() + i);
  b->dt.erase(b->dt.begin() + i);
  h->batch = nullptr;
  drop_batch_graphs(b);
  drop_plans(b);
  return rc;
}

int dim2d_batch_set_dt(dim2d_batch* b, dim2d_handle* h, double dt) {
  if (!b || !h) return set_error(DIM2D_ERR_ARG, "batch_set_dt: null argument");
  const int i = find(b, h);
  if (i < 0) return set_error(DIM2D_ERR_ARG, "batch_set_dt: field is not in this batch");
  if (!(dt >= 0) || !std::isfinite(dt)) return set_error(DIM2D_ERR_ARG, "batch_set_dt: bad dt");
  if (b->dt[i] != dt) {
    b->dt[i] = dt;
    drop_batch_graphs(b);
    drop_plans(b);
  }
  return DIM2D_OK;
}

int dim2d_batch_set_shape(dim2d_batch* b, int group, int shape) {
  if (!b || group < 0 || group >= NGROUPS || shape < 0 || shape >= NSHAPES)
    return set_error(DIM2D_ERR_ARG, "batch_set_shape: bad argument");
  if (b->shape[group] != shape) {
    b->shape[group] = shape;
    drop_batch_graphs(b);
  }
  return DIM2D_OK;
}

int dim2d_batch_set_persistent(dim2d_batch* b, int enable) {
  if (!b) return set_error(DIM2D_ERR_ARG, "batch_set_persistent: null batch");
  if (b->persistent != (enable != 0)) {
    b->persistent = enable != 0;
    drop_batch_graphs(b);
    drop_plans(b);
  }
  return DIM2D_OK;
}

int dim2d_batch_set_rows(dim2d_batch* b, int rows) {
  if (!b || (rows != 8 && rows != 16 && rows != 32))
    return set_error(DIM2D_ERR_ARG, "batch_set_rows: rows must be 8, 16 or 32");
  b->rows = rows;
  return DIM2D_OK;
}

int dim2d_batch_set_wait_limit(dim2d_batch* b, double seconds) {
  if (!b || !(seconds > 0) || !(seconds <= 60.0))
    return set_error(DIM2D_ERR_ARG, "batch_set_wait_limit: seconds must be in (0, 60]");
  b->wait_ns = (unsigned long long)(seconds * 1e9);
  return DIM2D_OK;
}

int dim2d_batch_withhold_item(dim2d_batch* b, long long item) {
  if (!b || item < -1) return set_error(DIM2D_ERR_ARG, "batch_withhold_item: bad argument");
  b->withhold = item;
  return DIM2D_OK;
}

int dim2d_batch_set_graphs(dim2d_batch* b, int enable) {
  if (!b) return set_error(DIM2D_ERR_ARG, "batch_set_graphs: null batch");
  b->use_graphs = enable != 0;
  return DIM2D_OK;
}

int dim2d_batch_step(dim2d_batch* b, int nsteps) {
  if (!b || nsteps < 0) return set_error(DIM2D_ERR_ARG, "batch_step: bad argument");
  if (b->m.empty() || nsteps == 0) return DIM2D_OK;
  if (b->persistent) {
    int rc = ensure_plans(b);
    if (rc) return rc;
    cudaError_t e = persistent_steps(b, nsteps, 1.0);
    if (e != cudaSuccess) return cuda_error(e, "batch persistent step");
    b->pparity += nsteps;
    if (nsteps & 1) swap_members(b);
    for (size_t i = 0; i < b->m.size(); i++)  // field_class.f:70, step by step
      for (int k = 0; k < nsteps; k++) b->m[i]->t += b->dt[i];
    return publish(b);
  }
  if (b->use_graphs && !b->graphs_valid) {
    int rc = build_graphs(b);
    if (rc && rc != DIM2D_ERR_UNSUPPORTED) return rc;
  }
  for (int s = 0; s < nsteps; s++) {
    if (b->use_graphs && b->graphs_valid) {
      cudaError_t e = cudaGraphLaunch(b->graph[b->parity], b->stream);
      if (e != cudaSuccess) return cuda_error(e, "batch step graph");
      b->launches += b->graph_launches[b->parity];
      b->parity ^= 1;
    } else {
      cudaError_t e = launch_step(b, 1.0);
      if (e != cudaSuccess) return cuda_error(e, "batch step");
      // the two graphs follow the buffer parity; a stream step flips it too
      b->parity ^= 1;
    }
    swap_members(b);  // the host side of rk3_step for every member
    for (size_t i = 0; i < b->m.size(); i++) b->m[i]->t += b->dt[i];  // field_class.f:70
  }
  return publish(b);
}

int dim2d_batch_sync(dim2d_batch* b) {
  if (!b) return set_error(DIM2D_ERR_ARG, "batch_sync: null batch");
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_error(e, "batch_sync");
  int rc0 = persistent_errors(b);
  if (rc0) return rc0;
  for (dim2d_handle* h : b->m) {
    int rc = check_status(h);
    if (rc) return rc;
  }
  return DIM2D_OK;
}

// persistent mode: dry launches (dt = 0, nsteps = 1: stage buffers only)
// with 8, 16 and 32 rows per strip item; keeps the fastest
static int autotune_persistent(dim2d_batch* b, int chosen[8], double* times_ms) {
  static const int opts[3] = {8, 16, 32};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double best = 1e300;
  int best_rows = b->rows;
  const int rows0 = b->rows;
  double t[3] = {0, 0, 0};
  for (int o = 0; o < 3 && e == cudaSuccess; o++) {
    b->rows = opts[o];
    int rc = ensure_plans(b);
    if (rc) {
      b->rows = rows0;
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      return rc;
    }
    e = persistent_steps(b, 1, 0.0);
    if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
    for (int r = 0; r < 3 && e == cudaSuccess; r++) e = persistent_steps(b, 1, 0.0);
    if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    t[o] = ms / 3.0;
    if (t[o] < best) {
      best = t[o];
      best_rows = opts[o];
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_error(e, "batch_autotune");
  b->rows = best_rows;
  int rc = persistent_errors(b);
  if (rc) return rc;
  for (int g = 0; g < NGROUPS; g++) {
    if (chosen) chosen[g] = best_rows;
    for (int o = 0; o < NSHAPES; o++)
      if (times_ms) times_ms[g * NSHAPES + o] = o < 3 ? t[o] : 0.0;
  }
  return DIM2D_OK;
}

int dim2d_batch_autotune(dim2d_batch* b, int chosen[8], double* times_ms) {
  if (!b) return set_error(DIM2D_ERR_ARG, "batch_autotune: null batch");
  if (b->persistent) return b->m.empty() ? DIM2D_OK : autotune_persistent(b, chosen, times_ms);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  for (int g = 0; g < NGROUPS && e == cudaSuccess; g++) {
    const std::vector<int> idx = members_of(b, g);
    double best = 1e300;
    int best_shape = b->shape[g];
    for (int sh = 0; sh < NSHAPES && e == cudaSuccess; sh++) {
      float ms = 0.f;
      if (!idx.empty()) {
        // dry steps (dt = 0) of this group alone: the stages write the
        // stage buffers B and C only; A, the state, is read
        auto dry = [&]() {
          cudaError_t r = cudaSuccess;
          for (int st = 1; st <= 3 && r == cudaSuccess; st++)
            r = group_stage(b, g, idx, st, sh, 0.0, b->stream);
          return r;
        };
        e = dry();
        if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
        for (int r = 0; r < 3 && e == cudaSuccess; r++) e = dry();
        if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        ms /= 3.0f;
        if (ms < best) {
          best = ms;
          best_shape = sh;
        }
      }
      if (times_ms) times_ms[g * NSHAPES + sh] = ms;
    }
    if (e == cudaSuccess && b->shape[g] != best_shape) {
      b->shape[g] = best_shape;
      drop_batch_graphs(b);
    }
    if (chosen) chosen[g] = b->shape[g];
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_error(e, "batch_autotune");
  return DIM2D_OK;
}

int dim2d_batch_size(const dim2d_batch* b) { return b ? (int)b->m.size() : -1; }

long long dim2d_batch_launch_count(const dim2d_batch* b) { return b ? b->launches : -1; }

long long dim2d_batch_cells(const dim2d_batch* b) {
  if (!b) return -1;
  long long n = 0;
  for (const dim2d_handle* h : b->m) n += (long long)(h->f.nx - 2 * BC) * (h->f.ny - 2 * BC);
  return n;
}

int dim2d_batch_set_stream(dim2d_batch* b, void* stream) {
  if (!b) return set_error(DIM2D_ERR_ARG, "batch_set_stream: null batch");
  b->stream = stream ? (cudaStream_t)stream : b->own_stream;
  return DIM2D_OK;
}

int dim2d_batch_destroy(dim2d_batch* b) {
  if (!b) return DIM2D_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  publish(b);
  for (dim2d_handle* h : b->m) h->batch = nullptr;
  drop_batch_graphs(b);
  drop_plans(b);
  for (int g = 0; g < NGROUPS; g++) {
    if (b->side[g]) cudaStreamDestroy(b->side[g]);
    if (b->join[g]) cudaEventDestroy(b->join[g]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->done) cudaEventDestroy(b->done);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return DIM2D_OK;
}

}  // extern "C"
