// dim2d_step.cu -- one RK3-TVD time step on the device
// (td_integrator_class.f:103-161 with rk3tvd_steps_module.f:52-490).
//
// Buffers: A holds u^n.  Stage 1 writes B = A + dt L(A); stage 2 writes
// C = 3/4 A + 1/4 (B + dt L(B)); stage 3 writes B = 1/3 A + 2/3 (C + dt L(C));
// then A and B swap.  u^n stays intact in A until the last boundary pass,
// which the wall operator reads as nodes_tmp (bc_operators_wall_xy_class.f).
// Each stage is followed by the node boundary pass; for periodic fields the
// stage kernel writes the ghost images itself, for open fields a second
// kernel integrates the ghost cells.
#include <utility>

#include "dim2d_internal.h"

using namespace dim2d;

StageArgs make_stage_args(const dim2d_handle* h, const double* uin, double* uout, double dt,
                          int st) {
  StageArgs a{};
  a.uin = uin;
  a.u0 = h->A;
  a.uout = uout;
  a.f = h->f;
  a.dx = h->dx;
  a.dy = h->dy;
  a.rdx = h->rdx;
  a.rdy = h->rdy;
  a.dt = dt;
  a.stage = st;
  a.b = st == 2 ? 0.75 : (st == 3 ? 1.0 / 3.0 : 0.0);  // rk3tvd_steps_module.f:225,444
  a.periodic = h->periodic;
  a.wall_s = h->south_wall;
  a.variant = h->variant;
  a.open = h->open_mask;
  a.mixed = h->precision == DIM2D_MIXED;
  a.t = h->t;
  a.xmap0 = h->xmap0;
  a.ymap0 = h->ymap0;
  // stages 2 and 3 follow the node pass of the stage before (stage()): they
  // may start while it runs, only the warps that read its ghosts wait
  a.node_sides = st >= 2 ? h->node_sides : 0;
  a.wall = h->wall;
  a.k = h->k;
  return a;
}

static NodeBcArgs make_node_args(const dim2d_handle* h, const double* utmp, double* u) {
  NodeBcArgs a{};
  a.utmp = utmp;
  a.u = u;
  a.f = h->f;
  a.dx = h->dx;
  a.dy = h->dy;
  a.rdx = h->rdx;
  a.rdy = h->rdy;
  a.t = h->t;
  a.xmap0 = h->xmap0;
  a.ymap0 = h->ymap0;
  a.south_wall = h->south_wall;
  a.corners_y = h->corners_y;
  a.open_w = h->open_w;
  a.open_e = h->open_e;
  a.open_n = h->open_n;
  a.status = h->status;
  a.wall = h->wall;
  a.k = h->k;
  return a;
}

int apply_bc_on_nodes(dim2d_handle* h, const double* nodes_tmp, double* nodes) {
  cudaError_t e = cudaSuccess;
  if (h->periodic) {
    e = launch_periodic_ghosts(nodes, h->f, h->stream);
    h->launches++;
  } else if (h->open_all) {
    return DIM2D_OK;  // no section of node type
  } else {
    e = launch_node_bc(make_node_args(h, nodes_tmp, nodes), h->stream);
    h->launches++;
  }
  if (e != cudaSuccess) return cuda_error(e, "apply_bc_on_nodes");
  return DIM2D_OK;
}

void prof_begin(dim2d_handle* h) {
  if (!h->prof) return;
  if (h->prof_used + 2 > h->prof_ev.size()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t ev;
      if (cudaEventCreate(&ev) != cudaSuccess) {
        h->prof = false;
        return;
      }
      h->prof_ev.push_back(ev);
    }
  }
  cudaEventRecord(h->prof_ev[h->prof_used], h->stream);
}

void prof_end(dim2d_handle* h) {
  if (!h->prof) return;
  cudaEventRecord(h->prof_ev[h->prof_used + 1], h->stream);
  h->prof_used += 2;
}

// Read the wall status word (synchronising).  Non-zero = a wall ghost cell
// had no bracketed / converged root, where the reference stops.
int check_status(dim2d_handle* h) {
  if (h->pplan) {  // a persistent launch that stopped at a wait that ran out
    int rc = persist_error(*h->pplan);
    if (rc) return rc;
  }
  if (!h->south_wall || !h->status) return DIM2D_OK;
  unsigned int st = 0;
  cudaError_t e = cudaMemcpyAsync(&st, h->status, sizeof st, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_error(e, "status");
  if (st)
    return set_error(DIM2D_ERR_WALL_ROOT,
                     "wall ghost cell: %s (status 0x%x)",
                     (st & 1u) ? "root not bracketed" : "Ridders' method did not converge", st);
  return DIM2D_OK;
}

cudaError_t launch_stage_work(dim2d_handle* h, const StageArgs& a, int mode) {
  prof_begin(h);
  cudaError_t e = mode == 0 ? launch_time_dev(a, h->stream) : launch_interior_stage(a, h->stream);
  prof_end(h);
  h->launches++;
  if (e == cudaSuccess && a.open && !stage_fuses_open(a)) {
    e = launch_open_ghosts(a, mode, h->stream);
    h->launches++;
  }
  return e;
}

static int stage(dim2d_handle* h, int st, const double* uin, double* uout, double dt) {
  // on open fields every ghost cell has a time derivative and is integrated
  // like the interior (x/y_borders widened, field_abstract_class.f:244-270)
  // and no node boundary pass follows; the mixed presets integrate their
  // open sections and run the node pass for the others
  cudaError_t e = launch_stage_work(h, make_stage_args(h, uin, uout, dt, st), 1);
  if (e != cudaSuccess) return cuda_error(e, "rk3 stage");
  if (h->periodic || h->open_all) return DIM2D_OK;  // periodic images: by the stage kernel
  return apply_bc_on_nodes(h, h->A, uout);
}

int rk3_step(dim2d_handle* h, double dt) {
  int rc = stage(h, 1, h->A, h->B, dt);
  if (!rc) rc = stage(h, 2, h->B, h->C, dt);
  if (!rc) rc = stage(h, 3, h->C, h->B, dt);
  if (rc) return rc;
  std::swap(h->A, h->B);
  h->t += dt;  // field_class.f:70
  return DIM2D_OK;
}

cudaError_t wait_copy_if(dim2d_handle* h, const double* target) {
  if (!h->copy_pending || target != h->copy_src) return cudaSuccess;
  h->copy_pending = false;
  return cudaStreamWaitEvent(h->stream, h->copy_done, 0);
}

void drop_graphs(dim2d_handle* h) {
  for (int i = 0; i < 2; i++) {
    if (h->graph_exec[i]) cudaGraphExecDestroy(h->graph_exec[i]);
    h->graph_exec[i] = nullptr;
    h->graph_A[i] = nullptr;
  }
}

// Capture one RK3 step into graph slot `slot`.  The capture runs
// rk3_step's host side (A/B swap, time += dt) without executing anything;
// on success the caller launches the graph once, which brings the device
// state to the host state.  On failure the host side is rolled back.  No
// kernel reads the field time, so one graph serves every time level.
static int capture_step(dim2d_handle* h, double dt, int slot) {
  if (h->graph_exec[slot]) cudaGraphExecDestroy(h->graph_exec[slot]);
  h->graph_exec[slot] = nullptr;
  h->graph_A[slot] = nullptr;
  double* const A0 = h->A;
  double* const B0 = h->B;
  const double t0 = h->t;
  const long long n0 = h->launches;
  cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DIM2D_ERR_UNSUPPORTED;  // e.g. the legacy default stream
  }
  const int rc = rk3_step(h, dt);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(h->stream, &g);
  const long long n = h->launches - n0;
  h->launches = n0;
  cudaGraphExec_t x = nullptr;
  if (!rc && e == cudaSuccess && g) e = cudaGraphInstantiate(&x, g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc || e != cudaSuccess || !x) {
    cudaGetLastError();
    h->A = A0;
    h->B = B0;
    h->t = t0;
    return rc ? rc : DIM2D_ERR_UNSUPPORTED;
  }
  h->graph_exec[slot] = x;
  h->graph_A[slot] = A0;
  h->graph_launches[slot] = n;
  return DIM2D_OK;
}

// Stage-kernel variant 6: nsteps steps as one launch of the persistent
// kernel (dim2d_persist.cu) over this field alone -- stages pipelined band
// by band, no stage boundary across the field.  The tables are built on
// first use for this dt and the field's buffers, and rebuilt when either
// changes; dt_scale 0 makes the autotuner's dry step (stage buffers only,
// no swap, no time advance).
int persist_steps(dim2d_handle* h, double dt, int nsteps, double dt_scale) {
  if (nsteps <= 0) return DIM2D_OK;
  // the launch writes both buffers of the pair: pending copies land first
  if (h->copy_pending) {
    cudaError_t ew = cudaStreamWaitEvent(h->stream, h->copy_done, 0);
    if (ew != cudaSuccess) return cuda_error(ew, "step");
    h->copy_pending = false;
  }
  // a dry step keeps whatever dt the tables hold (its stages use dt * 0)
  const double pdt = dt_scale == 0.0 ? (h->pplan && h->pdt >= 0.0 ? h->pdt : 0.0) : dt;
  bool rebuild = !h->pplan || !h->pplan->valid || h->pdt != pdt;
  int step0 = 0;
  if (!rebuild) {
    // the tables hold the buffers as built; A/B swap with every step
    const PDomain& d0 = h->pdom0;
    if (h->A == d0.buf[0] && h->B == d0.buf[1] && h->C == d0.buf[2]) step0 = 0;
    else if (h->A == d0.buf[1] && h->B == d0.buf[0] && h->C == d0.buf[2]) step0 = 1;
    else rebuild = true;
  }
  if (rebuild) {
    if (!h->pplan) h->pplan = new PersistPlan();
    std::vector<dim2d_handle*> hs{h};
    std::vector<double> dts{pdt};
    int rc = persist_build(*h->pplan, hs, dts, 16, h->stream);
    if (rc) return rc;
    h->pdt = pdt;
    h->pdom0.buf[0] = h->A;
    h->pdom0.buf[1] = h->B;
    h->pdom0.buf[2] = h->C;
    step0 = 0;
  }
  prof_begin(h);
  cudaError_t e = persist_launch(*h->pplan, nsteps, step0, dt_scale, 2000000000ull, -1, h->stream);
  prof_end(h);
  if (e != cudaSuccess) return cuda_error(e, "persistent step");
  h->launches++;
  if (dt_scale != 0.0) {
    if (nsteps & 1) std::swap(h->A, h->B);
    for (int s = 0; s < nsteps; s++) h->t += dt;  // field_class.f:70, step by step
  }
  return DIM2D_OK;
}

int rk3_steps(dim2d_handle* h, double dt, int nsteps) {
  if (h->variant == PERSIST_VARIANT) return persist_steps(h, dt, nsteps, 1.0);
  const bool graphs = h->use_graphs && !h->prof;
  if (graphs && h->graph_dt != dt) {
    drop_graphs(h);
    h->graph_dt = dt;
  }
  for (int s = 0; s < nsteps; s++) {
    // stage 1 writes B: a pending asynchronous copy of B must land first
    cudaError_t ew = wait_copy_if(h, h->B);
    if (ew != cudaSuccess) return cuda_error(ew, "step");
    if (graphs) {
      int slot = -1;
      for (int i = 0; i < 2; i++)
        if (h->graph_exec[i] && h->graph_A[i] == h->A) slot = i;
      bool fresh = false;
      if (slot < 0) {
        slot = (h->graph_exec[0] && h->graph_A[0] != h->A) ? 1 : 0;
        fresh = capture_step(h, dt, slot) == DIM2D_OK;
        if (!fresh) slot = -1;
      }
      if (slot >= 0) {
        cudaError_t e = cudaGraphLaunch(h->graph_exec[slot], h->stream);
        if (e != cudaSuccess) return cuda_error(e, "step graph");
        h->launches += h->graph_launches[slot];
        if (!fresh) {  // the host side of rk3_step
          std::swap(h->A, h->B);
          h->t += dt;  // field_class.f:70
        }
        continue;
      }
    }
    int rc = rk3_step(h, dt);
    if (rc) return rc;
  }
  return DIM2D_OK;
}
