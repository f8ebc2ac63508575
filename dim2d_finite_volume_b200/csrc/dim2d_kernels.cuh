// dim2d_kernels.cuh -- launch interface of the sm_100a kernels.
#pragma once
#include <cstdint>
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

// Wall constants (parameters_input.f:526-624): uniform micro contact angle
// (its cosine precomputed on the host, wall_xy_equilibrium_module.f:2262)
// and the wall heat source (no / constant / gaussian, :1645-1707).
struct WallConst {
  double cos_angle;
  int heat_choice;  // 0 none, 1 constant, 2 gaussian
  double qmax, qcenter, qvariance;
};

__host__ __device__ __forceinline__ double wall_heat_flux(const WallConst& w, double x) {
  if (w.heat_choice == 0) return 0.0;
  if (w.heat_choice == 1) return w.qmax;
  const double z = (x - w.qcenter) / w.qvariance;
  return w.qmax * exp(-0.5 * (z * z));
}

// Ghost sections integrated with the open (Hedstrom, bc_timedev) operator:
// bits of StageArgs::open.  hedstrom_xy sets all of them; wall_S_open sets
// N, W, E, NW, NE; half_wall_S_open sets N, E, NE (library_config.py:118-150).
enum OpenSection : int {
  OPEN_S = 1, OPEN_N = 2, OPEN_W = 4, OPEN_E = 8,
  OPEN_SW = 16, OPEN_SE = 32, OPEN_NW = 64, OPEN_NE = 128,
  OPEN_ALL = 255
};

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
  int variant;                         // 0 = 32x8 CTA tiles, 1..5 = warp strips (shape-1)
  int open;                            // OPEN_* mask of the time-integrated (Hedstrom)
                                       // ghost sections; strip launches integrate those
                                       // cells too (their first CTAs)
  int mixed;                           // DIM2D_MIXED: FP32 face pass (strip kernels)
  double t;                            // field time (constant over the stages)
  double xmap0, ymap0;                 // x_map(1), y_map(1): x_map(i) = xmap0 + (i-1) dx
  int node_sides;                      // NODE_* sides whose ghost cells the node pass just
                                       // before this launch writes; non-zero: the launch is
                                       // a programmatic dependent of that pass and the
                                       // warps that read those ghosts wait for it
  const int* __restrict__ mask;        // time derivative of a buffer-layer grid: its
                                       // grdpts_id map, written only where it is
                                       // interior_pt (1) inside [box_x0, box_x1] x
                                       // [box_y0, box_y1] (0-based, >= BC from the edges)
  int box_x0, box_x1, box_y0, box_y1;
  WallConst wall;
  DimConst k;
};

// sides of StageArgs::node_sides
enum NodeSide : int { NODE_W = 1, NODE_E = 2, NODE_S = 4, NODE_N = 8 };

// Node boundary pass of a field whose sides are mirrors (reflection_x/_y),
// open (nothing to do) or, on the south side, the wall operator.
struct NodeBcArgs {
  const double* __restrict__ utmp;  // nodes_tmp = u^n (wall temperature guess)
  double* __restrict__ u;           // field whose ghosts are set
  Field f;
  double dx, dy, rdx, rdy;
  double t, xmap0, ymap0;
  int south_wall;                   // 1: wall on S, 0: mirror
  int corners_y;                    // corners are reflection_y (reflection_xy) vs _x
  int open_w, open_e, open_n;       // side open (Hedstrom, integrated by the stage):
                                    // no node work there; with a south wall its S corner
                                    // is a wall corner (wall_S_open, half_wall_S_open)
  unsigned int* status;             // bit 0: root not bracketed, bits 1-3: Ridders
  WallConst wall;
  DimConst k;
};
cudaError_t launch_node_bc(const NodeBcArgs& a, cudaStream_t s);

// Tile of the fused interior kernel: TX x TY interior cells per CTA.
constexpr int TILE_X = 32;
constexpr int TILE_Y = 8;
size_t interior_smem_bytes();

cudaError_t launch_interior_stage(const StageArgs& a, cudaStream_t s);
// warp-streaming variant (dim2d_strip.cu); mode 0 = L(u), 1 = stage update;
// shape 0..4 = strip height / warps per CTA (8,4) (16,4) (32,4) (16,8) (8,8)
cudaError_t launch_strip_stage(const StageArgs& a, int mode, int shape, cudaStream_t s);
// The strip kernels read state rows as 16-byte pairs: they need an even
// pitch and 16-byte aligned input planes (fields allocated by the library
// always qualify; caller-provided layouts may not, and then use variant 0).
inline bool strip_layout_ok(const StageArgs& a) {
  return a.f.pitch % 2 == 0 && reinterpret_cast<uintptr_t>(a.uin) % 16 == 0;
}
// 1 if the stage launch of `a` runs a strip kernel (mixed precision always
// does: the tile kernel has no FP32 face pass)
inline bool stage_uses_strip(const StageArgs& a) {
  return (a.variant > 0 || a.mixed) && strip_layout_ok(a);
}
// strip shape of a stage launch (variant 1..5; mixed fields on variant 0
// use shape 1)
inline int strip_shape_of(const StageArgs& a) {
  return a.variant >= 1 && a.variant <= 5 ? a.variant - 1 : (a.variant == 6 ? 3 : 1);
}
// 1 if the stage launch of `a` also covers the open-boundary ghost cells
inline bool stage_fuses_open(const StageArgs& a) { return a.open && stage_uses_strip(a); }
// variants 0..5 as above; 6 = the persistent kernel (a whole step per
// launch, dim2d_persist.cu); its time derivative alone uses strip shape 3
constexpr int NUM_VARIANTS = 7;
// L(a.uin) of the interior cells into a.uout (stage fields ignored)
cudaError_t launch_time_dev(const StageArgs& a, cudaStream_t s);
// L(u) of a buffer-layer grid at its interior_pt points (StageArgs::mask):
// the strip kernel where strip_layout_ok (even nx, 16-byte aligned nodes),
// else the tile kernel
cudaError_t launch_time_dev_masked(const StageArgs& a, cudaStream_t s);
cudaError_t launch_strip_masked(const StageArgs& a, cudaStream_t s);
// open (Hedstrom) ghost cells of the sections in a.open; mode 0 writes
// L(u) into a.uout, mode 1 the RK stage update
cudaError_t launch_open_ghosts(const StageArgs& a, int mode, cudaStream_t s);
cudaError_t launch_fill(double* p, double v, size_t n, cudaStream_t s);
cudaError_t launch_periodic_ghosts(double* u, const Field& f, cudaStream_t s);
// The ghost frame of a field: every cell within BC of an edge, 4 planes.
// frame_cells counts them; frame_offset(f, i), 0 <= i < frame_cells(f), is
// the offset of cell i in the planar layout (per plane: the BC bottom rows,
// the BC top rows, then the BC left and BC right cells of each row between).
inline __host__ __device__ int frame_cells(const Field& f) {
  return 4 * (2 * BC * f.nx + (f.ny - 2 * BC) * 2 * BC);
}
inline __host__ __device__ size_t frame_offset(const Field& f, int i) {
  const int rows = 2 * BC * f.nx;
  const int per_plane = rows + (f.ny - 2 * BC) * 2 * BC;
  const int v = i / per_plane, j = i % per_plane;
  int x, y;
  if (j < rows) {
    const int r = j / f.nx;
    x = j % f.nx;
    y = r < BC ? r : f.ny - 2 * BC + r;
  } else {
    const int c = (j - rows) % (2 * BC);
    y = BC + (j - rows) / (2 * BC);
    x = c < BC ? c : f.nx - 2 * BC + c;
  }
  return (size_t)v * f.plane + (size_t)y * f.pitch + x;
}
// the ghost frame of src into d1 and d2
cudaError_t launch_copy_frame(const double* src, double* d1, double* d2, const Field& f,
                              cudaStream_t s);
cudaError_t launch_cfl_max(const double* u, const Field& f, const DimConst& k, double* out,
                           cudaStream_t s);

// ---- batched launches (dim2d_batch.cu): many fields of one boundary kind
// advanced by one launch per stage.  The per-domain tables travel as
// kernel parameters (read in place through __grid_constant__).
constexpr int BATCH_MAX = 64;  // domains per launch (larger groups are split)

struct BatchDomain {
  Field f;
  const double* uin;
  const double* u0;
  double* uout;
  double dx, dy, rdx, rdy, dt, xmap0;
  int periodic, wall_s;
  int open;                // OPEN_* mask of the time-integrated ghost sections
  int node_sides;          // as StageArgs::node_sides
  int ghost0, strip0, sx;  // first ghost CTA, first strip CTA, strips per row
};

struct BatchStageArgs {
  DimConst k;
  WallConst wall;
  int stage;
  double b;
  int ndom;
  int ghost_ctas;  // total ghost CTAs (open and wall kinds), placed before all strips
  BatchDomain d[BATCH_MAX];
};

// boundary kinds of a batched stage launch; BK_WALL launches also integrate
// the open sections of wall_S_open / half_wall_S_open members (their
// ghost CTAs first; wall_S_reflection members have none)
enum BatchKind : int { BK_PLAIN = 0, BK_WALL = 1, BK_OPEN = 2 };

// one stage of every domain in P (shape as launch_strip_stage; mixed: the
// DIM2D_MIXED face pass for all of them); fills the CTA geometry fields of P.d
cudaError_t launch_strip_batch(BatchStageArgs& P, int kind, int shape, bool mixed,
                               cudaStream_t s);

struct NodeBcDomain {
  const double* utmp;
  double* u;
  Field f;
  double dx, dy, rdx, rdy, xmap0, ymap0;
  int south_wall, corners_y;
  int open_w, open_e, open_n;
  unsigned int* status;
  int cta0;
};

struct NodeBcBatchArgs {
  DimConst k;
  WallConst wall;
  int ndom;
  NodeBcDomain d[BATCH_MAX];
};

// node boundary pass of every domain in P; fills P.d[].cta0
cudaError_t launch_node_bc_batch(NodeBcBatchArgs& P, cudaStream_t s);

// ---- persistent batched kernel (dim2d_strip.cu): one launch advances
// every domain of a batch (any mix of boundary kinds, one precision) by
// nsteps RK3 steps.  Its warps take work items in order from one counter:
// per step and stage, band by band, the open ghost cells and strips of every
// domain's row band, then the node boundary passes.  Dependencies are
// tracked per row band: a strip or ghost item of a band waits until the
// previous stage is complete on that band and its two neighbours (the
// stencil's reach; periodic fields wrap around) and, where the field has a
// node pass, until the previous stage's node pass is complete; a node item
// waits until its stage is complete on every band.  So stage s+1 starts on
// a band while stage s still runs elsewhere, fields advance independently,
// and no grid-wide barrier is needed.  Items are taken in dependency order,
// so warps that wait always wait on items that running warps hold.  Waits
// are bounded (wait_ns); one that runs out sets `error` and stops the launch.
enum PItemType : int { PI_GHOST = 0, PI_STRIP = 1, PI_NODE = 2 };

struct PDomain {
  Field f;
  double* buf[3];  // at launch: [0] = u^n, [1] = the other buffer of the pair, [2] = C
  double dx, dy, rdx, rdy, dt, xmap0, ymap0;
  int periodic, wall_s, open;                        // as StageArgs
  int south_wall, corners_y, open_w, open_e, open_n;  // as NodeBcArgs
  int sx;                                            // strips per row band
  int nb;                                            // row bands
  int band0;                                         // first of its band counters
  int nn;                                            // node items per stage (0: no pass)
  unsigned int* status;                              // wall root status word
};

struct PItem {
  int dom;
  int type;   // PItemType
  int stage;  // 1, 2, 3
  int index;  // strip: band * sx + column strip; ghost: first cell (open_ghost_cell
              // numbering); node: 32-cell group of node_bc_cell
  int count;  // ghost: cells of the item (<= 32)
  int band;   // row band (strip, ghost)
};

struct PersistArgs {
  DimConst k;
  WallConst wall;
  const PDomain* dom;
  const PItem* items;
  const int* sg;                  // strip + ghost items per stage of each band
  long long items_per_step;
  int nsteps;
  int step0;                      // buffer parity of the first step (0: u^n in buf[0])
  double dt_scale;                // 1, or 0 for the autotuner's dry steps
  int h_rows;                     // rows per strip item (= per band)
  unsigned long long* next;       // item counter (zero at launch)
  unsigned long long* done;       // per-band completion counters (zero at launch)
  unsigned long long* ndone;      // per-domain node-item completion counters (zero at launch)
  unsigned int* ctl;              // [0] abort flag, [1] error word (bit 0: a wait ran out)
  unsigned long long wait_ns;     // limit of one dependency wait
  long long withhold;             // item whose completion is never signalled (tests; -1: none)
};

// launch the persistent kernel with as many CTAs as fit on the device;
// *ctas receives that number
cudaError_t launch_batch_persistent(const PersistArgs& P, bool mixed, cudaStream_t s, int* ctas);

}  // namespace dim2d
