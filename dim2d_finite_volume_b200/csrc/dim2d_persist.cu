// dim2d_persist.cu -- work tables and launches of the persistent RK3
// kernel (k_batch_persistent, dim2d_strip.cu), shared by batches in
// persistent mode (dim2d_batch_set_persistent) and single fields on
// stage-kernel variant 6.  No counterpart in the reference, which advances
// one field by three separate stage loops per step
// (td_integrator_class.f:103-161).
//
// The per-step item table is the same for every step; the kernel maps
// item it of a launch to step it / items_per_step.  Buffer roles alternate
// with the step parity (the A/B swap of rk3_step), so a launch passes the
// parity of its first step relative to the buffers the tables were built
// with.
//
// Why the band dependencies order every access (X = u^n of step k, Y the
// other buffer of the pair, C; "(k,s,b)" = stage s of step k on band b;
// strips read rows y0-2 .. y1+2, so a band reads its neighbours' rows):
//   (k,1,b) reads X on b-1..b+1, writes Y on b;  (k,2,b) reads Y on
//   b-1..b+1 and X on b, writes C on b;  (k,3,b) reads C on b-1..b+1 and X
//   on b, writes Y on b.  Step k+1 swaps X and Y.
//   * read after write: every reader of stage s waits for stage s-1 on its
//     band and both neighbours -- the rows it reads;
//   * (k,3,b) writes Y rows of band b, read by (k,2,b-1..b+1): it waits
//     for exactly those;
//   * (k+1,1,b) writes X rows of band b (the old u^n), read by (k,1,b+-1)
//     and by (k,2,b), (k,3,b) as u^n: it waits for (k,3,b-1..b+1), which
//     waited for (k,2,b-2..b+2), which waited for (k,1,b-3..b+3);
//   * (k+1,2,b) writes C rows of band b, read by (k,3,b-1..b+1): it waits
//     for (k+1,1,b-1..b+1), which waited for (k,3,b-2..b+2);
//   * ghost images of periodic fields land in the opposite band: the
//     neighbour sets wrap around, so the same arguments hold;
//   * node passes write ghost cells of the stage output after the stage is
//     complete on every band, and every item of the next stage waits for
//     the whole pass; the wall pass reads u^n (ghost row 1 included), whose
//     next writer, stage 1 of the next step, waits for that pass too.
#include <algorithm>
#include <vector>

#include "dim2d_internal.h"
#include "dim2d_nodebc.cuh"
#include "dim2d_open.cuh"

using namespace dim2d;

namespace {

NodeBcArgs node_args_of(const dim2d_handle* h) {
  NodeBcArgs a{};
  a.f = h->f;
  a.south_wall = h->south_wall;
  a.corners_y = h->corners_y;
  a.open_w = h->open_w;
  a.open_e = h->open_e;
  a.open_n = h->open_n;
  return a;
}

// Ghost-cell items of one field's open sections, by row band: runs of at
// most 32 cells of open_ghost_cell's numbering (sections S, N, W, E, SW,
// SE, NW, NE in that order, skipping the closed ones), each inside one band:
// the S edge and S corners in band 0, the N edge and N corners in the last
// band, the W and E edge cells of the rows of each band in that band.
struct GhostRun {
  int first, count, band;
};
std::vector<GhostRun> ghost_runs(const dim2d_handle* h, int rows, int nb) {
  std::vector<GhostRun> out;
  const int mask = h->open_mask;
  if (!mask) return out;
  const int ey = h->f.ny - 2 * BC;
  auto add = [&](int first, int n, int band) {
    for (int o = 0; o < n; o += 32) out.push_back(GhostRun{first + o, std::min(32, n - o), band});
  };
  int off = 0;
  for (int sec = 0; sec < 8; sec++) {
    if (!(mask >> sec & 1)) continue;
    const int cells = open_section_cells(h->f, sec);
    if (sec == 0 || sec == 4 || sec == 5) {
      add(off, cells, 0);
    } else if (sec == 1 || sec == 6 || sec == 7) {
      add(off, cells, nb - 1);
    } else {  // W or E edge: BC columns of ey cells each
      for (int b = 0; b < nb; b++) {
        const int r0 = b * rows, n = b == nb - 1 ? ey - r0 : rows;
        for (int col = 0; col < BC; col++) add(off + col * ey + r0, n, b);
      }
    }
    off += cells;
  }
  return out;
}

// 1 if strip q of band `band` reads a ghost cell that the field's node
// pass writes (the strip reads columns c0-2 .. c0+31 and rows y0-2 ..
// y1+2).  Only those strips wait for the node pass of the previous stage;
// the cells the node pass reads (within two cells of its sides, and the
// u^n rows next to a wall) are written only by such strips, so the others
// need not wait for it either way.
int strip_reads_node_ghosts(const dim2d_handle* h, const PDomain& d, int band, int q, int rows) {
  const int sides = h->node_sides;
  if (!sides) return 0;
  const int c0 = BC + q * 30;
  const int y0 = BC + band * rows;
  const int y1 = band == d.nb - 1 ? h->f.ny - BC : y0 + rows;
  return ((sides & NODE_W) && c0 - 2 < BC) || ((sides & NODE_E) && c0 + 31 >= h->f.nx - BC) ||
         ((sides & NODE_S) && y0 - 2 < BC) || ((sides & NODE_N) && y1 + 2 >= h->f.ny - BC);
}

}  // namespace

// Row bands of ey interior rows: ey / rows rounded up, except that a last
// band of fewer than 2 rows joins the one before it (the last band then
// has up to rows + 1 rows).  The two last interior rows are the sources of
// a periodic field's ghost images across the domain; in one band, the
// neighbour dependencies (with wrap-around) cover them.
static int band_count(int ey, int rows) {
  int nb = (ey + rows - 1) / rows;
  if (nb > 1 && ey - (nb - 1) * rows < 2) nb--;
  return nb;
}

void persist_free(PersistPlan& pl) {
  if (pl.dom) cudaFree(pl.dom);
  if (pl.items) cudaFree(pl.items);
  if (pl.sg) cudaFree(pl.sg);
  if (pl.ctr) cudaFree(pl.ctr);
  if (pl.ctl) cudaFree(pl.ctl);
  pl = PersistPlan();
}

// Tables for fields hs (one precision) with time steps dts, bands (and
// strip items) of `rows` rows: per stage, band by band over all fields
// (largest first), each band's ghost-cell items then its strips; then the
// node boundary passes (wall fields first).  Synchronises `s` (the host
// tables are copied from pageable memory).
int persist_build(PersistPlan& pl, const std::vector<dim2d_handle*>& hs,
                  const std::vector<double>& dts, int rows, cudaStream_t s) {
  persist_free(pl);
  pl.rows = rows;
  pl.nfields = (int)hs.size();
  if (hs.empty()) {
    pl.valid = true;
    return DIM2D_OK;
  }
  const int n = (int)hs.size();
  std::vector<PDomain> dom(n);
  std::vector<std::vector<GhostRun>> ghosts(n);
  std::vector<int> sg;
  int maxnb = 0;
  for (int j = 0; j < n; j++) {
    const dim2d_handle* h = hs[j];
    PDomain& d = dom[j];
    d.f = h->f;
    d.buf[0] = h->A;
    d.buf[1] = h->B;
    d.buf[2] = h->C;
    d.dx = h->dx;
    d.dy = h->dy;
    d.rdx = h->rdx;
    d.rdy = h->rdy;
    d.dt = dts[j];
    d.xmap0 = h->xmap0;
    d.ymap0 = h->ymap0;
    d.periodic = h->periodic;
    d.wall_s = h->south_wall;
    d.open = h->open_mask;
    d.south_wall = h->south_wall;
    d.corners_y = h->corners_y;
    d.open_w = h->open_w;
    d.open_e = h->open_e;
    d.open_n = h->open_n;
    d.status = h->status;
    d.sx = (h->f.nx - 2 * BC + 29) / 30;  // 30 interior columns per strip
    d.nb = band_count(h->f.ny - 2 * BC, rows);
    d.band0 = (int)sg.size();
    d.nn = (h->periodic || h->open_all) ? 0 : (node_bc_count(node_args_of(h)) + 31) / 32;
    ghosts[j] = ghost_runs(h, rows, d.nb);
    for (int q = 0; q < d.nb; q++) sg.push_back(d.sx);
    for (const GhostRun& g : ghosts[j]) sg[d.band0 + g.band]++;
    maxnb = std::max(maxnb, d.nb);
  }
  std::vector<int> by_size(n), by_wall(n);
  for (int j = 0; j < n; j++) by_size[j] = by_wall[j] = j;
  std::stable_sort(by_size.begin(), by_size.end(), [&](int x, int y) {
    return (long long)dom[x].sx * dom[x].nb > (long long)dom[y].sx * dom[y].nb;
  });
  std::stable_sort(by_wall.begin(), by_wall.end(),
                   [&](int x, int y) { return dom[x].south_wall > dom[y].south_wall; });
  std::vector<PItem> items;
  for (int st = 1; st <= 3; st++) {
    for (int band = 0; band < maxnb; band++)
      for (int j : by_size) {
        if (band >= dom[j].nb) continue;
        for (const GhostRun& g : ghosts[j])
          if (g.band == band) items.push_back(PItem{j, PI_GHOST, st, g.first, g.count, band});
        for (int q = 0; q < dom[j].sx; q++)
          items.push_back(PItem{j, PI_STRIP, st, band * dom[j].sx + q,
                                strip_reads_node_ghosts(hs[j], dom[j], band, q, rows), band});
      }
    for (int j : by_wall)
      for (int q = 0; q < dom[j].nn; q++) items.push_back(PItem{j, PI_NODE, st, q, 0, 0});
  }
  pl.items_per_step = (long long)items.size();
  pl.nbands = (int)sg.size();
  pl.k = hs[0]->k;
  pl.wall = hs[0]->wall;
  pl.mixed = hs[0]->precision == DIM2D_MIXED;
  const size_t nctr = 1 + sg.size() + n;
  cudaError_t e = cudaMalloc(&pl.dom, sizeof(PDomain) * n);
  if (e == cudaSuccess) e = cudaMalloc(&pl.items, sizeof(PItem) * items.size());
  if (e == cudaSuccess) e = cudaMalloc(&pl.sg, sizeof(int) * sg.size());
  if (e == cudaSuccess) e = cudaMalloc(&pl.ctr, sizeof(unsigned long long) * nctr);
  if (e == cudaSuccess) e = cudaMalloc(&pl.ctl, sizeof(unsigned int) * 2);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(pl.dom, dom.data(), sizeof(PDomain) * n, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(pl.items, items.data(), sizeof(PItem) * items.size(),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(pl.sg, sg.data(), sizeof(int) * sg.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(pl.ctl, 0, sizeof(unsigned int) * 2, s);
  // the host tables go out of scope: the copies must land first
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    persist_free(pl);
    return cuda_error(e, "persistent kernel tables");
  }
  pl.valid = true;
  return DIM2D_OK;
}

cudaError_t persist_launch(PersistPlan& pl, int nsteps, int step0, double dt_scale,
                           unsigned long long wait_ns, long long withhold, cudaStream_t s) {
  if (pl.nfields == 0 || nsteps <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(
      pl.ctr, 0, sizeof(unsigned long long) * (1 + pl.nbands + pl.nfields), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(pl.ctl, 0, sizeof(unsigned int), s);  // abort flag
  if (e != cudaSuccess) return e;
  PersistArgs P{};
  P.k = pl.k;
  P.wall = pl.wall;
  P.dom = pl.dom;
  P.items = pl.items;
  P.sg = pl.sg;
  P.items_per_step = pl.items_per_step;
  P.nsteps = nsteps;
  P.step0 = step0 & 1;
  P.dt_scale = dt_scale;
  P.h_rows = pl.rows;
  P.next = pl.ctr;
  P.done = pl.ctr + 1;
  P.ndone = pl.ctr + 1 + pl.nbands;
  P.ctl = pl.ctl;
  P.wait_ns = wait_ns;
  P.withhold = withhold;
  return launch_batch_persistent(P, pl.mixed, s, &pl.ctas);
}

int persist_error(PersistPlan& pl) {
  if (!pl.ctl) return DIM2D_OK;
  unsigned int w = 0;
  cudaError_t e = cudaMemcpy(&w, pl.ctl + 1, sizeof w, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && w) e = cudaMemset(pl.ctl + 1, 0, sizeof(unsigned int));
  if (e != cudaSuccess) return cuda_error(e, "persistent kernel error word");
  if (w)
    return set_error(DIM2D_ERR_TIMEOUT,
                     "a work item of the persistent kernel waited longer than the limit for "
                     "the items before it (error word 0x%x); the launch stopped and the "
                     "fields' state is undefined", w);
  return DIM2D_OK;
}
