// Host emulation of the node boundary kernel: runs node_bc_cell() (the
// exact per-thread code of k_node_bc) on the CPU for every thread index of
// the launch plus out-of-range ones.  Reads and writes are checked against
// the two fields, and a read of a value that another thread index wrote
// counts as a race (threads of one launch are unordered on the GPU).
// Used by tests/test_nodebc_emulation.py.
#include <cstdio>
#include <cstdlib>
#include <vector>
static const double *g_lo0, *g_hi0, *g_lo1, *g_hi1;
static long g_bad = 0, g_race = 0, g_cur = 0;
static std::vector<long> g_writer;
static inline double chk(const double* p) {
  if (p >= g_lo1 && p < g_hi1) {
    long w = g_writer[p - g_lo1];
    if (w >= 0 && w != g_cur) g_race++;
    return *p;
  }
  if (p >= g_lo0 && p < g_hi0) return *p;
  g_bad++;
  return 0.0;
}
static inline void emu_store(double* p, double v) {
  if (p < g_lo1 || p >= g_hi1) { g_bad++; return; }
  g_writer[p - g_lo1] = g_cur;
  *p = v;
}
#define DIM2D_LDG_HOST(p) chk(p)
#define DIM2D_ST_HOST(p, v) emu_store(p, v)
#include "../../dim2d_finite_volume_b200/csrc/dim2d_nodebc.cu"
using namespace dim2d;
int main(int argc, char** argv) {
  FILE* fi = fopen(argv[1], "rb");
  int hdr[7];  // nx, ny, south_wall, corners_y, open_w, open_e, open_n
  double par[10];  // dx, dy, re, we, pr, cv_r, viscous_r, cos_angle, xmap0, qconst
  if (fread(hdr, 4, 7, fi) != 7 || fread(par, 8, 10, fi) != 10) return 2;
  const int nx = hdr[0], ny = hdr[1];
  const size_t plane = (size_t)nx * ny;
  std::vector<double> ut(4 * plane), u(4 * plane);
  if (fread(ut.data(), 8, 4 * plane, fi) != 4 * plane) return 2;
  if (fread(u.data(), 8, 4 * plane, fi) != 4 * plane) return 2;
  fclose(fi);
  g_lo0 = ut.data(); g_hi0 = ut.data() + 4 * plane;
  g_lo1 = u.data(); g_hi1 = u.data() + 4 * plane;
  g_writer.assign(4 * plane, -1);
  NodeBcArgs a{};
  a.utmp = ut.data(); a.u = u.data();
  a.f.nx = nx; a.f.ny = ny; a.f.pitch = nx; a.f.plane = plane;
  a.dx = par[0]; a.dy = par[1]; a.rdx = 1.0 / par[0]; a.rdy = 1.0 / par[1];
  a.south_wall = hdr[2]; a.corners_y = hdr[3];
  a.open_w = hdr[4]; a.open_e = hdr[5]; a.open_n = hdr[6];
  unsigned int status = 0; a.status = &status;
  DimConst& k = a.k;
  k.re = par[2]; k.we = par[3]; k.pr = par[4]; k.cv_r = par[5]; k.viscous_r = par[6];
  k.ire = 1.0 / k.re; k.iwe = 1.0 / k.we; k.ipr = 1.0 / k.pr; k.irepr = 1.0 / (k.re * k.pr);
  k.c15cv = 1.5 / k.cv_r; k.c3cv = 3.0 / k.cv_r; k.two_mu = 2.0 + k.viscous_r;
  k.c38cv = 3.0 / (8.0 * k.cv_r);
  a.wall.cos_angle = par[7]; a.xmap0 = par[8];
  a.wall.heat_choice = par[9] != 0.0 ? 1 : 0; a.wall.qmax = par[9];
  const int total = node_bc_count(a);
  for (int m = -3; m < total + 200; m++) { g_cur = m; node_bc_cell(a, m); }
  printf("total=%d bad=%ld race=%ld status=%u\n", total, g_bad, g_race, status);
  FILE* fo = fopen(argv[2], "wb");
  fwrite(u.data(), 8, 4 * plane, fo);
  fclose(fo);
  return 0;
}
