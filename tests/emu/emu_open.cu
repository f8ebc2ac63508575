// Host emulation of the open-boundary kernel: runs open_ghost_cell() (the
// exact per-cell code of the sm_100a kernel) on the CPU for every thread
// index of the launch plus out-of-range ones, with every read checked
// against the field and guard zones around the output.  Used by
// tests/test_open_emulation.py.
#include <cstdio>
#include <cstdlib>
#include <vector>
static const double* g_lo; static const double* g_hi; static long g_bad = 0;
static inline double chk(const double* p) { if (p < g_lo || p >= g_hi) { g_bad++; return 0.0; } return *p; }
#define DIM2D_LDG_HOST(p) chk(p)
#include "../../dim2d_finite_volume_b200/csrc/dim2d_open.cu"
using namespace dim2d;
int main(int argc, char** argv) {
  FILE* fi = fopen(argv[1], "rb");
  int nx, ny; double dx, dy; double par[5];
  fread(&nx, 4, 1, fi); fread(&ny, 4, 1, fi); fread(&dx, 8, 1, fi); fread(&dy, 8, 1, fi); fread(par, 8, 5, fi);
  size_t plane = (size_t)nx * ny;
  std::vector<double> u(4 * plane); fread(u.data(), 8, 4 * plane, fi); fclose(fi);
  std::vector<double> out(12 * plane, -777.0);  // guard zones before and after
  g_lo = u.data(); g_hi = u.data() + 4 * plane;
  StageArgs a{}; a.uin = u.data(); a.u0 = u.data(); a.uout = out.data() + 4 * plane;
  a.f.nx = nx; a.f.ny = ny; a.f.pitch = nx; a.f.plane = plane; a.rdx = 1.0 / dx; a.rdy = 1.0 / dy; a.dx = dx; a.dy = dy;
  DimConst& k = a.k; k.re = par[0]; k.we = par[1]; k.pr = par[2]; k.cv_r = par[3]; k.viscous_r = par[4];
  k.ire = 1.0 / k.re; k.iwe = 1.0 / k.we; k.ipr = 1.0 / k.pr; k.irepr = 1.0 / (k.re * k.pr); k.c15cv = 1.5 / k.cv_r; k.c3cv = 3.0 / k.cv_r; k.two_mu = 2.0 + k.viscous_r;
  k.c38cv = 3.0 / (8.0 * k.cv_r);
  // optional: open-section mask, south wall flag, x_map(1), constant wall heat flux
  a.open = argc > 3 ? atoi(argv[3]) : OPEN_ALL;
  a.wall_s = argc > 4 ? atoi(argv[4]) : 0;
  a.xmap0 = argc > 5 ? atof(argv[5]) : 0.0;
  const double qc = argc > 6 ? atof(argv[6]) : 0.0;
  a.wall.cos_angle = argc > 7 ? atof(argv[7]) : 0.0;
  a.wall.heat_choice = qc != 0.0 ? 1 : 0; a.wall.qmax = qc;
  int total = open_ghost_count(a.f, a.open);
  for (int m = -3; m < total + 300; m++) open_ghost_cell(a, m, 0);
  long guard = 0; for (size_t i = 0; i < 4 * plane; i++) { if (out[i] != -777.0) guard++; if (out[8 * plane + i] != -777.0) guard++; }
  long written = 0; for (size_t i = 4 * plane; i < 8 * plane; i++) if (out[i] != -777.0) written++;
  printf("total=%d bad_reads=%ld guard_writes=%ld written=%ld expected=%ld\n", total, g_bad, guard, written, 4L * total);
  FILE* fo = fopen(argv[2], "wb"); fwrite(out.data() + 4 * plane, 8, 4 * plane, fo); fclose(fo);
  return 0;
}
