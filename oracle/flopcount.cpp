// flopcount.cpp -- FP64 operations per cell-update of the oracle.
//
// TEST INFRASTRUCTURE ONLY.  Linked with the oracle's C sources compiled as
// C++ under flopcount.hpp (every double counts its arithmetic), it runs one
// RK3 step (compute_time_dev + stage, three times, with the boundary passes:
// td_integrator_class.f:103-161) of a 132 x 132 field (128^2 interior, the
// static-bubble size of the periodic workload) for the periodic_xy and
// hedstrom_xy presets, and one compute_time_dev alone, and prints the counts
// per interior cell as one JSON line.  The field is a tanh vapour bubble in
// liquid at T = 0.95 with a uniform x-velocity of 0.1 (the open preset's
// characteristic branches see a subsonic outflow on E and inflow on W).
// With an argument PREFIX it also writes the periodic field (PREFIX.nodes)
// and its time derivative (PREFIX.td) as raw doubles [4][ny][nx], so a test
// can check that the counting build computes what the oracle computes.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "dim2d_oracle.h"

// The oracle's prototypes above were read with double = fdouble; from here
// on double is the plain type again and fdouble names the counted one.
#undef double

FlopCounts g_flops;

namespace {

void reset() { g_flops = FlopCounts{0, 0, 0, 0, 0}; }

unsigned long long total() {
  return g_flops.add + g_flops.mul + g_flops.div + g_flops.sqrt + g_flops.transcendental;
}

void print_counts(const char* name, double cells, bool comma) {
  std::printf("\"%s\": {\"flops\": %.1f, \"add\": %.1f, \"mul\": %.1f, \"div\": %.1f, "
              "\"sqrt\": %.1f, \"transcendental\": %.1f}%s",
              name, (double)total() / cells, (double)g_flops.add / cells,
              (double)g_flops.mul / cells, (double)g_flops.div / cells,
              (double)g_flops.sqrt / cells, (double)g_flops.transcendental / cells,
              comma ? ", " : "");
}

// periodic_xy and hedstrom_xy as the library's presets number them
// (sections N,S,E,W,NE,NW,SE,SW; section ids SW=1 SE=2 NW=3 NE=4 S=5 E=6
// W=7 N=8; library_config.py:41-230)
orc_cfg preset(bool periodic, int n) {
  orc_cfg c;
  c.nx = n;
  c.ny = n;
  c.periodic = periodic ? 1 : 0;
  const int per_choice[8] = {ORC_PERIODIC_Y, ORC_PERIODIC_Y, ORC_PERIODIC_X, ORC_PERIODIC_X,
                             ORC_PERIODIC_X, ORC_PERIODIC_X, ORC_PERIODIC_X, ORC_PERIODIC_X};
  const int per_order[8] = {5, 8, 1, 2, 7, 6, 3, 4};
  const int open_order[8] = {1, 5, 2, 7, 6, 3, 8, 4};
  for (int s = 0; s < 8; s++) {
    c.bc_choice[s] = periodic ? per_choice[s] : ORC_HEDSTROM;
    c.bc_type[s] = periodic ? ORC_BC_NODES : ORC_BC_TIMEDEV;
    c.bc_order[s] = periodic ? per_order[s] : open_order[s];
  }
  return c;
}

void bubble(int n, const std::vector<fdouble>& x, const std::vector<fdouble>& y, double u0,
            std::vector<fdouble>& q) {
  const double T = 0.95, cv = 2.5, rl = 1.6, rv = 0.4, r0 = 0.1;
  const double w = 4.0 * (x[1].v - x[0].v);
  const size_t pl = (size_t)n * n;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      const double d = std::sqrt(x[i].v * x[i].v + y[j].v * y[j].v);
      const double r = 0.5 * (rl + rv) + 0.5 * (rl - rv) * std::tanh((d - r0) / w);
      const size_t o = (size_t)j * n + i;
      q[o] = r;
      q[o + pl] = r * u0;
      q[o + 2 * pl] = 0.0;
      q[o + 3 * pl] = r * (8.0 * cv * T / 3.0) - 3.0 * r * r + 0.5 * r * u0 * u0;
    }
}

void dump(const char* path, const std::vector<fdouble>& a) {
  std::FILE* fh = std::fopen(path, "wb");
  if (!fh) return;
  std::vector<double> plain(a.size());
  for (size_t i = 0; i < a.size(); i++) plain[i] = a[i].v;
  std::fwrite(plain.data(), sizeof(double), plain.size(), fh);
  std::fclose(fh);
}

}  // namespace

int main(int argc, char** argv) {
  const int n = 132;
  orc_params p;
  std::memset(&p, 0, sizeof p);
  p.re = 5.0;  // dim2d_parameters.f:179-199 (test set)
  p.we = 10.0;
  p.pr = 20.0;
  p.cv_r = 2.5;
  p.viscous_r = -1.5;
  p.wall_micro_contact_angle = 90.0;
  p.T0 = 0.95;
  p.flow_velocity = 0.1;
  orc_set_params(&p);
  orc_set_threads(1);

  std::vector<fdouble> x(n), y(n), q((size_t)4 * n * n), td((size_t)4 * n * n);
  orc_ini_coordinates(n, n, -0.5, 0.5, -0.5, 0.5, x.data(), y.data());
  const double cells = (double)(n - 4) * (n - 4);

  std::printf("{\"grid\": \"%dx%d\", \"interior_cells\": %d, ", n, n, (n - 4) * (n - 4));
  const char* names[2] = {"periodic_xy", "hedstrom_xy"};
  for (int k = 0; k < 2; k++) {
    const bool periodic = k == 0;
    const orc_cfg c = preset(periodic, n);
    bubble(n, x, y, periodic ? 0.0 : 0.1, q);
    if (periodic) orc_apply_bc_on_nodes(&c, 0.0, x.data(), y.data(), q.data(), q.data());
    reset();
    orc_compute_time_dev(&c, 0.0, q.data(), x.data(), y.data(), td.data());
    char nm[64];
    std::snprintf(nm, sizeof nm, "%s_time_dev", names[k]);
    print_counts(nm, cells, true);
    if (periodic && argc > 1) {
      std::string pre(argv[1]);
      dump((pre + ".nodes").c_str(), q);
      dump((pre + ".td").c_str(), td);
    }
    fdouble t = 0.0;
    reset();
    const int rc = orc_integrate(&c, q.data(), x.data(), y.data(), &t, 1e-5, 1);
    if (rc != 0) {
      std::fprintf(stderr, "flopcount: oracle integrate failed (%d)\n", rc);
      return 1;
    }
    std::snprintf(nm, sizeof nm, "%s_rk3_step", names[k]);
    print_counts(nm, cells, k == 0);
  }
  std::printf("}\n");
  return 0;
}
