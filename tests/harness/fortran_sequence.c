/*
 * fortran_sequence.c -- drives libdim2d.so through include/dim2d.h with the
 * call sequence of the Fortran drop-in integrator
 * (dim2d_finite_volume_b200/fortran/td_integrator_class.f) under the
 * reference's driver loop (src/main/sim_dim2d.f:50-92), and checks every
 * state the driver would read against the oracle.
 *
 * Sequence (what the Fortran module does, call for call):
 *   dim2d_default_params; the run's constants written over it
 *   dim2d_create(params, nx, ny, bc_choice, bc_type, bc_order, precision)
 *   dim2d_upload(nodes, x_map, y_map, time)          first integrate
 *   loop t = 1..nt:  dim2d_step(h, dt, 1)             integrate
 *                    dim2d_download at the driver's output steps
 *                    (every int(1/detail_print) steps) and at t = nt
 *   dim2d_destroy
 * The oracle (test infrastructure, oracle/liboracle.so) advances the same
 * initial state step by step; at each downloaded step the harness prints
 * the normwise error per conservative variable (max|gpu - oracle| /
 * max|oracle| over the cells the field integrates) and fails above `tol`.
 *
 * Input: a binary case file written by tests/test_fortran_harness.py:
 *   int32 nx, ny, nt, precision, bc_choice[8], bc_type[8], bc_order[8]
 *   float64 dt, detail_print, time, tol, and the 16 dim2d_params values
 *   (re, we, pr, cv_r, viscous_r, gravity_ac, gravity, contact angle,
 *   heat source choice, max heat flux, center, variance, obc strategies,
 *   T0, flow_velocity), x_map[nx], y_map[ny], nodes[4][ny][nx]
 *   (Fortran nodes(nx,ny,4) after field%ini).
 * Exit status: 0 = every compared state within tol, 1 = above tol,
 * 2 = a library or input error.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dim2d.h"
#include "dim2d_oracle.h"

static int fail(const char *what, int rc) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, dim2d_last_error());
  return 2;
}

static int read_all(FILE *f, void *p, size_t size, size_t n) {
  return fread(p, size, n, f) == n ? 0 : -1;
}

/* max|a-b|/max|b| per variable over [i0,i1) x [j0,j1) */
static double compare(const double *a, const double *b, int nx, int ny, int i0, int i1, int j0,
                      int j1, double err[4]) {
  double worst = 0.0;
  for (int k = 0; k < 4; k++) {
    double num = 0.0, den = 0.0;
    for (int j = j0; j < j1; j++)
      for (int i = i0; i < i1; i++) {
        const size_t o = ((size_t)k * ny + j) * nx + i;
        const double d = fabs(a[o] - b[o]);
        if (!(d <= num)) num = d; /* a NaN makes num NaN */
        if (fabs(b[o]) > den) den = fabs(b[o]);
      }
    err[k] = den > 0.0 ? num / den : num;
    if (!(err[k] <= worst)) worst = err[k];
  }
  return worst;
}

int main(int argc, char **argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s case.bin\n", argv[0]);
    return 2;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) {
    perror(argv[1]);
    return 2;
  }
  int hdr[4], bc_choice[8], bc_type[8], bc_order[8];
  double sc[4], pv[16];
  if (read_all(f, hdr, sizeof(int), 4) || read_all(f, bc_choice, sizeof(int), 8) ||
      read_all(f, bc_type, sizeof(int), 8) || read_all(f, bc_order, sizeof(int), 8) ||
      read_all(f, sc, sizeof(double), 4) || read_all(f, pv, sizeof(double), 16)) {
    fprintf(stderr, "short case file\n");
    return 2;
  }
  const int nx = hdr[0], ny = hdr[1], nt = hdr[2], precision = hdr[3];
  const double dt = sc[0], detail_print = sc[1], time0 = sc[2], tol = sc[3];
  const size_t n = (size_t)4 * nx * ny;
  double *x_map = malloc(sizeof(double) * nx), *y_map = malloc(sizeof(double) * ny);
  double *nodes = malloc(sizeof(double) * n), *ref = malloc(sizeof(double) * n);
  if (!x_map || !y_map || !nodes || !ref) return 2;
  if (read_all(f, x_map, sizeof(double), nx) || read_all(f, y_map, sizeof(double), ny) ||
      read_all(f, nodes, sizeof(double), n)) {
    fprintf(stderr, "short case file\n");
    return 2;
  }
  fclose(f);
  memcpy(ref, nodes, sizeof(double) * n);

  /* td_integrator_class.f, dim2d_gpu_upload_field: default params, then
   * the run's compile-time constants */
  dim2d_params p;
  dim2d_default_params(&p);
  p.re = pv[0];
  p.we = pv[1];
  p.pr = pv[2];
  p.cv_r = pv[3];
  p.viscous_r = pv[4];
  p.gravity_ac = (int)pv[5];
  p.gravity = pv[6];
  p.wall_micro_contact_angle = pv[7];
  p.wall_heat_source_choice = (int)pv[8];
  p.wall_maximum_heat_flux = pv[9];
  p.wall_heat_source_center = pv[10];
  p.wall_heat_source_variance = pv[11];
  p.obc_eigenqties_strategy = (int)pv[12];
  p.obc_edge_flux_strategy = (int)pv[13];
  p.T0 = pv[14];
  p.flow_velocity = pv[15];

  dim2d_handle *h = NULL;
  int rc = dim2d_create(&p, nx, ny, bc_choice, bc_type, bc_order, precision, &h);
  if (rc) return fail("dim2d_create", rc);
  rc = dim2d_upload(h, nodes, x_map, y_map, time0);
  if (rc) return fail("dim2d_upload", rc);

  /* the oracle with the same constants and sections */
  orc_params op;
  orc_get_params(&op);
  op.re = p.re;
  op.we = p.we;
  op.pr = p.pr;
  op.cv_r = p.cv_r;
  op.viscous_r = p.viscous_r;
  op.gravity_ac = p.gravity_ac;
  op.gravity = p.gravity;
  op.wall_micro_contact_angle = p.wall_micro_contact_angle;
  op.wall_heat_source_choice = p.wall_heat_source_choice;
  op.wall_maximum_heat_flux = p.wall_maximum_heat_flux;
  op.wall_heat_source_center = p.wall_heat_source_center;
  op.wall_heat_source_variance = p.wall_heat_source_variance;
  op.obc_eigenqties_strategy = p.obc_eigenqties_strategy;
  op.obc_edge_flux_strategy = p.obc_edge_flux_strategy;
  op.T0 = p.T0;
  op.flow_velocity = p.flow_velocity;
  orc_set_params(&op);
  orc_cfg cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.nx = nx;
  cfg.ny = ny;
  cfg.periodic = bc_choice[DIM2D_SIDE_N] == DIM2D_PERIODIC_Y;
  for (int s = 0; s < 8; s++) {
    cfg.bc_choice[s] = bc_choice[s];
    cfg.bc_type[s] = bc_type[s];
    cfg.bc_order[s] = bc_order[s];
  }
  orc_clear_status();

  /* sim_dim2d.f:55-60 and :81-92: output every int(1/detail_print) steps */
  const int output_print = detail_print > 0.0 ? (int)(1.0 / detail_print) : 0;
  /* cells compared: all for periodic / open fields (their ghosts are
   * images or time-integrated), the interior otherwise */
  int all = 1;
  for (int s = 0; s < 8; s++) all = all && bc_type[s] == DIM2D_BC_TIMEDEV;
  all = all || cfg.periodic;
  const int g = all ? 0 : 2;
  int compared = 0, status = 0;
  double t_orc = time0, t_dev = 0.0;
  for (int t = 1; t <= nt; t++) {
    rc = dim2d_step(h, dt, 1);
    if (rc) return fail("dim2d_step", rc);
    if (orc_integrate(&cfg, ref, x_map, y_map, &t_orc, dt, 1) != 0) {
      fprintf(stderr, "oracle integrate failed at step %d\n", t);
      return 2;
    }
    const int output = output_print == 1 || (output_print != 0 && t % output_print == 0);
    if (!output && t != nt) continue;
    rc = dim2d_download(h, nodes, &t_dev);
    if (rc) return fail("dim2d_download", rc);
    double err[4];
    const double worst = compare(nodes, ref, nx, ny, g, nx - g, g, ny - g, err);
    printf("step %d time %.9g (oracle %.9g): err %.3e %.3e %.3e %.3e\n", t, t_dev, t_orc,
           err[0], err[1], err[2], err[3]);
    compared++;
    if (!(worst <= tol) || fabs(t_dev - t_orc) > 1e-12 * (fabs(t_orc) + 1.0)) status = 1;
  }
  rc = dim2d_destroy(h);
  if (rc) return fail("dim2d_destroy", rc);
  printf("%d states compared, tol %.1e: %s\n", compared, tol, status ? "FAIL" : "ok");
  free(x_map);
  free(y_map);
  free(nodes);
  free(ref);
  return status;
}
