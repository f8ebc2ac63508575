/*
 * dim2d_oracle.h -- CPU restatement of the reference's DIM time-derivative
 * hot path (jdesmarais/dim2D_finite_volume, Fortran).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker used by tests/,
 * by __graft_entry__.smoke() and by the cpu_baseline / reference legs of
 * bench.py.  No product code path links, loads or calls it.
 *
 * Layout: nodes(nx,ny,ne) in Fortran column-major order, i.e. the C array
 * q[k][j][i] with i fastest; all indices taken by the functions below are
 * 1-based like the Fortran source.  FP64 throughout
 * (src/parameters/parameters_kind.f:24-28, rkind = selected_real_kind(8)).
 */
#ifndef DIM2D_ORACLE_H
#define DIM2D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* src/parameters/parameters_constant.f:145-176 */
enum {
  ORC_PERIODIC_X = 0, ORC_PERIODIC_Y = 1, ORC_REFLECTION_X = 2,
  ORC_REFLECTION_Y = 3, ORC_HEDSTROM = 4, ORC_WALL = 7
};
enum { ORC_BC_NODES = 0, ORC_BC_FLUXES = 1, ORC_BC_TIMEDEV = 2, ORC_BC_FLUX_AND_NODE = 3 };
enum {
  ORC_SW_CORNER = 1, ORC_SE_CORNER = 2, ORC_NW_CORNER = 3, ORC_NE_CORNER = 4,
  ORC_S_EDGE = 5, ORC_E_EDGE = 6, ORC_W_EDGE = 7, ORC_N_EDGE = 8
};
/* cardinal slots used by the bc arrays below */
enum { ORC_N = 0, ORC_S = 1, ORC_E = 2, ORC_W = 3, ORC_NE = 4, ORC_NW = 5, ORC_SE = 6, ORC_SW = 7 };

/* Physical constants: src/physical_models/dim2d/dim2d_parameters.f:146-199
 * and the gravity switch of src/parameters/parameters_input.f:197-202. */
typedef struct {
  double re, we, pr, cv_r, viscous_r;
  int gravity_ac;
  double gravity;
  /* wall: src/parameters/parameters_input.f:526-624 */
  double wall_micro_contact_angle;   /* degrees */
  int wall_heat_source_choice;       /* 0 = no_heat_source */
  double wall_maximum_heat_flux;
  double wall_heat_source_center, wall_heat_source_variance;
  /* open bc: src/parameters/parameters_input.f:630-662 */
  int obc_eigenqties_strategy;       /* 0 = obc_eigenqties_bc */
  int obc_edge_flux_strategy;        /* 0 = capillarity */
  double T0, flow_velocity;          /* far field for obc_eigenqties_lin */
} orc_params;

/* Boundary configuration: one dispatcher entry per cardinal section,
 * src/boundary_conditions/bc_operators_gen_class.f:95-148,1260-1276.
 * periodic != 0 selects the legacy periodic_xy class
 * (src/boundary_conditions/periodic_xy/bc_operators_class.f:116-199). */
typedef struct {
  int nx, ny;
  int periodic;
  int bc_choice[8];
  int bc_type[8];
  int bc_order[8];
} orc_cfg;

void orc_set_params(const orc_params *p);
void orc_get_params(orc_params *p);
void orc_set_threads(int n);

/* --- unit-level entry points used by the golden-vector tests ---------- */
/* Mattsson operator `op` of operator set `set` at (i,j) applied to
 * mass_density, with the gradient procedure that set pairs with.
 * set 0: interior (sd_operators_class.f).
 * op: 0 f,1 dfdx,2 dfdy,3 d2fdx2,4 d2fdy2,5 d2fdxdy,6 gradient_x,
 *     7 g,8 dgdx,9 dgdy,10 d2gdx2,11 d2gdy2,12 d2gdxdy,13 gradient_y,
 *     14 dfdx_nl, 15 dgdy_nl, both of the test's gradient_av procedure. */
double orc_sd_operator(int set, int op, const double *nodes, int nx, int ny,
                       int i, int j, double dx, double dy);
/* one of the 26 DIM flux functions of dim2d_fluxes_module.f, index as in
 * test_lernaeanhydra/test_dim2d_fluxes.f:291-316 (1-based) */
double orc_flux_function(int which, const double *nodes, int nx, int ny,
                         int i, int j, double dx, double dy);
/* hedstrom_xy_module.f:445-558 at node (i,j): direction 0 = x, 1 = y;
 * oneside_right selects the R0 (else L0) one-sided gradient; side_right
 * the incoming-wave test of a right (E/N) side; obc_prim = the 5
 * eigen-quantities (rho,u,v,P,c) or NULL for obc_eigenqties_bc. */
void orc_timedev_with_openbc(const double *nodes, int nx, int ny, int i, int j, int dir_y,
                             int oneside_right, double dn, int side_right,
                             const double *obc_prim, double td[4]);
/* primitive helpers */
double orc_classical_pressure_local(const double q[4]);
double orc_speed_of_sound(const double q[4]);

/* --- field-level entry points ----------------------------------------- */
/* td_operators_class.f:119-235 (debug_initialize_timedev on) */
void orc_compute_time_dev(const orc_cfg *c, double t, const double *nodes,
                          const double *x_map, const double *y_map,
                          double *time_dev);
/* masked ("_nopt") interior operators of buffer-layer grids
 * (dim2d_oracle_masked.c): grdpts_id(nx,ny) with no_pt 0, interior_pt 1,
 * bc_interior_pt 2, bc_pt 3; borders 1-based inclusive */
void orc_compute_time_dev_masked(int nx, int ny, const double *nodes, const int *grdpts_id,
                                 double dx, double dy, const int xb[2], const int yb[2],
                                 double *time_dev);
void orc_rk_stage_masked(int stage, int nx, int ny, double *nodes, double *nodes_tmp,
                         const double *time_dev, const int *grdpts_id, double dt,
                         const int xb[2], const int yb[2]);
/* field_abstract_class.f:447-463 -> bc dispatcher */
void orc_apply_bc_on_nodes(const orc_cfg *c, double t, const double *x_map,
                           const double *y_map, const double *nodes_tmp,
                           double *nodes);
/* td_integrator_class.f:103-161 + field_class.f:61-72, nsteps times;
 * x/y_borders from field_abstract_class.f:244-270.  Returns 0. */
int orc_integrate(const orc_cfg *c, double *nodes, const double *x_map,
                  const double *y_map, double *t, double dt, int nsteps);
/* field_abstract_class.f:286-315 */
void orc_ini_coordinates(int nx, int ny, double x_min, double x_max,
                         double y_min, double y_max, double *x_map,
                         double *y_map);

/* debug_real = NF90_FILL_DOUBLE, parameters_input.f:892 */
double orc_debug_real(void);

/* wall operator status: 0 ok, 1 root not bracketed, 2-4 Ridders failures
 * (where the reference stops the program) */
int orc_status(void);
void orc_clear_status(void);

/* wall_xy_equilibrium_module.f unit functions (known-answer tests) */
double orc_md_vapor(double T);
double orc_md_liquid(double T);
double orc_dwall_internal_energy_dmd(double md, double T, double micro_angle);
double orc_temperature_average(double T0, double delta_x, double q);
double orc_wall_temperature(double md, double g2, double vx, double vy, double Ed);
double orc_dmddx(double delta, const double tab[3], int grad_type);
double orc_wall_equilibrium_root_fct(double md, const double md_x[2], const double md_y[2],
                                     double vx, double vy, double Ed, double delta_x,
                                     double delta_y, double micro_angle, double q,
                                     int grad_type_x, int grad_type_y);
double orc_wall_heat_flux(double t, double x, double y);
/* compute_wall_flux_x at face (i,j) with the interior operators */
void orc_wall_flux_x_at(const double *nodes, int nx, int ny, int i, int j, double t,
                        const double *x_map, const double *y_map, int side_right, double f[4]);

#ifdef __cplusplus
}
#endif
#endif
