/*
 * dim2d.h -- C ABI of the B200 (sm_100a) DIM time-derivative library.
 *
 * Drop-in boundary for the reference's time integration of one field
 * (jdesmarais/dim2D_finite_volume, Fortran).  Each entry point names the
 * reference interface it replaces:
 *
 *   field%integrate(dt)                 src/field/field_class.f:61-72
 *   td_integrator%integrate(field, dt)  src/td_integrator/rungekutta3rdtvd/
 *                                       td_integrator_class.f:103-161
 *   field%compute_time_dev()            src/field/field_abstract_class.f:360-379
 *     -> td_operators%compute_time_dev  src/td_operators/finitevolume/
 *                                       td_operators_class.f:119-235
 *   field%apply_bc_on_nodes(nodes_tmp)  src/field/field_abstract_class.f:447-463
 *   field%ini_coordinates()             src/field/field_abstract_class.f:286-315
 *
 * Conventions
 *   - nodes(nx,ny,ne=4) FP64 in Fortran column-major order: the C array
 *     q[k][j][i], i fastest (what c_loc(field%nodes) points to).
 *   - nx, ny include bc_size = 2 ghost layers per side
 *     (src/parameters/parameters_input.f:81).
 *   - Every call returns DIM2D_OK (0) or a positive error code; the
 *     reference stops the process on errors (src/parameters/errors_module.f),
 *     a Fortran shim turns a non-zero status into `stop`.
 *   - A handle is used by one host thread at a time.  Calls are ordered on
 *     the handle's CUDA stream; dim2d_download and dim2d_sync synchronise.
 */
#ifndef DIM2D_H
#define DIM2D_H

#include <stddef.h>

#if defined(__GNUC__)
#define DIM2D_API __attribute__((visibility("default")))
#else
#define DIM2D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DIM2D_OK 0
#define DIM2D_ERR_ARG 1          /* invalid argument */
#define DIM2D_ERR_CUDA 2         /* CUDA runtime error (see dim2d_last_error) */
#define DIM2D_ERR_UNSUPPORTED 3  /* boundary configuration not provided */
#define DIM2D_ERR_NOMEM 4        /* device allocation refused */
#define DIM2D_ERR_WALL_ROOT 5    /* wall ghost-cell root not bracketed / not converged */
#define DIM2D_ERR_TIMEOUT 6      /* a bounded device wait expired */
#define DIM2D_ERR_NOT_READY 7    /* state not uploaded yet */
#define DIM2D_ERR_NONFINITE 8    /* a served request's state is no longer finite */

/* boundary choices: src/parameters/parameters_constant.f:145-152 */
#define DIM2D_PERIODIC_X 0
#define DIM2D_PERIODIC_Y 1
#define DIM2D_REFLECTION_X 2
#define DIM2D_REFLECTION_Y 3
#define DIM2D_HEDSTROM 4
#define DIM2D_WALL 7
/* boundary application types: parameters_constant.f:158-161 */
#define DIM2D_BC_NODES 0
#define DIM2D_BC_FLUXES 1
#define DIM2D_BC_TIMEDEV 2
#define DIM2D_BC_FLUX_AND_NODE 3
/* section types used by bc_order: parameters_constant.f:165-172 */
#define DIM2D_SW_CORNER 1
#define DIM2D_SE_CORNER 2
#define DIM2D_NW_CORNER 3
#define DIM2D_NE_CORNER 4
#define DIM2D_S_EDGE 5
#define DIM2D_E_EDGE 6
#define DIM2D_W_EDGE 7
#define DIM2D_N_EDGE 8
/* cardinal slots of the bc_choice / bc_type arrays */
#define DIM2D_SIDE_N 0
#define DIM2D_SIDE_S 1
#define DIM2D_SIDE_E 2
#define DIM2D_SIDE_W 3
#define DIM2D_SIDE_NE 4
#define DIM2D_SIDE_NW 5
#define DIM2D_SIDE_SE 6
#define DIM2D_SIDE_SW 7

/* precision of the stencil/flux pass.  DIM2D_MIXED: the node pass (van der
 * Waals inversion for velocities, pressure, temperatures) runs in FP64 and
 * leaves FP32 copies of the node state and quantities in shared memory; the
 * face pass (stencils and flux formulas) reads those FP32 copies and runs in
 * FP32, except the third-derivative capillary term (normal derivative of
 * the capillary temperature), which stays FP64; divergence and RK
 * accumulation are FP64 on the FP64 state in HBM.  Error against the FP64
 * path: <= 1e-5 normwise on the state (see the library's tests). */
#define DIM2D_FP64 0
#define DIM2D_MIXED 1

/* Physical and boundary constants.  The reference holds these as
 * compile-time Fortran parameters:
 *   re, we, pr, cv_r, viscous_r   src/physical_models/dim2d/dim2d_parameters.f:146-199
 *   gravity_ac, gravity           src/parameters/parameters_input.f:197-202
 *   wall_*                        src/parameters/parameters_input.f:526-624
 *   obc_*, T0, flow_velocity      src/parameters/parameters_input.f:127-157,630-662 */
typedef struct dim2d_params {
  double re, we, pr, cv_r, viscous_r;
  int gravity_ac;
  double gravity;
  double wall_micro_contact_angle; /* degrees */
  int wall_heat_source_choice;     /* 0 = no_heat_source */
  double wall_maximum_heat_flux;
  double wall_heat_source_center, wall_heat_source_variance;
  int obc_eigenqties_strategy;     /* 0 = obc_eigenqties_bc */
  int obc_edge_flux_strategy;      /* 0 = obc_edge_flux_capillarity */
  double T0, flow_velocity;
} dim2d_params;

typedef struct dim2d_handle dim2d_handle;

/* Fill *p with the reference's "for tests" constant set
 * (dim2d_parameters.f:179-187: Re=5, We=10, Pr=20, cv_r=2.5,
 * viscous_r=-1.5), no gravity, 90 degree contact angle, no heat source. */
DIM2D_API void dim2d_default_params(dim2d_params *p);

/* Create a solver for one nx x ny field (ghosts included) on the current
 * CUDA device.  bc_choice/bc_type are indexed by DIM2D_SIDE_*; bc_order
 * lists the 8 DIM2D_*_EDGE/CORNER section types in node-BC order
 * (parameters_input.f:397-453).  A periodic domain is bc_choice =
 * PERIODIC_Y on N/S and PERIODIC_X elsewhere (library_config.py:72-87),
 * all types DIM2D_BC_NODES; it selects the periodic_xy operator
 * (src/boundary_conditions/periodic_xy/bc_operators_class.f:116-199).
 * The other accepted configurations are the reference's presets
 * (library_config.py:58-150): hedstrom_xy, reflection_xy,
 * wall_S_reflection, wall_S_open and half_wall_S_open, each with the
 * types its choices imply (reflection: BC_NODES, wall: BC_FLUX_AND_NODE,
 * hedstrom: BC_TIMEDEV); anything else returns DIM2D_ERR_UNSUPPORTED, as
 * does a half_wall_S_open bc_order with the S edge before the W edge or
 * the SW corner before the S edge.
 * Allocates three device copies of the field.
 * Replaces: field%ini + td_integrator selection (field_abstract_class.f:148-198). */
DIM2D_API int dim2d_create(const dim2d_params *p, int nx, int ny, const int bc_choice[8],
                 const int bc_type[8], const int bc_order[8], int precision,
                 dim2d_handle **out);

/* Copy nodes(nx,ny,4), x_map(nx), y_map(ny) and the time to the device.
 * dx = x_map(2)-x_map(1), dy = y_map(2)-y_map(1) as in
 * td_operators_class.f:157-158. */
DIM2D_API int dim2d_upload(dim2d_handle *h, const double *nodes, const double *x_map,
                 const double *y_map, double t);

/* nsteps calls of field%integrate(dt): three RK3-TVD stages each with
 * compute_time_dev, the stage update and apply_bc_on_nodes
 * (td_integrator_class.f:103-161, rk3tvd_steps_module.f:52-490), time += dt.
 * Each step replays a CUDA graph captured on first use for this dt (one
 * per buffer parity; not while profiling or when disabled with
 * dim2d_set_graphs); launches and results are those of the stream path. */
DIM2D_API int dim2d_step(dim2d_handle *h, double dt, int nsteps);
/* No counterpart in the reference.  Enable (default) or disable the step
 * graphs of dim2d_step. */
DIM2D_API int dim2d_set_graphs(dim2d_handle *h, int enable);

/* time_dev(nx,ny,4) = L(nodes) of the resident state, interior cells (and
 * the ghost cells of time-derivative boundaries); other cells are written
 * with debug_real = NF90_FILL_DOUBLE like td_operators_class.f:150-154. */
DIM2D_API int dim2d_time_dev(dim2d_handle *h, double *time_dev);

/* field%apply_bc_on_nodes on the resident state, with nodes_tmp = nodes
 * (field_abstract_class.f:190-193). */
DIM2D_API int dim2d_apply_bc_on_nodes(dim2d_handle *h);

/* Copy the resident state (and time) back to the host; synchronises. */
DIM2D_API int dim2d_download(dim2d_handle *h, double *nodes, double *t);
/* No counterpart in the reference (its output is synchronous,
 * io_operators_class.f): queue a copy of the resident state into host
 * memory `nodes` (nodes(nx,ny,4) layout) on a side stream and return
 * without waiting; *t receives the time of that state.  The copy overlaps
 * the next dim2d_step; the step after it (the first to overwrite the
 * copied buffer) waits for the copy, as do uploads and boundary passes.
 * `nodes` must stay valid until the copy has landed: dim2d_copy_done
 * returns 1 (0 while in flight), or after dim2d_sync.  For overlap, `nodes`
 * must be pinned (dim2d_host_alloc).  Refused for batch members. */
DIM2D_API int dim2d_download_async(dim2d_handle *h, double *nodes, double *t);
DIM2D_API int dim2d_copy_done(dim2d_handle *h);
/* pinned host memory for dim2d_download_async / dim2d_upload */
DIM2D_API int dim2d_host_alloc(size_t bytes, void **p);
DIM2D_API int dim2d_host_free(void *p);

/* dt = cfl * min(dx,dy) / max over interior nodes of (c + |u|), speed of
 * sound from dim2d_prim_module.f:1179-1215, reduced on the device. */
DIM2D_API int dim2d_cfl_dt(dim2d_handle *h, double cfl, double *dt);

/* Run on the given CUDA stream (cudaStream_t) instead of the handle's own. */
DIM2D_API int dim2d_set_stream(dim2d_handle *h, void *stream);
/* Wait for all work queued on the handle (asynchronous downloads included). */
DIM2D_API int dim2d_sync(dim2d_handle *h);
/* Device pointer of the resident nodes (layout: 4 planes of ny rows of
 * `pitch` doubles) -- for callers that keep fields in HBM. */
DIM2D_API int dim2d_device_state(dim2d_handle *h, double **nodes, int *pitch);
/* Number of kernel launches issued by this handle so far. */
DIM2D_API long long dim2d_launch_count(const dim2d_handle *h);
/* Live kernel timing for roofline reports: while enabled, every launch of
 * the fused interior stage kernel is bracketed by CUDA events on the
 * handle's stream.  dim2d_profile_read synchronises and returns the summed
 * device time (ms) and the number of timed launches since enabling. */
DIM2D_API int dim2d_profile(dim2d_handle *h, int enable);
DIM2D_API int dim2d_profile_read(dim2d_handle *h, double *ms, long long *launches);

/* No counterpart in the reference (its stage loops have one fixed shape).
 * Stage-kernel variant: 0 = 32x8-cell CTA tiles; 1..5 = warp-streaming
 * strips 30 columns wide with (rows per warp, warps per CTA, resident CTAs
 * per SM) = (8,4,4), (16,4,4), (16,4,5), (16,2,8), (16,8,2) (FP64 fields
 * fit 16 warps per SM whatever the request; DIM2D_MIXED fields on (16,4,5)
 * run 20); 6 = the
 * persistent kernel of batches (dim2d_batch_set_persistent) over this field
 * alone: each dim2d_step call is one launch whose warps take 16-row strips
 * stage by stage, a band starting its next stage as soon as it and its
 * neighbours have finished the previous one (no field-wide stage
 * boundary); its tables are built on the first step with a new dt and
 * kept while dt and the grid are unchanged.  Every variant evaluates the
 * same face fluxes; results agree to rounding. */
#define DIM2D_NUM_VARIANTS 7
DIM2D_API int dim2d_set_variant(dim2d_handle *h, int variant);
DIM2D_API int dim2d_get_variant(const dim2d_handle *h);
/* Autotuner: times every variant on the resident field (dry RK3 steps with
 * dt = 0 that write only the two stage buffers; the state is not
 * modified), selects the fastest and caches the choice for fields of the
 * same size and boundary class in this process.  times_ms (optional,
 * DIM2D_NUM_VARIANTS entries) receives the average dry-step time of each
 * variant; passing it forces a new measurement. */
DIM2D_API int dim2d_autotune(dim2d_handle *h, int *chosen, double *times_ms);

DIM2D_API int dim2d_destroy(dim2d_handle *h);

/* No counterpart in the reference.  The RK3 time step for callers that
 * cannot allocate device memory -- hosts whose HBM is handed out by their
 * own pool or arena, or time-stepping loops that must not call cudaMalloc
 * because it synchronises the device.  The stages and boundary passes of
 * dim2d_step for the two configurations without a node boundary pass:
 * periodic_xy and hedstrom_xy (any other bc_choice / bc_type returns
 * DIM2D_ERR_UNSUPPORTED).  The caller passes the field as a device pointer
 * `nodes` (Fortran layout nodes(nx,ny,4), ghosts included, updated in
 * place) and x_map/y_map as host arrays.  The two stage copies live in one
 * file-scope __device__ array of 2 x 4 x DIM2D_NOALLOC_MAX_CELLS doubles
 * (16 MiB), held on every GPU that loads the library until exit; larger
 * fields (nx*ny > DIM2D_NOALLOC_MAX_CELLS) are rejected with
 * DIM2D_ERR_ARG.  Nothing is allocated: no cudaMalloc / cudaFree.  All
 * calls on a device share that array and it keeps the last call's
 * contents (each call clears what it uses first); calls that overlap on
 * the GPU race on it, so order them on one stream.  The first call in a
 * CUDA context looks up the array's address with that context current and
 * keeps it for that context (a new context, e.g. after cudaDeviceReset,
 * gets its own lookup): make that first call before any stream capture.
 * `stream` is a cudaStream_t (NULL = legacy default stream); the call
 * returns without synchronising.  After a non-zero return the contents of
 * `nodes` are undefined. */
#define DIM2D_NOALLOC_MAX_CELLS 262144
DIM2D_API int dim2d_step_noalloc(const dim2d_params *p, int nx, int ny, const int bc_choice[8],
                                 const int bc_type[8], const int bc_order[8], double *nodes,
                                 const double *x_map, const double *y_map, double dt,
                                 int nsteps, void *stream);

/* ---- Masked operators of buffer-layer grids.  A buffer layer carries its
 * own nodes(nx,ny,4) and grdpts_id(nx,ny) map: no_pt 0, interior_pt 1,
 * bc_interior_pt 2, bc_pt 3 (parameters_bf_layer.f:41-44).  These two calls
 * do the area-sized work of stepping one on the device; the layer's
 * boundary sections (bc_pt / bc_interior_pt points) remain the host-driven
 * layer code's.  All arrays are device pointers owned by the caller, in the
 * reference's layout (pitch nx); borders are 1-based inclusive, host arrays;
 * `stream` is a cudaStream_t (NULL = legacy default stream); the calls
 * return without synchronising and allocate nothing.
 *
 * Time derivative at the interior_pt points inside the borders (and at
 * least bc_size points from the grid's edges), written into time_dev;
 * every other point of time_dev is left as it is.  Every face of an
 * interior_pt point must lie between interior_pt / bc_interior_pt points,
 * as the reference's layers are built.
 * Replaces: the interior part of td_operators%compute_time_dev_nopt
 * (td_operators_class.f:293-417, fluxes pmodel_eq_class.f:1215-1360). */
DIM2D_API int dim2d_time_dev_masked(const dim2d_params *p, int nx, int ny, const double *nodes,
                                    const int *grdpts_id, double dx, double dy,
                                    const int x_borders[2], const int y_borders[2],
                                    double *time_dev, void *stream);
/* RK3-TVD stage `stage` (1, 2, 3) in place on nodes, nodes_tmp = u^n:
 * stage 1 over every point that is not no_pt (nodes_tmp receives u^n),
 * stages 2 and 3 over those inside the borders.
 * Replaces: compute_1st/2nd/3rd_step_nopt (rk3tvd_steps_module.f:130-614). */
DIM2D_API int dim2d_rk_stage_masked(int stage, int nx, int ny, double *nodes, double *nodes_tmp,
                                    const double *time_dev, const int *grdpts_id, double dt,
                                    const int x_borders[2], const int y_borders[2],
                                    void *stream);

/* ---- Batches: no counterpart in the reference (one field per process
 * there).  A batch advances many fields together: one launch per RK stage
 * per boundary kind covers all its fields, and a step is a captured CUDA
 * graph with one independent chain per kind (periodic_xy, hedstrom_xy,
 * wall_S_reflection, reflection_xy), so the kinds overlap on the device.
 * Members are fields created with dim2d_create and uploaded, on the
 * batch's device, sharing one dim2d_params (FP64 and DIM2D_MIXED fields
 * form separate groups); the batch borrows their
 * buffers and advances their state and time (wall_S_open and
 * half_wall_S_open fields join the wall_S_reflection chain).
 * While a field is a member,
 * dim2d_step on it is refused; dim2d_download/dim2d_time_dev of a member
 * are ordered after the batch's queued steps.  dim2d_destroy of a member
 * removes it first. */
typedef struct dim2d_batch dim2d_batch;
/* groups: periodic, open, wall_S, reflection (FP64), then the same four for
 * DIM2D_MIXED fields */
#define DIM2D_BATCH_GROUPS 8
DIM2D_API int dim2d_batch_create(dim2d_batch **out);
/* add a field that advances by dt per step */
DIM2D_API int dim2d_batch_add(dim2d_batch *b, dim2d_handle *h, double dt);
DIM2D_API int dim2d_batch_remove(dim2d_batch *b, dim2d_handle *h);
DIM2D_API int dim2d_batch_set_dt(dim2d_batch *b, dim2d_handle *h, double dt);
/* nsteps RK3 steps of every member (graph replays unless disabled) */
DIM2D_API int dim2d_batch_step(dim2d_batch *b, int nsteps);
/* wait for the batch and check the members' wall status words */
DIM2D_API int dim2d_batch_sync(dim2d_batch *b);
/* strip shape (0..4 = dim2d_set_variant 1..5) of one group */
DIM2D_API int dim2d_batch_set_shape(dim2d_batch *b, int group, int shape);
DIM2D_API int dim2d_batch_set_graphs(dim2d_batch *b, int enable);
/* Persistent mode (enable != 0): dim2d_batch_step(b, n) is one launch of a
 * persistent kernel per precision (FP64, DIM2D_MIXED) that advances every
 * member by n steps.  Its warps take work items from one queue -- per step
 * and stage, the ghost cells of open sections and the strips of every
 * member, then the node boundary passes -- and an item starts once the
 * items of its field that it depends on have completed (the previous stage
 * on its row band and the two next to it, the previous node pass), so fields
 * of every boundary kind and size advance together without grid-wide
 * barriers.  The per-cell code is the graph mode's; results agree with it to
 * rounding (the compiler may contract the two instantiations differently).
 * Each wait
 * is bounded (dim2d_batch_set_wait_limit, default 2 s); one that runs out
 * stops the launch and dim2d_batch_sync returns DIM2D_ERR_TIMEOUT. */
DIM2D_API int dim2d_batch_set_persistent(dim2d_batch *b, int enable);
/* rows of one strip work item of the persistent kernel: 8, 16 (default) or
 * 32; dim2d_batch_autotune picks it in persistent mode */
DIM2D_API int dim2d_batch_set_rows(dim2d_batch *b, int rows);
DIM2D_API int dim2d_batch_set_wait_limit(dim2d_batch *b, double seconds);
/* For tests of the bounded waits: in the next persistent launches, the
 * completion of work item `item` (an index into the launch's item order)
 * is not signalled, so the items of its field that follow wait until the
 * limit runs out; -1 (default) turns this off. */
DIM2D_API int dim2d_batch_withhold_item(dim2d_batch *b, long long item);
/* Autotuner: times dry steps (dt = 0, stage buffers only) of each group
 * for the 5 strip shapes and keeps the fastest; chosen[8] receives the
 * shapes, times_ms (optional) 8 x 5 dry-step times (0 for empty groups).
 * In persistent mode it times dry launches with 8, 16 and 32 rows per
 * strip item instead: chosen[g] receives the rows kept and times_ms[g*5 +
 * 0..2] the three times, for every g. */
DIM2D_API int dim2d_batch_autotune(dim2d_batch *b, int chosen[8], double *times_ms);
DIM2D_API int dim2d_batch_size(const dim2d_batch *b);
DIM2D_API long long dim2d_batch_launch_count(const dim2d_batch *b);
/* interior cells of all members (cell-updates per batch step) */
DIM2D_API long long dim2d_batch_cells(const dim2d_batch *b);
DIM2D_API int dim2d_batch_set_stream(dim2d_batch *b, void *stream);
DIM2D_API int dim2d_batch_destroy(dim2d_batch *b);

/* ---- Serving loop: no counterpart in the reference.  Requests (a
 * field's initial state, dt and step count) arrive at any time; the server
 * keeps their fields resident in HBM, admits them in arrival order while
 * their three device copies fit the memory budget, and advances all
 * admitted fields together in batched chunks of up to chunk_steps steps
 * (continuous batching: requests join and leave between chunks, the next
 * chunk is queued while the host admits and retires).  Fields come from
 * the device's stream-ordered pool; results land in pinned host memory.
 * dim2d_server_poll drives the loop (wait != 0: block until the oldest
 * queued chunk has finished); call it repeatedly.  Requests are FP64 or
 * DIM2D_MIXED, each in its own precision.  Behind every chunk the server
 * checks each member: a request whose interior state is no longer finite,
 * or whose wall ghost-cell root failed, leaves at the next chunk boundary
 * (one or two chunks later) with the state and time it has, instead of
 * being stepped to its last step. */
typedef struct dim2d_server dim2d_server;
/* mem_budget: bytes of device memory for fields (0 = free memory less a
 * reserve; larger values are capped the same way) */
DIM2D_API int dim2d_server_create(const dim2d_params *p, size_t mem_budget, int chunk_steps,
                                  dim2d_server **out);
/* copies the inputs; *id identifies the request */
DIM2D_API int dim2d_server_submit(dim2d_server *s, int nx, int ny, const int bc_choice[8],
                                  const int bc_type[8], const int bc_order[8], int precision,
                                  const double *nodes, const double *x_map, const double *y_map,
                                  double dt, long long nsteps, long long *id);
/* *completed = requests completed by this call */
DIM2D_API int dim2d_server_poll(dim2d_server *s, int wait, int *completed);
/* DIM2D_ERR_NOT_READY until the request is complete; then copies its final
 * nodes(nx,ny,4) and time, its latency (submit to completion, seconds),
 * and forgets the request.  DIM2D_ERR_WALL_ROOT (nodes and time still
 * copied) if a wall ghost-cell root failed during the solve, else
 * DIM2D_ERR_NONFINITE (likewise) if the state stopped being finite; the
 * time then says how far the solve got. */
DIM2D_API int dim2d_server_result(dim2d_server *s, long long id, double *nodes, double *t,
                                  double *latency_s);
/* out[8]: pending, active, copying, completed, cell-updates issued, bytes
 * in use, budget bytes, most requests active at once */
DIM2D_API int dim2d_server_stats(const dim2d_server *s, long long out[8]);
DIM2D_API int dim2d_server_destroy(dim2d_server *s);

/* field_abstract_class.f:286-315: dx = (x_max-x_min)/(nx-1-2*bc_size). */
DIM2D_API int dim2d_ini_coordinates(int nx, int ny, double x_min, double x_max, double y_min,
                          double y_max, double *x_map, double *y_map);

/* Message of the last error on the calling host thread. */
DIM2D_API const char *dim2d_last_error(void);
DIM2D_API const char *dim2d_version(void);

#ifdef __cplusplus
}
#endif
#endif
