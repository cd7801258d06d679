/*
 * mpsw.h — C ABI of the B200 MPAS shallow-water engine (RK4 forward, tangent linear, adjoint).
 *
 * The reference exposes its model as the f2py extension module `module_sw_mpas`, object
 * `mpas_sw_module`: argument-less subroutines acting on module variables that Python reads and
 * assigns as attributes (src/mpas_sw_module.f90:1-1218, called from src/mpas_sw_driver.py and
 * demo/run-*.py).  This header is that surface as plain C: one handle holds one module
 * instance; module variables are read and written by name in the reference's own layout
 * (Fortran column-major, index arrays 1-based, shapes as var_allocation* gives them); the
 * subroutines are entry points that run on the current CUDA device.  Handles are not
 * re-entrant: use one per thread.
 *
 * Every function returns 0 on success and a nonzero status otherwise; mpsw_last_error()
 * describes the failure.  No function aborts the process.
 */
#ifndef MPSW_H
#define MPSW_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mpsw_handle mpsw_handle;

enum {
  MPSW_OK = 0,
  MPSW_ERR_ARG = 1,      /* bad argument (unknown name, wrong count, null pointer) */
  MPSW_ERR_STATE = 2,    /* call out of order (not allocated, mesh not initialised) */
  MPSW_ERR_MESH = 3,     /* mesh failed validation */
  MPSW_ERR_CUDA = 4,     /* CUDA runtime error */
  MPSW_ERR_UNSUPPORTED = 5,
  MPSW_ERR_NONFINITE = 6 /* a routine formed a NaN or infinite tendency (or tendency adjoint): its
                            input state or members are corrupt, or the time step is unstable.
                            The reference has no such check; its Fortran carries the NaNs on. */
};

/* ---- lifecycle ------------------------------------------------------------------------ */
/* A new module instance with the reference's default scalars (src/mpas_sw_module.f90:23-55). */
int mpsw_create(mpsw_handle **out);
void mpsw_destroy(mpsw_handle *h);
/* Message of the last failure on this handle (or of mpsw_create when h is NULL). */
const char *mpsw_last_error(const mpsw_handle *h);
/* Library version string. */
const char *mpsw_version(void);

/* ---- module variables (f2py attribute access) ---------------------------------------- */
/* Scalars: dimensions (nCells, nEdges, ...), config_* switches, logicals as 0/1.  Names are
 * case-insensitive, as f2py attribute names are.  Constants (a, omega, gravity, pii, ...) are
 * readable only. */
int mpsw_set_scalar(mpsw_handle *h, const char *name, double value);
int mpsw_get_scalar(mpsw_handle *h, const char *name, double *value);

/* Allocatable arrays.  mpsw_var_info reports rank, Fortran dims, element type (0 = double,
 * 1 = int32) and whether the array is allocated.  mpsw_set_var/mpsw_get_var copy `count`
 * elements (must equal the allocated size) between a host buffer and the module variable. */
int mpsw_var_count(void);
const char *mpsw_var_name(int index);
int mpsw_var_info(mpsw_handle *h, const char *name, int *rank, long long dims[4], int *is_int,
                  int *allocated);
int mpsw_set_var(mpsw_handle *h, const char *name, const void *src, long long count);
int mpsw_get_var(mpsw_handle *h, const char *name, void *dst, long long count);

/* ---- module subroutines (src/mpas_sw_module.f90) -------------------------------------- */
int mpsw_var_allocation(mpsw_handle *h);      /* :211-367 */
int mpsw_var_allocation_tlm(mpsw_handle *h);  /* :369-429 */
int mpsw_var_allocation_adj(mpsw_handle *h);  /* :431-493 */
int mpsw_sw_mpas_init_block(mpsw_handle *h);  /* :495-526 */
/* :528-635, nsteps consecutive calls.  Tracers are carried unchanged, as in the reference,
 * unless the module scalar config_advect_tracers is nonzero (no counterpart in the reference):
 * then tracers(1) are transported with the flow (MPAS's order-2 scalar tendency, the call the
 * reference leaves out at :587, and its mass-weighted RK4), both levels of tracers receive the
 * result and tend_tracer the last stage's tendency.  mpsw_forward precision 1 refuses it. */
int mpsw_sw_rk4(mpsw_handle *h, int nsteps);
int mpsw_sw_rk4_tlm(mpsw_handle *h, int nsteps);  /* :637-781 */
int mpsw_sw_rk4_adj(mpsw_handle *h);              /* :783-1002 */
/* nsteps RK4 steps of the level-1 state, as nsteps calls of sw_rk4 (:528-635).  precision 0:
 * identical to mpsw_sw_rk4.  precision 1 (no counterpart in the reference): stencils in FP32
 * on h - h_ref (h_ref = the mean of h(1) at the call, rounded to a metre) and u, RK4 state and
 * accumulation in FP64; the module's diagnostics afterwards are the FP64 ones of the new state. */
int mpsw_forward(mpsw_handle *h, int precision, int nsteps);

/* ---- stencil routines on the level-1 state (module diagnostics in and out) ----------- */
int mpsw_solve_diagnostics(mpsw_handle *h);      /* sw_compute_solve_diagnostics, dyncore.f90:1-361 */
int mpsw_compute_tend(mpsw_handle *h);           /* sw_compute_tend, dyncore.f90:395-639 */
int mpsw_reconstruct_2d(mpsw_handle *h);         /* mpas_reconstruct_2d, operators.f90:283-370 */
int mpsw_solve_diagnostics_tlm(mpsw_handle *h);  /* dyncore_tlm.f90:1-447 */
int mpsw_compute_tend_tlm(mpsw_handle *h);       /* dyncore_tlm.f90:449-770 */
int mpsw_reconstruct_2d_tlm(mpsw_handle *h);     /* dyncore_tlm.f90:772-870 */
/* sw_compute_tend_adj (dyncore_adj.f90:455-738) + mpas_reconstruct_2d_adj (:740-831) +
 * sw_compute_solve_diagnostics_adj (:1-453) at the level-1 state, as the tail of
 * link_tlm_adj does them (module.f90:1163-1206): consumes tend_*_ad and the diagnostic /
 * reconstruction adjoints, accumulates into u_ad(1) and h_ad(1). */
int mpsw_adjoint_at_state(mpsw_handle *h);

/* ---- device-resident batched path ----------------------------------------------------- */
/* Member arrays are device buffers laid out [n][B] in the engine's internal (space-filling
 * curve) order; mpsw_to_internal / mpsw_to_reference convert from/to the reference order.
 * kind: 0 cells, 1 edges, 2 vertices.  stream: a cudaStream_t (NULL = legacy default). */
int mpsw_to_internal(mpsw_handle *h, int kind, int B, const double *src, double *dst, void *stream);
int mpsw_to_reference(mpsw_handle *h, int kind, int B, const double *src, double *dst, void *stream);

/* Level-1 prognostic state u(1), h(1) from / to device buffers in the reference order
 * (nEdges and nCells doubles); the time-2 level and the diagnostics follow as after a step. */
int mpsw_state_from_device(mpsw_handle *h, const double *u, const double *hh, void *stream);
int mpsw_state_to_device(mpsw_handle *h, double *u, double *hh, void *stream);

/* A window of `nsteps` RK4 steps starting from the current level-1 state u(1), h(1) (which is
 * left unchanged).  The nonlinear trajectory is kept as checkpoints every `ckpt_every` steps
 * and, as the storage mode selects, as the linearisation point of every RK stage of every
 * step; tangent-linear and adjoint sweeps read stored stages, or recompute states and stages
 * from the checkpoints where that precision is not stored (identical results either way).
 * The call copies the start state; the forward sweep itself runs in the first window call
 * that follows, alongside the members when that call is a tangent-linear sweep over a stored
 * precision, with the physics settings in force then.
 * precision: 0 = FP64 throughout, 1 = FP32 stencils with FP64 RK accumulation. */
int mpsw_window_init(mpsw_handle *h, int nsteps, int ckpt_every, void *stream);
/* Storage mode of the following mpsw_window_init calls.  No counterpart in the reference
 * (sw_rk4_adj recomputes a step's stages from its start state).  mode -1 (default): store the
 * FP64 and FP32 stage linearisation points when both fit in max_bytes (max_bytes 0: 40% of
 * the free device memory), else the FP32 ones alone if they fit, else none; mode 0: none
 * (checkpoints only); mode 1, 2, 3: FP64, FP32, both, regardless of size.  A stage slot holds
 * 6 nEdges + 2 nVertices + nCells values, nsteps * 4 slots per stored precision. */
int mpsw_window_storage(mpsw_handle *h, int mode, double max_bytes);
/* Launch choices of the eight member kernels (tl_vertex, tl_cell, tl_edge_diag, tl_edge_tend,
 * ad_edge, ad_cell, ad_vertex, ad_final) picked for (precision, B): v_block[2k] members per
 * thread, v_block[2k+1] threads per block; zeros when not tuned.  No counterpart in the
 * reference.  The first sweep of a window for a given (precision, B) times each kernel over the
 * pairs B allows on the window's own buffers and keeps the fastest (MPSW_TUNE=0 in the
 * environment keeps fixed defaults; MPSW_TUNE_CACHE=<file> keeps the choices in a text file
 * keyed by device, mesh size, precision and B, and reuses them). */
int mpsw_window_tuning(mpsw_handle *h, int precision, int B, int *v_block);
/* Checkpointing of the following mpsw_window_init calls, for windows whose stages are not
 * stored.  snapshots 0 (default): two-level checkpointing, a checkpoint every ckpt_every steps
 * and, in the adjoint sweep, one replay of each segment keeping its steps' states (one extra
 * forward over the window, ckpt_every states held).  snapshots s > 0: binomial reversal as in
 * Griewank's revolve: only the window's start state and s snapshot states are held, and the
 * adjoint sweep recomputes states by the schedule of fewest forward steps for s slots (the
 * sw_rk4_adj of each step then recomputes its four RK stages, as src/mpas_sw_module.f90:815-878
 * does).  Results are identical in every mode.  No counterpart in the reference, whose driver
 * keeps every step's state in a file (demo/run-adj.py:40-55). */
int mpsw_window_snapshots(mpsw_handle *h, int snapshots);
/* Nonlinear steps recomputed by the last adjoint sweep to re-form states (0 over stored stages). */
int mpsw_window_forward_steps(mpsw_handle *h, long long *steps);
/* Whether the window's sweeps of B members in `precision` run the fused member-stage kernels
 * (one kernel per tangent-linear or adjoint RK stage over halo tiles of the mesh) and with what
 * shape: *members_per_block 4 or 8 and *tile_cells the owned cells per tile, or both 0 when the
 * split member kernels run (FP64 members, del2 / del4 viscosity, bottom drag or wind stress,
 * meshes beyond 6 edges per cell or 10 edgesOnEdge, MPSW_FUSED=0 in the environment when the
 * mesh was built).  No counterpart in the reference. */
int mpsw_window_fused(mpsw_handle *h, int precision, int B, int *members_per_block, int *tile_cells);
/* Tangent linear over the window, B members in place: du [nEdges][B], dh [nCells][B]. */
int mpsw_window_tl(mpsw_handle *h, int precision, int B, double *du, double *dh, void *stream);
/* Adjoint over the window, B members in place: on entry the adjoint of the final state, on
 * exit the adjoint of the initial state. */
int mpsw_window_ad(mpsw_handle *h, int precision, int B, double *au, double *ah, void *stream);
/* Final nonlinear state of the window (device buffers, internal order). */
int mpsw_window_final_state(mpsw_handle *h, double *u, double *hh, void *stream);

/* ---- initial conditions ------------------------------------------------------------------
 * Williamson test case tc = 1, 2, 5 or 6 on the module's variables, as the reference's
 * sw_test_case_1/2/5/6 (src/mpas_sw_testcases.f90:1-398) set it up, with the per-entity
 * formulas evaluated by GPU kernels in FP64: the unit-sphere mesh is scaled by the Earth radius,
 * then u(1), h(1), and as the case has them fEdge, fVertex, h_s, tracers(1) and the shifted
 * lonCell are written.  Results agree with the host set-up to the last bits of sin / cos / pow. */
int mpsw_sw_test_case(mpsw_handle *h, int tc);
/*
 * Box average of a regular latitude-longitude field onto points, as the reference's grid2mpas
 * (src/grid2mpas.f90:21-70) does for its ERA5 initialisation: for each point (lat[k], lon[k], in
 * the units of the axes) the nearest axis entries (first minimum of the distance) and the mean
 * of the up to 3 x 3 grid values around them, clamped at the axis ends.  grid is [nlat][nlon]
 * (row-major, latitude rows), lat1d / lon1d the axes; all device buffers.  The reference shifts
 * negative longitudes of its arguments into latitudes by mistake (:46-47); callers here shift
 * longitudes into [0, 360) before the call (mpsw/ic.py: era_to_mpas). */
int mpsw_grid_to_points(mpsw_handle *h, int nlat, int nlon, const double *lat1d, const double *lon1d,
                        const double *grid, long long n, const double *lat, const double *lon, double *out,
                        void *stream);

/* ---- tendencies without device allocation ------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory when they
 * need the model (a host system that reserves all GPU memory for its own pool at start-up, or
 * code that must not synchronise the device the way cudaFree does): the tendencies tend_u,
 * tend_h of the state (u, hh), exactly as mpsw_compute_tend computes them, with the
 * intermediate diagnostics kept in a fixed 16 MiB array inside the library's device image
 * (held by every GPU that loads the library until the process exits).  All buffers are device
 * memory in the engine's internal order (see mpsw_to_internal): u and tend_u nEdges doubles,
 * hh and tend_h nCells doubles.  Needs sw_mpas_init_block to have put the mesh on the device;
 * the mesh must need at most 2,097,152 doubles of scratch, 3*nVertices + 3*nCells +
 * 2*nEdges (plus nEdges + nVertices + nCells with del4 viscosity), i.e. up to about 140,000
 * cells (100,000 with del4) on a quasi-uniform mesh; larger meshes are refused with
 * MPSW_ERR_UNSUPPORTED.  The call allocates nothing: sw_mpas_init_block, when it puts the
 * mesh on a device, also looks up the array's address there and loads the array and the
 * kernels this call launches (which lazy module loading, the CUDA default, would otherwise do
 * at the first call), so run that set-up before the device's memory is reserved.  The current
 * device must be the one the handle's mesh was built on (else MPSW_ERR_STATE).  Every call on a
 * device shares the array, so calls whose work overlaps on the GPU (other streams, other
 * threads, other handles) race; order them. */
int mpsw_compute_tend_noalloc(mpsw_handle *h, const double *u, const double *hh, double *tend_u,
                              double *tend_h, void *stream);

/* ---- measurement ----------------------------------------------------------------------- */
/* The stream the handle's module subroutines run on (a cudaStream_t), so a caller can time
 * them with events on it. */
int mpsw_get_stream(mpsw_handle *h, void **stream);
/* Number of kernels the library has launched in this process (all handles). */
long long mpsw_launch_count(void);
/* Average time of `iters` launches of one member stencil kernel on the buffers of the last
 * window sweep (same precision and B): which = 0 tl_vertex, 1 tl_cell, 2 tl_edge_diag,
 * 3 tl_edge_tend, 4 ad_edge, 5 ad_cell, 6 ad_vertex, 7 ad_final; or of a whole stage:
 * 8 tangent-linear stage, 9 adjoint stage.  Each launch is timed alone with CUDA events on the
 * engine's stream, after a 256 MiB write that evicts L2 (a cold start, as in a sweep). */
int mpsw_time_kernel(mpsw_handle *h, int which, int precision, int B, int iters, double *ms_per_launch);

#ifdef __cplusplus
}
#endif
#endif /* MPSW_H */
