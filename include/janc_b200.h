/*
 * janc_b200 C ABI: the per-step reacting-flow path of JANC (luofx23/JANC,
 * src/janc_v2) on NVIDIA B200 (sm_100a).
 *
 * All arrays are device pointers to C-contiguous float64 in the reference's
 * layout:
 *   U    [nv][nx][ny]  nv = 12 in 2D: rho, rho*u, rho*v, rho*E, rho*Y_1..8
 *                      nv = 11 in 1D (ny = 1): rho, rho*u, rho*E, rho*Y_1..8
 *   aux  [2][nx][ny]   gamma, T
 * Species order is the mechanism's; the last species (N2) is implicit,
 * Y_N2 = 1 - sum(Y).  Every call returns 0 or a jb_status bit set.
 *
 * Two kinds of call.  Configuration calls (jb_create, jb_destroy,
 * jb_set_transport, jb_adjoint_reserve and the jb_ens_* set-up calls) may
 * allocate or free device memory and may synchronise the device.  Every
 * other call (jb_flux_func, jb_update_aux, jb_reaction_source_terms,
 * jb_advance, jb_advance_ex, jb_rk3, jb_u_to_prim, jb_cfl_dt, jb_get_thermo,
 * jb_boundary_conditions, jb_adjoint_step, jb_state_from_PTY_vjp, ...)
 * allocates nothing, is asynchronous on the given CUDA stream (a
 * cudaStream_t passed as void*; NULL = legacy default stream) and does not
 * synchronise, except jb_status, which synchronises its stream by design.
 * The handle owns its tables and the workspaces its configuration calls
 * sized; it never frees caller memory.  Calls on one handle are
 * stream-ordered and not thread-safe.
 */
#ifndef JANC_B200_H
#define JANC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#include "../janc_b200/csrc/jb_types.h"

typedef struct jb_handle jb_handle;

/* Library version string. */
const char* jb_version(void);

/* Configure one solver: mechanism tables (preprocess/load.py:8-135 packing,
 * already non-dimensionalised), grid, the four side boundary kinds
 * (jb_bc_kind; 1D uses bc[0..1]) and the arithmetic variant (jb_precision).
 * Replaces the module-global set_thermo / set_reaction / set_flux_solver /
 * set_boundary calls made by Simulator.__init__
 * (src/janc_v2/simulation/set_simulator.py:384-390). */
int jb_create(const jb_mech_params* mech, int dim, int nx, int ny, double dx, double dy,
              const int bc[4], int precision, jb_handle** out);
int jb_destroy(jb_handle* h);

/* theta of the reference's boundary callables: pressure_outlet back pressure
 * 'Pb' (boundary_conditions_2D/pressure_outlet.py:25) and the injector's
 * 'Yinj' [8][nx] device array (examples/janc_basic_example2.ipynb) with the
 * blocked-injector pressure (1.0 in the notebook's nondimensional units). */
int jb_set_theta(jb_handle* h, double Pb, const double* Yinj, double inj_block_p);

/* flux_func(U, aux, dx, dy, dt, theta) -> dt * total_flux(BC(U, aux))
 * (src/janc_v2/simulation/set_simulator.py:26-29 1D, :44-47 2D). */
int jb_flux_func(jb_handle* h, const double* U, const double* aux, double dt, double* rhs,
                 void* stream);

/* update_aux(U, aux) -> aux (src/janc_v2/solver_2D/aux_func.py:21-29,
 * solver_1D/aux_func.py:21-28; Halley solve thermo_model.py:135-153 with the
 * reference's global stopping rule). */
int jb_update_aux(jb_handle* h, const double* U, const double* aux_in, double* aux_out,
                  void* stream);

/* reaction_source_terms(U, aux, dt) -> dU
 * (src/janc_v2/model/reaction_model.py:202-203 -> detailed_reaction :183-193). */
int jb_reaction_source_terms(jb_handle* h, const double* U, const double* aux, double dt,
                             double* S, void* stream);

/* nsteps of advance_one_step (set_simulator.py:117-122: SSP-RK3 flux stages
 * TVD_RK3.py:5-12, chemistry, temperature solve).  cfl > 0: each step's dt is
 * cfl * min(...) as Simulator.advance_func (set_simulator.py:420-447);
 * otherwise dt_fixed.  dt_hist (device, nsteps doubles, may be NULL) receives
 * each step's dt.  U/aux are not modified; U_out/aux_out receive the result. */
int jb_advance(jb_handle* h, const double* U, const double* aux, double* U_out, double* aux_out,
               double dt_fixed, double cfl, int nsteps, double* dt_hist, void* stream);

/* One SSP-RK3 step of the flux alone, followed by update_aux after each
 * stage: time_step_dict['TVD_RK3'](U, aux, dx, dy, dt, theta, flux_func,
 * update_aux) (src/janc_v2/simulation/time_step/TVD_RK3.py:5-12), i.e. the
 * advance_flux of set_simulator.py:83-84 without the chemistry split. */
int jb_rk3(jb_handle* h, const double* U, const double* aux, double* U_out, double* aux_out,
           double dt, void* stream);

/* U_to_prim(U, aux) -> rho, u, [v,] Y, p, a (src/janc_v2/solver_2D/aux_func.py:39-51,
 * solver_1D/aux_func.py:39-50); each output is [ncell] except Y [8][ncell];
 * v is ignored in 1D. */
int jb_u_to_prim(jb_handle* h, const double* U, const double* aux, double* rho, double* u, double* v,
                 double* Y, double* p, double* a, void* stream);

/* CFL_1D / CFL_2D (set_simulator.py:420-443): *dt_out (device) =
 * cfl * min(dx/(|u|+a)) resp. cfl * min(1/((|u|+a)/dx + (|v|+a)/dy)). */
int jb_cfl_dt(jb_handle* h, const double* U, const double* aux, double cfl, double* dt_out,
              void* stream);

/* get_thermo(T, Y) -> cp, gamma, h, R, dcp for n points
 * (src/janc_v2/model/thermo_model.py:115-126); Y is [8][n]. */
int jb_get_thermo(jb_handle* h, long long n, const double* T, const double* Y, double* cp,
                  double* gamma, double* hh, double* R, double* dcp, void* stream);

/* Synchronise `stream` and return the device status bits accumulated since
 * the last call (non-finite state, singular chemistry matrix), then clear. */
int jb_status(jb_handle* h, unsigned* status, void* stream);

/* Bytes of device workspace the handle holds. */
long long jb_workspace_bytes(const jb_handle* h);

/* Change the grid spacing of a configured handle (the reference passes dx, dy
 * on every call: set_simulator.py:26,44). */
int jb_set_spacing(jb_handle* h, double dx, double dy);

/* Select the advective flux (replaces set_flux_solver, solver_1D/flux.py:18-35,
 * solver_2D/flux.py:19-40): JB_FLUX_LF = flux splitting with LF and WENO5-JS
 * (the default), JB_FLUX_HLLC / JB_FLUX_AUSMPW = godunov_flux
 * (solver_2D/flux.py:43-54) with WENO5-JS on the primitives and the HLLC
 * (riemann_solver/HLLC.py) or AUSMPW+ (riemann_solver/AUSMPW_plus.py)
 * Riemann solver, JB_FLUX_SW = flux splitting with Steger-Warming
 * (flux_splitting/SW.py; the 1D form with the Jacobian and metric of 1, which
 * the reference's 1D flux_splitting cannot call: its split_flux takes a third
 * `metrics` argument it is not given).  The mixed variant reconstructs in
 * float32; the Riemann solver, RK and temperature solve are float64 in every
 * variant.  jb_adjoint_step supports JB_FLUX_LF only. */
int jb_set_flux_scheme(jb_handle* h, int scheme);

/* Select the face reconstruction of both flux paths (the
 * 'interface_reconstruction' entry of set_flux_solver,
 * solver_2D/reconstruction/__init__.py): JB_RECON_WENO5 (WENO5-JS, the
 * default) or JB_RECON_MUSCL (reconstruction/MUSCL.py: minmod limiter,
 * kappa = 1/3, beta = 1).  jb_adjoint_step supports WENO5-JS only. */
int jb_set_reconstruction(jb_handle* h, int recon);

/* Viscous fluxes (flux_solver_config 'viscosity': 'on'; replaces
 * transport_model.set_transport, model/transport_model.py:26-104, and
 * viscous_flux, solver_2D/flux.py:70-115 / solver_1D/flux.py:67-99): the
 * laminar transport model of *tr is used by every later flux evaluation of
 * the handle (added to the advective flux as NS_flux does, solver_2D/flux.py:117).
 * tr->turbulence_model = 1 adds the LES sub-grid viscosity of the 2D Vreman
 * model (model/LES/Verman.py; JB_ERR_UNSUPPORTED on a 1D handle, where the
 * reference has no model).  tr = NULL switches back to Euler fluxes (and frees
 * the scratch).  A configuration call: the first call with a model allocates
 * the viscous scratch.  jb_adjoint_step supports the inviscid path only. */
int jb_set_transport(jb_handle* h, const jb_transport* tr);

/* x-slab decomposition (replaces the reference's is_parallel mode:
 * parallel/boundary_padding.py exchange_halo, parallel/boundary.py
 * boundary_conditions_{1D,2D}, the jax.lax.pmin of CFL_1D / CFL_2D in
 * simulation/set_simulator.py:413-436).  A handle holds one slab of
 * nx columns; a left / right side created with JB_BC_HALO takes its 3 ghost
 * columns from the neighbouring slab, a physical side keeps its boundary
 * condition (the first and last slab of a non-periodic x axis).  Before each
 * flux evaluation the handle packs its 3 edge columns of (U, aux) into
 * send[2][nv+2][3][ny] (side 0: columns 0..2, side 1: columns nx-3..nx-1)
 * and calls fn(user, flags, stream) on the launch stream; with JB_XCH_HALO
 * the transport must deliver into halo[0] the left neighbour's send[1] and
 * into halo[1] the right neighbour's send[0] (the ring wraps for every x
 * side, as exchange_halo does; a physical side's halo supplies only its
 * padded corners), with JB_XCH_DT replace red[0..1] by their MIN over the
 * ranks (the CFL minimum).  Both stream-ordered on `stream`; fn returns 0 on
 * success.  LF alpha and the temperature solve's stop stay per slab, as in
 * the reference.  Buffers are caller-owned device memory and must outlive
 * the handle's calls; fn = NULL detaches.  The adjoint is single-domain. */
typedef int (*jb_exchange_fn)(void* user, int flags, void* stream);
int jb_set_exchange(jb_handle* h, double* send, double* halo, long long* red, jb_exchange_fn fn,
                    void* user);

/* The ghost-padded arrays (replaces boundary_conditions_1D / _2D,
 * boundary/boundary.py:120-132, and parallel/boundary.py:6-25 on a slab):
 * Up [nv][nx+6][ny+6] and auxp [2][nx+6][ny+6] (1D: [nv][nx+6], [2][nx+6]),
 * every entry as the flux kernels see it, padded corners included. */
int jb_boundary_conditions(jb_handle* h, const double* U, const double* aux, double* Up, double* auxp,
                           void* stream);

/* Caller-computed ghost layers on the sides created with JB_BC_HALO, for
 * boundary conditions given as functions (boundary/boundary.py:16-21,
 * 37-42, 58-63, 79-84: a callable receives the 3 boundary-adjacent layers of
 * U and aux and returns the 3 ghost layers).  Before each flux evaluation
 * the handle packs the x sides' edge columns into sendx[2][nv+2][3][ny] (as
 * jb_set_exchange does) and the y sides' edge rows into
 * sendy[2][nv+2][nx][3] (bottom: rows 0..2, top: rows ny-3..ny-1), then
 * calls fn(user, JB_XCH_HALO, stream); fn writes halox[side] / haloy[side]
 * with ghost layer l at padded position l (left, bottom) or n + l (right,
 * top), in the same layouts.  The padded corners keep the single-domain
 * periodic wrap; no reduction is asked for.  Buffers of a direction without
 * a JB_BC_HALO side may be NULL; fn = NULL detaches. */
int jb_set_ghost_cells(jb_handle* h, double* sendx, double* halox, double* sendy, double* haloy,
                       jb_exchange_fn fn, void* user);

/* Block-structured AMR (2D, flux splitting with LF; WENO5-JS or MUSCL from
 * the handle; no viscosity).  Blocks are [nb][nv+2][X][Y] float64: U fields,
 * then gamma, T (the reference's blk_data), each block's own layout.
 *
 * jb_amr_stage replaces one stage of advance_one_step_amr
 * (simulation/time_step/TVD_RK3.py:15-36) with the vmapped block flux and
 * update functions of set_rhs(is_amr=True) (simulation/set_simulator.py:
 * 37-42): G is the stage input with its 3-cell ghost layers filled by the
 * block layer (X = bx + 6, Y = by + 6), U0 the step's first stage input (the
 * same layout; read for stage 2 and 3, may be NULL for stage 1), out
 * (same layout, not overlapping G or U0) receives
 *   stage 1: G + pad(dt L(G)),  2: 3/4 U0 + 1/4 (G + pad(dt L(G))),
 *   3: 1/3 U0 + 2/3 (G + pad(dt L(G)))
 * over the whole padded block (the ghost entries with a zero rhs, as the
 * reference pads its rhs) and its update_aux started from G's temperature.
 * Every reduction is per block, as vmap makes it: the LF wave-speed maxima
 * over the block's padded array and the temperature solve's stop over the
 * block's padded cells.  dx, dy: the level's spacing.
 *
 * jb_amr_chem replaces the detailed-chemistry part of the AMR
 * advance_one_step (set_simulator.py:106-113): blk and out are unpadded
 * blocks (X = bx, Y = by; out may equal blk); out = U + S(U, T, dt) and its
 * update_aux with each block's own stop.
 *
 * jb_amr_flux is the block flux function alone (set_simulator.py:37-40, for
 * time schemes composed by the caller, e.g. RK2.advance_one_step_amr,
 * simulation/time_step/RK2.py:14-32): U [nb][nv][bx+6][by+6] and aux
 * [nb][2][bx+6][by+6] of padded blocks -> rhs [nb][nv][bx+6][by+6] =
 * pad(dt * total_flux(U, aux), 3) with zeros in the ghost entries.
 * jb_amr_update_aux is vmap(update_aux) (set_simulator.py:41): U [nb][nv][nx]
 * [ny], aux_in / aux_out [nb][2][nx][ny] (padded or not), each block's
 * temperature solve stopping on its own residuals.
 *
 * All need a 2D handle (its grid is not used; its mechanism, precision and
 * reconstruction are); the flux calls return JB_ERR_UNSUPPORTED for Godunov,
 * Steger-Warming or viscous configurations.  A mixed-precision handle
 * computes the blocks in float64. */
int jb_amr_stage(jb_handle* h, int nb, int bx, int by, double dx, double dy, int stage, const double* G,
                 const double* U0, double dt, double* out, void* stream);
int jb_amr_chem(jb_handle* h, int nb, int bx, int by, const double* blk, double dt, double* out, void* stream);
int jb_amr_flux(jb_handle* h, int nb, int bx, int by, double dx, double dy, const double* U, const double* aux,
                double dt, double* rhs, void* stream);
int jb_amr_update_aux(jb_handle* h, int nb, int nx, int ny, const double* U, const double* aux_in, double* aux_out,
                      void* stream);

/* sizeof(jb_mech_params) and sizeof(jb_grid) as compiled, for binding checks. */
int jb_sizeof_mech_params(void);
int jb_sizeof_grid(void);

/* update_aux without any device allocation (no counterpart in the reference,
 * whose JAX functions always allocate their results through XLA).  For
 * callers that cannot allocate device memory themselves - a plugin inside a
 * host code that reserves all device memory at start-up, or a call made from
 * within another runtime's operator whose memory that runtime owns - and so
 * cannot call jb_create().  Same result as jb_update_aux() on a solver of
 * that grid and precision, with U, aux_in and aux_out supplied by the
 * caller.  precision is JB_PREC_STRICT or JB_PREC_FP64; JB_PREC_MIXED returns
 * JB_ERR_UNSUPPORTED (the mixed variant's temperature solve is the fp64 one,
 * so pass JB_PREC_FP64 for it).  Its scratch lives in one static device array inside the
 * library, sized for at most JB_NOALLOC_MAX_CELLS cells (about 3.1 MB, held
 * on every GPU that loads the library until exit); larger grids return
 * JB_ERR_ARG.  Outside stream capture every call looks up the array's device
 * address (cudaGetSymbolAddress), so a device reset between calls is safe; a
 * captured call reuses the address of the device's last uncaptured call, so
 * make the first call on a device before any stream capture (a captured
 * first call returns JB_ERR_ARG).  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
#define JB_NOALLOC_MAX_CELLS 65536
int jb_update_aux_noalloc(const jb_mech_params* mech, int dim, int nx, int ny, int precision,
                          const double* U, const double* aux_in, double* aux_out, void* stream);

/* Measurement helpers (no reference counterpart).  jb_set_kernel_timing
 * enables CUDA events around each launch of jb_advance (at most JB_TIMED_MAX
 * launches between reads) and clears the totals; jb_kernel_times waits for
 * the recorded events and returns accumulated milliseconds and launch counts
 * per jb_kernel_cat (arrays of JB_KCAT_COUNT). */
int jb_set_kernel_timing(jb_handle* h, int enable);
int jb_kernel_times(jb_handle* h, double* ms, long long* launches);

/* Measurement helper (no reference counterpart): launches `blocks` x 256
 * threads, each doing iters*128 float64 FMAs (2 FLOP each), for measuring
 * the device's FP64 peak.  `scratch` is a device buffer of `blocks` doubles. */
int jb_probe_fp64_fma(int blocks, int iters, double* scratch, void* stream);

/* Human-readable description of the last error on this handle. */
const char* jb_last_error(const jb_handle* h);

/* ------------------------------------------------------------------------
 * Reverse mode (the adjoint), 2D and 1D grids with periodic, slip, no-slip,
 * zero-gradient or pressure-outlet sides (back pressure Pb held fixed) and
 * the rotating-detonation injector on the bottom side (2D; Yinj held fixed).
 * The reference gets these derivatives from jax.grad
 * through advance_one_step and the CFL time step (set_simulator.py:117-122,
 * 420-447; 1D: CFL min dx / (|u| + a)) with get_T's custom VJP
 * (src/janc_v2/model/thermo_model.py:155-190); these calls compute the same
 * vector-Jacobian products with hand-written kernels.
 * ------------------------------------------------------------------------ */
/* Pressure probe: mean p over the wx x wy cells from (x0, y0) (1D: y0 = 0,
 * wy = 1). */
int jb_set_probe(jb_handle* h, int x0, int y0, int wx, int wy);
/* Scale every pre-exponential factor A_i of the handle's mechanism by
 * exp(offset[i]) relative to the tables given to jb_create (NULL restores
 * them); offset is a host array of nreac doubles. */
int jb_set_log_A_offset(jb_handle* h, const double* offset);
/* Doubles of one step's record (U, aux and the three RK stages' states). */
long long jb_record_doubles(const jb_handle* h);
/* jb_advance (chemistry on) plus: probe_p (device, nsteps doubles, may be
 * NULL) receives the probe pressure after each step; rec (device,
 * (nsteps + 1) * jb_record_doubles doubles, may be NULL) receives every
 * step's record and the final state, and rec_slots (device, nsteps *
 * sizeof(jb_slots) bytes) each step's time step and LF alphas. */
int jb_advance_ex(jb_handle* h, const double* U, const double* aux, double* U_out, double* aux_out,
                  double dt_fixed, double cfl, int nsteps, double* dt_hist, double* probe_p, double* rec,
                  double* rec_slots, void* stream);
/* Configuration call: allocate the adjoint's workspace (stage adjoints,
 * primitives, face scratch, reductions) and upload the padded-grid
 * multiplicity of the handle's sides; synchronous.  Returns
 * JB_ERR_UNSUPPORTED for what jb_adjoint_step cannot differentiate.  Call it
 * once before the first jb_adjoint_step, outside any stream capture. */
int jb_adjoint_reserve(jb_handle* h);
/* One step of the adjoint (needs jb_adjoint_reserve; allocates nothing).
 * rec points at step n's record (step n+1's
 * record follows it), rec_slots at step n's slots; cfl as given to the
 * forward (<= 0: fixed time step).  On entry Ubar / Abar hold the adjoint
 * of the state after the step (U_{n+1}: nv x ncell, aux_{n+1}: 2 x ncell);
 * on return that of the state before it.  dt_bar, pp_bar (device scalars,
 * may be NULL) are the adjoints of the step's time step and probe
 * pressure; lnA_bar (device, nreac doubles) accumulates the adjoint of
 * ln A. */
int jb_adjoint_step(jb_handle* h, const double* rec, const double* rec_slots, double cfl, double* Ubar,
                    double* Abar, const double* dt_bar, const double* pp_bar, double* lnA_bar, void* stream);
/* Adjoint of the initial-state builder (rho = P/(R T), rho E = rho h - P,
 * aux = [gamma, T]; examples/janc_basic_example1.ipynb) with respect to T:
 * Tbar (ncell) from Ubar, Abar of the built state. */
int jb_state_from_PTY_vjp(jb_handle* h, const double* P, const double* T, const double* Y, const double* Ubar,
                          const double* Abar, double* Tbar, void* stream);

/* ------------------------------------------------------------------------
 * Batched ensemble of 1D instances (no single reference counterpart: the
 * reference advances one case per Simulator; each instance here follows
 * Simulator.advance_func, src/janc_v2/simulation/set_simulator.py:412-447,
 * with its own CFL time step and LF alpha).  All instances use the same
 * mechanism; they differ in length, spacing, side boundaries (bc[2i],
 * bc[2i+1]: left, right; not the injector) and initial state.  The ensemble
 * owns the state: U [11][nx_i] and aux [2][nx_i] of instance i live at the
 * device pointers jb_ens_instance returns and are advanced in place.
 * Precision: JB_PREC_FP64 or JB_PREC_MIXED.  cfl[i] > 0 selects the CFL time
 * step, else dt[i] (dt may be NULL when every cfl[i] > 0).  Unlike the calls
 * above, jb_ens_create, jb_ens_configure and jb_ens_autotune allocate device
 * memory, and the first jb_ens_advance of a launch shape builds its graph.
 * ------------------------------------------------------------------------ */
typedef struct jb_ensemble jb_ensemble;

int jb_ens_create(const jb_mech_params* mech, int n, const int* nx, const double* dx, const int* bc,
                  const double* cfl, const double* dt, int precision, jb_ensemble** out);
int jb_ens_destroy(jb_ensemble* e);
/* Device pointers to instance i's state and its cell count. */
int jb_ens_instance(jb_ensemble* e, int i, double** U, double** aux, int* nx);
long long jb_ens_total_cells(const jb_ensemble* e);
/* Launch shape: block = 64, 128 or 256 threads, blocks_per_sm resident CTAs
 * per SM; CTAs are assigned to instances in proportion to their flux tiles. */
int jb_ens_configure(jb_ensemble* e, int block, int blocks_per_sm);
/* Back pressure of each instance's pressure-outlet sides, pb[n] (theta['Pb']
 * of boundary_conditions_1D/pressure_outlet.py:5-22, in the ensemble's
 * units); 0 until set.  A set-up call: it uploads the instance table. */
int jb_ens_set_back_pressure(jb_ensemble* e, const double* pb);
/* Times every launch shape the device fits on `trial_steps` steps (the
 * state is restored afterwards) and keeps the fastest. */
int jb_ens_autotune(jb_ensemble* e, int trial_steps, void* stream, int* best_block, int* best_bpsm,
                    double* best_ms);
int jb_ens_launch_shape(const jb_ensemble* e, int* block, int* blocks_per_sm, int* nblocks, int* max_tiles,
                        int* graph_mode);
/* Advance every instance nsteps steps with one persistent cooperative
 * launch, replayed from a CUDA graph (rebuilt when nsteps, dt_hist or the
 * launch shape change).  dt_hist: NULL or device [n][nsteps] time steps. */
int jb_ens_advance(jb_ensemble* e, int nsteps, double* dt_hist, void* stream);
/* The same launch without the graph. */
int jb_ens_advance_direct(jb_ensemble* e, int nsteps, double* dt_hist, void* stream);
/* Synchronises `stream`, returns the status bits seen per instance (array of
 * n, or NULL) and combined (JB_ERR_TIMEOUT when a barrier wait gave up; the
 * kernel then stopped early and later launches return at once until this
 * call has reported it), and clears them. */
int jb_ens_status(jb_ensemble* e, unsigned* per_instance, unsigned* combined, void* stream);
const char* jb_ens_last_error(const jb_ensemble* e);
/* Test hook for the timeout path: one launch in which instance 0's CTA
 * group waits for a CTA that is never launched, so its first barrier gives
 * up after wait_limit_ms (at most 1000) and every CTA returns; *combined
 * then holds JB_ERR_TIMEOUT.  Leaves the ensemble's state undefined. */
int jb_ens_selftest_timeout(jb_ensemble* e, double wait_limit_ms, unsigned* combined, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* JANC_B200_H */
