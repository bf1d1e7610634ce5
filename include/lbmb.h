/*
 * lbmb.h — C ABI of the B200 (sm_100a) LBMFlow single-GPU time step.
 *
 * One opaque handle = one solver = one CUDA device + one stream. Every entry
 * point returns an int status: 0 (LBMB_OK) or a negative lbmb_status; the
 * text of the last failure on the calling thread is lbmb_last_error().
 * Nothing throws across the ABI. Host buffers are caller-owned; device
 * buffers are owned by the handle. A handle is not thread-safe; distinct
 * handles may be driven from distinct threads.
 *
 * Arrays use the reference's compact global cell order
 *   cell = (z * ny + y) * nx + x
 * and populations are in the reference's deviation form (f_q - w_q),
 * q-major: f[q * ncells + cell] (crates/lbm-core/src/fields.rs:3-15).
 * Populations read or written through this ABI are always the reference's
 * logical post-stream state, whatever in-place layout the device uses.
 *
 * Each entry point names the reference interface it replaces
 * (path:line inside the reference project).
 */
#ifndef LBMB_H
#define LBMB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbmb_solver lbmb_solver;

enum lbmb_status {
  LBMB_OK = 0,
  LBMB_ERR_INVALID = -1,     /* invalid argument / spec (SpecError) */
  LBMB_ERR_CUDA = -2,        /* CUDA runtime failure */
  LBMB_ERR_UNSUPPORTED = -3, /* UnsupportedReason::NotImplemented */
  LBMB_ERR_DIVERGED = -4,    /* non-finite mass detected (Diverged) */
  LBMB_ERR_STATE = -5,       /* call out of order (e.g. scalar not enabled) */
  LBMB_ERR_NOMEM = -6,       /* device allocation failed */
  LBMB_ERR_CHECKPOINT = -7   /* CheckpointError: lbmb_last_error() reads
                              * "<code>: <message>" with the reference's
                              * stable code (CKPT_IO, CKPT_BAD_MAGIC,
                              * CKPT_VERSION_MISMATCH, ...) */
};

enum lbmb_collision { LBMB_BGK = 0, LBMB_TRT = 1, LBMB_CENTRAL_MOMENT = 2 };

/* Population storage precision. Arithmetic is fp32 for F32/F16/BF16 and
 * fp64 for F64. F16/BF16 store the deviation (f_q - w_q). */
enum lbmb_storage { LBMB_STORE_F32 = 0, LBMB_STORE_F16 = 1, LBMB_STORE_BF16 = 2, LBMB_STORE_F64 = 3 };

/* Backend reduction kinds (crates/lbm-core/src/params.rs:411-419). */
enum lbmb_reduction { LBMB_RED_FLUID_CELLS = 0, LBMB_RED_MASS_DEV = 1, LBMB_RED_MOMENTUM = 2 };

/* GlobalSpec subset on the hot path (crates/lbm-core/src/solver.rs:131-148). */
typedef struct lbmb_config {
  int32_t lattice;     /* 19 (D3Q19) or 27 (D3Q27) */
  int32_t collision;   /* lbmb_collision */
  int32_t storage;     /* lbmb_storage */
  int32_t dims[3];     /* nx, ny, nz */
  int32_t periodic[3]; /* per axis; non-periodic faces must be full solid rims */
  int32_t device;      /* CUDA ordinal */
  double nu;           /* lattice viscosity */
  double magic;        /* TRT magic parameter (3/16 standard) */
  double omega_shear;  /* central-moment shear rate in (0, 2] */
  double force[3];     /* uniform Guo body force */
  double smagorinsky_cs; /* 0: off (the reference's operators). > 0: Smagorinsky
                          * LES, tau_eff = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2
                          * |Pi_neq| / rho)) / 2 applied to the shear rate (no
                          * reference counterpart; stabilises under-resolved
                          * high-Re tanks) */
  int32_t free_slip_top;  /* nonzero: the solid layer z = nz - 1 is a free-slip
                           * (specular) wall: a population leaving a cell of
                           * layer nz - 2 upwards with velocity (cx, cy, 1)
                           * arrives at cell x + (cx, cy, 0) with (cx, cy, -1)
                           * when that cell is fluid (half-way bounce-back
                           * otherwise); no reference counterpart (the
                           * reference tank has a no-slip lid) */
} lbmb_config;

/* DirectForcingConfig (crates/lbm-core/src/rotating_ibm.rs:106-130). */
typedef struct lbmb_ibm_config {
  int32_t max_iterations; /* default 3 */
  double slip_tolerance;  /* default 1e-2 */
  int32_t kernel_radius;  /* 1 (2-point linear) or 2 (3-point quadratic) */
  double relaxation;      /* (0, 1], default 1 */
} lbmb_ibm_config;

/* IbmDiagnostics (crates/lbm-core/src/rotating_ibm.rs:134-153). */
typedef struct lbmb_ibm_diag {
  int32_t iterations;
  double slip_max, slip_rms, slip_max_rel, slip_rms_rel;
  double torque[3];
  double fluid_force[3];
  double marker_force[3];
  double momentum_error_rel;
} lbmb_ibm_diag;

/* Impeller marker generators for lbmb_build_stirred_tank. */
enum lbmb_impeller_kind {
  LBMB_IMPELLER_RUSHTON = 0,    /* reference generator, geometry.rs:815-906 */
  LBMB_IMPELLER_PITCHED = 1,    /* reference generator, 45-degree blades */
  LBMB_IMPELLER_FLAT_BLADE = 2  /* disc + flat blades sampled at a uniform spacing */
};

/* Stirred-tank set-up (crates/lbm-core/src/geometry.rs:84-132), SI units. */
typedef struct lbmb_tank_spec {
  int32_t dims[3];
  double dx_m;
  double vessel_diameter_m;
  double liquid_height_m;
  int32_t baffle_count; /* 0 or 4 (wall attached) */
  double baffle_width_m;
  double baffle_thickness_m;
  int32_t impeller_kind; /* lbmb_impeller_kind */
  double impeller_diameter_m;
  double clearance_m;
  int32_t blade_count;
  double omega_rad_s;          /* rotational speed (rad/s, SI) */
  double marker_spacing_cells; /* LBMB_IMPELLER_FLAT_BLADE only */
  double min_cells;            /* resolution floor; <= 0 -> 32 (STIRRED_TANK_MIN_CELLS) */
} lbmb_tank_spec;

/* Text of the last failure on this thread ("" if none). */
const char* lbmb_last_error(void);

/* Library version string. */
const char* lbmb_version(void);

/* Solver::try_new + Backend::alloc (solver.rs:1754-1900, backend.rs:138).
 * solid: ncells bytes (nonzero = solid), may be NULL (all fluid).
 * wall_u: ncells x 3 wall velocities (meaningful on solids), may be NULL.
 * State after creation: quiescent f = 0 (rho = 1, u = 0). */
int lbmb_create(const lbmb_config* cfg, const uint8_t* solid, const double* wall_u,
                lbmb_solver** out);
int lbmb_destroy(lbmb_solver* h);

/* Cell count and lattice size of a handle. */
int lbmb_shape(const lbmb_solver* h, int64_t* ncells, int32_t* q);

/* Solver::init_with (solver.rs:2474-2605): f = feq(rho, u) + f_neq(grad u)
 * from sampled fields (rho: ncells, u: ncells x 3), then moments refresh. */
int lbmb_init_fields(lbmb_solver* h, const double* rho, const double* u);

/* Backend::stage_in / stage_out (backend.rs:146-155): q-major deviation
 * populations (Q x ncells, f64 view of the storage precision). stage_in
 * also refreshes the cached moments, like the reference's init path. */
int lbmb_stage_in(lbmb_solver* h, const double* f);
int lbmb_stage_out(lbmb_solver* h, double* f);

/* Solver::run (solver.rs:2283-2343): `steps` x {collide, stream, moments}
 * (+ every enabled passive scalar, solver.rs:2113-2205). */
int lbmb_step(lbmb_solver* h, int64_t steps);

/* Solver::run_guarded (solver.rs:2346-2356): runs in chunks of check_every
 * and checks the f64 mass after each; returns LBMB_ERR_DIVERGED with
 * *completed = steps done at the failing check. */
int lbmb_run_guarded(lbmb_solver* h, int64_t steps, int64_t check_every, int64_t* completed);

/* Backend::read_moments (backend.rs:355-362): rho and the physical velocity
 * (with the Guo half-force) of the current state; any pointer may be NULL.
 * Solid cells report the values they were initialised with. */
int lbmb_read_moments(lbmb_solver* h, double* rho, double* ux, double* uy, double* uz);

/* Backend::reduce (backend.rs:347-353, 920-970): f64 accumulation over
 * fluid cells. axis is used by LBMB_RED_MOMENTUM only. */
int lbmb_reduce(lbmb_solver* h, int32_t kind, int32_t axis, double* out);

/* Solver::total_mass_f64 (solver.rs:5114-5117). */
int lbmb_total_mass(lbmb_solver* h, double* out);

/* Solver::clear_body_force_field (solver.rs:2805-2822). */
int lbmb_clear_body_force_field(lbmb_solver* h);

/* Current per-cell force field (ncells x 3, zeros where absent). */
int lbmb_get_force_field(lbmb_solver* h, double* out);

/* ---- Per-cell relaxation field and WALE LES ------------------------------ */

/* Solver::set_omega_field (solver.rs:4443-4473): a per-cell relaxation
 * rate (n values; NULL removes it) for the following collisions: TRT/BGK
 * take omega+ = field and c+ = 1 - omega+/2 with omega- unchanged
 * (kernels.rs:151-156), the central moment takes it as its shear rate
 * (kernels.rs:481). Not combined with smagorinsky_cs > 0. While a field
 * is set the sweep runs on the direct, bulk or window kernel (a solver on
 * another kind moves to window, or direct where window cannot run);
 * batches and the adjoint do not take it. */
int lbmb_set_omega_field(lbmb_solver* h, const double* omega);

/* Solver::gather_velocity_gradient (solver.rs:5482-5582): n x 9 row-major,
 * g[i][j] = du_i/dx_j (lattice units); symmetric off-diagonal part from the
 * native strain rate, diagonal and rotation from velocity differences with
 * the half-way wall stencil; solid cells zero. */
int lbmb_gather_velocity_gradient(lbmb_solver* h, double* g9);

/* WaleLesDiagnostics (les.rs:19-31). tau_eff_max and nu_t_max are NaN
 * without a bound. */
typedef struct {
  int64_t clipped_cells;
  double clipped_fraction;
  double max_nu_t_before_clipping;
  double tau_eff_max;
  double nu_t_max;
} lbmb_wale_diag;

/* WaleLes::update (les.rs:120-211; Cw = 0.325, Delta = 1): WALE eddy
 * viscosity nu_t from the velocity gradient, clipped at
 * (tau_eff_max - tau0) / 3 when tau_eff_max is not NaN, and the field
 * omega+ = 1 / (3 (nu + nu_t) + 1/2) installed for the next collision on
 * the device (one-step lag). nu_t (n values) may be NULL. */
int lbmb_wale_update(lbmb_solver* h, double tau_eff_max, double* nu_t, lbmb_wale_diag* diag);

/* ---- Shear-rate and stress QOIs ----------------------------------------- */

/* Solver::gather_strain_rate / gather_shear_rate (solver.rs:5464-5480,
 * 5588-5599; per cell solver.rs:5393-5447): the native strain rate from the
 * non-equilibrium second moment of the current post-stream populations and
 * the cached moments, Pi_neq + 0.5 (uF + Fu), scaled by
 * -1 / (2 cs^2 rho tau_eff) with tau_eff = 1 / omega+ (lattice units).
 * s6 = n x 6 [S_xx, S_yy, S_zz, S_xy, S_xz, S_yz], gamma = n values of
 * sqrt(2 S:S); either may be NULL. Solid cells report zeros. */
int lbmb_gather_strain_rate(lbmb_solver* h, double* s6, double* gamma);

/* stress.rs compute_stress_field (stress.rs:32-82) on the cached velocity in
 * SI units (lattice velocity x dx_m / dt_s), as the bioprocess runner calls
 * it (runner.rs:1648-1676) with a uniform viscosity mu_pa_s: central
 * differences, one-sided next to a solid or the domain edge (not periodic),
 * s6 = n x 6 strain-rate tensor, gamma = gamma_dot [1/s], viscous =
 * mu gamma_dot [Pa]; any output may be NULL; solid cells report zeros. */
int lbmb_stress_field(lbmb_solver* h, double dx_m, double dt_s, double mu_pa_s, double* s6, double* gamma,
                      double* viscous);

/* stress.rs PercentileSummary (stress.rs:12-20) with the number of finite
 * values it is taken over; valid = 0 when there is none (the reference's
 * None). fraction_above_threshold is NaN without a threshold. */
typedef struct {
  double p50, p90, p95, p99, max;
  double fraction_above_threshold;
  int64_t count;
  int32_t valid;
} lbmb_percentiles;

/* The stress QOI of write_stress_and_wall_outputs (runner.rs:1648-1690):
 * percentile_summary (stress.rs:84-100) of gamma_dot and of the viscous
 * stress over the fluid cells, sorted on the device. Thresholds: NaN for
 * none (the runner passes 0). device_ms (may be NULL): device time of the
 * moments, stress field, sort and counts. */
int lbmb_stress_summary(lbmb_solver* h, double dx_m, double dt_s, double mu_pa_s, double gamma_threshold,
                        double tau_threshold, lbmb_percentiles* gamma, lbmb_percentiles* viscous,
                        double* device_ms);

/* stress.rs WallShearProxy (stress.rs:22-30). */
typedef struct {
  int64_t cell_index;
  double tau_w_pa, y_plus, u_parallel_m_s, y_m;
  double normal[3];
} lbmb_wall_shear;

/* stress.rs wall_shear_proxy (stress.rs:102-165, 228-294): every fluid cell
 * with a solid among its 26 in-domain neighbours, in cell order; the wall
 * velocity is the solver's wall velocity x dx_m / dt_s. Writes up to
 * capacity entries to out (may be NULL) and the total to *count. */
int lbmb_wall_shear_proxy(lbmb_solver* h, double dx_m, double dt_s, double rho_kg_m3, double mu_pa_s,
                          lbmb_wall_shear* out, int64_t capacity, int64_t* count);

/* RotatingBody::from_markers (rotating_ibm.rs:32-58): upload body `body`
 * (0-based slot): n markers at lattice coordinates (n x 3), quadrature
 * weights, rotation centre and angular velocity (rad/step). */
int lbmb_ibm_set_body(lbmb_solver* h, int32_t body, const double* pos, const double* weight,
                      int64_t n, const double center[3], const double omega[3]);

/* Solver::apply_rotating_ibm (solver.rs:3016-3282): direct-forcing sweeps
 * on the device; the spread is added to the force field and the
 * diagnostics are returned. diag may be NULL. */
int lbmb_apply_rotating_ibm(lbmb_solver* h, int32_t body, const lbmb_ibm_config* cfg,
                            lbmb_ibm_diag* diag);

/* One iteration of the runner loop with the caller's marker set
 * (crates/lbm-cli/src/runner.rs:1080-1085: clear_body_force_field, apply the
 * impeller marker set, step): the same device work and results as
 * lbmb_clear_body_force_field + lbmb_ibm_set_body + lbmb_apply_rotating_ibm
 * + lbmb_step(h, 1), with the direct forcing and the IBM-forced cells on a
 * side stream beside the full-grid sweep. The call returns once the
 * diagnostics are on the host (through a pinned staging copy); the step's
 * sweep may still be running, as after lbmb_step, and later calls queue
 * behind it (entry points that return data synchronise). The marker arrays
 * are copied every call and may be changed once it returns (pinned host
 * memory makes the copy asynchronous). diag may be NULL. Not with a uniform
 * body force. */
int lbmb_runner_step(lbmb_solver* h, int32_t body, const double* pos, const double* weight, int64_t n,
                     const double center[3], const double omega[3], const lbmb_ibm_config* cfg,
                     lbmb_ibm_diag* diag);

/* Solver::enable_scalar_distribution (solver.rs:2856-2890): q = 7 (D3Q7,
 * cs^2 = 1/4) or the hydro lattice size (the reference's choice). */
int lbmb_enable_scalar(lbmb_solver* h, int32_t q, double diffusivity, int32_t* index);

/* Solver::set_scalar_concentration (solver.rs:2910-2966). */
int lbmb_set_scalar_concentration(lbmb_solver* h, int32_t k, const double* c);

/* Solver::gather_scalar_concentration (solver.rs:2892-2908). */
int lbmb_gather_scalar_concentration(lbmb_solver* h, int32_t k, double* c);

/* ---- Oxygen transfer and uptake sources on a scalar --------------------- */

/* OxygenDiagnostics (oxygen.rs:18-23) of the negative clip. */
typedef struct {
  int64_t clipped_cells;
  double clipped_fraction;
  double min_before_clip;
} lbmb_oxygen_diag;

/* OxygenFluxLedger (oxygen.rs:25-31); cumulative_mol is read and updated. */
typedef struct {
  double cumulative_mol, last_step_mol, source_integral_mol_s;
  int64_t active_interface_cells;
} lbmb_oxygen_ledger;

/* OurLedger (reaction.rs:23-27); cumulative_kmol_consumed is read and updated. */
typedef struct {
  double cumulative_kmol_consumed, last_step_kmol_consumed;
} lbmb_our_ledger;

/* OurModel (reaction.rs:7-21). */
typedef enum { LBMB_OUR_CONSTANT = 0, LBMB_OUR_MONOD = 1, LBMB_OUR_CELL_DENSITY = 2 } lbmb_our_kind;
typedef struct {
  int32_t kind;
  double our_kmol_m3_s;                 /* constant */
  double our_max, ks, c_ref;            /* Monod: our_max (C/c_ref) / (ks + C/c_ref) */
  double specific_our;                  /* cell-density scaled: specific_our x density */
} lbmb_our_model;

/* The reference's composition gather_scalar_concentration ->
 * apply_interfacial_flux_sources (oxygen.rs:124-191, kL of a constant or
 * calibrated model) -> set_scalar_concentration, on the device for scalar
 * k: C += kL a (C* - C) dt over every cell, negative values clipped to 0,
 * the scalar reset to the equilibrium of the new C with the current
 * velocity. c_star / cell_volume: n values or NULL for the uniform value;
 * area_density: n values (1/m). Invalid inputs return LBMB_ERR_INVALID and
 * leave the scalar unchanged. Solid cells hold concentration 0 here (the
 * reference keeps the value last set there). */
int lbmb_scalar_interfacial_flux(lbmb_solver* h, int32_t k, const double* c_star, double c_star_uniform,
                                 const double* area_density, const double* cell_volume, double cell_volume_uniform,
                                 double dt_s, double kl_m_s, lbmb_oxygen_ledger* ledger, lbmb_oxygen_diag* diag);

/* Same composition with apply_oxygen_reaction_source (reaction.rs:95-137):
 * C -= OUR(C) dt, clip, ledger of kmol consumed. cell_density: n values,
 * required by LBMB_OUR_CELL_DENSITY, else ignored (may be NULL). */
int lbmb_scalar_oxygen_uptake(lbmb_solver* h, int32_t k, const lbmb_our_model* model, const double* cell_density,
                              const double* cell_volume, double cell_volume_uniform, double dt_s,
                              lbmb_our_ledger* ledger, lbmb_oxygen_diag* diag);

/* qoi::scalar_cv over fluid cells (crates/lbm-core/src/qoi.rs:507-532);
 * *cv = NaN where the reference returns None. */
int lbmb_scalar_cv(lbmb_solver* h, int32_t k, double* cv);

/* Runner hot loop (crates/lbm-cli/src/runner.rs:1079-1129) on the device:
 * `steps` x {clear force field, IBM of `body`, step}, recording per step
 * torque_lu = -diag.torque[2] (runner.rs:1396-1425), the fluid force
 * (steps x 3) and the IBM iteration count; and, if scalar >= 0, the scalar
 * CV every probe_every steps (NaN elsewhere). Any output may be NULL.
 * As the reference runner (runner.rs:1125-1128), the f64 total mass is
 * checked after every 1000th step of the call; a non-finite value stops the
 * run there (status "diverged"): the call returns LBMB_ERR_DIVERGED, the
 * outputs hold the executed steps (NaN, iterations 0, after them) and
 * lbmb_run_impeller_status reports the executed step count. Between checks
 * the loop replays a CUDA graph of 16 steps, captured on the first call and
 * kept by the handle (with its series buffers) while the body, the IBM
 * configuration, the sweep kernel and the scalar set are unchanged; the
 * device time of lbmb_last_timing covers the steps only. */
int lbmb_run_impeller(lbmb_solver* h, int32_t body, const lbmb_ibm_config* cfg, int64_t steps,
                      int32_t scalar, int64_t probe_every, double* torque_lu, double* fluid_force,
                      double* cv, int32_t* ibm_iterations);

/* Outcome of the last lbmb_run_impeller call on this handle (the runner's
 * `executed` and `status`, runner.rs:1077-1129): *executed = steps taken,
 * *diverged = 1 when the run stopped on a non-finite total mass. Either
 * pointer may be NULL. */
int lbmb_run_impeller_status(lbmb_solver* h, int64_t* executed, int32_t* diverged);

/* No counterpart in the reference (failure detection of the device path).
 * Bound on every mbarrier wait of the bulk-copy sweep kernel
 * (LBMB_SWEEP_BULK), in SM clock cycles; 0 restores the
 * default (2^31, about a second). A wait that runs out sets a device error
 * flag, waits (bounded) for the kernel's own copies and returns; the call
 * that launched the step then fails with LBMB_ERR_CUDA ("device wait timed
 * out") and the context stays usable. A negative value is a self-test: the
 * next such sweep waits -cycles on a barrier nothing arrives at, reports the
 * timeout and leaves the populations untouched. */
int lbmb_set_wait_limit(lbmb_solver* h, int64_t cycles);

/* Device time of the last lbmb_step / lbmb_run_impeller call in ms (CUDA
 * events on the solver stream), and the hydro kernel's share of it. */
int lbmb_last_timing(lbmb_solver* h, double* total_ms, double* hydro_ms, int64_t* hydro_launches);

/* build_wall_rims (crates/lbm-core/src/solver.rs:1357-1404): one-cell solid
 * rims on the faces with is_wall set (face order XNeg, XPos, YNeg, YPos,
 * ZNeg, ZPos; u = 6 x 3 wall velocities); corner cells keep the fastest
 * wall. Outputs solid (ncells) and wall_u (ncells x 3). */
int lbmb_build_wall_rims(const int32_t dims[3], const int32_t is_wall[6], const double u[18], uint8_t* solid,
                         double* wall_u);

/* build_stirred_tank_geometry + generate_impeller_marker_set
 * (crates/lbm-core/src/geometry.rs:207-345, 657-916): voxel flags,
 * baffle mask, stamped wall velocity (SI) and impeller markers (lattice
 * coordinates). Call once with marker_pos = marker_weight = NULL to read
 * *n_markers, then again with capacity >= *n_markers. Outputs may be NULL. */
int lbmb_build_stirred_tank(const lbmb_tank_spec* spec, uint8_t* solid, uint8_t* baffle_mask,
                            double* wall_velocity, double* marker_pos, double* marker_weight, int64_t capacity,
                            int64_t* n_markers, double center[3], double omega[3]);

/* No counterpart in the reference. The f64 reduction of lbmb_reduce over
 * populations the caller already holds in device memory, for callers that
 * cannot allocate device memory while they run (an application that owns
 * every device byte through its own arena, a process under a hard memory
 * quota, a stepping loop that must not call cudaMalloc/cudaFree). It
 * allocates nothing: its block partials live in a fixed file-scope device
 * array of about 640 KiB that every device loading this library keeps
 * until exit.
 *   f:      device, q-major populations f[q * plane + cell] (normal layout),
 *           element type per `storage`; plane >= ncells.
 *   solid:  device, ncells bytes (nonzero = solid, skipped), or NULL.
 *   force:  host, uniform body force for the F/2 momentum term, or NULL.
 *   out:    host, {fluid cells, sum f_dev, momentum x, y, z}.
 *   stream: cudaStream_t to run on (NULL: the legacy default stream).
 * ncells above 33,554,432 (2^25) is rejected with LBMB_ERR_INVALID. Each
 * call looks up the array's address in the current device context (a
 * lookup, not an allocation); the first call on a device loads the array's
 * module, so make it before any stream capture. Calls share the array:
 * calls that overlap on the GPU race and must be serialized by the caller. */
int lbmb_reduce_populations_noalloc(const void* f, int32_t storage, int32_t q, int64_t ncells, int64_t plane,
                                    const uint8_t* solid, const double force[3], double out[5], void* stream);

/* Sweep kernel of the fused collide-stream (no reference counterpart: the
 * reference has one CPU row loop per operator). All kinds compute the same
 * update; they differ in how populations reach the registers:
 *   LBMB_SWEEP_DIRECT  one cell per thread, direct loads (every config);
 *   LBMB_SWEEP_BULK    bulk asynchronous copies staged in shared memory;
 *   LBMB_SWEEP_ASYNC   per-thread cp.async ring (4/8-byte storage);
 *   LBMB_SWEEP_PAIR    two x-adjacent cells per thread, 2-element accesses
 *                      (4 bytes and more for 16-bit storage) and packed
 *                      fp32x2 arithmetic (TRT/BGK or central moment on
 *                      D3Q27, fp32/fp16/bf16 storage, even nx, no uniform
 *                      body force);
 *   LBMB_SWEEP_TILE    the pair update fed by 16-byte cp.async windows
 *                      staged in shared memory several tiles ahead (same
 *                      conditions as LBMB_SWEEP_PAIR);
 *   LBMB_SWEEP_LEAN    one cell per thread with a small register footprint
 *                      for high occupancy (TRT/BGK, fp32/fp16/bf16 storage,
 *                      no uniform body force);
 *   LBMB_SWEEP_WINDOW  one cell per thread, tiles of 256 cells staged in
 *                      shared memory by 16-byte cp.async windows several
 *                      tiles ahead (TRT/BGK or central moment, fp32/fp16/
 *                      bf16 storage, no uniform body force).
 * A kind that cannot run the solver's configuration returns
 * LBMB_ERR_UNSUPPORTED and leaves the current kind in place. */
typedef enum {
  LBMB_SWEEP_DIRECT = 0,
  LBMB_SWEEP_BULK = 1,
  LBMB_SWEEP_ASYNC = 2,
  LBMB_SWEEP_PAIR = 3,
  LBMB_SWEEP_TILE = 4,
  LBMB_SWEEP_LEAN = 5,
  LBMB_SWEEP_WINDOW = 6
} lbmb_sweep_kind;
int lbmb_set_sweep_kernel(lbmb_solver* h, int32_t kind);
int lbmb_get_sweep_kernel(lbmb_solver* h, int32_t* kind);
/* Launch variant of the current sweep kernel (no reference counterpart).
 * Lean kernel: register budget per parity, as resident 128-thread blocks per
 * SM the kernel is compiled for: 10 (48 registers), 9 (56), 8 (64), 7 (72)
 * or 6 (80); more
 * registers avoid spills, fewer keep more warps resident. cp.async kernel
 * (fp32 storage): the same per parity with 4 (128 registers, 3-tile ring,
 * the default), 5 (96, 3 tiles) or 6 (80, 2 tiles); its persistent grid
 * fills every resident slot, less 32 block slots in the sweep of a runner
 * step, where the IBM kernels run concurrently on a side stream. Window
 * kernel: resident 256-thread blocks per SM per parity, 2 (128 registers),
 * 3 (80) or 4 (64), with a tile ring of 3 where shared memory allows, else
 * 2; default 2 for the central moment, 3 for TRT/BGK. Pair kernel (TRT/BGK,
 * D3Q27 central moment): resident 128-thread blocks per SM per parity, 3 (168
 * registers), 4 (128, the default) or 5 (96); 13, 14 or 15 name the same
 * budgets with the populations of the next tile staged in shared memory by
 * cp.async while the warp computes the current one (two stages of Q x 32
 * 8-byte slots per warp; the grid holds as many blocks as shared memory
 * allows, at most the budget's). The persistent pair grid leaves 32 block
 * slots free in a runner step as the cp.async kernel does. */
int lbmb_set_sweep_variant(lbmb_solver* h, int32_t even_blocks_per_sm, int32_t odd_blocks_per_sm);

/* Sweep autotuner (no reference counterpart): times every sweep kernel kind
 * that can run this solver's configuration, and every register budget of
 * the lean kernel, for steps_per_trial hydro steps each on the solver's own
 * grid and state, selects the fastest and restores the populations, so the
 * simulation continues exactly as before the call. Optional per-trial
 * outputs (capacity entries): trial_desc[3 i] = {kind, even, odd blocks per
 * SM (0 for kinds without a register budget)}, trial_ms[i] = ms per step.
 * Needs one extra population buffer of device memory while it runs. */
typedef struct {
  int32_t kind;
  int32_t even_blocks_per_sm;
  int32_t odd_blocks_per_sm;
  int32_t n_trials;
  double best_ms_per_step;
  double default_ms_per_step; /* the kernel in place before the call */
} lbmb_autotune_result;
int lbmb_autotune_sweep(lbmb_solver* h, int32_t steps_per_trial, lbmb_autotune_result* out,
                        int32_t* trial_desc, double* trial_ms, int32_t capacity);

/* Batched runner for sweeps (replaces the sequential per-case loop of
 * crates/lbm-cli/src/sweep.rs:47-106, each case being runner.rs:1079-1129).
 * ncases solvers of one lattice and storage type (TRT/BGK, fp32/fp16/bf16,
 * no uniform force, no scalar distributions, one device, same step parity)
 * are advanced in lockstep: per step one launch per kernel family covers
 * every case (IBM prep / interp / spread / diag / commit, forced cells, the
 * full-grid sweep, the cached-field refresh), captured in CUDA graphs. Each
 * case runs the runner step of its own body (bodies[k], NULL = body 0, set
 * with lbmb_ibm_set_body) with cfg; per-case results equal running the case
 * alone with the lean sweep kernel. The solvers must outlive the batch and
 * must not be stepped on their own while a batch call runs. */
typedef struct lbmb_batch lbmb_batch;
int lbmb_batch_create(lbmb_solver* const* solvers, const int32_t* bodies, int32_t ncases,
                      const lbmb_ibm_config* cfg, lbmb_batch** out);
/* Register budget of the batched sweep picked by timing every candidate on
 * the cases' own grids (populations restored afterwards). */
int lbmb_batch_autotune(lbmb_batch* b, int32_t steps_per_trial, int32_t* even_blocks_per_sm,
                        int32_t* odd_blocks_per_sm, double* best_ms_per_step);
/* steps runner steps of every case; torque_lu (may be NULL) receives
 * ncases x steps values, case-major (-torque_z, runner.rs:1396-1425);
 * device_ms (may be NULL) the device time of the whole call. */
int lbmb_batch_run(lbmb_batch* b, int64_t steps, double* torque_lu, double* device_ms);
int lbmb_batch_destroy(lbmb_batch* b);

/* Adjoint of the runner loop (no reference counterpart: the reference has
 * no differentiation). Runs `steps` runner steps from the solver's current
 * state with the body's IBM at a fixed sweep count (cfg->max_iterations,
 * slip tolerance ignored: no early exit), J = mean of the per-step torque
 * (runner.rs:1396-1425 convention) over steps [window_begin, steps). The
 * populations are checkpointed every checkpoint_every steps; the backward
 * pass recomputes each segment from its checkpoint and runs the discrete
 * adjoint of the IBM + TRT collide-stream step in reverse, giving dJ/dnu,
 * dJ/dOmega_z (rad/step) and dJ/d(marker position) (3 per marker, NULL to
 * skip). torque (may be NULL) receives the forward series (steps values).
 * Needs TRT/BGK, no subgrid model, no uniform force, no scalars. The solver
 * ends in the state after the forward run. Device memory: one population
 * buffer per checkpoint and per step of a segment. */
typedef struct {
  int64_t steps;
  int64_t window_begin;
  int32_t checkpoint_every; /* default 100 when <= 0; rounded up to even */
  int32_t body;
} lbmb_adjoint_config;
typedef struct {
  double J;
  double dJ_dnu;
  double dJ_domega_z;
  double dJ_domega_plus;  /* w.r.t. the TRT rates, for reference */
  double dJ_domega_minus;
  double forward_ms;      /* device time of the checkpointed forward run */
  double adjoint_ms;      /* device time of recomputation + backward pass */
  int64_t markers;
} lbmb_adjoint_result;
int lbmb_adjoint_torque(lbmb_solver* h, const lbmb_ibm_config* cfg, const lbmb_adjoint_config* ac,
                        lbmb_adjoint_result* out, double* dJ_dpos, double* torque);

/* Synchronize the solver stream. */
int lbmb_sync(lbmb_solver* h);

/* ---- Checkpoint/restart (the reference's v3 file format) -----------------
 * A checkpoint is a directory: manifest.json and rank_0000_part_0000.bin
 * (crates/lbm-core/src/solver.rs:29-44, 84-118, 4536-4724). Populations are
 * written over the reference's halo-padded box (halo cells zero) in the
 * run's dtype: "f64" for F64 storage, "f32" for F32 / F16 / BF16 storage
 * (16-bit values widen exactly). The stale stash is written as zero planes.
 * Restoring validates the manifest and the rank file (kind, format version,
 * dtype, lattice, extents, scenario hash, decomposition hash, rank count,
 * part geometry, mask hash, payload hash, section lengths, solid mask) and
 * installs nothing on any failure. */

/* Solver::time (solver.rs:4642): hydro steps taken since creation or
 * installed by a restore. */
int lbmb_get_time(const lbmb_solver* h, uint64_t* step);

/* Name of a scalar distribution as the checkpoint records it (the
 * reference's enable_scalar_distribution name, solver.rs:2856); default
 * "scalar<k>". At most 63 bytes. */
int lbmb_set_scalar_name(lbmb_solver* h, int32_t k, const char* name);

/* QoiCheckpointState carried opaque (a JSON object) through save/restore
 * (Solver::set_qoi_checkpoint_state / qoi_checkpoint_state; section
 * QOI_ACCUMULATORS, solver.rs:4583-4585). json = NULL clears. get: len
 * receives the byte length (-1 when none is set); at most cap bytes are
 * copied. */
int lbmb_set_qoi_checkpoint_state(lbmb_solver* h, const char* json, int64_t len);
int lbmb_get_qoi_checkpoint_state(lbmb_solver* h, char* buf, int64_t cap, int64_t* len);

/* Solver::save (solver.rs:4715-4724). */
int lbmb_checkpoint_save(lbmb_solver* h, const char* dir);

/* Solver::restore (solver.rs:4739-4742, load_into 4759-5060) into this
 * solver, whose configuration and masks are the authority the checkpoint is
 * checked against. The scalar distributions of the file replace the
 * solver's: an enabled scalar is overwritten when its lattice matches,
 * further ones are enabled; a solver with more scalars than the file, or
 * with a different scalar lattice, is refused (CKPT_SCENARIO_MISMATCH). The
 * body-force field of the file becomes the solver's field, both the one the
 * next collision applies and the one inside the cached moments; solid-cell
 * moments are installed as carried values. The relaxation field is not part
 * of the format and is left as it is. */
int lbmb_checkpoint_restore(lbmb_solver* h, const char* dir);

/* The format on caller-owned compact host arrays, no device involved (the
 * reference's write_part_checkpoint / read_rank_file on one part). */
typedef struct {
  int32_t lattice;    /* 19 | 27 */
  int32_t collision;  /* lbmb_collision */
  int32_t dtype_bits; /* 32 | 64: the run's arithmetic type */
  int32_t dims[3];
  int32_t periodic[3];
  double nu, magic, omega_shear;
  double force[3];
} lbmb_checkpoint_spec;

typedef struct {
  char name[64];
  double diffusivity;
  int32_t q;          /* 7 or the hydro lattice */
  double* h;          /* q x ncells, ordinary form, logical post-stream */
  int64_t h_capacity; /* elements of h (read) */
  double* conc;       /* ncells */
} lbmb_checkpoint_scalar;

typedef struct {
  uint64_t step;
  double* f;           /* Q x ncells, deviation form */
  double* moments;     /* 4 x ncells: rho, ux, uy, uz */
  int32_t has_force_field;
  double* force_field; /* ncells x 3 */
  int32_t n_scalars;
  int32_t scalar_capacity; /* entries of scalars (read) */
  lbmb_checkpoint_scalar* scalars;
  int32_t has_qoi;
  char* qoi_json;
  int64_t qoi_len;
  int64_t qoi_capacity; /* bytes of qoi_json (read) */
} lbmb_checkpoint_data;

int lbmb_checkpoint_write_host(const char* dir, const lbmb_checkpoint_spec* spec, const uint8_t* solid,
                               const double* wall_u, const lbmb_checkpoint_data* data);
int lbmb_checkpoint_read_host(const char* dir, const lbmb_checkpoint_spec* spec, const uint8_t* solid,
                              const double* wall_u, lbmb_checkpoint_data* data);

/* FNV-1a 64 of a byte buffer (the checkpoint payload hash, solver.rs:
 * 831-835). */
uint64_t lbmb_fnv1a64(const void* data, uint64_t len);


/* ---- Runner QOIs, unit report, scalar pulse, capabilities -------------- */

/* qoi::PowerQoiResult (crates/lbm-core/src/qoi.rs:455-468), nq omitted
 * (the reference runner skips it: no discharge surface). */
typedef struct {
  double torque_n_m;
  double power_w;
  double rotational_speed_hz;
  double np;            /* P / (rho N^3 D^5) */
  double p_over_v_w_m3; /* P / V */
} lbmb_power_result;

/* qoi::power_qois (crates/lbm-core/src/qoi.rs:477-505): P = omega Tq,
 * N = omega / 2 pi. LBMB_ERR_INVALID for non-finite or non-positive
 * dimensional inputs, or N <= 0 (the reference's Err). */
int lbmb_power_qois(double torque_n_m, double omega_rad_s, double rho_kg_m3, double impeller_diameter_m,
                    double working_volume_m3, lbmb_power_result* out);

/* torque_record_from_ibm + write_power_qois (crates/lbm-cli/src/runner.rs:
 * 1396-1425, 1514-1543) over the per-step lattice torque series that
 * lbmb_run_impeller writes (entry s - 1 = step s): the runner records steps
 * with s % probe_every == 0 or s == run_steps, converts each to N m with
 * rho dx^5 / dt^2, averages the records with s >= run_steps / 2 (all
 * records when none is that late) and applies power_qois with the
 * impeller's SI angular speed. executed = steps the run took (a diverged
 * run stops early); *records_used (may be NULL) = records averaged. */
int lbmb_power_from_torque_series(const double* torque_lu, int64_t executed, int64_t run_steps, int64_t probe_every,
                                  double rho_kg_m3, double dx_m, double dt_s, double omega_rad_s,
                                  double impeller_diameter_m, double working_volume_m3, lbmb_power_result* out,
                                  int64_t* records_used);

/* Inputs of bioprocess_unit_report for a single-phase stirred tank
 * (crates/lbm-scenario/src/units.rs:116-208). */
typedef struct {
  double vessel_diameter_m;
  double liquid_height_m;
  double impeller_diameter_m;
  double rotational_speed_rpm;
  double liquid_density_kg_m3;
  double liquid_viscosity_pa_s;
  double dt_s;
  int32_t grid[3];
  double scalar_diffusivity_m2_s; /* passive scalar diffusivity; <= 0: no scalar model */
} lbmb_unit_input;

/* Feasibility codes of the unit report (units.rs:8-31, 210-305), as bits. */
enum lbmb_unit_issue {
  LBMB_UNIT_MA_LATTICE_HIGH = 1,            /* warning: Ma > 0.10 */
  LBMB_UNIT_MA_LATTICE_TOO_HIGH = 2,        /* rejection: Ma > 0.30 */
  LBMB_UNIT_TAU_NEAR_HALF = 4,              /* warning: 0.5 < tau <= 0.55 */
  LBMB_UNIT_TAU_NON_POSITIVE_VISCOSITY = 8, /* rejection: tau <= 0.5 */
  LBMB_UNIT_GRID_REYNOLDS_HIGH = 16,        /* warning: u_lu / nu_lu > 15 */
  LBMB_UNIT_SCALAR_DIFFUSION_UNSTABLE = 32  /* warning: nu_lu / D_lu > 25 */
};

/* UnitReport's lattice mapping and single-phase groups (units.rs:33-95). */
typedef struct {
  double dx_m;    /* vessel diameter / nx */
  double dt_s;
  double u_ref_lu; /* N D dt / dx */
  double nu_lu;    /* (mu / rho) dt / dx^2 */
  double tau_lu;   /* 3 nu_lu + 1/2 */
  double cs2_lu;   /* 1/3 */
  double reynolds; /* rho N D^2 / mu */
  double froude;   /* N^2 D / g */
  double mach_lattice;
  double schmidt;  /* NaN without a scalar */
  double peclet;   /* u_ref T / D; NaN without a scalar */
  double scalar_diffusivity_lu; /* D dt / dx^2; NaN without a scalar */
  double grid_reynolds;         /* u_ref_lu / nu_lu */
  uint32_t warnings;            /* lbmb_unit_issue bits */
  uint32_t rejections;          /* lbmb_unit_issue bits */
} lbmb_unit_mapping;

/* bioprocess_unit_report (units.rs:96-325), single-phase subset: fills
 * *out; LBMB_ERR_INVALID for a non-positive input (require_positive),
 * LBMB_ERR_UNSUPPORTED with *out filled when a rejection fired (the
 * checked report's OutOfValidityRange). */
int lbmb_unit_report(const lbmb_unit_input* in, lbmb_unit_mapping* out);

/* scalar_initial_condition, pulse branch (crates/lbm-cli/src/runner.rs:
 * 1317-1377): values[cell] = concentration on fluid cells whose centre
 * ((x + 0.5) dx, ...) lies within radius_m of center_m, else 0 (solid may
 * be NULL: no solids). */
int lbmb_scalar_top_hat_pulse(const int32_t dims[3], const uint8_t* solid, double dx_m, const double center_m[3],
                              double radius_m, double concentration, double* values);

/* The pulse's lattice diffusivity D dt / dx^2 (runner.rs:1371-1375), the
 * value lbmb_enable_scalar takes. */
int lbmb_scalar_diffusivity_lu(double diffusivity_m2_s, double dt_s, double dx_m, double* d_lu);

/* Reasons a distribution family is unsupported (UnsupportedReason,
 * crates/lbm-core/src/solver.rs:174). */
enum lbmb_unsupported_reason { LBMB_SUPPORTED = 0, LBMB_UNSUPPORTED_NOT_IMPLEMENTED = 1 };

/* The Backend trait's capability hooks (crates/lbm-core/src/backend.rs:
 * 162-199, 343-345) for this device backend, plus what the handle's
 * configuration enables here. */
typedef struct {
  int32_t handles_single_part_periodic_halo; /* 1: periodic axes wrap inside the sweep */
  int32_t supports_localized_features;       /* 0: no volume sources or masked face patches */
  int32_t supports_d3q27_open_faces;         /* 0: no open faces */
  int32_t supports_two_pass;                 /* 0: the collide-stream is one fused sweep */
  int32_t supports_gravity_body_force;       /* 0: uniform and IBM force fields only */
  int32_t distribution_hydro;                /* lbmb_unsupported_reason */
  int32_t distribution_phase;
  int32_t distribution_scalar;
  int64_t run_chunk_size;                    /* steps one call takes without a host sync (INT64_MAX: any) */
  uint32_t lattices;                         /* bit 0: D3Q19, bit 1: D3Q27, bit 2: D3Q7 scalars */
  uint32_t storages;                         /* bit k: lbmb_storage k */
  uint32_t collisions;                       /* bit k: lbmb_collision k */
  int32_t adjoint;                           /* the handle's configuration allows lbmb_adjoint_torque */
  int32_t batch;                             /* ... lbmb_batch_create */
  int32_t checkpoint;                        /* ... lbmb_checkpoint_save / restore */
} lbmb_backend_caps;

/* Capability query (Backend::distribution_support and supports_* hooks,
 * backend.rs:162-199). h may be NULL: the backend's general answers, with
 * adjoint / batch / checkpoint reporting what some configuration allows. */
int lbmb_capabilities(lbmb_solver* h, lbmb_backend_caps* out);

#ifdef __cplusplus
}
#endif

#endif /* LBMB_H */
