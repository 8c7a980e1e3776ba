/*
 * orchard_b200.h -- C ABI of the B200 (sm_100a) projection time step.
 *
 * Drop-in boundary for the CPU path of Orchard Flow (zfifteen/solver).  The
 * reference has no FFI layer; its seams are C++ free functions, and each entry
 * point below replaces one of them (cited as file:line in the reference).  The
 * Python binding (solver_b200/_capi.py) is a thin layer over this header.
 *
 * Conventions
 *  - All arrays are the reference's padded MAC storage, double precision,
 *    one ghost layer, index i + sx*(j + sy*k), i unit-stride
 *    (core/field_layout.hpp:178-183).  A cell field has storage
 *    (nx+2, ny+2, nz+2); the face field normal to axis a has one more entry
 *    along a (core/field_layout.hpp:75-86).
 *  - Host arrays are borrowed for the duration of a call only.  Calls are
 *    synchronous: they return after results and diagnostics are on the host.
 *  - One context per host thread; a context owns one CUDA stream and all
 *    device memory for its grid (state, scratch, multigrid hierarchy).
 *  - Every entry point returns an of_status; of_last_error() gives the text of
 *    the last failure on the calling thread, worded as the reference's
 *    exceptions so that the C++ layer can rethrow them unchanged.
 *  - There is no CPU fallback: a missing or unusable GPU is an error.
 */
#ifndef ORCHARD_B200_H
#define ORCHARD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OF_ABI_VERSION 1

typedef enum {
  OF_OK = 0,
  OF_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  OF_RUNTIME_ERROR = 2,    /* std::runtime_error: zero pivot, singular coarse matrix */
  OF_NOT_CONVERGED = 3,    /* require_converged_pressure_projection (solver/projection.cpp:1133) */
  OF_NONFINITE = 4,        /* "... solve produced a non-finite state" (solver/taylor_green.cpp:614) */
  OF_CUDA_ERROR = 5,
  OF_TIMEOUT = 6           /* a device-side wait gave up (never expected) */
} of_status;

/* Grid (core/grid.hpp:57-87); ghost_layers is always 1. */
typedef struct {
  int nx, ny, nz;
  double dx, dy, dz;
} of_grid;

/* PhysicalBoundaryType (bc/boundary_conditions.hpp:10-16) */
enum { OF_NO_SLIP_WALL = 0, OF_PRESCRIBED_VELOCITY = 1, OF_SYMMETRY = 2, OF_FIXED_PRESSURE = 3,
       OF_PERIODIC = 4 };
/* PressureBoundaryType (bc/boundary_conditions.hpp:18-22) */
enum { OF_P_NEUMANN = 0, OF_P_DIRICHLET = 1, OF_P_PERIODIC = 2 };

/* BoundaryCondition (bc/boundary_conditions.hpp:24-29) */
typedef struct {
  int type;
  double velocity[3];
  double pressure;
  double pressure_gradient;
} of_face_bc;

/* BoundaryConditionSet; faces x_min, x_max, y_min, y_max, z_min, z_max. */
typedef struct {
  of_face_bc faces[6];
} of_bc;

/* PressureBoundaryCondition / PressureBoundarySet (bc/boundary_conditions.hpp:46-62) */
typedef struct {
  int type;
  double value;
  double gradient;
} of_pface_bc;

typedef struct {
  of_pface_bc faces[6];
} of_pbc;

/* PoissonSolveDiagnostics (solver/projection.hpp:22-39); the four label
 * strings ("mgpcg", "geometric_multigrid", "v_cycle", "damped_jacobi") and
 * the residual history are supplied separately. */
typedef struct {
  int iterations;
  double initial_residual_l2;
  double final_residual_l2;
  double relative_residual;
  double removed_rhs_mean;
  int multigrid_levels;
  int coarse_unknowns;
  int pre_smoothing_steps;
  int post_smoothing_steps;
  int converged;
  int zero_mean_enforced;
} of_poisson_diag;

/* ProjectionDiagnostics (solver/projection.hpp:41-47) */
typedef struct {
  double rhs_l2;
  double divergence_l2_before;
  double divergence_l2_after;
  double pressure_mean;
  of_poisson_diag pressure_solve;
} of_projection_diag;

/* TaylorGreenStepMetrics (solver/taylor_green.hpp:32-42); the cavity's
 * SimulationStepMetrics (solver/lid_driven_cavity.hpp:27-36) is the same
 * without max_divergence_l2. */
typedef struct {
  int step;
  double time;
  double dt;
  double max_cfl;
  double max_velocity_change;
  double divergence_l2;
  double max_divergence_l2;
  int pressure_iterations;
  double pressure_relative_residual;
} of_step_metrics;

/* Arithmetic of the pressure solve.  OF_FP64 follows the reference; OF_MIXED
 * runs the multigrid V-cycle in FP32 storage and arithmetic inside the FP64
 * conjugate-gradient loop (residual, search direction, dot products, mean
 * removal and the coarsest-grid solve stay FP64). */
enum { OF_FP64 = 0, OF_MIXED = 1 };

/* Predictor factorisation-correction variant: the Taylor-Green form
 * (solver/taylor_green.cpp:196-225, 3D terms when nz > 1) or the cavity's 2D
 * form (solver/lid_driven_cavity.cpp:219-252). */
enum { OF_CORRECTION_TAYLOR_GREEN = 0, OF_CORRECTION_CAVITY = 1 };

/* Parameters of one projection time step (the locals of
 * run_taylor_green_steps, solver/taylor_green.cpp:556-564, and of
 * advance_lid_driven_cavity_impl, solver/lid_driven_cavity.cpp:538-547). */
typedef struct {
  double viscosity;
  double dt;
  double density;
  int poisson_max_iterations;
  double poisson_tolerance;
  int correction_variant;    /* OF_CORRECTION_* */
  int track_max_divergence;  /* 1: update max_divergence_l2 (Taylor-Green) */
  const char* solver_name;   /* "Taylor-Green" / "lid-driven cavity" for messages */
} of_step_params;

typedef struct of_ctx of_ctx;

/* ---- library / context ------------------------------------------------- */

int of_abi_version(void);
/* Text of the last failure on this thread (empty if none). */
const char* of_last_error(void);

/* Creates a context for one grid and velocity boundary set on `device`
 * (a CUDA ordinal).  Validates the grid like Grid's constructor
 * (core/grid.hpp:76-86) and the pairing of periodic faces. */
of_status of_create(const of_grid* grid, const of_bc* bc, int device, of_ctx** out);
of_status of_destroy(of_ctx* ctx);
of_status of_set_precision(of_ctx* ctx, int precision);
/* Bytes of device memory the context holds. */
of_status of_device_bytes(of_ctx* ctx, size_t* bytes);
/* The grid the context was created on. */
of_status of_get_grid(of_ctx* ctx, of_grid* grid);

/* ---- operator entry points (host buffers) ------------------------------- */

/* compute_advection_term, TVD/van Leer (solver/momentum_terms.hpp:36-38,
 * solver/momentum_terms.cpp:307-314).  Writes the active entries of a*;
 * their ghost entries are left as passed in. */
of_status of_compute_advection_term(of_ctx* ctx, const double* u, const double* v,
                                    const double* w, double* au, double* av, double* aw);

/* solve_predictor_adi (solver/projection.hpp:49-52, solver/projection.cpp:1028-1047). */
of_status of_solve_predictor_adi(of_ctx* ctx, double alpha, const double* rhs_u,
                                 const double* rhs_v, const double* rhs_w, double* pred_u,
                                 double* pred_v, double* pred_w, int* line_solves);

/* linsolve::solve_pressure_poisson (linsolve/poisson_solver.hpp:34-37,
 * linsolve/poisson_solver.cpp:678-809).  `pressure` is in/out (its active
 * entries are the initial guess).  `history` receives up to history_cap
 * residual norms (may be NULL). */
of_status of_solve_pressure_poisson(of_ctx* ctx, const of_pbc* pbc, int max_iterations,
                                    double tolerance, const double* rhs, double* pressure,
                                    of_poisson_diag* diag, double* history, int history_cap);

/* project_velocity (solver/projection.hpp:65-70, solver/projection.cpp:1097-1131).
 * pressure_correction is in/out; pressure_rhs may be NULL. */
of_status of_project_velocity(of_ctx* ctx, double dt, double density, int max_iterations,
                              double tolerance, const double* pred_u, const double* pred_v,
                              const double* pred_w, double* pressure_correction,
                              double* corr_u, double* corr_v, double* corr_w,
                              double* pressure_rhs, of_projection_diag* diag);

/* ---- resident state (run_taylor_green_steps / run_lid_driven_cavity_steps) */

/* Copies a TaylorGreenState / LidDrivenCavityState (solver/taylor_green.hpp:44-57)
 * to the device.  adv_* is the AB2 history (advection_previous). */
of_status of_state_upload(of_ctx* ctx, const double* u, const double* v, const double* w,
                          const double* adv_u, const double* adv_v, const double* adv_w,
                          const double* p_total, int has_previous_advection,
                          const of_step_metrics* metrics);
of_status of_state_download(of_ctx* ctx, double* u, double* v, double* w, double* adv_u,
                            double* adv_v, double* adv_w, double* p_total,
                            int* has_previous_advection, of_step_metrics* metrics);

/* Taylor-Green initial state on the device (solver/taylor_green.cpp:335-395)
 * for the context's grid.  mode 0: the reference's phase; mode 1: the same
 * flow shifted by (pi/2, pi/2): u = sin x cos y [cos z],
 * v = -cos x sin y [cos z], p = +1/4 (cos 2x + cos 2y) [2D] or
 * +1/16 (cos 2x + cos 2y)(cos 2z + 2) [3D]. */
of_status of_tg_init(of_ctx* ctx, double viscosity, double dt, int mode);

/* Fluid at rest with the boundary conditions applied: zero velocity, history
 * and total pressure, then the velocity ghost fills and the total-pressure
 * ghosts from viscosity * Laplacian (initialize_lid_driven_cavity_state,
 * solver/lid_driven_cavity.cpp:390-408).  Metrics reset, metrics.dt = dt. */
of_status of_rest_init(of_ctx* ctx, double viscosity, double dt);

/* ---- diagnostics of the resident state (case-driver validation) --------- */

/* kinetic_energy (solver/taylor_green.cpp:269-289): the mean over cells of
 * 1/2 |face-averaged velocity|^2, reduced on the device. */
of_status of_kinetic_energy(of_ctx* ctx, double* energy);

/* velocity_relative_l2_error (solver/taylor_green.cpp:291-333) of the
 * resident velocity against the Taylor-Green field of phase `mode` (as
 * of_tg_init) decayed by exp(-rate * viscosity * time), rate 3 in 3D and 2 in
 * 2D; reduced on the device. */
of_status of_tg_velocity_error(of_ctx* ctx, double viscosity, double time, int mode,
                               double* error);

/* Copies one storage line of a resident field to the host: field 0 = total
 * pressure, 1..3 = velocity u, v, w; the line runs along `axis` (0..2) over
 * the whole storage extent n of that axis, through the storage indices
 * (i, j, k) of the other two axes (the index along `axis` is ignored).
 * `out` holds n doubles; *n_out (optional) receives n.  The centreline
 * samples of the cavity (solver/lid_driven_cavity.cpp:100-131) are such lines. */
of_status of_sample_line(of_ctx* ctx, int field, int axis, int i, int j, int k, double* out,
                         int* n_out);

/* Runs `steps` projection steps on the resident state: the loop body of
 * run_taylor_green_steps (solver/taylor_green.cpp:577-633) and of
 * advance_lid_driven_cavity_impl (solver/lid_driven_cavity.cpp:562-623).
 * Fails with OF_NOT_CONVERGED / OF_NONFINITE at the step where the
 * reference throws; the state then holds the last completed step. */
of_status of_run_steps(of_ctx* ctx, const of_step_params* params, int steps,
                       of_step_metrics* metrics);

/* One step of a host-resident state: of_state_upload of the arrays,
 * of_run_steps(1) and of_state_download back into the same arrays, with
 * has_previous_advection and metrics in/out -- the call a caller that keeps
 * its TaylorGreenState / LidDrivenCavityState on the host makes per step
 * (run_taylor_green_steps with step_count 1).  When the three adv_* arrays
 * are pinned (cudaHostAlloc / cudaHostRegister), the new AB2 history is copied
 * back while the pressure solve runs.  On failure the arrays hold the state
 * they were called with. */
of_status of_step_host(of_ctx* ctx, const of_step_params* params, double* u, double* v, double* w,
                       double* adv_u, double* adv_v, double* adv_w, double* p_total,
                       int* has_previous_advection, of_step_metrics* metrics);

/* ---- tangent-linear and adjoint runs -------------------------------------- */

/* No counterpart in the reference: the discrete derivatives of of_run_steps
 * on periodic grids with the Taylor-Green predictor.  Both start from the
 * context's resident state and leave it `steps` steps later, as of_run_steps
 * does.  The advection is linearised with its limiter, upwind and
 * first-order branches frozen at the base trajectory. */

/* Diagnostics of an adjoint run. */
typedef struct {
  double loss;             /* 1/2 |u(T) - target|^2 over the unique velocity entries */
  double grad_viscosity;   /* d loss / d viscosity */
  int forward_steps;       /* forward steps run, recomputation included */
  double forward_ms;       /* device time of the first forward pass */
  double backward_ms;      /* device time of the recomputation and reverse steps */
  size_t device_bytes;     /* device memory held by the tangent-linear / adjoint buffers */
  int snapshots;           /* saved states besides the initial one */
  size_t device_bytes_in_use; /* device memory in use after the forward pass (all allocations) */
} of_adjoint_info;

/* du, dv, dw (host, padded): a perturbation of the active entries of the
 * resident velocity.  out_*: the tangent-linear velocity after `steps` steps
 * (ghosts filled). */
of_status of_tangent_linear(of_ctx* ctx, const of_step_params* params, int steps, const double* du,
                            const double* dv, const double* dw, double* out_u, double* out_v,
                            double* out_w);

/* Gradient of loss = 1/2 sum over the unique velocity entries (the duplicated
 * periodic face excluded) of (u(T) - target)^2 with respect to the active
 * entries of the resident velocity (grad_*, host, padded, ghosts zero) and to
 * the viscosity (info->grad_viscosity).  The state before every
 * `checkpoint_every` steps is kept; each segment is recomputed from it during
 * the reverse sweep. */
of_status of_adjoint_gradient(of_ctx* ctx, const of_step_params* params, int steps,
                              int checkpoint_every, const double* target_u,
                              const double* target_v, const double* target_w, double* grad_u,
                              double* grad_v, double* grad_w, of_adjoint_info* info);

/* The same gradient with the optimal binomial checkpoint schedule ("revolve",
 * Griewank & Walther, ACM TOMS 26, 2000): `snapshots` saved states besides the
 * initial one, placed so that the number of recomputed forward steps is the
 * least possible; snapshots = 0 takes as many as fit in the free device memory
 * (2 GiB kept free, at most 64), and at most 128 are used in any case (with
 * 128, no step of a 4096-step horizon is advanced more than twice; the
 * schedule's dynamic program costs O(steps^2 snapshots) host operations,
 * about a second at 4096 steps and 128 snapshots).  The work set is leaner than
 * of_adjoint_gradient's (no tangent-linear buffers; the working state shares
 * the context's scratch), which is what lets 512^3 runs of hundreds of steps
 * fit one device.  steps <= 4096.  Every reverse step sees the same
 * recomputed state as in of_adjoint_gradient, so the results agree to
 * rounding (the transposed advection accumulates with atomics). */
of_status of_adjoint_gradient_binomial(of_ctx* ctx, const of_step_params* params, int steps,
                                       int snapshots, const double* target_u,
                                       const double* target_v, const double* target_w,
                                       double* grad_u, double* grad_v, double* grad_w,
                                       of_adjoint_info* info);

/* Host-only: forward steps the binomial schedule recomputes to reverse
 * `steps` steps with `snapshots` free snapshots -- from a saved initial state
 * alone (reverse_cost; Griewank's closed form for snapshots + 1 checkpoints)
 * and right after the forward pass that placed the first snapshots
 * (after_forward_cost, what of_adjoint_gradient_binomial runs beyond its
 * forward pass).  Snapshots beyond 128 are not used (as above).  Either
 * pointer may be NULL. */
of_status of_adjoint_schedule_cost(int steps, int snapshots, long long* reverse_cost,
                                   long long* after_forward_cost);

/* ---- allocation-free entry point ---------------------------------------- */

/* No counterpart in the reference (it has no device path).  The pressure
 * right-hand side pass of project_velocity on DEVICE buffers, without a
 * context: pressure_rhs = (density/dt) div(u) on the active cells
 * (build_pressure_rhs, solver/projection.cpp:1049-1064) and, when norms is
 * not NULL, norms[0] = divergence_l2_before and norms[1] = rhs_l2 (host
 * doubles; solver/projection.cpp:1110-1116).
 *
 * For callers that cannot allocate device memory: a framework that owns all
 * device memory through its own pool and calls this inside its step loop,
 * where a context's allocations and the device-wide synchronisation of
 * cudaMalloc/cudaFree are not acceptable.  The call allocates nothing: its
 * scratch (reduction partials, ticket, norms; 131,104 bytes) is a static
 * device array of the library, found by cudaGetSymbolAddress on the first
 * call on each device (setup; make that first call before any stream capture)
 * and cached until the process exits: do not reset the device
 * (cudaDeviceReset) between calls.
 *
 *  - u, v, w: device face fields in padded storage whose boundary conditions
 *    are already applied (project_velocity's `working` after
 *    apply_velocity_boundary_conditions); only active faces are read.
 *  - pressure_rhs: device cell field; active entries written, ghosts untouched.
 *  - Runs on the current CUDA device and on `stream` (a cudaStream_t; NULL is
 *    the default stream).  With norms == NULL the call only enqueues work;
 *    otherwise it returns after the norms are on the host.
 *  - Limits: at most 8192 blocks of 32 x 8 cells per k plane
 *    (ceil(nx/32) * ceil(ny/8) <= 8192, i.e. 2,097,152 cells per plane) and
 *    (nx+3)(ny+3)(nz+3) < 2^31; larger grids fail with OF_INVALID_ARGUMENT.
 *  - Calls on one device share the scratch: calls that overlap in time (two
 *    streams, two host threads) race and give wrong norms.  Serialise them. */
of_status of_pressure_rhs_noalloc(const of_grid* grid, double dt, double density,
                                  const double* u, const double* v, const double* w,
                                  double* pressure_rhs, double* norms, void* stream);

/* ---- instrumentation ---------------------------------------------------- */

/* The context's CUDA stream (cudaStream_t) for callers that time on it. */
of_status of_stream(of_ctx* ctx, void** stream);

/* Kernel classes (predictor_rhs, adi_sweep, ..., see of_kernel_class_name).
 * Every launch is counted; with profiling enabled each launch of a class is
 * also bracketed by CUDA events on its stream and its device time summed. */
int of_kernel_class_count(void);
const char* of_kernel_class_name(int id);
of_status of_profile_enable(int enable);
of_status of_profile_reset(void);
of_status of_profile_read(int id, long long* launches, long long* timed_launches,
                          double* total_ms);

/* Device time of the V-cycle's coarse-level chain (every level below the
 * finest, as each CG iteration runs it after the finest level's restriction)
 * inside a CUDA graph: the chain alone is captured once and replayed `reps`
 * times on the level-1 rhs of the context's last solve (a diagnostic: it
 * changes no state that a later solve reads).  *us_per_chain = microseconds
 * per chain, *launches_per_chain = its kernels.  Per-launch event timing
 * (of_profile_enable) cannot measure these short kernels inside the graph. */
of_status of_profile_coarse_chain(of_ctx* ctx, int reps, double* us_per_chain,
                                  int* launches_per_chain);

#ifdef __cplusplus
}
#endif

#endif /* ORCHARD_B200_H */
