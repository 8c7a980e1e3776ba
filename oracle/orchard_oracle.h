/*
 * CPU oracle interface for the Orchard Flow projection step.
 *
 * TEST INFRASTRUCTURE ONLY.  Two libraries export exactly this interface:
 *   - oracle/liborchard_oracle.so : a plain-C restatement of the reference
 *     algorithm (orchard_oracle.c), the checker used by the parity tests;
 *   - oracle/_ref/liborchard_ref.so : the reference's own C++ sources compiled
 *     in place (ref_shim.cpp adapts them to this interface), used to pin the
 *     restatement bit-for-bit.
 * Nothing in the product path may link or call either library.
 *
 * Arrays are the reference's padded MAC storage: double, one ghost layer,
 * index i + sx*(j + sy*k) with i unit-stride (core/field_layout.hpp:178-183).
 * Cell fields are (nx+2, ny+2, nz+2); the face field normal to axis a has
 * one more entry along a (core/field_layout.hpp:75-86).
 */
#ifndef ORCHARD_ORACLE_H
#define ORCHARD_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;
  double dx, dy, dz;
} oo_grid;

/* PhysicalBoundaryType (bc/boundary_conditions.hpp:10-16) */
enum { OO_NO_SLIP_WALL = 0, OO_PRESCRIBED_VELOCITY = 1, OO_SYMMETRY = 2, OO_FIXED_PRESSURE = 3,
       OO_PERIODIC = 4 };
/* PressureBoundaryType (bc/boundary_conditions.hpp:18-22) */
enum { OO_P_NEUMANN = 0, OO_P_DIRICHLET = 1, OO_P_PERIODIC = 2 };

typedef struct {
  int type;
  double velocity[3];
  double pressure;
  double pressure_gradient;
} oo_face_bc;

/* faces ordered x_min, x_max, y_min, y_max, z_min, z_max (core/grid.hpp:14-21) */
typedef struct {
  oo_face_bc faces[6];
} oo_bc;

typedef struct {
  int type;
  double value;
  double gradient;
} oo_pface_bc;

typedef struct {
  oo_pface_bc faces[6];
} oo_pbc;

/* PoissonSolveDiagnostics (solver/projection.hpp:22-39) without the strings */
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
} oo_poisson_diag;

/* ProjectionDiagnostics (solver/projection.hpp:41-47) */
typedef struct {
  double rhs_l2;
  double divergence_l2_before;
  double divergence_l2_after;
  double pressure_mean;
  oo_poisson_diag pressure_solve;
} oo_projection_diag;

/* TaylorGreenStepMetrics (solver/taylor_green.hpp:32-42); the cavity's
 * SimulationStepMetrics is the same without max_divergence_l2. */
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
} oo_step_metrics;

/* TaylorGreenConfig numeric keys (solver/taylor_green.hpp:18-30) */
typedef struct {
  int nx, ny, nz;
  double viscosity;
  double cfl_limit;
  double final_time;
  int poisson_max_iterations;
  double poisson_tolerance;
} oo_tg_config;

/* LidDrivenCavityConfig numeric keys (solver/lid_driven_cavity.hpp:12-25) */
typedef struct {
  int nx, ny;
  double reynolds;
  double lid_velocity;
  double cfl_limit;
  int max_steps;
  int min_steps;
  double steady_tolerance;
  int poisson_max_iterations;
  double poisson_tolerance;
} oo_cavity_config;

/* State arrays of a Taylor-Green or cavity run, all padded storage. */
typedef struct {
  double* u;
  double* v;
  double* w;
  double* adv_u;
  double* adv_v;
  double* adv_w;
  double* p;
  int has_previous_advection;
  oo_step_metrics metrics;
} oo_state;

/* Return codes: 0 ok, 1 invalid argument, 2 runtime error (pivot, non-finite,
 * non-convergence).  oo_last_error() holds the exception text. */
const char* oo_last_error(void);

/* TVD/van Leer advection term, active entries written (solver/momentum_terms.cpp:307). */
int oo_advection(const oo_grid* g, const double* u, const double* v, const double* w,
                 double* au, double* av, double* aw);
/* nu * Laplacian, active entries (solver/momentum_terms.cpp:316). */
int oo_diffusion(const oo_grid* g, double nu, const double* u, const double* v, const double* w,
                 double* du, double* dv, double* dw);
/* Ghost/duplicate-face fill in place (solver/projection.cpp:966). */
int oo_apply_velocity_bc(const oo_grid* g, const oo_bc* bc, double* u, double* v, double* w);
/* Pressure ghost fill in place (solver/projection.cpp:973). */
int oo_apply_pressure_bc(const oo_grid* g, const oo_pbc* pbc, double* p);
/* (solver/projection.cpp:934) */
int oo_derive_pressure_correction_bc(const oo_bc* bc, oo_pbc* out);
/* Total-pressure ghosts from the wall-normal source (solver/projection.cpp:986). */
int oo_apply_total_pressure_bc(const oo_grid* g, const oo_bc* bc, const double* su,
                               const double* sv, const double* sw, double* p);
/* MAC gradient / divergence (operators/discrete_operators.cpp:64,98). */
int oo_gradient(const oo_grid* g, const double* p, double* gu, double* gv, double* gw);
int oo_divergence(const oo_grid* g, const double* u, const double* v, const double* w,
                  double* div);
/* ADI predictor; out = rhs then per-component ADI (solver/projection.cpp:1028). */
int oo_predictor_adi(const oo_grid* g, const oo_bc* bc, double alpha, const double* ru,
                     const double* rv, const double* rw, double* pu, double* pv, double* pw,
                     int* line_solves);
/* MG-PCG Poisson solve (linsolve/poisson_solver.cpp:678); residual history
 * written to hist (capacity hist_cap, may be NULL). */
int oo_poisson_solve(const oo_grid* g, const oo_pbc* pbc, int max_iterations, double tolerance,
                     const double* rhs, double* pressure, oo_poisson_diag* diag, double* hist,
                     int hist_cap);
/* Projection (solver/projection.cpp:1097); rhs_out may be NULL. */
int oo_project_velocity(const oo_grid* g, const oo_bc* bc, double dt, double density,
                        int max_iterations, double tolerance, const double* pu,
                        const double* pv, const double* pw, double* phi, double* cu,
                        double* cv, double* cw, double* rhs_out, oo_projection_diag* diag);

/* Taylor-Green driver (solver/taylor_green.cpp:497-634). */
int oo_tg_grid(const oo_tg_config* c, oo_grid* g);
double oo_tg_dt(const oo_tg_config* c);
int oo_tg_bc(const oo_tg_config* c, oo_bc* bc);
/* mode 0: the reference's own initial state (solver/taylor_green.cpp:335);
 * mode 1: the same flow shifted by (pi/2, pi/2): u = sin x cos y [cos z],
 * v = -cos x sin y [cos z], p = +1/4 (cos 2x + cos 2y) [2D] or
 * +1/16 (cos 2x + cos 2y)(cos 2z + 2) [3D]. */
int oo_tg_init(const oo_tg_config* c, int mode, oo_state* s);
/* Re-runs the initial-state tail on caller-filled u, v, w (active) and p:
 * velocity BC, diffusion, total-pressure BC (solver/taylor_green.cpp:391-394). */
int oo_tg_init_tail(const oo_tg_config* c, oo_state* s);
int oo_tg_steps(const oo_tg_config* c, int steps, oo_state* s);
/* Validation of finalize_taylor_green_result (solver/taylor_green.cpp:258-333,
 * 403-417): kinetic energy, exact kinetic energy at `time`, normalized energy
 * error and velocity relative L2 error against the analytic decay.  mode as
 * in oo_tg_init (the analytic field is shifted the same way). */
typedef struct {
  double kinetic_energy;
  double exact_kinetic_energy;
  double normalized_energy_error;
  double velocity_relative_l2_error;
} oo_tg_validation;
int oo_tg_validate(const oo_tg_config* c, int mode, const double* u, const double* v,
                   const double* w, double time, oo_tg_validation* out);

/* Lid-driven cavity driver (solver/lid_driven_cavity.cpp:339-624). */
int oo_cavity_grid(const oo_cavity_config* c, oo_grid* g);
double oo_cavity_dt(const oo_cavity_config* c);
int oo_cavity_bc(const oo_cavity_config* c, oo_bc* bc);
int oo_cavity_init(const oo_cavity_config* c, oo_state* s);
int oo_cavity_steps(const oo_cavity_config* c, int steps, oo_state* s);

/* ---- reference build only (oracle/_ref/liborchard_ref.so) -------------------
 * The reference's drivers and I/O around the step, exported for the golden
 * fixtures of the case layer: config files, describe(), the SLVCHKP1
 * checkpoint, finalize and the VTK writer.  validate_* are the configs'
 * boolean keys (they enter describe() and the checkpoint). */
int oo_ref_tg_config_load(const char* path, oo_tg_config* c, int* validate_energy, char* describe,
                          size_t cap);
int oo_ref_cavity_config_load(const char* path, oo_cavity_config* c, int* validate_reference,
                              char* describe, size_t cap);
/* "name|version|compiler_id|compiler_version|profile|strict" of get_build_info. */
int oo_ref_build_description(char* buf, size_t cap);
int oo_ref_cavity_checkpoint_write(const char* path, const oo_cavity_config* c, int validate_reference,
                                   const oo_state* s);
/* meta[0..2] = checksum, build hash, configuration hash. */
int oo_ref_cavity_checkpoint_load(const char* path, const oo_cavity_config* c, int validate_reference,
                                  oo_state* s, unsigned long long meta[3]);
/* finalize_lid_driven_cavity_result on a state: extrema (u max, u min, v max,
 * v min), the four envelope samples and errors, the worst error and pass. */
int oo_ref_cavity_finalize(const oo_cavity_config* c, int validate_reference, const oo_state* s,
                           double extrema[4], double samples[4], double errors[4], double* max_error,
                           int* pass);
int oo_ref_write_vtk(const char* path, const oo_grid* g, const oo_state* s);

#ifdef __cplusplus
}
#endif

#endif
