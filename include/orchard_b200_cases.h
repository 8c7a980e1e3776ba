/*
 * orchard_b200_cases.h -- the callers of the projection step: the
 * Taylor-Green and lid-driven-cavity case drivers, their config files and
 * validation, the SLVCHKP1 checkpoint and the legacy-VTK export.
 *
 * These mirror the reference's drivers and I/O (solver/taylor_green.*,
 * solver/lid_driven_cavity.*, io/checkpoint.*, io/vtk_export.*) on top of the
 * step ABI of orchard_b200.h: a case context is an of_ctx created on the
 * case's grid and boundary conditions, whose resident state is the case state
 * (TaylorGreenState / LidDrivenCavityState).  Error texts are the
 * reference's exception messages; file formats are byte-compatible.
 */
#ifndef ORCHARD_B200_CASES_H
#define ORCHARD_B200_CASES_H

#include <stdint.h>

#include "orchard_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* AdvectionScheme / FluxLimiter (solver/momentum_terms.hpp:9-22).  The step
 * implements the TVD / van Leer scheme, the only one the config files reach. */
enum { OF_ADVECTION_TVD = 0, OF_ADVECTION_UPWIND = 1, OF_ADVECTION_CENTRAL = 2 };
enum { OF_LIMITER_VAN_LEER = 0 };
/* ExecutionBackend (solver/taylor_green.hpp:10-13); only "cpu" (the step on
 * this library's device) is accepted by the drivers. */
enum { OF_BACKEND_CPU = 0, OF_BACKEND_METAL = 1 };

/* ---- Taylor-Green -------------------------------------------------------- */

/* TaylorGreenConfig (solver/taylor_green.hpp:18-30). */
typedef struct {
  int nx, ny, nz;
  double viscosity;
  double cfl_limit;
  double final_time;
  int poisson_max_iterations;
  double poisson_tolerance;
  int validate_energy;
  int backend;
  int advection_scheme;
  int advection_limiter;
} of_tg_config;

/* TaylorGreenResult (solver/taylor_green.hpp:66-76) with its validation. */
typedef struct {
  of_step_metrics final_step;
  double initial_kinetic_energy;
  double final_kinetic_energy;
  char reference_dataset[64];     /* empty when validation is off */
  double normalized_energy_error;
  double velocity_relative_l2_error;
  double exact_kinetic_energy;
  int pass;
  char accelerator_name[64];      /* the CUDA device that ran the steps */
  double elapsed_seconds;         /* wall time of the steps run by of_tg_run */
} of_tg_result;

/* default_taylor_green_config / load_taylor_green_config
 * (solver/taylor_green.cpp:421-481): `key = value` lines, '#' comments. */
of_status of_tg_config_default(of_tg_config* config);
of_status of_tg_config_load(const char* path, of_tg_config* config);
/* describe (solver/taylor_green.cpp:483-495) into buf (NUL-terminated;
 * *len, optional, receives the full length). */
of_status of_tg_config_describe(const of_tg_config* config, char* buf, size_t cap, size_t* len);
/* make_taylor_green_grid, make_taylor_green_boundary_conditions and
 * taylor_green_dt (solver/taylor_green.cpp:497-525); *steps = the step count
 * that reaches final_time.  Any output pointer may be NULL. */
of_status of_tg_case(const of_tg_config* config, of_grid* grid, of_bc* bc, double* dt, int* steps);
/* A context on the case grid holding initialize_taylor_green_state
 * (solver/taylor_green.cpp:527-538). */
of_status of_tg_create(const of_tg_config* config, int device, of_ctx** out);
/* run_taylor_green_steps (solver/taylor_green.cpp:540-634). */
of_status of_tg_run_steps(of_ctx* ctx, const of_tg_config* config, int steps,
                          of_step_metrics* metrics);
/* finalize_taylor_green_result (solver/taylor_green.cpp:636-651). */
of_status of_tg_finalize(of_ctx* ctx, const of_tg_config* config, of_tg_result* result);
/* run_taylor_green (solver/taylor_green.cpp:667-735) on the CPU backend:
 * re-initialises the resident state, runs ceil(final_time / dt) steps and
 * finalizes; the resident state is the final state afterwards. */
of_status of_tg_run(of_ctx* ctx, const of_tg_config* config, of_tg_result* result);

/* ---- lid-driven cavity ---------------------------------------------------- */

/* LidDrivenCavityConfig (solver/lid_driven_cavity.hpp:12-25). */
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
  int validate_reference;
  int advection_scheme;
  int advection_limiter;
} of_cavity_config;

/* CenterlineSampleKind (solver/lid_driven_cavity.hpp:51-54) */
enum { OF_U_VERTICAL = 0, OF_V_HORIZONTAL = 1 };

/* LidDrivenCavityValidationPoint (solver/lid_driven_cavity.hpp:71-80). */
typedef struct {
  char label[32];
  int line;
  double coordinate;
  double reference_value;
  double reference_lower_bound;
  double reference_upper_bound;
  double sample_value;
  double relative_error;
} of_cavity_point;

/* LidDrivenCavityResult (solver/lid_driven_cavity.hpp:95-102) without the
 * profiles themselves (of_cavity_centerlines returns those). */
typedef struct {
  of_step_metrics final_step;
  double u_vertical_max, u_vertical_min;
  double v_horizontal_max, v_horizontal_min;
  char reference_dataset[64];     /* empty when validation is off */
  of_cavity_point points[4];
  double max_relative_error;
  double divergence_l2;
  int pass;
  double elapsed_seconds;         /* wall time of the steps run by of_cavity_run */
} of_cavity_result;

of_status of_cavity_config_default(of_cavity_config* config);
/* load_lid_driven_cavity_config (solver/lid_driven_cavity.cpp:296-336). */
of_status of_cavity_config_load(const char* path, of_cavity_config* config);
/* describe (solver/lid_driven_cavity.cpp:338-349). */
of_status of_cavity_config_describe(const of_cavity_config* config, char* buf, size_t cap,
                                    size_t* len);
/* make_lid_driven_cavity_grid / _boundary_conditions / _viscosity / _dt
 * (solver/lid_driven_cavity.cpp:362-388).  Output pointers may be NULL. */
of_status of_cavity_case(const of_cavity_config* config, of_grid* grid, of_bc* bc,
                         double* viscosity, double* dt);
/* A context holding initialize_lid_driven_cavity_state
 * (solver/lid_driven_cavity.cpp:390-408). */
of_status of_cavity_create(const of_cavity_config* config, int device, of_ctx** out);
/* run_lid_driven_cavity_steps (solver/lid_driven_cavity.cpp:625-630). */
of_status of_cavity_run_steps(of_ctx* ctx, const of_cavity_config* config, int steps,
                              of_step_metrics* metrics);
/* The solver_cavity loop (tools/lid_driven_cavity_main.cpp:65-74): one step
 * at a time until max_steps or, after min_steps, until max_velocity_change
 * <= steady_tolerance.  The step count is the resident state's. */
of_status of_cavity_run_to_steady(of_ctx* ctx, const of_cavity_config* config,
                                  of_step_metrics* metrics);
/* finalize_lid_driven_cavity_result (solver/lid_driven_cavity.cpp:632-656)
 * including the Re 100 envelope gate (validate_lid_driven_cavity_re100,
 * solver/lid_driven_cavity.cpp:445-480). */
of_status of_cavity_finalize(of_ctx* ctx, const of_cavity_config* config, of_cavity_result* result);
/* run_lid_driven_cavity (solver/lid_driven_cavity.cpp:658-662): re-initialises
 * the resident state, steps to steady state or max_steps and finalizes. */
of_status of_cavity_run(of_ctx* ctx, const of_cavity_config* config, of_cavity_result* result);
/* The two centreline profiles of finalize (coordinates and values; ny and nx
 * entries, ghosts excluded).  Any pointer may be NULL. */
of_status of_cavity_centerlines(of_ctx* ctx, double* u_coordinate, double* u_value,
                                double* v_coordinate, double* v_value);

/* ---- SLVCHKP1 checkpoint (io/checkpoint.cpp) ------------------------------ */

/* CheckpointMetadata (io/checkpoint.hpp:10-17) */
typedef struct {
  uint32_t format_version;
  uint32_t scalar_bytes;
  uint64_t checksum;
  uint64_t build_hash;
  uint64_t configuration_hash;
} of_checkpoint_meta;

/* FNV-1a 64 (io/checkpoint.cpp:29-36), the hash of both checkpoint hashes. */
uint64_t of_fnv1a64(const void* data, size_t size);
/* build_hash (io/checkpoint.cpp:42-49) of a BuildInfo: FNV-1a of
 * "name|version|compiler_id|compiler_version|profile|fast-math or strict". */
uint64_t of_build_hash(const char* project_name, const char* project_version,
                       const char* compiler_id, const char* compiler_version,
                       const char* build_profile, int fast_math_enabled);
/* This library's own build hash (project "Orchard Flow B200"). */
uint64_t of_library_build_hash(void);

/* write_lid_driven_cavity_checkpoint (io/checkpoint.cpp:313-349) of the
 * context's resident state.  build_hash 0 means of_library_build_hash(). */
of_status of_cavity_checkpoint_write(of_ctx* ctx, const char* path, const of_cavity_config* config,
                                     uint64_t build_hash);
/* load_lid_driven_cavity_checkpoint (io/checkpoint.cpp:351-461) into the
 * context's resident state.  The file is validated completely (framing,
 * checksum, metadata, config, grid and field extents, in the reference's
 * order and with its messages) before anything is uploaded.  build_hash 0
 * means of_library_build_hash().  meta may be NULL. */
of_status of_cavity_checkpoint_load(of_ctx* ctx, const char* path, const of_cavity_config* config,
                                    uint64_t build_hash, of_checkpoint_meta* meta);

/* The same two on host arrays (padded storage of the cavity grid), with no
 * device involved. */
of_status of_cavity_checkpoint_write_host(const char* path, const of_cavity_config* config,
                                          uint64_t build_hash, const double* u, const double* v,
                                          const double* w, const double* adv_u,
                                          const double* adv_v, const double* adv_w,
                                          const double* p_total, int has_previous_advection,
                                          const of_step_metrics* metrics);
of_status of_cavity_checkpoint_load_host(const char* path, const of_cavity_config* config,
                                         uint64_t build_hash, double* u, double* v, double* w,
                                         double* adv_u, double* adv_v, double* adv_w,
                                         double* p_total, int* has_previous_advection,
                                         of_step_metrics* metrics, of_checkpoint_meta* meta);

/* The Taylor-Green state under the same framing: sections META, TGCF (the
 * TaylorGreenConfig fields in declaration order, u32 / f64 little-endian),
 * GRID, VELX..PRST as the cavity's, and MDIV (max_divergence_l2, f64).  The
 * configuration hash is FNV-1a of describe(config). */
of_status of_tg_checkpoint_write(of_ctx* ctx, const char* path, const of_tg_config* config,
                                 uint64_t build_hash);
of_status of_tg_checkpoint_load(of_ctx* ctx, const char* path, const of_tg_config* config,
                                uint64_t build_hash, of_checkpoint_meta* meta);

/* ---- legacy VTK (io/vtk_export.cpp:18-73) -------------------------------- */

/* write_mac_fields_vtk of the resident velocity (cell-averaged) and total
 * pressure: ASCII STRUCTURED_POINTS, values in the reference's stream format. */
of_status of_write_vtk(of_ctx* ctx, const char* path);

#ifdef __cplusplus
}
#endif

#endif /* ORCHARD_B200_CASES_H */
