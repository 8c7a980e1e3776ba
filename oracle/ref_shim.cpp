// Adapter from the oracle interface (orchard_oracle.h) to the reference's own
// C++ functions, compiled in place from the reference sources by
// oracle/Makefile into oracle/_ref/liborchard_ref.so.  TEST INFRASTRUCTURE
// ONLY: it pins the plain-C restatement (orchard_oracle.c) and generates the
// golden fixtures; the product never links it.

#include "orchard_oracle.h"

#include "core/fields.hpp"
#include "core/runtime.hpp"
#include "io/checkpoint.hpp"
#include "io/vtk_export.hpp"
#include "linsolve/poisson_solver.hpp"
#include "operators/discrete_operators.hpp"
#include "solver/lid_driven_cavity.hpp"
#include "solver/momentum_terms.hpp"
#include "solver/projection.hpp"
#include "solver/taylor_green.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

namespace {

thread_local std::string g_error;

solver::Grid make_grid(const oo_grid* g) {
  return solver::Grid{g->nx, g->ny, g->nz, g->dx, g->dy, g->dz, 1};
}

void load(solver::StructuredField& f, const double* src) {
  std::memcpy(f.data(), src, f.size() * sizeof(double));
}

void store(const solver::StructuredField& f, double* dst) {
  std::memcpy(dst, f.data(), f.size() * sizeof(double));
}

void load_velocity(solver::VelocityField& f, const double* u, const double* v, const double* w) {
  load(f.x, u);
  load(f.y, v);
  load(f.z, w);
}

void store_velocity(const solver::VelocityField& f, double* u, double* v, double* w) {
  store(f.x, u);
  store(f.y, v);
  store(f.z, w);
}

solver::BoundaryConditionSet make_bc(const oo_bc* bc) {
  solver::BoundaryConditionSet out;
  for(int f = 0; f < 6; ++f) {
    out.faces[f].type = static_cast<solver::PhysicalBoundaryType>(bc->faces[f].type);
    for(int c = 0; c < 3; ++c) {
      out.faces[f].velocity[c] = bc->faces[f].velocity[c];
    }
    out.faces[f].pressure = bc->faces[f].pressure;
    out.faces[f].pressure_gradient = bc->faces[f].pressure_gradient;
  }
  return out;
}

void export_bc(const solver::BoundaryConditionSet& in, oo_bc* bc) {
  for(int f = 0; f < 6; ++f) {
    bc->faces[f].type = static_cast<int>(in.faces[f].type);
    for(int c = 0; c < 3; ++c) {
      bc->faces[f].velocity[c] = in.faces[f].velocity[c];
    }
    bc->faces[f].pressure = in.faces[f].pressure;
    bc->faces[f].pressure_gradient = in.faces[f].pressure_gradient;
  }
}

solver::PressureBoundarySet make_pbc(const oo_pbc* pbc) {
  solver::PressureBoundarySet out;
  for(int f = 0; f < 6; ++f) {
    out.faces[f].type = static_cast<solver::PressureBoundaryType>(pbc->faces[f].type);
    out.faces[f].value = pbc->faces[f].value;
    out.faces[f].gradient = pbc->faces[f].gradient;
  }
  return out;
}

void export_poisson(const solver::PoissonSolveDiagnostics& d, oo_poisson_diag* out) {
  out->iterations = d.iterations;
  out->initial_residual_l2 = d.initial_residual_l2;
  out->final_residual_l2 = d.final_residual_l2;
  out->relative_residual = d.relative_residual;
  out->removed_rhs_mean = d.removed_rhs_mean;
  out->multigrid_levels = d.multigrid_levels;
  out->coarse_unknowns = d.coarse_unknowns;
  out->pre_smoothing_steps = d.pre_smoothing_steps;
  out->post_smoothing_steps = d.post_smoothing_steps;
  out->converged = d.converged ? 1 : 0;
  out->zero_mean_enforced = d.zero_mean_enforced ? 1 : 0;
}

solver::TaylorGreenConfig make_tg(const oo_tg_config* c) {
  solver::TaylorGreenConfig config = solver::default_taylor_green_config();
  config.nx = c->nx;
  config.ny = c->ny;
  config.nz = c->nz;
  config.viscosity = c->viscosity;
  config.cfl_limit = c->cfl_limit;
  config.final_time = c->final_time;
  config.poisson_max_iterations = c->poisson_max_iterations;
  config.poisson_tolerance = c->poisson_tolerance;
  config.validate_energy = false;
  return config;
}

solver::LidDrivenCavityConfig make_cavity(const oo_cavity_config* c) {
  solver::LidDrivenCavityConfig config = solver::default_lid_driven_cavity_config();
  config.nx = c->nx;
  config.ny = c->ny;
  config.reynolds = c->reynolds;
  config.lid_velocity = c->lid_velocity;
  config.cfl_limit = c->cfl_limit;
  config.max_steps = c->max_steps;
  config.min_steps = c->min_steps;
  config.steady_tolerance = c->steady_tolerance;
  config.poisson_max_iterations = c->poisson_max_iterations;
  config.poisson_tolerance = c->poisson_tolerance;
  config.validate_reference = false;
  return config;
}

template <typename State>
void load_state(State& st, const oo_state* s) {
  load_velocity(st.velocity, s->u, s->v, s->w);
  load_velocity(st.advection_previous, s->adv_u, s->adv_v, s->adv_w);
  load(st.pressure_total, s->p);
  st.has_previous_advection = s->has_previous_advection != 0;
}

template <typename State>
void store_state(const State& st, oo_state* s) {
  store_velocity(st.velocity, s->u, s->v, s->w);
  store_velocity(st.advection_previous, s->adv_u, s->adv_v, s->adv_w);
  store(st.pressure_total, s->p);
  s->has_previous_advection = st.has_previous_advection ? 1 : 0;
}

void load_metrics(solver::TaylorGreenStepMetrics& m, const oo_step_metrics& s) {
  m.step = s.step;
  m.time = s.time;
  m.dt = s.dt;
  m.max_cfl = s.max_cfl;
  m.max_velocity_change = s.max_velocity_change;
  m.divergence_l2 = s.divergence_l2;
  m.max_divergence_l2 = s.max_divergence_l2;
  m.pressure_iterations = s.pressure_iterations;
  m.pressure_relative_residual = s.pressure_relative_residual;
}

void store_metrics(const solver::TaylorGreenStepMetrics& m, oo_step_metrics& s) {
  s.step = m.step;
  s.time = m.time;
  s.dt = m.dt;
  s.max_cfl = m.max_cfl;
  s.max_velocity_change = m.max_velocity_change;
  s.divergence_l2 = m.divergence_l2;
  s.max_divergence_l2 = m.max_divergence_l2;
  s.pressure_iterations = m.pressure_iterations;
  s.pressure_relative_residual = m.pressure_relative_residual;
}

void load_metrics(solver::SimulationStepMetrics& m, const oo_step_metrics& s) {
  m.step = s.step;
  m.time = s.time;
  m.dt = s.dt;
  m.max_cfl = s.max_cfl;
  m.max_velocity_change = s.max_velocity_change;
  m.divergence_l2 = s.divergence_l2;
  m.pressure_iterations = s.pressure_iterations;
  m.pressure_relative_residual = s.pressure_relative_residual;
}

void store_metrics(const solver::SimulationStepMetrics& m, oo_step_metrics& s) {
  s.step = m.step;
  s.time = m.time;
  s.dt = m.dt;
  s.max_cfl = m.max_cfl;
  s.max_velocity_change = m.max_velocity_change;
  s.divergence_l2 = m.divergence_l2;
  s.max_divergence_l2 = 0.0;
  s.pressure_iterations = m.pressure_iterations;
  s.pressure_relative_residual = m.pressure_relative_residual;
}

template <typename Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    return 0;
  } catch(const std::invalid_argument& e) {
    g_error = e.what();
    return 1;
  } catch(const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}

}  // namespace

extern "C" {

const char* oo_last_error(void) {
  return g_error.c_str();
}

int oo_advection(const oo_grid* g, const double* u, const double* v, const double* w,
                 double* au, double* av, double* aw) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField vel(grid), out(grid);
    load_velocity(vel, u, v, w);
    load_velocity(out, au, av, aw);
    solver::compute_advection_term(vel, solver::AdvectionOptions{}, out);
    store_velocity(out, au, av, aw);
  });
}

int oo_diffusion(const oo_grid* g, double nu, const double* u, const double* v, const double* w,
                 double* du, double* dv, double* dw) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField vel(grid), out(grid);
    load_velocity(vel, u, v, w);
    load_velocity(out, du, dv, dw);
    solver::compute_diffusion_term(vel, nu, out);
    store_velocity(out, du, dv, dw);
  });
}

int oo_apply_velocity_bc(const oo_grid* g, const oo_bc* bc, double* u, double* v, double* w) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField vel(grid);
    load_velocity(vel, u, v, w);
    solver::apply_velocity_boundary_conditions(make_bc(bc), vel);
    store_velocity(vel, u, v, w);
  });
}

int oo_apply_pressure_bc(const oo_grid* g, const oo_pbc* pbc, double* p) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::PressureField pf(grid);
    load(pf, p);
    solver::apply_pressure_boundary_conditions(make_pbc(pbc), pf);
    store(pf, p);
  });
}

int oo_derive_pressure_correction_bc(const oo_bc* bc, oo_pbc* out) {
  return guarded([&] {
    const solver::PressureBoundarySet mapped =
        solver::derive_pressure_correction_boundary_conditions(make_bc(bc));
    for(int f = 0; f < 6; ++f) {
      out->faces[f].type = static_cast<int>(mapped.faces[f].type);
      out->faces[f].value = mapped.faces[f].value;
      out->faces[f].gradient = mapped.faces[f].gradient;
    }
  });
}

int oo_apply_total_pressure_bc(const oo_grid* g, const oo_bc* bc, const double* su,
                               const double* sv, const double* sw, double* p) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField src(grid);
    load_velocity(src, su, sv, sw);
    solver::PressureField pf(grid);
    load(pf, p);
    solver::apply_total_pressure_boundary_conditions(make_bc(bc), src, pf);
    store(pf, p);
  });
}

int oo_gradient(const oo_grid* g, const double* p, double* gu, double* gv, double* gw) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::PressureField pf(grid);
    load(pf, p);
    solver::VelocityField out(grid);
    load_velocity(out, gu, gv, gw);
    solver::operators::compute_gradient(pf, out);
    store_velocity(out, gu, gv, gw);
  });
}

int oo_divergence(const oo_grid* g, const double* u, const double* v, const double* w,
                  double* div) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField vel(grid);
    load_velocity(vel, u, v, w);
    solver::ScalarField out(grid);
    load(out, div);
    solver::operators::compute_divergence(vel, out);
    store(out, div);
  });
}

int oo_predictor_adi(const oo_grid* g, const oo_bc* bc, double alpha, const double* ru,
                     const double* rv, const double* rw, double* pu, double* pv, double* pw,
                     int* line_solves) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField rhs(grid), out(grid);
    load_velocity(rhs, ru, rv, rw);
    load_velocity(out, pu, pv, pw);
    const solver::HelmholtzDiagnostics d = solver::solve_predictor_adi(rhs, alpha, make_bc(bc), out);
    store_velocity(out, pu, pv, pw);
    if(line_solves != nullptr) {
      *line_solves = d.line_solves;
    }
  });
}

int oo_poisson_solve(const oo_grid* g, const oo_pbc* pbc, int max_iterations, double tolerance,
                     const double* rhs, double* pressure, oo_poisson_diag* diag, double* hist,
                     int hist_cap) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::ScalarField r(grid);
    load(r, rhs);
    solver::PressureField p(grid);
    load(p, pressure);
    solver::ProjectionOptions options{};
    options.poisson_max_iterations = max_iterations;
    options.poisson_tolerance = tolerance;
    const solver::PoissonSolveDiagnostics d =
        solver::linsolve::solve_pressure_poisson(r, make_pbc(pbc), options, p);
    store(p, pressure);
    if(diag != nullptr) {
      export_poisson(d, diag);
    }
    if(hist != nullptr) {
      for(int i = 0; i < hist_cap && i < static_cast<int>(d.residual_history.size()); ++i) {
        hist[i] = d.residual_history[static_cast<std::size_t>(i)];
      }
    }
  });
}

int oo_project_velocity(const oo_grid* g, const oo_bc* bc, double dt, double density,
                        int max_iterations, double tolerance, const double* pu,
                        const double* pv, const double* pw, double* phi, double* cu,
                        double* cv, double* cw, double* rhs_out, oo_projection_diag* diag) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField predicted(grid), corrected(grid);
    load_velocity(predicted, pu, pv, pw);
    load_velocity(corrected, cu, cv, cw);
    solver::PressureField p(grid);
    load(p, phi);
    solver::ScalarField rhs(grid);
    if(rhs_out != nullptr) {
      load(rhs, rhs_out);
    }
    const solver::ProjectionOptions options{
        .dt = dt,
        .density = density,
        .poisson_max_iterations = max_iterations,
        .poisson_tolerance = tolerance,
    };
    const solver::ProjectionDiagnostics d = solver::project_velocity(
        predicted, make_bc(bc), options, p, corrected, rhs_out != nullptr ? &rhs : nullptr);
    store(p, phi);
    store_velocity(corrected, cu, cv, cw);
    if(rhs_out != nullptr) {
      store(rhs, rhs_out);
    }
    if(diag != nullptr) {
      diag->rhs_l2 = d.rhs_l2;
      diag->divergence_l2_before = d.divergence_l2_before;
      diag->divergence_l2_after = d.divergence_l2_after;
      diag->pressure_mean = d.pressure_mean;
      export_poisson(d.pressure_solve, &diag->pressure_solve);
    }
  });
}

int oo_tg_grid(const oo_tg_config* c, oo_grid* g) {
  return guarded([&] {
    const solver::Grid grid = solver::make_taylor_green_grid(make_tg(c));
    *g = oo_grid{grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz};
  });
}

double oo_tg_dt(const oo_tg_config* c) {
  double dt = 0.0;
  guarded([&] { dt = solver::taylor_green_dt(make_tg(c)); });
  return dt;
}

int oo_tg_bc(const oo_tg_config* c, oo_bc* bc) {
  return guarded([&] { export_bc(solver::make_taylor_green_boundary_conditions(make_tg(c)), bc); });
}

int oo_tg_init(const oo_tg_config* c, int mode, oo_state* s) {
  return guarded([&] {
    const solver::TaylorGreenConfig config = make_tg(c);
    if(mode != 0) {
      throw std::invalid_argument("the reference only provides its own initial state (mode 0)");
    }
    const solver::TaylorGreenState st = solver::initialize_taylor_green_state(config);
    store_state(st, s);
    store_metrics(st.metrics, s->metrics);
  });
}

int oo_tg_init_tail(const oo_tg_config* c, oo_state* s) {
  return guarded([&] {
    // Same three calls as the reference's initial-state tail
    // (solver/taylor_green.cpp:391-394), on caller-filled fields.
    const solver::TaylorGreenConfig config = make_tg(c);
    const solver::Grid grid = solver::make_taylor_green_grid(config);
    const solver::BoundaryConditionSet bc = solver::make_taylor_green_boundary_conditions(config);
    solver::VelocityField vel(grid);
    load_velocity(vel, s->u, s->v, s->w);
    solver::PressureField p(grid);
    load(p, s->p);
    solver::apply_velocity_boundary_conditions(bc, vel);
    solver::VelocityField diffusion(grid);
    solver::compute_diffusion_term(vel, config.viscosity, diffusion);
    solver::apply_total_pressure_boundary_conditions(bc, diffusion, p);
    store_velocity(vel, s->u, s->v, s->w);
    store(p, s->p);
  });
}

int oo_tg_steps(const oo_tg_config* c, int steps, oo_state* s) {
  return guarded([&] {
    const solver::TaylorGreenConfig config = make_tg(c);
    solver::TaylorGreenState st(solver::make_taylor_green_grid(config));
    load_state(st, s);
    load_metrics(st.metrics, s->metrics);
    solver::run_taylor_green_steps(config, steps, st);
    store_state(st, s);
    store_metrics(st.metrics, s->metrics);
  });
}

int oo_tg_validate(const oo_tg_config* c, int mode, const double* u, const double* v,
                   const double* w, double time, oo_tg_validation* out) {
  return guarded([&] {
    if(mode != 0) {
      throw std::invalid_argument("the reference validates its own initial state only (mode 0)");
    }
    solver::TaylorGreenConfig config = make_tg(c);
    config.validate_energy = true;
    solver::TaylorGreenState st(solver::make_taylor_green_grid(config));
    load_velocity(st.velocity, u, v, w);
    st.metrics.time = time;
    const solver::TaylorGreenResult r = solver::finalize_taylor_green_result(config, st);
    out->kinetic_energy = r.final_kinetic_energy;
    out->exact_kinetic_energy = r.validation.exact_kinetic_energy;
    out->normalized_energy_error = r.validation.normalized_energy_error;
    out->velocity_relative_l2_error = r.validation.velocity_relative_l2_error;
  });
}

int oo_cavity_grid(const oo_cavity_config* c, oo_grid* g) {
  return guarded([&] {
    const solver::Grid grid = solver::make_lid_driven_cavity_grid(make_cavity(c));
    *g = oo_grid{grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz};
  });
}

double oo_cavity_dt(const oo_cavity_config* c) {
  double dt = 0.0;
  guarded([&] { dt = solver::lid_driven_cavity_dt(make_cavity(c)); });
  return dt;
}

int oo_cavity_bc(const oo_cavity_config* c, oo_bc* bc) {
  return guarded(
      [&] { export_bc(solver::make_lid_driven_cavity_boundary_conditions(make_cavity(c)), bc); });
}

int oo_cavity_init(const oo_cavity_config* c, oo_state* s) {
  return guarded([&] {
    const solver::LidDrivenCavityState st = solver::initialize_lid_driven_cavity_state(make_cavity(c));
    store_state(st, s);
    store_metrics(st.metrics, s->metrics);
  });
}

int oo_cavity_steps(const oo_cavity_config* c, int steps, oo_state* s) {
  return guarded([&] {
    const solver::LidDrivenCavityConfig config = make_cavity(c);
    solver::LidDrivenCavityState st(solver::make_lid_driven_cavity_grid(config));
    load_state(st, s);
    load_metrics(st.metrics, s->metrics);
    solver::run_lid_driven_cavity_steps(config, steps, st);
    store_state(st, s);
    store_metrics(st.metrics, s->metrics);
  });
}

}  // extern "C"

// ---- reference build only: drivers and I/O around the step ----------------

namespace {

void copy_text(char* dst, size_t cap, const std::string& text) {
  if(dst == nullptr || cap == 0) return;
  const size_t n = std::min(cap - 1, text.size());
  std::memcpy(dst, text.data(), n);
  dst[n] = '\0';
}

solver::LidDrivenCavityConfig make_cavity_full(const oo_cavity_config* c, int validate_reference) {
  solver::LidDrivenCavityConfig config = make_cavity(c);
  config.validate_reference = validate_reference != 0;
  return config;
}

}  // namespace

extern "C" {

int oo_ref_tg_config_load(const char* path, oo_tg_config* c, int* validate_energy, char* describe,
                          size_t cap) {
  return guarded([&] {
    const solver::TaylorGreenConfig config = solver::load_taylor_green_config(path);
    *c = oo_tg_config{config.nx, config.ny, config.nz, config.viscosity, config.cfl_limit,
                      config.final_time, config.poisson_max_iterations, config.poisson_tolerance};
    if(validate_energy) *validate_energy = config.validate_energy ? 1 : 0;
    copy_text(describe, cap, solver::describe(config));
  });
}

int oo_ref_cavity_config_load(const char* path, oo_cavity_config* c, int* validate_reference,
                              char* describe, size_t cap) {
  return guarded([&] {
    const solver::LidDrivenCavityConfig config = solver::load_lid_driven_cavity_config(path);
    *c = oo_cavity_config{config.nx, config.ny, config.reynolds, config.lid_velocity, config.cfl_limit,
                          config.max_steps, config.min_steps, config.steady_tolerance,
                          config.poisson_max_iterations, config.poisson_tolerance};
    if(validate_reference) *validate_reference = config.validate_reference ? 1 : 0;
    copy_text(describe, cap, solver::describe(config));
  });
}

int oo_ref_build_description(char* buf, size_t cap) {
  return guarded([&] {
    const solver::BuildInfo b = solver::get_build_info();
    copy_text(buf, cap,
              b.project_name + "|" + b.project_version + "|" + b.compiler_id + "|" + b.compiler_version +
                  "|" + b.build_profile + "|" + (b.fast_math_enabled ? "fast-math" : "strict"));
  });
}

int oo_ref_cavity_checkpoint_write(const char* path, const oo_cavity_config* c, int validate_reference,
                                   const oo_state* s) {
  return guarded([&] {
    const solver::LidDrivenCavityConfig config = make_cavity_full(c, validate_reference);
    solver::LidDrivenCavityState st(solver::make_lid_driven_cavity_grid(config));
    load_state(st, s);
    load_metrics(st.metrics, s->metrics);
    solver::io::write_lid_driven_cavity_checkpoint(path, config, st);
  });
}

int oo_ref_cavity_checkpoint_load(const char* path, const oo_cavity_config* c, int validate_reference,
                                  oo_state* s, unsigned long long meta[3]) {
  return guarded([&] {
    const solver::LidDrivenCavityConfig config = make_cavity_full(c, validate_reference);
    const solver::io::LidDrivenCavityCheckpoint ck = solver::io::load_lid_driven_cavity_checkpoint(path, config);
    store_state(ck.state, s);
    store_metrics(ck.state.metrics, s->metrics);
    meta[0] = ck.metadata.checksum;
    meta[1] = ck.metadata.build_hash;
    meta[2] = ck.metadata.configuration_hash;
  });
}

int oo_ref_cavity_finalize(const oo_cavity_config* c, int validate_reference, const oo_state* s,
                           double extrema[4], double samples[4], double errors[4], double* max_error,
                           int* pass) {
  return guarded([&] {
    const solver::LidDrivenCavityConfig config = make_cavity_full(c, validate_reference);
    solver::LidDrivenCavityState st(solver::make_lid_driven_cavity_grid(config));
    load_state(st, s);
    load_metrics(st.metrics, s->metrics);
    const solver::LidDrivenCavityResult r = solver::finalize_lid_driven_cavity_result(config, st);
    extrema[0] = r.extrema.u_vertical_max;
    extrema[1] = r.extrema.u_vertical_min;
    extrema[2] = r.extrema.v_horizontal_max;
    extrema[3] = r.extrema.v_horizontal_min;
    for(int q = 0; q < 4; ++q) {
      samples[q] = r.validation.points[q].sample_value;
      errors[q] = r.validation.points[q].relative_error;
    }
    *max_error = r.validation.max_relative_error;
    *pass = r.validation.pass ? 1 : 0;
  });
}

int oo_ref_write_vtk(const char* path, const oo_grid* g, const oo_state* s) {
  return guarded([&] {
    const solver::Grid grid = make_grid(g);
    solver::VelocityField velocity(grid);
    solver::PressureField pressure(grid);
    load_velocity(velocity, s->u, s->v, s->w);
    load(pressure, s->p);
    solver::io::write_mac_fields_vtk(path, velocity, pressure);
  });
}

}  // extern "C"
