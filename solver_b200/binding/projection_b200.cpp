// B200 bodies of the reference's projection-step seams, for the reference tree.
//
// A maintainer adds this file to Orchard Flow's build in place of the CPU
// bodies of four free functions and links the B200 library
// (-L<this repo>/solver_b200 -lorchard_b200):
//
//   solver::compute_advection_term            solver/momentum_terms.hpp:36-38
//   solver::solve_predictor_adi               solver/projection.hpp:49-52
//   solver::project_velocity                  solver/projection.hpp:65-70
//   solver::linsolve::solve_pressure_poisson  linsolve/poisson_solver.hpp:34-37
//
// Every other function of the reference (case drivers, BC fills, operators,
// checkpoint, CLI) is unchanged and calls these four as before.  Field storage
// is the same on both sides (StructuredField::data(), padded, i + sx*(j + sy*k)),
// so arrays cross the C ABI without repacking.  Errors come back as the
// reference's exception types with its messages (of_last_error holds the
// reference's wording).
//
// Contexts: one per (grid, velocity boundary set) and host thread, created on
// CUDA device 0 on first use and cached (at most kCachedContexts per thread,
// least recently used first out).  The advection term and the standalone
// pressure solve take no velocity boundary set; they use a context with all
// faces periodic (their ABI calls do not read it).
//
// Differences from the CPU bodies, by design: compute_advection_term
// supports the TVD / van Leer scheme (the reference's default and the only
// scheme its case drivers use) and rejects the others; project_velocity
// leaves pressure_solve.residual_history empty (solve_pressure_poisson fills
// it).  Set ORCHARD_B200_BINDING_VERBOSE=1 to have each new context reported
// on stderr.
#include "linsolve/poisson_solver.hpp"
#include "solver/momentum_terms.hpp"
#include "solver/projection.hpp"

#include "orchard_b200.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <list>
#include <stdexcept>
#include <string>
#include <vector>

namespace solver {
namespace b200_binding {

constexpr std::size_t kCachedContexts = 4;

void throw_on(const of_status status) {
  if(status == OF_OK) {
    return;
  }
  if(status == OF_INVALID_ARGUMENT) {
    throw std::invalid_argument(of_last_error());
  }
  throw std::runtime_error(of_last_error());
}

of_grid to_abi(const Grid& grid) {
  of_grid out{};
  out.nx = grid.nx;
  out.ny = grid.ny;
  out.nz = grid.nz;
  out.dx = grid.dx;
  out.dy = grid.dy;
  out.dz = grid.dz;
  return out;
}

of_bc to_abi(const BoundaryConditionSet& in) {
  of_bc out{};
  for(int face = 0; face < 6; ++face) {
    out.faces[face].type = static_cast<int>(in.faces[face].type);
    for(int c = 0; c < 3; ++c) {
      out.faces[face].velocity[c] = in.faces[face].velocity[c];
    }
    out.faces[face].pressure = in.faces[face].pressure;
    out.faces[face].pressure_gradient = in.faces[face].pressure_gradient;
  }
  return out;
}

of_pbc to_abi(const PressureBoundarySet& in) {
  of_pbc out{};
  for(int face = 0; face < 6; ++face) {
    out.faces[face].type = static_cast<int>(in.faces[face].type);
    out.faces[face].value = in.faces[face].value;
    out.faces[face].gradient = in.faces[face].gradient;
  }
  return out;
}

of_bc all_periodic() {
  of_bc out{};
  for(int face = 0; face < 6; ++face) {
    out.faces[face].type = OF_PERIODIC;
  }
  return out;
}

struct CachedContext {
  of_grid grid{};
  of_bc bc{};
  of_ctx* ctx = nullptr;
};

struct ContextCache {
  std::list<CachedContext> entries;  // most recently used first
  ~ContextCache() {
    for(CachedContext& e : entries) {
      of_destroy(e.ctx);
    }
  }
};

of_ctx* context_for(const Grid& grid, const of_bc& bc) {
  thread_local ContextCache cache;
  const of_grid g = to_abi(grid);
  for(auto it = cache.entries.begin(); it != cache.entries.end(); ++it) {
    if(std::memcmp(&it->grid, &g, sizeof g) == 0 && std::memcmp(&it->bc, &bc, sizeof bc) == 0) {
      cache.entries.splice(cache.entries.begin(), cache.entries, it);
      return cache.entries.front().ctx;
    }
  }
  CachedContext e;
  e.grid = g;
  e.bc = bc;
  throw_on(of_create(&g, &bc, /*device=*/0, &e.ctx));
  if(const char* v = std::getenv("ORCHARD_B200_BINDING_VERBOSE"); v != nullptr && v[0] == '1') {
    std::fprintf(stderr, "b200 binding: context on CUDA device 0 for grid %dx%dx%d\n", g.nx, g.ny,
                 g.nz);
  }
  cache.entries.push_front(e);
  if(cache.entries.size() > kCachedContexts) {
    of_destroy(cache.entries.back().ctx);
    cache.entries.pop_back();
  }
  return e.ctx;
}

PoissonSolveDiagnostics from_abi(const of_poisson_diag& d) {
  PoissonSolveDiagnostics out;
  out.iterations = d.iterations;
  out.initial_residual_l2 = d.initial_residual_l2;
  out.final_residual_l2 = d.final_residual_l2;
  out.relative_residual = d.relative_residual;
  out.removed_rhs_mean = d.removed_rhs_mean;
  out.multigrid_levels = d.multigrid_levels;
  out.coarse_unknowns = d.coarse_unknowns;
  out.pre_smoothing_steps = d.pre_smoothing_steps;
  out.post_smoothing_steps = d.post_smoothing_steps;
  out.converged = d.converged != 0;
  out.zero_mean_enforced = d.zero_mean_enforced != 0;
  return out;
}

}  // namespace b200_binding

void compute_advection_term(const VelocityField& velocity,
                            const AdvectionOptions& options,
                            VelocityField& advection) {
  if(options.scheme != AdvectionScheme::tvd || options.limiter != FluxLimiter::van_leer) {
    throw std::invalid_argument(
        "compute_advection_term: the B200 path implements the tvd scheme with the van_leer limiter");
  }
  const Grid& grid = velocity.x.layout().grid();
  of_ctx* ctx = b200_binding::context_for(grid, b200_binding::all_periodic());
  b200_binding::throw_on(of_compute_advection_term(ctx, velocity.x.data(), velocity.y.data(),
                                                   velocity.z.data(), advection.x.data(),
                                                   advection.y.data(), advection.z.data()));
}

HelmholtzDiagnostics solve_predictor_adi(const VelocityField& rhs,
                                         const double alpha,
                                         const BoundaryConditionSet& boundary_conditions,
                                         VelocityField& predicted_velocity) {
  const Grid& grid = rhs.x.layout().grid();
  of_ctx* ctx = b200_binding::context_for(grid, b200_binding::to_abi(boundary_conditions));
  HelmholtzDiagnostics diagnostics;
  b200_binding::throw_on(of_solve_predictor_adi(
      ctx, alpha, rhs.x.data(), rhs.y.data(), rhs.z.data(), predicted_velocity.x.data(),
      predicted_velocity.y.data(), predicted_velocity.z.data(), &diagnostics.line_solves));
  return diagnostics;
}

ProjectionDiagnostics project_velocity(const VelocityField& predicted_velocity,
                                       const BoundaryConditionSet& boundary_conditions,
                                       const ProjectionOptions& options,
                                       PressureField& pressure_correction,
                                       VelocityField& corrected_velocity,
                                       ScalarField* pressure_rhs) {
  const Grid& grid = pressure_correction.layout().grid();
  of_ctx* ctx = b200_binding::context_for(grid, b200_binding::to_abi(boundary_conditions));
  of_projection_diag d{};
  b200_binding::throw_on(of_project_velocity(
      ctx, options.dt, options.density, options.poisson_max_iterations, options.poisson_tolerance,
      predicted_velocity.x.data(), predicted_velocity.y.data(), predicted_velocity.z.data(),
      pressure_correction.data(), corrected_velocity.x.data(), corrected_velocity.y.data(),
      corrected_velocity.z.data(), pressure_rhs != nullptr ? pressure_rhs->data() : nullptr, &d));
  ProjectionDiagnostics out;
  out.rhs_l2 = d.rhs_l2;
  out.divergence_l2_before = d.divergence_l2_before;
  out.divergence_l2_after = d.divergence_l2_after;
  out.pressure_mean = d.pressure_mean;
  out.pressure_solve = b200_binding::from_abi(d.pressure_solve);
  return out;
}

namespace linsolve {

PoissonSolveDiagnostics solve_pressure_poisson(const ScalarField& rhs,
                                               const PressureBoundarySet& boundary_conditions,
                                               const ProjectionOptions& options,
                                               PressureField& pressure) {
  const Grid& grid = rhs.layout().grid();
  of_ctx* ctx = b200_binding::context_for(grid, b200_binding::all_periodic());
  const of_pbc pbc = b200_binding::to_abi(boundary_conditions);
  of_poisson_diag d{};
  std::vector<double> history(
      static_cast<std::size_t>(options.poisson_max_iterations > 0 ? options.poisson_max_iterations : 0) + 1);
  b200_binding::throw_on(of_solve_pressure_poisson(
      ctx, &pbc, options.poisson_max_iterations, options.poisson_tolerance, rhs.data(),
      pressure.data(), &d, history.data(), static_cast<int>(history.size())));
  PoissonSolveDiagnostics out = b200_binding::from_abi(d);
  history.resize(std::min(history.size(), static_cast<std::size_t>(d.iterations) + 1));
  out.residual_history = std::move(history);
  return out;
}

}  // namespace linsolve
}  // namespace solver
