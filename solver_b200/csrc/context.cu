// C ABI (include/orchard_b200.h): contexts, state residency and the step
// driver.  One context owns one stream and every device buffer of its grid;
// each entry point validates its arguments with the reference's messages,
// enqueues the kernels and returns after the diagnostics are on the host.
#include "../../include/orchard_b200.h"
#include "kernels.hpp"

#include <cmath>
#include <cstring>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_last_error;

struct StatusError : std::runtime_error {
  of_status status;
  StatusError(of_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void fail(of_status s, const std::string& msg) { throw StatusError(s, msg); }

template <typename Fn>
of_status guarded(Fn&& fn) {
  try {
    fn();
    g_last_error.clear();
    return OF_OK;
  } catch(const StatusError& e) {
    g_last_error = e.what();
    return e.status;
  } catch(const ofb::CudaError& e) {
    g_last_error = e.what();
    return OF_CUDA_ERROR;
  } catch(const std::invalid_argument& e) {
    g_last_error = e.what();
    return OF_INVALID_ARGUMENT;
  } catch(const std::bad_alloc& e) {
    g_last_error = std::string("host allocation failed: ") + e.what();
    return OF_RUNTIME_ERROR;
  } catch(const std::exception& e) {
    g_last_error = e.what();
    return OF_RUNTIME_ERROR;
  }
}

}  // namespace

using ofb::Grid;
using ofb::Lay;
using ofb::PBC;
using ofb::VBC;

struct of_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Grid g{};
  VBC bc{};
  PBC pbc{};  // derived pressure-correction conditions
  Lay lay[4];  // cell, u, v, w
  int precision = OF_FP64;

  // resident state (TaylorGreenState / LidDrivenCavityState)
  double* vel[3] = {nullptr, nullptr, nullptr};
  double* adv_prev[3] = {nullptr, nullptr, nullptr};
  double* adv_cur[3] = {nullptr, nullptr, nullptr};
  double* p_total = nullptr;
  int has_prev = 0;
  bool state_clean = false;  // velocity ghosts already filled (BC idempotent)
  of_step_metrics metrics{};

  // scratch
  double* rhs[3] = {nullptr, nullptr, nullptr};
  double* adi_b[3] = {nullptr, nullptr, nullptr};
  double* corrected[3] = {nullptr, nullptr, nullptr};
  double* prhs = nullptr;       // padded pressure rhs
  double* phi = nullptr;        // padded pressure correction (operator API)

  ofb::RedBuf rb{};
  ofb::SolveScalars* sc = nullptr;       // device
  ofb::SolveScalars* sc_host = nullptr;  // pinned

  ofb::PoissonPlan* poisson = nullptr;
  int poisson_types[6] = {-1, -1, -1, -1, -1, -1};
  int poisson_precision = -1;
  ofb::AdiPlan* adi = nullptr;
  double adi_alpha = -1.0;
  size_t bytes = 0;

  ~of_ctx() {
    cudaSetDevice(device);
    if(stream) cudaStreamSynchronize(stream);
    for(int c = 0; c < 3; ++c) {
      cudaFree(vel[c]);
      cudaFree(adv_prev[c]);
      cudaFree(adv_cur[c]);
      cudaFree(rhs[c]);
      cudaFree(adi_b[c]);
      cudaFree(corrected[c]);
    }
    cudaFree(p_total);
    cudaFree(prhs);
    cudaFree(phi);
    cudaFree(rb.partials);
    cudaFree(rb.ticket);
    cudaFree(sc);
    if(sc_host) cudaFreeHost(sc_host);
    ofb::poisson_plan_destroy(poisson);
    ofb::adi_plan_destroy(adi);
    if(stream) cudaStreamDestroy(stream);
  }

  double* alloc(size_t n) {
    double* p = nullptr;
    OFB_CHECK(cudaMalloc(&p, n * sizeof(double)));
    OFB_CHECK(cudaMemsetAsync(p, 0, n * sizeof(double), stream));
    bytes += n * sizeof(double);
    return p;
  }

  size_t size(int loc) const { return lay[loc].size(); }

  void upload(double* dst, const double* src, int loc) {
    OFB_CHECK(cudaMemcpyAsync(dst, src, size(loc) * sizeof(double), cudaMemcpyHostToDevice, stream));
  }
  void download(double* dst, const double* src, int loc) {
    OFB_CHECK(cudaMemcpyAsync(dst, src, size(loc) * sizeof(double), cudaMemcpyDeviceToHost, stream));
  }
  void d2d(double* dst, const double* src, int loc) {
    OFB_CHECK(cudaMemcpyAsync(dst, src, size(loc) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  }
  void sync() { OFB_CHECK(cudaStreamSynchronize(stream)); }

  ofb::PoissonPlan* poisson_for(const PBC& p) {
    bool same = poisson != nullptr && poisson_precision == precision;
    for(int f = 0; f < 6 && same; ++f) same = poisson_types[f] == p.type[f];
    if(!same) {
      sync();
      ofb::poisson_plan_destroy(poisson);
      poisson = nullptr;
      poisson = ofb::poisson_plan_create(g, p, precision);
      for(int f = 0; f < 6; ++f) poisson_types[f] = p.type[f];
      poisson_precision = precision;
    }
    return poisson;
  }

  ofb::AdiPlan* adi_for(double alpha) {
    if(adi == nullptr || adi_alpha != alpha) {
      sync();
      ofb::adi_plan_destroy(adi);
      adi = nullptr;
      adi = ofb::adi_plan_create(g, bc, alpha);
      adi_alpha = alpha;
    }
    return adi;
  }
};

namespace {

void require_ctx(of_ctx* ctx) {
  if(ctx == nullptr) fail(OF_INVALID_ARGUMENT, "null context");
  OFB_CHECK(cudaSetDevice(ctx->device));
}

void require_ptr(const void* p, const char* what) {
  if(p == nullptr) fail(OF_INVALID_ARGUMENT, std::string(what) + " must not be null");
}

void check_pressure_pairing(const int* types, bool pressure) {
  const int periodic = pressure ? static_cast<int>(ofb::kPPeriodic) : static_cast<int>(ofb::kPeriodic);
  for(int a = 0; a < 3; ++a) {
    if((types[2 * a] == periodic) != (types[2 * a + 1] == periodic)) {
      fail(OF_INVALID_ARGUMENT, pressure ? "periodic pressure boundaries must be paired on both sides"
                                         : "periodic velocity boundaries must be paired on both sides");
    }
  }
}

// derive_pressure_correction_boundary_conditions (solver/projection.cpp:934-964)
PBC derive_pbc(const VBC& bc) {
  PBC p{};
  for(int f = 0; f < 6; ++f) {
    switch(bc.type[f]) {
      case ofb::kNoSlip:
      case ofb::kPrescribed:
      case ofb::kSymmetry:
        p.type[f] = ofb::kPNeumann;
        break;
      case ofb::kFixedPressure:
        p.type[f] = ofb::kPDirichlet;
        break;
      default:
        p.type[f] = ofb::kPPeriodic;
        break;
    }
    p.value[f] = 0.0;
    p.gradient[f] = 0.0;
  }
  check_pressure_pairing(p.type, true);
  return p;
}

PBC to_pbc(const of_pbc* in) {
  PBC p{};
  for(int f = 0; f < 6; ++f) {
    p.type[f] = in->faces[f].type;
    p.value[f] = in->faces[f].value;
    p.gradient[f] = in->faces[f].gradient;
    if(p.type[f] < 0 || p.type[f] > 2) fail(OF_INVALID_ARGUMENT, "unknown pressure boundary type");
  }
  return p;
}

void export_poisson(of_ctx* ctx, const ofb::SolveScalars& s, of_poisson_diag* d) {
  if(d == nullptr) return;
  d->iterations = s.iterations;
  d->initial_residual_l2 = s.r0;
  d->final_residual_l2 = s.iterations > 0 ? s.rnorm : s.r0;
  d->relative_residual = s.rel;
  d->removed_rhs_mean = s.removed_rhs_mean;
  d->multigrid_levels = ofb::poisson_levels(ctx->poisson);
  d->coarse_unknowns = ofb::poisson_coarse_unknowns(ctx->poisson);
  d->pre_smoothing_steps = 2;
  d->post_smoothing_steps = 2;
  d->converged = s.converged;
  d->zero_mean_enforced = s.zero_mean;
}

// The pressure solve of project_velocity / solve_pressure_poisson on the
// context's compact b (shift set) with initial guess x (shift set).
ofb::SolveScalars run_poisson(of_ctx* ctx, int max_iterations, double tolerance, double* history,
                              int history_cap) {
  ofb::poisson_solve(ctx->poisson, max_iterations, tolerance, ctx->sc, ctx->sc_host, ctx->rb,
                     ctx->stream, history, history_cap);
  return *ctx->sc_host;
}

// solve_predictor_adi on the context's rhs buffers; returns pointers to the
// three predicted components (rhs[] or adi_b[]).
void predictor_adi(of_ctx* ctx, double alpha, double* out[3], int* line_solves) {
  ofb::AdiPlan* plan = alpha != 0.0 ? ctx->adi_for(alpha) : nullptr;
  int lines = 0;
  for(int c = 0; c < 3; ++c) {
    double* a = ctx->rhs[c];
    double* b = ctx->adi_b[c];
    ofb::launch_component_bc(ctx->g, ctx->bc, c, a, ctx->stream);
    if(alpha == 0.0) {
      out[c] = a;
      continue;
    }
    for(int axis = 0; axis < 3; ++axis) {
      if(ofb::adi_axis_active(plan, c, axis)) {
        ofb::launch_adi_sweep(plan, c, axis, a, b, ctx->stream);
        lines += ofb::adi_line_count(plan, c, axis);
        std::swap(a, b);
      }
      ofb::launch_component_bc(ctx->g, ctx->bc, c, a, ctx->stream);
    }
    out[c] = a;
  }
  if(line_solves) *line_solves = lines;
}

}  // namespace

extern "C" {

int of_abi_version(void) { return OF_ABI_VERSION; }

const char* of_last_error(void) { return g_last_error.c_str(); }

of_status of_create(const of_grid* grid, const of_bc* bc, int device, of_ctx** out) {
  return guarded([&] {
    require_ptr(grid, "grid");
    require_ptr(bc, "boundary conditions");
    require_ptr(out, "output context pointer");
    *out = nullptr;
    // Grid constructor checks (core/grid.hpp:76-86)
    if(grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0)
      fail(OF_INVALID_ARGUMENT, "grid dimensions must be positive");
    if(grid->dx <= 0.0 || grid->dy <= 0.0 || grid->dz <= 0.0)
      fail(OF_INVALID_ARGUMENT, "grid spacing must be positive");
    const long long cells = static_cast<long long>(grid->nx + 3) * (grid->ny + 3) * (grid->nz + 3);
    if(cells >= (1LL << 31)) fail(OF_INVALID_ARGUMENT, "grid too large for 32-bit indexing");
    int ndev = 0;
    if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      fail(OF_CUDA_ERROR, "no CUDA device is available (the B200 path has no CPU fallback)");
    if(device < 0 || device >= ndev) fail(OF_INVALID_ARGUMENT, "CUDA device ordinal out of range");
    auto ctx = std::make_unique<of_ctx>();
    ctx->device = device;
    OFB_CHECK(cudaSetDevice(device));
    OFB_CHECK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->g = Grid{grid->nx, grid->ny, grid->nz, grid->dx, grid->dy, grid->dz};
    for(int f = 0; f < 6; ++f) {
      ctx->bc.type[f] = bc->faces[f].type;
      if(ctx->bc.type[f] < 0 || ctx->bc.type[f] > 4)
        fail(OF_INVALID_ARGUMENT, "unknown physical boundary type");
      for(int c = 0; c < 3; ++c) ctx->bc.vel[f][c] = bc->faces[f].velocity[c];
      ctx->bc.pressure[f] = bc->faces[f].pressure;
    }
    check_pressure_pairing(ctx->bc.type, false);
    ctx->pbc = derive_pbc(ctx->bc);
    for(int loc = 0; loc < 4; ++loc) ctx->lay[loc] = ofb::make_lay(ctx->g, loc);
    for(int c = 0; c < 3; ++c) {
      const size_t n = ctx->size(1 + c);
      ctx->vel[c] = ctx->alloc(n);
      ctx->adv_prev[c] = ctx->alloc(n);
      ctx->adv_cur[c] = ctx->alloc(n);
      ctx->rhs[c] = ctx->alloc(n);
      ctx->adi_b[c] = ctx->alloc(n);
      ctx->corrected[c] = ctx->alloc(n);
    }
    ctx->p_total = ctx->alloc(ctx->size(0));
    ctx->prhs = ctx->alloc(ctx->size(0));
    ctx->phi = ctx->alloc(ctx->size(0));
    OFB_CHECK(cudaMalloc(&ctx->rb.partials, sizeof(double) * ofb::kMaxRed * ofb::kMaxBlocks));
    OFB_CHECK(cudaMalloc(&ctx->rb.ticket, sizeof(unsigned int)));
    OFB_CHECK(cudaMemsetAsync(ctx->rb.ticket, 0, sizeof(unsigned int), ctx->stream));
    OFB_CHECK(cudaMalloc(&ctx->sc, sizeof(ofb::SolveScalars)));
    OFB_CHECK(cudaMemsetAsync(ctx->sc, 0, sizeof(ofb::SolveScalars), ctx->stream));
    OFB_CHECK(cudaMallocHost(&ctx->sc_host, sizeof(ofb::SolveScalars)));
    ctx->sync();
    *out = ctx.release();
  });
}

of_status of_destroy(of_ctx* ctx) {
  return guarded([&] { delete ctx; });
}

of_status of_set_precision(of_ctx* ctx, int precision) {
  return guarded([&] {
    require_ctx(ctx);
    if(precision != OF_FP64 && precision != OF_MIXED)
      fail(OF_INVALID_ARGUMENT, "precision must be OF_FP64 or OF_MIXED");
    ctx->precision = precision;
  });
}

of_status of_stream(of_ctx* ctx, void** stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(stream, "stream");
    *stream = static_cast<void*>(ctx->stream);
  });
}

of_status of_device_bytes(of_ctx* ctx, size_t* bytes) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(bytes, "bytes");
    *bytes = ctx->bytes + (ctx->poisson ? ofb::poisson_device_bytes(ctx->poisson) : 0) +
             sizeof(double) * ofb::kMaxRed * ofb::kMaxBlocks;
  });
}

of_status of_compute_advection_term(of_ctx* ctx, const double* u, const double* v,
                                    const double* w, double* au, double* av, double* aw) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(u, "u");
    require_ptr(v, "v");
    require_ptr(w, "w");
    require_ptr(au, "advection x");
    require_ptr(av, "advection y");
    require_ptr(aw, "advection z");
    const double* in[3] = {u, v, w};
    double* out[3] = {au, av, aw};
    for(int c = 0; c < 3; ++c) {
      ctx->upload(ctx->corrected[c], in[c], 1 + c);
      ctx->upload(ctx->adv_cur[c], out[c], 1 + c);
    }
    ofb::launch_advection(ctx->g, ctx->corrected[0], ctx->corrected[1], ctx->corrected[2],
                          ctx->adv_cur[0], ctx->adv_cur[1], ctx->adv_cur[2], ctx->stream);
    for(int c = 0; c < 3; ++c) ctx->download(out[c], ctx->adv_cur[c], 1 + c);
    ctx->sync();
    ctx->state_clean = false;
  });
}

of_status of_solve_predictor_adi(of_ctx* ctx, double alpha, const double* rhs_u,
                                 const double* rhs_v, const double* rhs_w, double* pred_u,
                                 double* pred_v, double* pred_w, int* line_solves) {
  return guarded([&] {
    require_ctx(ctx);
    if(alpha < 0.0) fail(OF_INVALID_ARGUMENT, "solve_predictor_adi expects a non-negative alpha");
    const double* in[3] = {rhs_u, rhs_v, rhs_w};
    double* outp[3] = {pred_u, pred_v, pred_w};
    for(int c = 0; c < 3; ++c) {
      require_ptr(in[c], "predictor rhs");
      require_ptr(outp[c], "predicted velocity");
      ctx->upload(ctx->rhs[c], in[c], 1 + c);
      ctx->d2d(ctx->adi_b[c], ctx->rhs[c], 1 + c);  // edge ghosts follow the input
    }
    double* res[3];
    predictor_adi(ctx, alpha, res, line_solves);
    for(int c = 0; c < 3; ++c) ctx->download(outp[c], res[c], 1 + c);
    ctx->sync();
  });
}

of_status of_solve_pressure_poisson(of_ctx* ctx, const of_pbc* pbc_in, int max_iterations,
                                    double tolerance, const double* rhs, double* pressure,
                                    of_poisson_diag* diag, double* history, int history_cap) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(pbc_in, "pressure boundary conditions");
    require_ptr(rhs, "rhs");
    require_ptr(pressure, "pressure");
    if(max_iterations <= 0) fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects iterations > 0");
    if(tolerance <= 0.0) fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects tolerance > 0");
    const PBC p = to_pbc(pbc_in);
    check_pressure_pairing(p.type, true);
    ofb::PoissonPlan* plan = ctx->poisson_for(p);
    int zm = 1;
    for(int f = 0; f < 6; ++f)
      if(p.type[f] == ofb::kPDirichlet) zm = 0;
    ctx->upload(ctx->prhs, rhs, 0);
    ctx->upload(ctx->phi, pressure, 0);
    ofb::launch_rhs_to_system(ctx->g, p, ctx->prhs, ofb::poisson_b(plan), ctx->sc, ctx->rb, ctx->stream);
    ofb::launch_pressure_to_compact(ctx->g, ctx->phi, ofb::poisson_x(plan), ctx->sc, zm, ctx->rb,
                                    ctx->stream);
    const ofb::SolveScalars s = run_poisson(ctx, max_iterations, tolerance, history, history_cap);
    ofb::launch_compact_to_pressure(ctx->g, ofb::poisson_x(plan), ctx->sc, ctx->phi, ctx->stream);
    ctx->download(pressure, ctx->phi, 0);
    ctx->sync();
    export_poisson(ctx, s, diag);
  });
}

of_status of_project_velocity(of_ctx* ctx, double dt, double density, int max_iterations,
                              double tolerance, const double* pred_u, const double* pred_v,
                              const double* pred_w, double* pressure_correction,
                              double* corr_u, double* corr_v, double* corr_w,
                              double* pressure_rhs, of_projection_diag* diag) {
  return guarded([&] {
    require_ctx(ctx);
    const double* in[3] = {pred_u, pred_v, pred_w};
    double* outp[3] = {corr_u, corr_v, corr_w};
    for(int c = 0; c < 3; ++c) {
      require_ptr(in[c], "predicted velocity");
      require_ptr(outp[c], "corrected velocity");
    }
    require_ptr(pressure_correction, "pressure correction");
    // build_pressure_rhs and solve_pressure_poisson argument checks, in the
    // order project_velocity reaches them (solver/projection.cpp:1053-1058,
    // linsolve/poisson_solver.cpp:682-687)
    if(dt <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects dt > 0");
    if(density <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects density > 0");
    if(max_iterations <= 0) fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects iterations > 0");
    if(tolerance <= 0.0) fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects tolerance > 0");
    ofb::PoissonPlan* plan = ctx->poisson_for(ctx->pbc);
    int zm = 1;
    for(int f = 0; f < 6; ++f)
      if(ctx->pbc.type[f] == ofb::kPDirichlet) zm = 0;
    for(int c = 0; c < 3; ++c) ctx->upload(ctx->rhs[c], in[c], 1 + c);
    ofb::launch_velocity_bc(ctx->g, ctx->bc, ctx->rhs[0], ctx->rhs[1], ctx->rhs[2], ctx->stream);
    ctx->upload(ctx->phi, pressure_correction, 0);
    if(pressure_rhs) ctx->upload(ctx->prhs, pressure_rhs, 0);
    ofb::launch_divergence_rhs(ctx->g, ctx->pbc, ctx->rhs[0], ctx->rhs[1], ctx->rhs[2],
                               density / dt, ctx->prhs, ofb::poisson_b(plan), ctx->sc, ctx->rb,
                               ctx->stream);
    ofb::launch_pressure_to_compact(ctx->g, ctx->phi, ofb::poisson_x(plan), ctx->sc, zm, ctx->rb,
                                    ctx->stream);
    ofb::SolveScalars s = run_poisson(ctx, max_iterations, tolerance, nullptr, 0);
    // correct_velocity: corrected = working (full copy), active faces updated, BC
    for(int c = 0; c < 3; ++c) ctx->d2d(ctx->corrected[c], ctx->rhs[c], 1 + c);
    ofb::launch_correct_velocity(ctx->g, ctx->pbc, ofb::poisson_x(plan), ctx->sc, ctx->rhs[0],
                                 ctx->rhs[1], ctx->rhs[2], -dt / density, ctx->corrected[0],
                                 ctx->corrected[1], ctx->corrected[2], nullptr, nullptr, nullptr,
                                 ctx->sc, ctx->rb, ctx->stream);
    ofb::launch_velocity_bc(ctx->g, ctx->bc, ctx->corrected[0], ctx->corrected[1],
                            ctx->corrected[2], ctx->stream);
    ofb::CellPassArgs cp{};
    cp.g = ctx->g;
    cp.u = ctx->corrected[0];
    cp.v = ctx->corrected[1];
    cp.w = ctx->corrected[2];
    cp.x = ofb::poisson_x(plan);
    cp.phi_padded = ctx->phi;
    ofb::launch_cell_pass(cp, ctx->sc, ctx->rb, ctx->stream);
    OFB_CHECK(cudaMemcpyAsync(ctx->sc_host, ctx->sc, sizeof(ofb::SolveScalars),
                              cudaMemcpyDeviceToHost, ctx->stream));
    for(int c = 0; c < 3; ++c) ctx->download(outp[c], ctx->corrected[c], 1 + c);
    ctx->download(pressure_correction, ctx->phi, 0);
    if(pressure_rhs) ctx->download(pressure_rhs, ctx->prhs, 0);
    ctx->sync();
    s = *ctx->sc_host;
    if(diag) {
      diag->rhs_l2 = s.rhs_l2;
      diag->divergence_l2_before = s.div_before_l2;
      diag->divergence_l2_after = s.div_after_l2;
      diag->pressure_mean = s.pressure_mean;
      export_poisson(ctx, s, &diag->pressure_solve);
    }
    ctx->state_clean = false;
  });
}

of_status of_state_upload(of_ctx* ctx, const double* u, const double* v, const double* w,
                          const double* adv_u, const double* adv_v, const double* adv_w,
                          const double* p_total, int has_previous_advection,
                          const of_step_metrics* metrics) {
  return guarded([&] {
    require_ctx(ctx);
    const double* vin[3] = {u, v, w};
    const double* ain[3] = {adv_u, adv_v, adv_w};
    for(int c = 0; c < 3; ++c) {
      require_ptr(vin[c], "velocity");
      require_ptr(ain[c], "previous advection");
      ctx->upload(ctx->vel[c], vin[c], 1 + c);
      ctx->upload(ctx->adv_prev[c], ain[c], 1 + c);
      ctx->upload(ctx->adv_cur[c], ain[c], 1 + c);
      // Edge and corner ghosts are never written by any kernel; every
      // velocity-shaped buffer carries the state's so that full-copy
      // semantics of the reference hold without per-step copies.
      ctx->d2d(ctx->rhs[c], ctx->vel[c], 1 + c);
      ctx->d2d(ctx->adi_b[c], ctx->vel[c], 1 + c);
      ctx->d2d(ctx->corrected[c], ctx->vel[c], 1 + c);
    }
    require_ptr(p_total, "total pressure");
    ctx->upload(ctx->p_total, p_total, 0);
    ctx->has_prev = has_previous_advection ? 1 : 0;
    ctx->metrics = metrics ? *metrics : of_step_metrics{};
    ctx->state_clean = false;
    ctx->sync();
  });
}

of_status of_state_download(of_ctx* ctx, double* u, double* v, double* w, double* adv_u,
                            double* adv_v, double* adv_w, double* p_total,
                            int* has_previous_advection, of_step_metrics* metrics) {
  return guarded([&] {
    require_ctx(ctx);
    double* vout[3] = {u, v, w};
    double* aout[3] = {adv_u, adv_v, adv_w};
    for(int c = 0; c < 3; ++c) {
      if(vout[c]) ctx->download(vout[c], ctx->vel[c], 1 + c);
      if(aout[c]) ctx->download(aout[c], ctx->adv_prev[c], 1 + c);
    }
    if(p_total) ctx->download(p_total, ctx->p_total, 0);
    ctx->sync();
    if(has_previous_advection) *has_previous_advection = ctx->has_prev;
    if(metrics) *metrics = ctx->metrics;
  });
}

of_status of_tg_init(of_ctx* ctx, double viscosity, double dt, int mode) {
  return guarded([&] {
    require_ctx(ctx);
    if(mode != 0 && mode != 1) fail(OF_INVALID_ARGUMENT, "Taylor-Green initial-state mode must be 0 or 1");
    for(int c = 0; c < 3; ++c) {
      OFB_CHECK(cudaMemsetAsync(ctx->vel[c], 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
      OFB_CHECK(cudaMemsetAsync(ctx->adv_prev[c], 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
      OFB_CHECK(cudaMemsetAsync(ctx->adv_cur[c], 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
      OFB_CHECK(cudaMemsetAsync(ctx->rhs[c], 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
      OFB_CHECK(cudaMemsetAsync(ctx->adi_b[c], 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
      OFB_CHECK(cudaMemsetAsync(ctx->corrected[c], 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
    }
    OFB_CHECK(cudaMemsetAsync(ctx->p_total, 0, ctx->size(0) * sizeof(double), ctx->stream));
    ofb::launch_tg_init(ctx->g, mode, ctx->vel[0], ctx->vel[1], ctx->vel[2], ctx->p_total, ctx->stream);
    // initial-state tail (solver/taylor_green.cpp:391-394)
    ofb::launch_velocity_bc(ctx->g, ctx->bc, ctx->vel[0], ctx->vel[1], ctx->vel[2], ctx->stream);
    ofb::launch_total_pressure_bc(ctx->g, ctx->bc, viscosity, ctx->vel[0], ctx->vel[1], ctx->vel[2],
                                  ctx->p_total, ctx->stream);
    ctx->has_prev = 0;
    ctx->metrics = of_step_metrics{};
    ctx->metrics.dt = dt;
    ctx->state_clean = true;
    ctx->sync();
  });
}

of_status of_run_steps(of_ctx* ctx, const of_step_params* prm, int steps, of_step_metrics* out) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(prm, "step parameters");
    if(steps < 0) fail(OF_INVALID_ARGUMENT, "run_taylor_green_steps expects a non-negative step count");
    if(prm->dt <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects dt > 0");
    if(prm->density <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects density > 0");
    if(prm->poisson_max_iterations <= 0)
      fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects iterations > 0");
    if(prm->poisson_tolerance <= 0.0)
      fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects tolerance > 0");
    const std::string name = prm->solver_name ? prm->solver_name : "Taylor-Green";
    const double dt = prm->dt;
    const double nu = prm->viscosity;
    const double alpha = 0.5 * nu * dt;
    ofb::PoissonPlan* plan = ctx->poisson_for(ctx->pbc);
    cudaStream_t s = ctx->stream;
    const Grid& g = ctx->g;
    for(int step = 0; step < steps; ++step) {
      // current = state.velocity with boundary conditions (solver/taylor_green.cpp:578-579)
      const double* cur[3] = {ctx->vel[0], ctx->vel[1], ctx->vel[2]};
      if(!ctx->state_clean) {
        for(int c = 0; c < 3; ++c) ctx->d2d(ctx->corrected[c], ctx->vel[c], 1 + c);
        ofb::launch_velocity_bc(g, ctx->bc, ctx->corrected[0], ctx->corrected[1], ctx->corrected[2], s);
        for(int c = 0; c < 3; ++c) cur[c] = ctx->corrected[c];
      }
      // assemble_predictor_rhs (fused)
      ofb::PredictorArgs pa{};
      pa.g = g;
      for(int c = 0; c < 3; ++c) {
        pa.cur[c] = cur[c];
        pa.prev[c] = ctx->adv_prev[c];
        pa.adv[c] = ctx->adv_cur[c];
        pa.rhs[c] = ctx->rhs[c];
      }
      pa.p = ctx->p_total;
      pa.nu = nu;
      pa.dt = dt;
      pa.alpha = alpha;
      pa.has_prev = ctx->has_prev;
      pa.variant = prm->correction_variant;
      ofb::launch_predictor_rhs(pa, s);
      // solve_predictor_adi
      double* pred[3];
      predictor_adi(ctx, alpha, pred, nullptr);
      // project_velocity with a zero initial pressure correction
      ofb::launch_divergence_rhs(g, ctx->pbc, pred[0], pred[1], pred[2], prm->density / dt, ctx->prhs,
                                 ofb::poisson_b(plan), ctx->sc, ctx->rb, s);
      // pressure_correction.fill(0.0) (solver/taylor_green.cpp:596): x = 0, mean 0
      OFB_CHECK(cudaMemsetAsync(ofb::poisson_x(plan), 0, sizeof(double) * g.nx * g.ny * g.nz, s));
      OFB_CHECK(cudaMemsetAsync(&ctx->sc->sx, 0, sizeof(double), s));
      const ofb::SolveScalars ps =
          run_poisson(ctx, prm->poisson_max_iterations, prm->poisson_tolerance, nullptr, 0);
      if(!ps.converged) {
        std::ostringstream m;
        m << name << " pressure solve did not converge at step " << (step + 1)
          << " (iterations=" << ps.iterations << ", relative_residual=" << ps.rel
          << ", tolerance=" << prm->poisson_tolerance << ")";
        fail(OF_NOT_CONVERGED, m.str());
      }
      ofb::launch_correct_velocity(g, ctx->pbc, ofb::poisson_x(plan), ctx->sc, pred[0], pred[1],
                                   pred[2], -dt / prm->density, ctx->corrected[0], ctx->corrected[1],
                                   ctx->corrected[2], ctx->vel[0], ctx->vel[1], ctx->vel[2], ctx->sc,
                                   ctx->rb, s);
      ofb::launch_velocity_bc(g, ctx->bc, ctx->corrected[0], ctx->corrected[1], ctx->corrected[2], s);
      ofb::CellPassArgs cp{};
      cp.g = g;
      cp.u = ctx->corrected[0];
      cp.v = ctx->corrected[1];
      cp.w = ctx->corrected[2];
      cp.x = ofb::poisson_x(plan);
      cp.p_total = ctx->p_total;
      cp.rhs_padded = ctx->prhs;
      cp.p_rhs_scale = -0.5 * nu * dt;
      cp.dt = dt;
      ofb::launch_cell_pass(cp, ctx->sc, ctx->rb, s);
      ofb::launch_total_pressure_bc(g, ctx->bc, nu, ctx->corrected[0], ctx->corrected[1],
                                    ctx->corrected[2], ctx->p_total, s);
      OFB_CHECK(cudaMemcpyAsync(ctx->sc_host, ctx->sc, sizeof(ofb::SolveScalars),
                                cudaMemcpyDeviceToHost, s));
      ctx->sync();
      const ofb::SolveScalars d = *ctx->sc_host;
      if(d.nonfinite) fail(OF_NONFINITE, name + " solve produced a non-finite state");
      for(int c = 0; c < 3; ++c) {
        std::swap(ctx->vel[c], ctx->corrected[c]);
        std::swap(ctx->adv_prev[c], ctx->adv_cur[c]);
      }
      ctx->has_prev = 1;
      ctx->state_clean = true;
      of_step_metrics& m = ctx->metrics;
      m.step += 1;
      m.time += dt;
      m.dt = dt;
      m.max_cfl = d.max_cfl;
      m.max_velocity_change = d.max_dv;
      m.divergence_l2 = d.div_after_l2;
      if(prm->track_max_divergence)
        m.max_divergence_l2 = m.max_divergence_l2 < d.div_after_l2 ? d.div_after_l2 : m.max_divergence_l2;
      m.pressure_iterations = d.iterations;
      m.pressure_relative_residual = d.rel;
    }
    if(out) *out = ctx->metrics;
  });
}

// Allocation-free pressure rhs for callers whose device memory is owned by
// their own allocator and who cannot let a call allocate or synchronise the
// device inside their step loop (ofb::launch_pressure_rhs_noalloc, noalloc.cu).
of_status of_pressure_rhs_noalloc(const of_grid* grid, double dt, double density,
                                  const double* u, const double* v, const double* w,
                                  double* pressure_rhs, double* norms, void* stream) {
  return guarded([&] {
    require_ptr(grid, "grid");
    require_ptr(u, "velocity u");
    require_ptr(v, "velocity v");
    require_ptr(w, "velocity w");
    require_ptr(pressure_rhs, "pressure rhs");
    if(grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0)
      fail(OF_INVALID_ARGUMENT, "grid dimensions must be positive");
    if(grid->dx <= 0.0 || grid->dy <= 0.0 || grid->dz <= 0.0)
      fail(OF_INVALID_ARGUMENT, "grid spacing must be positive");
    const long long cells = static_cast<long long>(grid->nx + 3) * (grid->ny + 3) * (grid->nz + 3);
    if(cells >= (1LL << 31)) fail(OF_INVALID_ARGUMENT, "grid too large for 32-bit indexing");
    // the scratch holds the block partials of one launch; a launch has
    // ceil(nx/32) * ceil(ny/8) blocks per k plane at least
    const long long plane_blocks = static_cast<long long>((grid->nx + ofb::kTX - 1) / ofb::kTX) *
                                   ((grid->ny + ofb::kTY - 1) / ofb::kTY);
    if(plane_blocks > ofb::noalloc_max_plane_blocks()) {
      std::ostringstream m;
      m << "of_pressure_rhs_noalloc: a " << grid->nx << " x " << grid->ny
        << " k plane needs " << plane_blocks << " reduction blocks of 32 x 8 cells; the static "
        << "scratch holds " << ofb::noalloc_max_plane_blocks() << " (at most "
        << ofb::noalloc_max_plane_blocks() * ofb::kTX * ofb::kTY << " cells per k plane)";
      fail(OF_INVALID_ARGUMENT, m.str());
    }
    if(dt <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects dt > 0");
    if(density <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects density > 0");
    const Grid g{grid->nx, grid->ny, grid->nz, grid->dx, grid->dy, grid->dz};
    ofb::launch_pressure_rhs_noalloc(g, u, v, w, density / dt, pressure_rhs, ofb::noalloc_scratch(),
                                     norms, static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"
