// C ABI (include/orchard_b200.h): contexts, state residency and the step
// driver.  One context owns one stream and every device buffer of its grid;
// each entry point validates its arguments with the reference's messages,
// enqueues the kernels and returns after the diagnostics are on the host.
#include "../../include/orchard_b200.h"
#include "kernels.hpp"

#include <algorithm>
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
  } catch(const ofb::TimeoutError& e) {
    g_last_error = e.what();
    return OF_TIMEOUT;
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

namespace ofb {
// Lets the case layer (cases.cpp) report through of_last_error().
void set_last_error(const std::string& message) { g_last_error = message; }
}  // namespace ofb

using ofb::Grid;
using ofb::Lay;
using ofb::PBC;
using ofb::VBC;

namespace {

// Device buffers of the tangent-linear and adjoint runs, allocated on first
// use and kept with the context.
struct SavedState {
  double* vel[3] = {nullptr, nullptr, nullptr};
  double* adv_prev[3] = {nullptr, nullptr, nullptr};
  double* p = nullptr;
  int has_prev = 0;
  bool clean = false;
};

// What a work set serves: the tangent-linear run, the adjoint with a
// checkpoint every `every` steps, or the adjoint with a binomial schedule
// (lean: no tangent buffers, the working state and the recomputed
// intermediates share the context's scratch, `slots` saved states).
enum AdjKind { kAdjTangent = 0, kAdjSegments = 1, kAdjBinomial = 2 };

struct AdjWork {
  std::vector<double*> owned;
  size_t bytes = 0;
  int steps = 0, every = 0, kind = -1, snapshots = 0;
  bool auto_snapshots = false;  // kAdjBinomial: snapshots sized to the free memory
  // tangent-linear state and the base velocity it is linearised about
  double *t_vel[3] = {}, *t_adv_prev[3] = {}, *t_adv_cur[3] = {}, *t_corr[3] = {}, *t_p = nullptr,
         *base_cur[3] = {};
  // adjoint variables
  double *lam_vel[3] = {}, *lam_corr[3] = {}, *lam_pred[3] = {}, *lam_b[3] = {}, *lam_cur[3] = {},
         *lam_prev[3] = {}, *lam_advtot[3] = {}, *target[3] = {}, *out[3] = {};
  double *lam_p = nullptr, *lam_phi = nullptr, *lam_q = nullptr;
  // recomputed intermediates of the step being differentiated
  double *y[3][3] = {}, *rc_adv[3] = {}, *rc_corr[3] = {};
  // working state of a recomputation
  double *w_vel[3] = {}, *w_adv_prev[3] = {}, *w_adv_cur[3] = {}, *w_corr[3] = {}, *w_p = nullptr;
  std::vector<SavedState> ckpt, seg, slots;
  std::vector<double*> phi;  // per step: compact pressure correction + its shift (may be empty)
  double* acc = nullptr;  // [0] loss, [1] d/dnu (direct), [2] sum mu.D y of the sweeps
  ~AdjWork() {
    for(double* p : owned) cudaFree(p);
  }
  double* alloc(size_t n, cudaStream_t s) {
    double* p = nullptr;
    OFB_CHECK(cudaMalloc(&p, n * sizeof(double)));
    OFB_CHECK(cudaMemsetAsync(p, 0, n * sizeof(double), s));
    owned.push_back(p);
    bytes += n * sizeof(double);
    return p;
  }
};

}  // namespace

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
  double* diag = nullptr;       // diagnostics reductions (4 doubles)
  cudaStream_t side = nullptr;  // of_step_host: download of the AB2 history
  cudaEvent_t adv_ready = nullptr;

  ofb::RedBuf rb{};
  ofb::SolveScalars* sc = nullptr;       // device
  ofb::SolveScalars* sc_host = nullptr;  // pinned

  ofb::PoissonPlan* poisson = nullptr;
  int poisson_types[6] = {-1, -1, -1, -1, -1, -1};
  int poisson_precision = -1;
  ofb::AdiPlan* adi = nullptr;
  double adi_alpha = -1.0;
  size_t bytes = 0;
  AdjWork* adj = nullptr;

  ~of_ctx() {
    cudaSetDevice(device);
    if(stream) cudaStreamSynchronize(stream);
    delete adj;
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
    cudaFree(diag);
    cudaFree(rb.partials);
    cudaFree(rb.ticket);
    cudaFree(sc);
    if(sc_host) cudaFreeHost(sc_host);
    ofb::poisson_plan_destroy(poisson);
    ofb::adi_plan_destroy(adi);
    if(side) {
      cudaStreamSynchronize(side);
      cudaStreamDestroy(side);
    }
    if(adv_ready) cudaEventDestroy(adv_ready);
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
// three predicted components (rhs[] or adi_b[]).  With sweep_out, sweep
// (component, axis) writes into sweep_out[component][axis] instead of the
// ping-pong buffers, so every sweep's output survives the call (the adjoint
// needs them for the viscosity derivative).
void predictor_adi(of_ctx* ctx, double alpha, double* out[3], int* line_solves,
                   double* const (*sweep_out)[3] = nullptr) {
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
        if(sweep_out != nullptr) {
          ofb::launch_adi_sweep(plan, c, axis, a, sweep_out[c][axis], ctx->stream);
          a = sweep_out[c][axis];
        } else {
          ofb::launch_adi_sweep(plan, c, axis, a, b, ctx->stream);
          std::swap(a, b);
        }
        lines += ofb::adi_line_count(plan, c, axis);
      }
      ofb::launch_component_bc(ctx->g, ctx->bc, c, a, ctx->stream);
    }
    out[c] = a;
  }
  if(line_solves) *line_solves = lines;
}

// A time-step state: velocity, AB2 advection history, total pressure, and the
// velocity buffer the step writes before the buffers are exchanged.  The
// context's resident state is one; the tangent-linear run keeps another.
struct StepState {
  double* vel[3];
  double* adv_prev[3];
  double* adv_cur[3];
  double* p;
  double* corrected[3];
  int has_prev;
  bool clean;  // velocity ghosts already filled
};

StepState resident_state(of_ctx* ctx) {
  StepState st{};
  for(int c = 0; c < 3; ++c) {
    st.vel[c] = ctx->vel[c];
    st.adv_prev[c] = ctx->adv_prev[c];
    st.adv_cur[c] = ctx->adv_cur[c];
    st.corrected[c] = ctx->corrected[c];
  }
  st.p = ctx->p_total;
  st.has_prev = ctx->has_prev;
  st.clean = ctx->state_clean;
  return st;
}

void set_resident_state(of_ctx* ctx, const StepState& st) {
  for(int c = 0; c < 3; ++c) {
    ctx->vel[c] = st.vel[c];
    ctx->adv_prev[c] = st.adv_prev[c];
    ctx->adv_cur[c] = st.adv_cur[c];
    ctx->corrected[c] = st.corrected[c];
  }
  ctx->p_total = st.p;
  ctx->has_prev = st.has_prev;
  ctx->state_clean = st.clean;
}

// Options of one step for the adjoint machinery.
struct StepHooks {
  // tangent-linear step: the advection is linearised about these velocities
  // (the base trajectory's current velocity) and applied to the state's
  const double* const* lin_base = nullptr;
  // when set, every ADI sweep output is kept (predictor_adi's sweep_out)
  double* const (*sweep_out)[3] = nullptr;
  // stop after the pressure rhs (ctx->prhs) is formed: no solve, no update
  bool stop_after_rhs = false;
  // pressure-solve result of this step: when phi_store is set the solution
  // (compact x and its mean shift) is copied there after the solve; when
  // phi_load is set the solve is skipped and the stored result used instead
  // (a recomputed step then reproduces the original bit for bit)
  double* phi_store = nullptr;
  const double* phi_load = nullptr;
  // when set, this step's advection term (the next step's AB2 history) is
  // copied to these host arrays on `side` as soon as the predictor has
  // formed it, overlapping the rest of the step
  double* const* adv_host = nullptr;
  cudaStream_t side = nullptr;
  cudaEvent_t adv_ready = nullptr;
};

// One projection step on `st` (the loop body of run_taylor_green_steps,
// solver/taylor_green.cpp:577-633, and of advance_lid_driven_cavity_impl,
// solver/lid_driven_cavity.cpp:562-623).  Returns the step's diagnostics.
ofb::SolveScalars forward_step(of_ctx* ctx, const of_step_params* prm, const std::string& name,
                               int step_no, StepState& st, const StepHooks* hk = nullptr) {
  const double dt = prm->dt;
  const double nu = prm->viscosity;
  const double alpha = 0.5 * nu * dt;
  ofb::PoissonPlan* plan = ctx->poisson_for(ctx->pbc);
  cudaStream_t s = ctx->stream;
  const Grid& g = ctx->g;
  // current = state.velocity with boundary conditions (solver/taylor_green.cpp:578-579)
  const double* cur[3] = {st.vel[0], st.vel[1], st.vel[2]};
  if(!st.clean) {
    for(int c = 0; c < 3; ++c) ctx->d2d(st.corrected[c], st.vel[c], 1 + c);
    ofb::launch_velocity_bc(g, ctx->bc, st.corrected[0], st.corrected[1], st.corrected[2], s);
    for(int c = 0; c < 3; ++c) cur[c] = st.corrected[c];
  }
  // assemble_predictor_rhs (fused)
  ofb::PredictorArgs pa{};
  pa.g = g;
  for(int c = 0; c < 3; ++c) {
    pa.cur[c] = cur[c];
    pa.prev[c] = st.adv_prev[c];
    pa.adv[c] = st.adv_cur[c];
    pa.rhs[c] = ctx->rhs[c];
  }
  pa.p = st.p;
  pa.nu = nu;
  pa.dt = dt;
  pa.alpha = alpha;
  pa.has_prev = st.has_prev;
  pa.variant = prm->correction_variant;
  if(hk != nullptr && hk->lin_base != nullptr) {
    ofb::launch_advection_jvp(g, hk->lin_base, cur, st.adv_cur, s);
    ofb::launch_predictor_rest(pa, s);
  } else {
    ofb::launch_predictor_rhs(pa, s);
  }
  if(hk != nullptr && hk->adv_host != nullptr) {
    OFB_CHECK(cudaEventRecord(hk->adv_ready, s));
    OFB_CHECK(cudaStreamWaitEvent(hk->side, hk->adv_ready, 0));
    for(int c = 0; c < 3; ++c)
      OFB_CHECK(cudaMemcpyAsync(hk->adv_host[c], st.adv_cur[c], ctx->size(1 + c) * sizeof(double),
                                cudaMemcpyDeviceToHost, hk->side));
  }
  // solve_predictor_adi
  double* pred[3];
  predictor_adi(ctx, alpha, pred, nullptr, hk != nullptr ? hk->sweep_out : nullptr);
  // project_velocity with a zero initial pressure correction
  ofb::launch_divergence_rhs(g, ctx->pbc, pred[0], pred[1], pred[2], prm->density / dt, ctx->prhs,
                             ofb::poisson_b(plan), ctx->sc, ctx->rb, s);
  if(hk != nullptr && hk->stop_after_rhs) return ofb::SolveScalars{};
  const size_t ncell = static_cast<size_t>(g.nx) * g.ny * g.nz;
  if(hk != nullptr && hk->phi_load != nullptr) {
    OFB_CHECK(cudaMemcpyAsync(ofb::poisson_x(plan), hk->phi_load, sizeof(double) * ncell,
                              cudaMemcpyDeviceToDevice, s));
    OFB_CHECK(cudaMemcpyAsync(&ctx->sc->sx, hk->phi_load + ncell, sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
  } else {
    // pressure_correction.fill(0.0) (solver/taylor_green.cpp:596): x = 0, mean 0
    OFB_CHECK(cudaMemsetAsync(ofb::poisson_x(plan), 0, sizeof(double) * ncell, s));
    OFB_CHECK(cudaMemsetAsync(&ctx->sc->sx, 0, sizeof(double), s));
    const ofb::SolveScalars ps =
        run_poisson(ctx, prm->poisson_max_iterations, prm->poisson_tolerance, nullptr, 0);
    if(!ps.converged) {
      std::ostringstream m;
      m << name << " pressure solve did not converge at step " << step_no
        << " (iterations=" << ps.iterations << ", relative_residual=" << ps.rel
        << ", tolerance=" << prm->poisson_tolerance << ")";
      fail(OF_NOT_CONVERGED, m.str());
    }
    if(hk != nullptr && hk->phi_store != nullptr) {
      OFB_CHECK(cudaMemcpyAsync(hk->phi_store, ofb::poisson_x(plan), sizeof(double) * ncell,
                                cudaMemcpyDeviceToDevice, s));
      OFB_CHECK(cudaMemcpyAsync(hk->phi_store + ncell, &ctx->sc->sx, sizeof(double),
                                cudaMemcpyDeviceToDevice, s));
    }
  }
  ofb::launch_correct_velocity(g, ctx->pbc, ofb::poisson_x(plan), ctx->sc, pred[0], pred[1],
                               pred[2], -dt / prm->density, st.corrected[0], st.corrected[1],
                               st.corrected[2], st.vel[0], st.vel[1], st.vel[2], ctx->sc,
                               ctx->rb, s);
  ofb::launch_velocity_bc(g, ctx->bc, st.corrected[0], st.corrected[1], st.corrected[2], s);
  ofb::CellPassArgs cp{};
  cp.g = g;
  cp.u = st.corrected[0];
  cp.v = st.corrected[1];
  cp.w = st.corrected[2];
  cp.x = ofb::poisson_x(plan);
  cp.p_total = st.p;
  cp.rhs_padded = ctx->prhs;
  cp.p_rhs_scale = -0.5 * nu * dt;
  cp.dt = dt;
  ofb::launch_cell_pass(cp, ctx->sc, ctx->rb, s);
  ofb::launch_total_pressure_bc(g, ctx->bc, nu, st.corrected[0], st.corrected[1],
                                st.corrected[2], st.p, s);
  OFB_CHECK(cudaMemcpyAsync(ctx->sc_host, ctx->sc, sizeof(ofb::SolveScalars),
                            cudaMemcpyDeviceToHost, s));
  ctx->sync();
  const ofb::SolveScalars d = *ctx->sc_host;
  if(d.nonfinite) fail(OF_NONFINITE, name + " solve produced a non-finite state");
  for(int c = 0; c < 3; ++c) {
    std::swap(st.vel[c], st.corrected[c]);
    std::swap(st.adv_prev[c], st.adv_cur[c]);
  }
  st.has_prev = 1;
  st.clean = true;
  return d;
}

// ---------------------------------------------------------------------------
// Tangent-linear and adjoint runs (periodic grids, Taylor-Green predictor).
// ---------------------------------------------------------------------------

size_t g_cells(of_ctx* ctx) { return static_cast<size_t>(ctx->g.nx) * ctx->g.ny * ctx->g.nz; }

SavedState alloc_saved(of_ctx* ctx, AdjWork* W) {
  SavedState t;
  for(int c = 0; c < 3; ++c) {
    t.vel[c] = W->alloc(ctx->size(1 + c), ctx->stream);
    t.adv_prev[c] = W->alloc(ctx->size(1 + c), ctx->stream);
  }
  t.p = W->alloc(ctx->size(0), ctx->stream);
  return t;
}

size_t saved_bytes(of_ctx* ctx) {
  return sizeof(double) * (ctx->size(0) + 2 * (ctx->size(1) + ctx->size(2) + ctx->size(3)));
}

// Keeps every step's pressure-solve result when it fits comfortably (under
// 40% of the free device memory): recomputed steps then skip their pressure
// solves.
void keep_pressure_results(of_ctx* ctx, AdjWork* W, int steps) {
  size_t free_b = 0, total_b = 0;
  OFB_CHECK(cudaMemGetInfo(&free_b, &total_b));
  const size_t per = (static_cast<size_t>(g_cells(ctx)) + 1) * sizeof(double);
  if(static_cast<double>(per) * steps < 0.4 * static_cast<double>(free_b))
    for(int n = 0; n < steps; ++n) W->phi.push_back(W->alloc(per / sizeof(double), ctx->stream));
}

constexpr int kMaxSnapshots = 64;
// The binomial schedule places at most this many snapshots: with 128 free
// snapshots every one of up to kMaxBinomialSteps = 4096 steps is advanced at
// most twice in the reverse sweep (binom(131, 2) >= 4096), and the schedule's
// dynamic program stays near 1e9 cheap operations (it is O(steps^2 snapshots)).
constexpr int kMaxScheduleSnapshots = 128;
constexpr size_t kSnapshotReserve = size_t(2) << 30;  // device memory left free by the auto sizing

// Work set of a tangent-linear or adjoint run; kept on the context while the
// same kind of run repeats.  `every`: checkpoint interval (kAdjSegments);
// `snapshots`: saved states besides the initial one (kAdjBinomial; 0 sizes
// them to the free device memory).
AdjWork* adj_work(of_ctx* ctx, int kind, int steps, int every, int snapshots = 0) {
  AdjWork* W = ctx->adj;
  if(W != nullptr && W->kind == kind && W->steps == steps && W->every == every &&
     (kind != kAdjBinomial ||
      (snapshots == 0 ? W->auto_snapshots
                      : !W->auto_snapshots && W->snapshots == std::min(snapshots, steps - 1))))
    return W;
  ctx->sync();
  delete W;
  ctx->adj = nullptr;
  W = new AdjWork();
  ctx->adj = W;  // owned by the context from here, so a failed allocation frees it
  cudaStream_t s = ctx->stream;
  auto face = [&](int c) { return ctx->size(1 + c); };
  const size_t cell = ctx->size(0);
  for(int c = 0; c < 3; ++c) {
    for(double** b : {&W->lam_vel[c], &W->lam_corr[c], &W->lam_pred[c], &W->lam_b[c], &W->lam_cur[c],
                      &W->lam_prev[c], &W->lam_advtot[c], &W->w_vel[c], &W->w_adv_prev[c]})
      *b = W->alloc(face(c), s);
    for(int a = 0; a < 3; ++a) W->y[c][a] = W->alloc(face(c), s);
    if(kind == kAdjBinomial) {
      // the target is read once, into lam_corr, before the reverse steps use
      // it; the gradient is assembled in lam_b after the last of them
      W->target[c] = W->lam_corr[c];
      W->out[c] = W->lam_b[c];
      continue;
    }
    for(double** b : {&W->target[c], &W->out[c], &W->rc_adv[c], &W->rc_corr[c], &W->w_adv_cur[c],
                      &W->w_corr[c]})
      *b = W->alloc(face(c), s);
    if(kind == kAdjTangent)
      for(double** b : {&W->t_vel[c], &W->t_adv_prev[c], &W->t_adv_cur[c], &W->t_corr[c], &W->base_cur[c]})
        *b = W->alloc(face(c), s);
  }
  if(kind == kAdjTangent) W->t_p = W->alloc(cell, s);
  W->w_p = W->alloc(cell, s);
  W->lam_p = W->alloc(cell, s);
  W->lam_phi = W->alloc(cell, s);
  W->lam_q = W->alloc(cell, s);
  W->acc = W->alloc(4, s);
  if(kind == kAdjSegments) {
    const int nseg = (steps + every - 1) / every;
    for(int k = 0; k < nseg; ++k) W->ckpt.push_back(alloc_saved(ctx, W));
    for(int k = 0; k < every && k < steps; ++k) W->seg.push_back(alloc_saved(ctx, W));
    if(every > 1) keep_pressure_results(ctx, W, steps);
  } else if(kind == kAdjBinomial) {
    W->slots.push_back(alloc_saved(ctx, W));  // the initial state
    if(steps > 1) keep_pressure_results(ctx, W, steps);
    int want = std::min(steps - 1, snapshots > 0 ? std::min(snapshots, kMaxScheduleSnapshots) : kMaxSnapshots);
    if(snapshots == 0) {
      size_t free_b = 0, total_b = 0;
      OFB_CHECK(cudaMemGetInfo(&free_b, &total_b));
      const size_t room = free_b > kSnapshotReserve ? (free_b - kSnapshotReserve) / saved_bytes(ctx) : 0;
      want = std::min<long long>(want, static_cast<long long>(room));
    }
    for(int k = 0; k < want; ++k) W->slots.push_back(alloc_saved(ctx, W));
    W->snapshots = want;
    W->auto_snapshots = snapshots == 0;
  }
  W->kind = kind;
  W->steps = steps;
  W->every = every;
  return W;
}

// The base-trajectory velocity buffers of the work set take the resident
// velocity's edge and corner ghosts (constants of every step), as the
// context's own velocity buffers do.
void adopt_edges(of_ctx* ctx, AdjWork* W) {
  for(int c = 0; c < 3; ++c)
    for(double* b : {W->w_vel[c], W->w_corr[c], W->rc_corr[c], W->base_cur[c]})
      if(b != nullptr) ctx->d2d(b, ctx->vel[c], 1 + c);
}

void save_state(of_ctx* ctx, const StepState& st, SavedState& out) {
  for(int c = 0; c < 3; ++c) {
    ctx->d2d(out.vel[c], st.vel[c], 1 + c);
    ctx->d2d(out.adv_prev[c], st.adv_prev[c], 1 + c);
  }
  ctx->d2d(out.p, st.p, 0);
  out.has_prev = st.has_prev;
  out.clean = st.clean;
}

void load_state(of_ctx* ctx, const SavedState& in, StepState& st) {
  for(int c = 0; c < 3; ++c) {
    ctx->d2d(st.vel[c], in.vel[c], 1 + c);
    ctx->d2d(st.adv_prev[c], in.adv_prev[c], 1 + c);
  }
  ctx->d2d(st.p, in.p, 0);
  st.has_prev = in.has_prev;
  st.clean = in.clean;
}

void require_adjoint_case(of_ctx* ctx, const of_step_params* prm) {
  for(int f = 0; f < 6; ++f)
    if(ctx->bc.type[f] != ofb::kPeriodic)
      fail(OF_INVALID_ARGUMENT, "the tangent-linear and adjoint runs support periodic boundaries only");
  if(prm->correction_variant != OF_CORRECTION_TAYLOR_GREEN)
    fail(OF_INVALID_ARGUMENT, "the tangent-linear and adjoint runs support the Taylor-Green predictor only");
}

void zero(of_ctx* ctx, double* p, int loc) {
  OFB_CHECK(cudaMemsetAsync(p, 0, ctx->size(loc) * sizeof(double), ctx->stream));
}

// The velocity the step at state `st` advects: the state's own buffers when
// clean, else a ghost-filled copy in `scratch`.
void current_velocity(of_ctx* ctx, const StepState& st, double* const* scratch, const double* cur[3]) {
  if(st.clean) {
    for(int c = 0; c < 3; ++c) cur[c] = st.vel[c];
    return;
  }
  for(int c = 0; c < 3; ++c) ctx->d2d(scratch[c], st.vel[c], 1 + c);
  ofb::launch_velocity_bc(ctx->g, ctx->bc, scratch[0], scratch[1], scratch[2], ctx->stream);
  for(int c = 0; c < 3; ++c) cur[c] = scratch[c];
}

// Reverse step: given the adjoints of the step's outputs (W->lam_vel, the
// AB2 history W->lam_prev, the total pressure W->lam_p), forms those of its
// inputs in the same buffers.  `S` is the state the step started from.
void adjoint_step(of_ctx* ctx, const of_step_params* prm, AdjWork* W, const SavedState& S) {
  const Grid& g = ctx->g;
  cudaStream_t s = ctx->stream;
  const double dt = prm->dt, nu = prm->viscosity, rho = prm->density;
  const double alpha = 0.5 * nu * dt;
  ofb::PoissonPlan* plan = ctx->poisson_for(ctx->pbc);
  // recompute the step's predictor, sweeps and pressure rhs from S
  StepState rs{};
  for(int c = 0; c < 3; ++c) {
    rs.vel[c] = S.vel[c];
    rs.adv_prev[c] = S.adv_prev[c];
    rs.adv_cur[c] = W->rc_adv[c];
    rs.corrected[c] = W->rc_corr[c];
  }
  rs.p = S.p;
  rs.has_prev = S.has_prev;
  rs.clean = S.clean;
  StepHooks hk;
  hk.sweep_out = W->y;
  hk.stop_after_rhs = true;
  forward_step(ctx, prm, "adjoint", 0, rs, &hk);
  const double* cur[3];
  for(int c = 0; c < 3; ++c) cur[c] = S.clean ? S.vel[c] : W->rc_corr[c];
  // total pressure: ghost fill, then p += phi - 0.5 nu dt q
  ofb::launch_pressure_bc_T(g, W->lam_p, s);
  zero(ctx, W->lam_phi, 0);
  zero(ctx, W->lam_q, 0);
  ofb::launch_axpby_active(g, ofb::kCell, 1.0, W->lam_p, 0.0, nullptr, W->lam_phi, s);
  ofb::launch_axpby_active(g, ofb::kCell, -0.5 * nu * dt, W->lam_p, 0.0, nullptr, W->lam_q, s);
  ofb::launch_dot_active(g, ofb::kCell, W->lam_p, ctx->prhs, -0.5 * dt, W->acc + 1, ctx->rb, s);
  // velocity ghost fill and correction u = u* - (dt/rho) G phi
  for(int c = 0; c < 3; ++c) {
    ctx->d2d(W->lam_corr[c], W->lam_vel[c], 1 + c);
    zero(ctx, W->lam_pred[c], 1 + c);
  }
  ofb::launch_velocity_bc_T(g, W->lam_corr[0], W->lam_corr[1], W->lam_corr[2], s);
  for(int c = 0; c < 3; ++c)
    ofb::launch_axpby_active(g, ofb::kFaceX + c, 1.0, W->lam_corr[c], 0.0, nullptr, W->lam_pred[c], s);
  ofb::launch_correct_T(g, -dt / rho, W->lam_corr, W->lam_phi, s);
  // pressure solve: phi = M q with M symmetric, so lam_q += M lam_phi.  The
  // rhs is scaled to unit RMS first: adjoint magnitudes are arbitrary and the
  // solve's breakdown test |p.Ap| < 1e-30 is absolute.
  OFB_CHECK(cudaMemsetAsync(W->acc + 3, 0, sizeof(double), s));
  ofb::launch_dot_active(g, ofb::kCell, W->lam_phi, W->lam_phi, 1.0, W->acc + 3, ctx->rb, s);
  double ss = 0.0;
  OFB_CHECK(cudaMemcpyAsync(&ss, W->acc + 3, sizeof(double), cudaMemcpyDeviceToHost, s));
  ctx->sync();
  const double rms = std::sqrt(ss / (static_cast<double>(g.nx) * g.ny * g.nz));
  if(rms > 0.0) {
    ofb::launch_axpby_active(g, ofb::kCell, 1.0 / rms, W->lam_phi, 0.0, nullptr, W->lam_phi, s);
    ofb::launch_rhs_to_system(g, ctx->pbc, W->lam_phi, ofb::poisson_b(plan), ctx->sc, ctx->rb, s);
    OFB_CHECK(cudaMemsetAsync(ofb::poisson_x(plan), 0, sizeof(double) * g.nx * g.ny * g.nz, s));
    OFB_CHECK(cudaMemsetAsync(&ctx->sc->sx, 0, sizeof(double), s));
    const ofb::SolveScalars ps =
        run_poisson(ctx, prm->poisson_max_iterations, prm->poisson_tolerance, nullptr, 0);
    if(!ps.converged) {
      std::ostringstream m;
      m << "adjoint pressure solve did not converge (iterations=" << ps.iterations
        << ", relative_residual=" << ps.rel << ")";
      fail(OF_NOT_CONVERGED, m.str());
    }
    ofb::launch_add_compact(g, ofb::poisson_x(plan), ctx->sc, rms, W->lam_q, s);
  }
  // divergence q = (rho/dt) D u*
  ofb::launch_divergence_T(g, rho / dt, W->lam_q, W->lam_pred, s);
  // ADI: BC(rhs), then per axis sweep + BC, undone in reverse
  ofb::AdiPlan* adi = ctx->adi_for(alpha);
  double* lam_rhs[3];
  for(int c = 0; c < 3; ++c) {
    double* a = W->lam_pred[c];
    double* b = W->lam_b[c];
    for(int axis = 2; axis >= 0; --axis) {
      ofb::launch_component_bc_T(g, c, a, s);
      if(!ofb::adi_axis_active(adi, c, axis)) continue;
      const bool dup = axis == c;  // periodic normal component: duplicated face
      if(dup) ofb::launch_duplicate(g, c, true, a, s);
      zero(ctx, b, 1 + c);
      ofb::launch_adi_sweep(adi, c, axis, a, b, s);
      if(dup) ofb::launch_duplicate(g, c, false, b, s);
      int begin = 0, n = 0;
      ofb::adi_axis_geometry(adi, c, axis, &begin, &n);
      ofb::launch_adi_alpha_dot(g, c, axis, begin, n, b, W->y[c][axis], W->acc + 2, ctx->rb, s);
      std::swap(a, b);
    }
    ofb::launch_component_bc_T(g, c, a, s);
    lam_rhs[c] = a;
    W->lam_b[c] = b;
    W->lam_pred[c] = a;
  }
  // predictor rhs: 27-point operator, pressure gradient, AB2 combination
  for(int c = 0; c < 3; ++c) zero(ctx, W->lam_cur[c], 1 + c);
  ofb::launch_predictor_T(g, nu, dt, alpha, lam_rhs, W->lam_cur, W->lam_p, s);
  const double s_adv = S.has_prev ? -1.5 * dt : -dt;
  for(int c = 0; c < 3; ++c) {
    ofb::launch_axpby_active(g, ofb::kFaceX + c, s_adv, lam_rhs[c], 1.0, W->lam_prev[c],
                             W->lam_advtot[c], s);
    ofb::launch_axpby_active(g, ofb::kFaceX + c, S.has_prev ? 0.5 * dt : 0.0, lam_rhs[c], 0.0,
                             nullptr, W->lam_prev[c], s);
  }
  ofb::launch_predictor_nu_dot(g, dt, alpha, cur, lam_rhs, W->acc + 1, ctx->rb, s);
  ofb::launch_advection_vjp(g, cur, W->lam_advtot, W->lam_cur, s);
  if(!S.clean) ofb::launch_velocity_bc_T(g, W->lam_cur[0], W->lam_cur[1], W->lam_cur[2], s);
  for(int c = 0; c < 3; ++c) std::swap(W->lam_vel[c], W->lam_cur[c]);
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

of_status of_get_grid(of_ctx* ctx, of_grid* grid) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(grid, "grid");
    *grid = of_grid{ctx->g.nx, ctx->g.ny, ctx->g.nz, ctx->g.dx, ctx->g.dy, ctx->g.dz};
  });
}

of_status of_stream(of_ctx* ctx, void** stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(stream, "stream");
    *stream = static_cast<void*>(ctx->stream);
  });
}

of_status of_profile_coarse_chain(of_ctx* ctx, int reps, double* us_per_chain, int* launches_per_chain) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(us_per_chain, "us_per_chain");
    require_ptr(launches_per_chain, "launches_per_chain");
    if(reps < 1) throw std::invalid_argument("reps must be >= 1");
    ofb::PoissonPlan* plan = ctx->poisson_for(ctx->pbc);
    *us_per_chain = ofb::poisson_time_coarse_chain(plan, ctx->rb, ctx->stream, reps, launches_per_chain);
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
      ctx->d2d(ctx->adv_cur[c], ctx->adv_prev[c], 1 + c);
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

namespace {

// Shared tail of the initial states: zero every velocity-shaped buffer and the
// total pressure, fill the analytic Taylor-Green field (mode 0/1) or leave the
// fluid at rest (mode < 0), then the ghost fills of the reference's init
// (solver/taylor_green.cpp:391-394, solver/lid_driven_cavity.cpp:401-406).
void init_state(of_ctx* ctx, double viscosity, double dt, int mode) {
  for(int c = 0; c < 3; ++c) {
    double* bufs[6] = {ctx->vel[c], ctx->adv_prev[c], ctx->adv_cur[c],
                       ctx->rhs[c], ctx->adi_b[c], ctx->corrected[c]};
    for(double* b : bufs) OFB_CHECK(cudaMemsetAsync(b, 0, ctx->size(1 + c) * sizeof(double), ctx->stream));
  }
  OFB_CHECK(cudaMemsetAsync(ctx->p_total, 0, ctx->size(0) * sizeof(double), ctx->stream));
  if(mode >= 0)
    ofb::launch_tg_init(ctx->g, mode, ctx->vel[0], ctx->vel[1], ctx->vel[2], ctx->p_total, ctx->stream);
  ofb::launch_velocity_bc(ctx->g, ctx->bc, ctx->vel[0], ctx->vel[1], ctx->vel[2], ctx->stream);
  ofb::launch_total_pressure_bc(ctx->g, ctx->bc, viscosity, ctx->vel[0], ctx->vel[1], ctx->vel[2],
                                ctx->p_total, ctx->stream);
  ctx->has_prev = 0;
  ctx->metrics = of_step_metrics{};
  ctx->metrics.dt = dt;
  ctx->state_clean = true;
  ctx->sync();
}

// Device scratch of the diagnostics reductions (4 doubles), made on first use.
double* diag_buffer(of_ctx* ctx) {
  if(ctx->diag == nullptr) {
    OFB_CHECK(cudaMalloc(&ctx->diag, 4 * sizeof(double)));
    ctx->bytes += 4 * sizeof(double);
  }
  return ctx->diag;
}

}  // namespace

of_status of_tg_init(of_ctx* ctx, double viscosity, double dt, int mode) {
  return guarded([&] {
    require_ctx(ctx);
    if(mode != 0 && mode != 1) fail(OF_INVALID_ARGUMENT, "Taylor-Green initial-state mode must be 0 or 1");
    init_state(ctx, viscosity, dt, mode);
  });
}

of_status of_rest_init(of_ctx* ctx, double viscosity, double dt) {
  return guarded([&] {
    require_ctx(ctx);
    init_state(ctx, viscosity, dt, -1);
  });
}

of_status of_kinetic_energy(of_ctx* ctx, double* energy) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(energy, "energy");
    double* d = diag_buffer(ctx);
    ofb::launch_kinetic_energy(ctx->g, ctx->vel[0], ctx->vel[1], ctx->vel[2], ctx->rb, d, ctx->stream);
    double sum = 0.0;
    OFB_CHECK(cudaMemcpyAsync(&sum, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ctx->sync();
    *energy = sum / static_cast<double>(ctx->lay[0].active_count());
  });
}

of_status of_tg_velocity_error(of_ctx* ctx, double viscosity, double time, int mode, double* error) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(error, "error");
    if(mode != 0 && mode != 1) fail(OF_INVALID_ARGUMENT, "Taylor-Green initial-state mode must be 0 or 1");
    // exact_decay (solver/taylor_green.cpp:258-261)
    const double rate = ctx->g.nz > 1 ? 3.0 : 2.0;
    const double decay = std::exp(-rate * viscosity * time);
    double* d = diag_buffer(ctx);
    double num = 0.0, den = 0.0;
    for(int c = 0; c < 3; ++c) {
      ofb::launch_tg_error(ctx->g, 1 + c, mode, decay, ctx->vel[c], ctx->rb, d, ctx->stream);
      double part[2];
      OFB_CHECK(cudaMemcpyAsync(part, d, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      ctx->sync();
      num += part[0];
      den += part[1];
    }
    *error = den > 0.0 ? std::sqrt(num / den) : std::sqrt(num);
  });
}

of_status of_sample_line(of_ctx* ctx, int field, int axis, int i, int j, int k, double* out,
                         int* n_out) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(out, "output line");
    if(field < 0 || field > 3) fail(OF_INVALID_ARGUMENT, "field must be 0 (pressure) or 1..3 (velocity)");
    if(axis < 0 || axis > 2) fail(OF_INVALID_ARGUMENT, "axis must be 0, 1 or 2");
    const Lay& L = ctx->lay[field];
    int idx[3] = {i, j, k};
    idx[axis] = 0;
    for(int a = 0; a < 3; ++a)
      if(idx[a] < 0 || idx[a] >= L.s(a)) throw std::out_of_range("storage coordinate index outside field extent");
    const double* base = field == 0 ? ctx->p_total : ctx->vel[field - 1];
    const int n = L.s(axis);
    const size_t stride = static_cast<size_t>(L.stride(axis)) * sizeof(double);
    OFB_CHECK(cudaMemcpy2DAsync(out, sizeof(double), base + L.idx(idx[0], idx[1], idx[2]), stride,
                                sizeof(double), n, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->sync();
    if(n_out) *n_out = n;
  });
}

namespace {

// Parameter checks of run_*_steps (the messages of the reference's callees).
void check_step_params(const of_step_params* prm, int steps) {
  require_ptr(prm, "step parameters");
  if(steps < 0) fail(OF_INVALID_ARGUMENT, "run_taylor_green_steps expects a non-negative step count");
  if(prm->dt <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects dt > 0");
  if(prm->density <= 0.0) fail(OF_INVALID_ARGUMENT, "build_pressure_rhs expects density > 0");
  if(prm->poisson_max_iterations <= 0)
    fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects iterations > 0");
  if(prm->poisson_tolerance <= 0.0)
    fail(OF_INVALID_ARGUMENT, "solve_pressure_poisson expects tolerance > 0");
}

// One step of the resident state and its metrics update; on failure the
// state stays at the last completed step.
void resident_step(of_ctx* ctx, const of_step_params* prm, const std::string& name, const StepHooks* hk) {
  StepState st = resident_state(ctx);
  ofb::SolveScalars d;
  try {
    d = forward_step(ctx, prm, name, ctx->metrics.step + 1, st, hk);
  } catch(...) {
    set_resident_state(ctx, st);
    throw;
  }
  set_resident_state(ctx, st);
  of_step_metrics& m = ctx->metrics;
  m.step += 1;
  m.time += prm->dt;
  m.dt = prm->dt;
  m.max_cfl = d.max_cfl;
  m.max_velocity_change = d.max_dv;
  m.divergence_l2 = d.div_after_l2;
  if(prm->track_max_divergence)
    m.max_divergence_l2 = m.max_divergence_l2 < d.div_after_l2 ? d.div_after_l2 : m.max_divergence_l2;
  m.pressure_iterations = d.iterations;
  m.pressure_relative_residual = d.rel;
}

bool pinned_host(const void* p) {
  cudaPointerAttributes a{};
  if(cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

of_status of_run_steps(of_ctx* ctx, const of_step_params* prm, int steps, of_step_metrics* out) {
  return guarded([&] {
    require_ctx(ctx);
    check_step_params(prm, steps);
    const std::string name = prm->solver_name ? prm->solver_name : "Taylor-Green";
    for(int step = 0; step < steps; ++step) resident_step(ctx, prm, name, nullptr);
    if(out) *out = ctx->metrics;
  });
}

of_status of_step_host(of_ctx* ctx, const of_step_params* prm, double* u, double* v, double* w,
                       double* adv_u, double* adv_v, double* adv_w, double* p_total,
                       int* has_previous_advection, of_step_metrics* metrics) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(has_previous_advection, "has_previous_advection");
    check_step_params(prm, 1);
    const of_status up = of_state_upload(ctx, u, v, w, adv_u, adv_v, adv_w, p_total, *has_previous_advection,
                                         metrics);
    if(up != OF_OK) fail(up, of_last_error());
    const std::string name = prm->solver_name ? prm->solver_name : "Taylor-Green";
    double* adv[3] = {adv_u, adv_v, adv_w};
    StepHooks hk;
    const bool overlap = pinned_host(adv_u) && pinned_host(adv_v) && pinned_host(adv_w);
    if(overlap) {
      if(ctx->side == nullptr) OFB_CHECK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
      if(ctx->adv_ready == nullptr) OFB_CHECK(cudaEventCreateWithFlags(&ctx->adv_ready, cudaEventDisableTiming));
      hk.adv_host = adv;
      hk.side = ctx->side;
      hk.adv_ready = ctx->adv_ready;
    }
    try {
      resident_step(ctx, prm, name, overlap ? &hk : nullptr);
    } catch(...) {
      // the history copies may have written this failed step's advection:
      // put the resident (uploaded) history back into the caller's arrays
      if(overlap) {
        cudaStreamSynchronize(ctx->side);
        for(int c = 0; c < 3; ++c)
          cudaMemcpyAsync(adv[c], ctx->adv_prev[c], ctx->size(1 + c) * sizeof(double),
                          cudaMemcpyDeviceToHost, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
      }
      throw;
    }
    double* vout[3] = {u, v, w};
    for(int c = 0; c < 3; ++c) {
      ctx->download(vout[c], ctx->vel[c], 1 + c);
      if(!overlap) ctx->download(adv[c], ctx->adv_prev[c], 1 + c);
    }
    ctx->download(p_total, ctx->p_total, 0);
    if(overlap) OFB_CHECK(cudaStreamSynchronize(ctx->side));
    ctx->sync();
    *has_previous_advection = ctx->has_prev;
    if(metrics) *metrics = ctx->metrics;
  });
}

of_status of_tangent_linear(of_ctx* ctx, const of_step_params* prm, int steps, const double* du,
                            const double* dv, const double* dw, double* out_u, double* out_v,
                            double* out_w) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(prm, "step parameters");
    const double* din[3] = {du, dv, dw};
    double* dout[3] = {out_u, out_v, out_w};
    for(int c = 0; c < 3; ++c) {
      require_ptr(din[c], "velocity perturbation");
      require_ptr(dout[c], "tangent-linear output");
    }
    if(steps < 1) fail(OF_INVALID_ARGUMENT, "the tangent-linear run needs at least one step");
    require_adjoint_case(ctx, prm);
    const std::string name = prm->solver_name ? prm->solver_name : "Taylor-Green";
    AdjWork* W = adj_work(ctx, kAdjTangent, steps, steps);
    StepState st = resident_state(ctx);
    adopt_edges(ctx, W);
    StepState t{};
    for(int c = 0; c < 3; ++c) {
      t.vel[c] = W->t_vel[c];
      t.adv_prev[c] = W->t_adv_prev[c];
      t.adv_cur[c] = W->t_adv_cur[c];
      t.corrected[c] = W->t_corr[c];
      // only the active entries of the perturbation count (ghosts are refilled,
      // edges are constants of the step)
      ctx->upload(W->out[c], din[c], 1 + c);
      zero(ctx, t.vel[c], 1 + c);
      ofb::launch_axpby_active(ctx->g, ofb::kFaceX + c, 1.0, W->out[c], 0.0, nullptr, t.vel[c],
                               ctx->stream);
      zero(ctx, t.adv_prev[c], 1 + c);
      zero(ctx, t.adv_cur[c], 1 + c);
      zero(ctx, t.corrected[c], 1 + c);
    }
    t.p = W->t_p;
    zero(ctx, t.p, 0);
    t.has_prev = st.has_prev;
    t.clean = false;
    try {
      for(int n = 0; n < steps; ++n) {
        const double* base[3];
        current_velocity(ctx, st, W->base_cur, base);
        StepHooks hk;
        hk.lin_base = base;
        forward_step(ctx, prm, name + " tangent-linear", n + 1, t, &hk);
        forward_step(ctx, prm, name, ctx->metrics.step + 1, st);
        ctx->metrics.step += 1;
        ctx->metrics.time += prm->dt;
      }
    } catch(...) {
      set_resident_state(ctx, st);
      for(int c = 0; c < 3; ++c) {
        W->t_vel[c] = t.vel[c];
        W->t_adv_prev[c] = t.adv_prev[c];
        W->t_adv_cur[c] = t.adv_cur[c];
        W->t_corr[c] = t.corrected[c];
      }
      throw;
    }
    set_resident_state(ctx, st);
    for(int c = 0; c < 3; ++c) {
      W->t_vel[c] = t.vel[c];
      W->t_adv_prev[c] = t.adv_prev[c];
      W->t_adv_cur[c] = t.adv_cur[c];
      W->t_corr[c] = t.corrected[c];
      ctx->download(dout[c], t.vel[c], 1 + c);
    }
    ctx->sync();
  });
}

}  // extern "C"

namespace {

size_t device_in_use() {
  size_t free_b = 0, total_b = 0;
  OFB_CHECK(cudaMemGetInfo(&free_b, &total_b));
  return total_b - free_b;
}

constexpr int kMaxBinomialSteps = 4096;

// Optimal binomial checkpoint schedule (the "revolve" schedule: Griewank,
// Optimization Methods and Software 1 (1992); Griewank & Walther, ACM TOMS 26
// (2000)), by dynamic programming over the n steps still to reverse and the s
// snapshots still free.  With the state at the start of the n steps saved and
// the adjoint at their end known, reversing them costs
//   C(1, s) = 0,   C(n, 0) = n (n - 1) / 2   (advance from the start for each step),
//   C(n, s) = min over 0 < m < n of  m + C(n - m, s - 1) + C(m, s)
// forward steps: advance m steps and save, reverse the right part with one
// snapshot fewer, then the left part with that snapshot free again.  C(n, s)
// equals the published minimum t n - binom(s + t + 1, t - 1) for s + 1
// checkpoints, t the smallest with binom(s + t + 1, t) >= n.  D is the same
// recursion right after the forward pass that reached the end: that pass saved
// the first split of every level on its way ("spine"), so those advances are
// free:  D(1, s) = 0,  D(n, 0) = C(n, 0),  D(n, s) = min over m of D(n - m, s - 1) + C(m, s).
struct Schedule {
  int n = 0, s = 0;
  std::vector<long long> C, D;
  std::vector<int> Cm, Dm;
  // snapshot-major: row j holds C(., j), so the split search reads two rows
  // contiguously
  size_t at(int i, int j) const { return static_cast<size_t>(j) * (n + 1) + i; }
  Schedule(int steps, int snaps) : n(steps), s(snaps) {
    const size_t size = static_cast<size_t>(n + 1) * (s + 1);
    C.assign(size, 0);
    D.assign(size, 0);
    Cm.assign(size, 0);
    Dm.assign(size, 0);
    for(int i = 2; i <= n; ++i) C[at(i, 0)] = D[at(i, 0)] = static_cast<long long>(i) * (i - 1) / 2;
    for(int j = 1; j <= s; ++j) {
      const long long* cj = &C[at(0, j)];
      const long long* cp = &C[at(0, j - 1)];
      const long long* dp = &D[at(0, j - 1)];
      for(int i = 2; i <= n; ++i) {
        if(j >= i - 1) {
          // enough snapshots to save every state on the way: advance one step
          // at a time (C = i - 1; right after the forward pass nothing is left
          // to advance, D = 0)
          C[at(i, j)] = i - 1;
          Cm[at(i, j)] = 1;
          D[at(i, j)] = 0;
          Dm[at(i, j)] = 1;
          continue;
        }
        long long best_c = -1, best_d = -1;
        int m_c = 1, m_d = 1;
        for(int m = 1; m < i; ++m) {
          const long long left = cj[m];
          const long long c = m + cp[i - m] + left;
          const long long d = dp[i - m] + left;
          if(best_c < 0 || c < best_c) {
            best_c = c;
            m_c = m;
          }
          if(best_d < 0 || d < best_d) {
            best_d = d;
            m_d = m;
          }
        }
        C[at(i, j)] = best_c;
        Cm[at(i, j)] = m_c;
        D[at(i, j)] = best_d;
        Dm[at(i, j)] = m_d;
      }
    }
  }
  // the steps before which the forward pass saves the spine snapshots 1, 2, ...
  std::vector<int> spine() const {
    std::vector<int> pos;
    int start = 0, left = n, free = s;
    while(left > 1 && free > 0) {
      const int m = Dm[at(left, free)];
      start += m;
      left -= m;
      --free;
      pos.push_back(start);
    }
    return pos;
  }
};

// The reverse sweep of a binomial schedule.  The working state `ws` holds the
// recomputed states; the adjoint step's recomputed intermediates use its
// scratch halves (AB2 term, corrected velocity), which hold nothing between
// steps.
struct BinomialSweep {
  of_ctx* ctx;
  const of_step_params* prm;
  AdjWork* W;
  const Schedule* sch;
  std::string name;
  StepState ws{};
  int top = 1;
  long long forward = 0;

  void advance(const SavedState& from, int n0, int k) {
    load_state(ctx, from, ws);
    for(int i = 0; i < k; ++i) {
      StepHooks hk;
      if(!W->phi.empty()) hk.phi_load = W->phi[n0 + i];
      forward_step(ctx, prm, name, n0 + i + 1, ws, &hk);
      ++forward;
    }
  }
  SavedState working() const {
    SavedState v;
    for(int c = 0; c < 3; ++c) {
      v.vel[c] = ws.vel[c];
      v.adv_prev[c] = ws.adv_prev[c];
    }
    v.p = ws.p;
    v.has_prev = ws.has_prev;
    v.clean = ws.clean;
    return v;
  }
  void reverse_step(const SavedState& S) {
    for(int c = 0; c < 3; ++c) {
      W->rc_adv[c] = ws.adv_cur[c];
      W->rc_corr[c] = ws.corrected[c];
    }
    adjoint_step(ctx, prm, W, S);
  }
  // Reverses steps n0 .. n0 + n - 1; the state before step n0 is in
  // slots[slot], snapshots top .. top + free - 1 are free; on the spine the
  // state at the split is already in slots[top].
  void run(int slot, int n0, int n, int free, bool on_spine) {
    const SavedState& S = W->slots[slot];
    if(n == 1) {
      reverse_step(S);
      return;
    }
    if(free == 0) {
      for(int k = n - 1; k >= 1; --k) {
        advance(S, n0, k);
        reverse_step(working());
      }
      reverse_step(S);
      return;
    }
    const int m = on_spine ? sch->Dm[sch->at(n, free)] : sch->Cm[sch->at(n, free)];
    const int mine = top++;
    if(!on_spine) {
      advance(S, n0, m);
      save_state(ctx, ws, W->slots[mine]);
    }
    run(mine, n0 + m, n - m, free - 1, on_spine);
    --top;
    run(slot, n0, m, free, false);
  }
};

}  // namespace

extern "C" {

of_status of_adjoint_schedule_cost(int steps, int snapshots, long long* reverse_cost,
                                   long long* after_forward_cost) {
  return guarded([&] {
    if(steps < 1 || steps > kMaxBinomialSteps)
      fail(OF_INVALID_ARGUMENT, "the binomial schedule supports 1 to 4096 steps");
    if(snapshots < 0) fail(OF_INVALID_ARGUMENT, "snapshots must be non-negative");
    const int s = std::min(std::min(snapshots, kMaxScheduleSnapshots), std::max(steps - 1, 0));
    const Schedule sch(steps, s);
    if(reverse_cost) *reverse_cost = sch.C[sch.at(steps, s)];
    if(after_forward_cost) *after_forward_cost = sch.D[sch.at(steps, s)];
  });
}

of_status of_adjoint_gradient_binomial(of_ctx* ctx, const of_step_params* prm, int steps,
                                       int snapshots, const double* target_u,
                                       const double* target_v, const double* target_w,
                                       double* grad_u, double* grad_v, double* grad_w,
                                       of_adjoint_info* info) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(prm, "step parameters");
    const double* tin[3] = {target_u, target_v, target_w};
    double* gout[3] = {grad_u, grad_v, grad_w};
    for(int c = 0; c < 3; ++c) {
      require_ptr(tin[c], "target velocity");
      require_ptr(gout[c], "gradient output");
    }
    if(steps < 1) fail(OF_INVALID_ARGUMENT, "the adjoint run needs at least one step");
    if(steps > kMaxBinomialSteps)
      fail(OF_INVALID_ARGUMENT, "the binomial schedule supports 1 to 4096 steps");
    if(snapshots < 0) fail(OF_INVALID_ARGUMENT, "snapshots must be non-negative");
    require_adjoint_case(ctx, prm);
    const std::string name = prm->solver_name ? prm->solver_name : "Taylor-Green";
    // the pressure and ADI plans exist before the snapshots are sized
    ctx->poisson_for(ctx->pbc);
    ctx->adi_for(0.5 * prm->viscosity * prm->dt);
    AdjWork* W = adj_work(ctx, kAdjBinomial, steps, 0, snapshots);
    adopt_edges(ctx, W);
    const Schedule sch(steps, W->snapshots);
    const std::vector<int> spine = sch.spine();
    const Grid& g = ctx->g;
    cudaStream_t s = ctx->stream;
    cudaEvent_t e0, e1, e2;
    OFB_CHECK(cudaEventCreate(&e0));
    OFB_CHECK(cudaEventCreate(&e1));
    OFB_CHECK(cudaEventCreate(&e2));
    struct EventGuard {
      cudaEvent_t a, b, c;
      ~EventGuard() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaEventDestroy(c);
      }
    } guard{e0, e1, e2};
    OFB_CHECK(cudaMemsetAsync(W->acc, 0, 4 * sizeof(double), s));
    // forward run: the initial state and the spine snapshots are saved on the way
    OFB_CHECK(cudaEventRecord(e0, s));
    StepState st = resident_state(ctx);
    size_t next = 0;
    try {
      for(int n = 0; n < steps; ++n) {
        if(n == 0) save_state(ctx, st, W->slots[0]);
        if(next < spine.size() && spine[next] == n) save_state(ctx, st, W->slots[1 + next++]);
        StepHooks hk;
        if(!W->phi.empty()) hk.phi_store = W->phi[n];
        forward_step(ctx, prm, name, ctx->metrics.step + 1, st, &hk);
        ctx->metrics.step += 1;
        ctx->metrics.time += prm->dt;
      }
    } catch(...) {
      set_resident_state(ctx, st);
      throw;
    }
    set_resident_state(ctx, st);
    OFB_CHECK(cudaEventRecord(e1, s));
    const size_t in_use = device_in_use();
    // loss 1/2 |u(T) - target|^2 on the unique entries and its seed
    for(int c = 0; c < 3; ++c) {
      ctx->upload(W->target[c], tin[c], 1 + c);
      zero(ctx, W->lam_vel[c], 1 + c);
      zero(ctx, W->lam_prev[c], 1 + c);
    }
    zero(ctx, W->lam_p, 0);
    const double* vel_t[3] = {st.vel[0], st.vel[1], st.vel[2]};
    const double* tgt[3] = {W->target[0], W->target[1], W->target[2]};
    ofb::launch_loss_seed(g, ctx->bc, vel_t, tgt, W->lam_vel, W->acc, ctx->rb, s);
    // reverse sweep; the working state borrows the context's scratch halves.
    // Its steps swap the halves with the work set's buffers, so each buffer
    // goes back to its owner afterwards (contents are scratch; all four carry
    // the state's edge ghosts).
    BinomialSweep sw{ctx, prm, W, &sch, name};
    double* own_vel[3];
    double* own_adv[3];
    double* own_cur[3];
    double* own_corr[3];
    for(int c = 0; c < 3; ++c) {
      sw.ws.vel[c] = own_vel[c] = W->w_vel[c];
      sw.ws.adv_prev[c] = own_adv[c] = W->w_adv_prev[c];
      sw.ws.adv_cur[c] = own_cur[c] = ctx->adv_cur[c];
      sw.ws.corrected[c] = own_corr[c] = ctx->corrected[c];
    }
    sw.ws.p = W->w_p;
    auto give_back = [&] {
      for(int c = 0; c < 3; ++c) {
        W->w_vel[c] = own_vel[c];
        W->w_adv_prev[c] = own_adv[c];
        ctx->adv_cur[c] = own_cur[c];
        ctx->corrected[c] = own_corr[c];
        W->rc_adv[c] = W->rc_corr[c] = nullptr;
      }
    };
    try {
      sw.run(0, 0, steps, W->snapshots, true);
    } catch(...) {
      give_back();
      throw;
    }
    give_back();
    // the initial state's ghosts were filled from its active entries
    if(W->slots[0].clean) ofb::launch_velocity_bc_T(g, W->lam_vel[0], W->lam_vel[1], W->lam_vel[2], s);
    for(int c = 0; c < 3; ++c) {
      zero(ctx, W->out[c], 1 + c);
      ofb::launch_axpby_active(g, ofb::kFaceX + c, 1.0, W->lam_vel[c], 0.0, nullptr, W->out[c], s);
      ctx->download(gout[c], W->out[c], 1 + c);
    }
    OFB_CHECK(cudaEventRecord(e2, s));
    double acc[4];
    OFB_CHECK(cudaMemcpyAsync(acc, W->acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    ctx->sync();
    if(info != nullptr) {
      info->loss = acc[0];
      info->grad_viscosity = acc[1] + 0.5 * prm->dt * acc[2];
      info->forward_steps = static_cast<int>(steps + sw.forward);
      float f_ms = 0.0f, b_ms = 0.0f;
      OFB_CHECK(cudaEventElapsedTime(&f_ms, e0, e1));
      OFB_CHECK(cudaEventElapsedTime(&b_ms, e1, e2));
      info->forward_ms = f_ms;
      info->backward_ms = b_ms;
      info->device_bytes = W->bytes;
      info->snapshots = W->snapshots;
      info->device_bytes_in_use = in_use;
    }
  });
}

of_status of_adjoint_gradient(of_ctx* ctx, const of_step_params* prm, int steps,
                              int checkpoint_every, const double* target_u,
                              const double* target_v, const double* target_w, double* grad_u,
                              double* grad_v, double* grad_w, of_adjoint_info* info) {
  return guarded([&] {
    require_ctx(ctx);
    require_ptr(prm, "step parameters");
    const double* tin[3] = {target_u, target_v, target_w};
    double* gout[3] = {grad_u, grad_v, grad_w};
    for(int c = 0; c < 3; ++c) {
      require_ptr(tin[c], "target velocity");
      require_ptr(gout[c], "gradient output");
    }
    if(steps < 1) fail(OF_INVALID_ARGUMENT, "the adjoint run needs at least one step");
    if(checkpoint_every < 1) fail(OF_INVALID_ARGUMENT, "checkpoint_every must be positive");
    require_adjoint_case(ctx, prm);
    const std::string name = prm->solver_name ? prm->solver_name : "Taylor-Green";
    const int every = checkpoint_every < steps ? checkpoint_every : steps;
    AdjWork* W = adj_work(ctx, kAdjSegments, steps, every);
    adopt_edges(ctx, W);
    const Grid& g = ctx->g;
    cudaStream_t s = ctx->stream;
    cudaEvent_t e0, e1, e2;
    OFB_CHECK(cudaEventCreate(&e0));
    OFB_CHECK(cudaEventCreate(&e1));
    OFB_CHECK(cudaEventCreate(&e2));
    struct EventGuard {
      cudaEvent_t a, b, c;
      ~EventGuard() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaEventDestroy(c);
      }
    } guard{e0, e1, e2};
    for(int c = 0; c < 3; ++c) ctx->upload(W->target[c], tin[c], 1 + c);
    OFB_CHECK(cudaMemsetAsync(W->acc, 0, 4 * sizeof(double), s));
    int forward_steps = 0;
    // forward run, keeping the state before every segment of `every` steps
    OFB_CHECK(cudaEventRecord(e0, s));
    StepState st = resident_state(ctx);
    const int nseg = (steps + every - 1) / every;
    const int last0 = (nseg - 1) * every;  // first step of the last segment
    try {
      for(int n = 0; n < steps; ++n) {
        if(n % every == 0) save_state(ctx, st, W->ckpt[n / every]);
        // the last segment's states are kept now, so it needs no recomputation
        if(n >= last0) save_state(ctx, st, W->seg[n - last0]);
        StepHooks hk;
        if(!W->phi.empty()) hk.phi_store = W->phi[n];
        forward_step(ctx, prm, name, ctx->metrics.step + 1, st, &hk);
        ctx->metrics.step += 1;
        ctx->metrics.time += prm->dt;
        ++forward_steps;
      }
    } catch(...) {
      set_resident_state(ctx, st);
      throw;
    }
    set_resident_state(ctx, st);
    OFB_CHECK(cudaEventRecord(e1, s));
    const size_t in_use = device_in_use();
    // loss 1/2 |u(T) - target|^2 on the unique entries and its seed
    for(int c = 0; c < 3; ++c) {
      zero(ctx, W->lam_vel[c], 1 + c);
      zero(ctx, W->lam_prev[c], 1 + c);
    }
    zero(ctx, W->lam_p, 0);
    const double* vel_t[3] = {st.vel[0], st.vel[1], st.vel[2]};
    const double* tgt[3] = {W->target[0], W->target[1], W->target[2]};
    ofb::launch_loss_seed(g, ctx->bc, vel_t, tgt, W->lam_vel, W->acc, ctx->rb, s);
    // backward over the segments: recompute the states of a segment from its
    // checkpoint, then run the reverse steps
    StepState ws{};
    for(int c = 0; c < 3; ++c) {
      ws.vel[c] = W->w_vel[c];
      ws.adv_prev[c] = W->w_adv_prev[c];
      ws.adv_cur[c] = W->w_adv_cur[c];
      ws.corrected[c] = W->w_corr[c];
    }
    ws.p = W->w_p;
    for(int k = nseg - 1; k >= 0; --k) {
      const int n0 = k * every;
      const int n1 = std::min(steps, n0 + every);
      if(k < nseg - 1) {
        load_state(ctx, W->ckpt[k], ws);
        for(int n = n0; n < n1; ++n) {
          save_state(ctx, ws, W->seg[n - n0]);
          if(n + 1 < n1) {
            StepHooks hk;
            if(!W->phi.empty()) hk.phi_load = W->phi[n];
            forward_step(ctx, prm, name, n + 1, ws, &hk);
            ++forward_steps;
          }
        }
      }
      for(int n = n1 - 1; n >= n0; --n) adjoint_step(ctx, prm, W, W->seg[n - n0]);
    }
    // the initial state's ghosts were filled from its active entries
    if(W->ckpt[0].clean) ofb::launch_velocity_bc_T(g, W->lam_vel[0], W->lam_vel[1], W->lam_vel[2], s);
    for(int c = 0; c < 3; ++c) {
      zero(ctx, W->out[c], 1 + c);
      ofb::launch_axpby_active(g, ofb::kFaceX + c, 1.0, W->lam_vel[c], 0.0, nullptr, W->out[c], s);
      ctx->download(gout[c], W->out[c], 1 + c);
    }
    OFB_CHECK(cudaEventRecord(e2, s));
    double acc[4];
    OFB_CHECK(cudaMemcpyAsync(acc, W->acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    ctx->sync();
    if(info != nullptr) {
      info->loss = acc[0];
      info->grad_viscosity = acc[1] + 0.5 * prm->dt * acc[2];
      info->forward_steps = forward_steps;
      float f_ms = 0.0f, b_ms = 0.0f;
      OFB_CHECK(cudaEventElapsedTime(&f_ms, e0, e1));
      OFB_CHECK(cudaEventElapsedTime(&b_ms, e1, e2));
      info->forward_ms = f_ms;
      info->backward_ms = b_ms;
      info->device_bytes = W->bytes;
      info->snapshots = static_cast<int>(W->ckpt.size() + W->seg.size());
      info->device_bytes_in_use = in_use;
    }
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
