// Host-side launchers of the B200 projection-step kernels.  Every launcher
// enqueues on the given stream and returns immediately; the context code
// (context.cu) sequences them into the reference's step.
#pragma once

#include "common.cuh"
#include "prof.hpp"

namespace ofb {

// Device scalars shared by the pressure solve and the step diagnostics.  All
// reductions land here; the host reads the block back once per iteration or
// step.
struct SolveScalars {
  // pressure solve (linsolve/poisson_solver.cpp:678-809)
  double sb, sx, sr, sp, sap, sz;  // pending mean shifts of b, x, r, p, Ap, z
  double rz, pap, alpha, beta;
  double sum_r;                    // sum of the stored residual
  double r0, rnorm, rel;
  double removed_rhs_mean;
  double pressure_mean;
  int iterations;
  int converged;
  int stop;                        // |p.Ap| < 1e-30 (linsolve/poisson_solver.cpp:757)
  int zero_mean;
  int n;                           // fine unknowns
  double tol;
  // projection / step diagnostics (solver/projection.cpp:1097-1131)
  double div_before_l2, div_after_l2, rhs_l2;
  double max_cfl, max_dv;
  int nonfinite;
  // loop control of the rotated CG loop (one body = V-cycle, p, A p, x/r)
  int first;      // the next p update is the first (p = z)
  int max_it;
  int cont;       // run another body
  int body_runs;
  double* hist;   // device residual history, hist[0] = r0
  int hist_cap;
  int outer;      // mixed path: defect-correction steps taken
};

// Per-level mean shifts of the V-cycle vectors.
struct LevelScalars {
  double sb;  // rhs
  double sa;  // smoother output a
  double sx;  // smoother output b (the level's correction)
  double sum_x;
};

// ---- boundary conditions (bc.cu) ----
// apply_velocity_boundary_conditions (solver/projection.cpp:966-971) on three
// face fields in place.
void launch_velocity_bc(const Grid& g, const VBC& bc, double* u, double* v, double* w,
                        cudaStream_t s);
// Same on a single component (solve_component_adi's per-component calls).
void launch_component_bc(const Grid& g, const VBC& bc, int comp, double* f, cudaStream_t s);
// apply_total_pressure_boundary_conditions (solver/projection.cpp:986-1026) with
// the wall-normal source nu * Laplacian(velocity) evaluated at the wall faces.
void launch_total_pressure_bc(const Grid& g, const VBC& bc, double nu, const double* u,
                              const double* v, const double* w, double* p, cudaStream_t s);

// ---- momentum (momentum.cu) ----
struct PredictorArgs {
  Grid g;
  const double* cur[3];   // current velocity (ghosts filled)
  const double* p;        // total pressure (ghosts filled)
  const double* prev[3];  // previous advection (AB2 history), may be unused
  double* adv[3];         // out: advection at this step
  double* rhs[3];         // out: predictor rhs (active entries)
  double nu, dt, alpha;
  int has_prev;
  int variant;            // 0 Taylor-Green, 1 cavity
};
void launch_predictor_rhs(const PredictorArgs& a, cudaStream_t s);
// The predictor rhs from a.adv already computed (everything but the advection);
// linear in (cur, p, adv, prev).
void launch_predictor_rest(const PredictorArgs& a, cudaStream_t s);
void launch_advection(const Grid& g, const double* u, const double* v, const double* w,
                      double* au, double* av, double* aw, cudaStream_t s);
void launch_tg_init(const Grid& g, int mode, double* u, double* v, double* w, double* p,
                    cudaStream_t s);

// ---- ADI (adi.cu) ----
struct AdiPlan;  // per-(component, axis) Thomas coefficients, built on the host
AdiPlan* adi_plan_create(const Grid& g, const VBC& bc, double alpha);
void adi_plan_destroy(AdiPlan* p);
// One sweep of solve_component_adi (solver/projection.cpp:868-888): reads the
// active lines of `in`, writes the solved lines of `out`.
void launch_adi_sweep(const AdiPlan* p, int comp, int axis, const double* in, double* out,
                      cudaStream_t s);
int adi_line_count(const AdiPlan* p, int comp, int axis);
bool adi_axis_active(const AdiPlan* p, int comp, int axis);

// ---- projection (projection.cu) ----
// Divergence of the predicted velocity -> pressure rhs (rho/dt) div (padded,
// active entries) and the compact system rhs b = -rhs - source
// (solver/projection.cpp:1049-1064, linsolve/poisson_solver.cpp:701-705).
void launch_divergence_rhs(const Grid& g, const PBC& pbc, const double* u, const double* v,
                           const double* w, double scale, double* rhs_padded, double* b,
                           SolveScalars* sc, RedBuf rb, cudaStream_t s);
// System rhs from a caller-provided padded rhs (standalone Poisson solve).
void launch_rhs_to_system(const Grid& g, const PBC& pbc, const double* rhs_padded, double* b,
                          SolveScalars* sc, RedBuf rb, cudaStream_t s);
// Compact initial guess from the padded pressure; sum -> sx.
void launch_pressure_to_compact(const Grid& g, const double* p_padded, double* x,
                                SolveScalars* sc, int zm, RedBuf rb, cudaStream_t s);
// correct_velocity (solver/projection.cpp:1066-1095) active faces, and the
// max |corrected - previous| reduction when prev != nullptr.
void launch_correct_velocity(const Grid& g, const PBC& pbc, const double* x,
                             const SolveScalars* sc, const double* pu, const double* pv,
                             const double* pw, double scale, double* cu, double* cv, double* cw,
                             const double* prev_u, const double* prev_v, const double* prev_w,
                             SolveScalars* sc_out, RedBuf rb, cudaStream_t s);
// Post-correction cell pass: divergence after, pressure mean, optional write of
// the padded pressure correction, optional total-pressure update and CFL.
struct CellPassArgs {
  Grid g;
  const double* u;
  const double* v;
  const double* w;
  const double* x;           // compact pressure correction (shift sc->sx)
  double* phi_padded;        // out (active), may be null
  double* p_total;           // in/out, may be null
  const double* rhs_padded;  // pressure rhs for the total-pressure update
  double p_rhs_scale;        // -0.5 nu dt
  double dt;                 // for the CFL diagnostic (0: skip)
};
void launch_cell_pass(const CellPassArgs& a, SolveScalars* sc, RedBuf rb, cudaStream_t s);

// ---- Poisson (poisson.cu) ----
struct PoissonPlan;  // hierarchy, coarse factorisation, work vectors
PoissonPlan* poisson_plan_create(const Grid& g, const PBC& pbc, int precision);
void poisson_plan_destroy(PoissonPlan* p);
int poisson_levels(const PoissonPlan* p);
int poisson_coarse_unknowns(const PoissonPlan* p);
size_t poisson_device_bytes(const PoissonPlan* p);
double* poisson_b(PoissonPlan* p);  // compact system rhs
double* poisson_x(PoissonPlan* p);  // compact solution
// Runs the MG-PCG loop on b (with shift sc->sb) and x (shift sc->sx).  Returns
// after the device scalars hold the final diagnostics.  `history` (host) gets
// the residual norms when non-null.
void poisson_solve(PoissonPlan* p, int max_iterations, double tolerance, SolveScalars* sc_dev,
                   SolveScalars* sc_host, RedBuf rb, cudaStream_t s, double* history,
                   int history_cap);
// Device time (us) of the V-cycle's coarse-level chain -- levels 1 .. coarsest,
// as each CG iteration runs it -- replayed `reps` times from a CUDA graph of
// that chain alone on the level-1 rhs of the last solve (nothing it writes is
// read before the next solve's V-cycles overwrite it); *launches = kernels per
// chain.
double poisson_time_coarse_chain(PoissonPlan* p, RedBuf rb, cudaStream_t s, int reps, int* launches);
// Writes x - sx into the active entries of a padded pressure field.
void launch_compact_to_pressure(const Grid& g, const double* x, const SolveScalars* sc,
                                double* p_padded, cudaStream_t s);

// ---- tangent-linear and adjoint pieces (adjoint.cu), periodic grids ----
// out = A'(base) dir: the advection's Jacobian-vector product (branches frozen).
void launch_advection_jvp(const Grid& g, const double* const* base, const double* const* dir,
                          double* const* out, cudaStream_t s);
// lam_cur += A'(base)^T lam_adv (atomics; ghost positions included).
void launch_advection_vjp(const Grid& g, const double* const* base, const double* const* lam_adv,
                          double* const* lam_cur, cudaStream_t s);
// lam_cur += W^T lam_rhs (the predictor's 27-point operator on the velocity)
// and lam_p += (-dt G)^T lam_rhs (cells, ghosts included).
void launch_predictor_T(const Grid& g, double nu, double dt, double alpha, const double* const* lam_rhs,
                        double* const* lam_cur, double* lam_p, cudaStream_t s);
// *acc += lam_rhs . d(rhs)/d(nu) at the base velocity cur.
void launch_predictor_nu_dot(const Grid& g, double dt, double alpha, const double* const* cur,
                             const double* const* lam_rhs, double* acc, RedBuf rb, cudaStream_t s);
// out = a x + b y on the active entries of a padded field at `loc` (y may be null).
void launch_axpby_active(const Grid& g, int loc, double a, const double* x, double b,
                         const double* y, double* out, cudaStream_t s);
// Transposes of the periodic velocity and total-pressure ghost fills.
void launch_velocity_bc_T(const Grid& g, double* u, double* v, double* w, cudaStream_t s);
void launch_component_bc_T(const Grid& g, int comp, double* f, cudaStream_t s);
void launch_pressure_bc_T(const Grid& g, double* p, cudaStream_t s);
// Duplicated periodic face of the normal component: fold into the first
// unknown (fold) and clear, or just clear.
void launch_duplicate(const Grid& g, int comp, bool fold, double* f, cudaStream_t s);
// *acc += sum over lines of mu . D y (cyclic second difference on the unknowns).
void launch_adi_alpha_dot(const Grid& g, int comp, int axis, int begin, int n, const double* mu,
                          const double* y, double* acc, RedBuf rb, cudaStream_t s);
// lam_pred += (scale D)^T lam_q ; lam_phi += (scale G_periodic)^T lam_corr.
void launch_divergence_T(const Grid& g, double scale, const double* lam_q, double* const* lam_pred,
                         cudaStream_t s);
void launch_correct_T(const Grid& g, double scale, const double* const* lam_corr, double* lam_phi,
                      cudaStream_t s);
// lam = vel - target on the unique active entries; *loss += 1/2 |lam|^2.
void launch_loss_seed(const Grid& g, const VBC& bc, const double* const* vel,
                      const double* const* target, double* const* lam, double* loss, RedBuf rb,
                      cudaStream_t s);
// lam_q += scale (x - sc->sx) on the active cells.
void launch_add_compact(const Grid& g, const double* x, const SolveScalars* sc, double scale,
                        double* lam_q, cudaStream_t s);
// *acc += scale * sum over active entries of a * b.
void launch_dot_active(const Grid& g, int loc, const double* a, const double* b, double scale,
                       double* acc, RedBuf rb, cudaStream_t s);
// Geometry of one ADI sweep (begin, unknowns) for the viscosity derivative.
void adi_axis_geometry(const AdiPlan* p, int comp, int axis, int* begin, int* n);

// ---- validation reductions of the case drivers (diagnostics.cu) ----
// out[0] = sum over cells of 1/2 |face-averaged velocity|^2.
void launch_kinetic_energy(const Grid& g, const double* u, const double* v, const double* w,
                           RedBuf rb, double* out, cudaStream_t s);
// out[0] = sum (f - exact)^2, out[1] = sum exact^2 over the active entries of
// the face field at `loc`, exact = the Taylor-Green state of phase `mode` x decay.
void launch_tg_error(const Grid& g, int loc, int mode, double decay, const double* f, RedBuf rb,
                     double* out, cudaStream_t s);

// ---- allocation-free pressure rhs (noalloc.cu) ----
// Device address of the file-scope scratch on the current device (looked up
// once per device with cudaGetSymbolAddress, then cached).
double* noalloc_scratch();
// Most reduction blocks the scratch holds for one k plane (32 x 8 cells each).
long long noalloc_max_plane_blocks();
// rhs = scale div(u) on the active cells of a padded cell field, plus
// norms_host[0] = divergence L2, norms_host[1] = rhs L2 (active means) when
// norms_host != nullptr, in which case the stream is synchronised.
void launch_pressure_rhs_noalloc(const Grid& g, const double* u, const double* v, const double* w,
                                 double scale, double* rhs, double* scratch, double* norms_host,
                                 cudaStream_t s);

}  // namespace ofb
