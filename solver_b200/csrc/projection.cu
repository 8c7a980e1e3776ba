// Projection-side kernels (solver/projection.cpp:1049-1131): divergence to
// pressure right-hand side, the Poisson system right-hand side with its
// boundary source, the velocity correction u = u* - (dt/rho) grad(phi) with the
// pressure-correction ghost rules folded in, and one post-correction cell pass
// that produces every step diagnostic and the total-pressure update.
#include "kernels.hpp"

namespace ofb {

namespace {

#define CELL_PROLOGUE(g)                                   \
  const int i = blockIdx.x * kTX + threadIdx.x;            \
  const int j = blockIdx.y * kTY + threadIdx.y;            \
  const bool valid = i < (g).nx && j < (g).ny;             \
  const int k0 = blockIdx.z * kchunk;                      \
  const int k1 = min(k0 + kchunk, (g).nz);

// build_boundary_source (linsolve/poisson_solver.cpp:635-642): the operator
// applied to a zero field with the actual boundary values.
__device__ __forceinline__ double boundary_source(const Grid& g, const PBC& pbc, int i, int j,
                                                  int k) {
  const int pos[3] = {i, j, k};
  double acc = 0.0;
#pragma unroll
  for(int a = 0; a < 3; ++a) {
    double nb = 0.0;
    const double h = g.h(a);
    const int n = g.n(a);
#pragma unroll
    for(int s = 0; s < 2; ++s) {
      const bool upper = s == 1;
      if((!upper && pos[a] > 0) || (upper && pos[a] < n - 1)) continue;
      const int type = pbc.type[2 * a + s];
      if(type == kPNeumann) nb += upper ? 0.0 + pbc.gradient[2 * a + s] * h : 0.0 - pbc.gradient[2 * a + s] * h;
      else if(type == kPDirichlet) nb += 2.0 * pbc.value[2 * a + s] - 0.0;
    }
    acc -= nb / (h * h);
  }
  return acc;
}

__global__ void __launch_bounds__(kTX* kTY)
    k_divergence_rhs(Grid g, PBC pbc, const double* __restrict__ u, const double* __restrict__ v,
                     const double* __restrict__ w, double scale, double* __restrict__ rhs,
                     double* __restrict__ b, SolveScalars* sc, int zm, int with_source,
                     int kchunk, RedBuf rb) {
  CELL_PROLOGUE(g)
  const Lay P = make_lay(g, kCell), U = make_lay(g, kFaceX), V = make_lay(g, kFaceY),
            W = make_lay(g, kFaceZ);
  const CLay C = make_clay(g.nx, g.ny, g.nz);
  const double idx = 1.0 / g.dx, idy = 1.0 / g.dy, idz = 1.0 / g.dz;
  double acc[3] = {0.0, 0.0, 0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const int uq = U.idx(i + 1, j + 1, k + 1), vq = V.idx(i + 1, j + 1, k + 1),
                wq = W.idx(i + 1, j + 1, k + 1);
      // compute_divergence (operators/discrete_operators.cpp:98-113)
      const double div = (u[uq + 1] - u[uq]) * idx + (v[vq + V.sx] - v[vq]) * idy +
                         (w[wq + W.sxy] - w[wq]) * idz;
      const double r = div * scale;
      rhs[P.idx(i + 1, j + 1, k + 1)] = r;
      double bv = -r;
      if(with_source) bv -= boundary_source(g, pbc, i, j, k);
      b[C.idx(i, j, k)] = bv;
      acc[0] += div * div;
      acc[1] += r * r;
      acc[2] += bv;
    }
  }
  const bool mx[3] = {false, false, false};
  const int n = C.count();
  reduce_finish<3>(acc, mx, rb, [=](const Sums<3>& s) {
    sc->div_before_l2 = sqrt(s.v[0] / n);
    sc->rhs_l2 = sqrt(s.v[1] / n);
    sc->sb = zm ? s.v[2] / n : 0.0;
    sc->removed_rhs_mean = sc->sb;
  });
}

__global__ void __launch_bounds__(kTX* kTY)
    k_rhs_to_system(Grid g, PBC pbc, const double* __restrict__ rhs, double* __restrict__ b,
                    SolveScalars* sc, int zm, int kchunk, RedBuf rb) {
  CELL_PROLOGUE(g)
  const Lay P = make_lay(g, kCell);
  const CLay C = make_clay(g.nx, g.ny, g.nz);
  double acc[1] = {0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const double bv = -rhs[P.idx(i + 1, j + 1, k + 1)] - boundary_source(g, pbc, i, j, k);
      b[C.idx(i, j, k)] = bv;
      acc[0] += bv;
    }
  }
  const bool mx[1] = {false};
  const int n = C.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) {
    sc->sb = zm ? s.v[0] / n : 0.0;
    sc->removed_rhs_mean = sc->sb;
  });
}

__global__ void __launch_bounds__(kTX* kTY)
    k_pressure_to_compact(Grid g, const double* __restrict__ p, double* __restrict__ x,
                          SolveScalars* sc, int zm, int kchunk, RedBuf rb) {
  CELL_PROLOGUE(g)
  const Lay P = make_lay(g, kCell);
  const CLay C = make_clay(g.nx, g.ny, g.nz);
  double acc[1] = {0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const double v = p[P.idx(i + 1, j + 1, k + 1)];
      x[C.idx(i, j, k)] = v;
      acc[0] += v;
    }
  }
  const bool mx[1] = {false};
  const int n = C.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { sc->sx = zm ? s.v[0] / n : 0.0; });
}

// Pressure correction at compact cell c along `axis` with the ghost rules of
// apply_pressure_boundary_conditions (solver/projection.cpp:302-337, 973-984):
// periodic image, Neumann active -/+ gradient * h, Dirichlet 2 value - active.
__device__ __forceinline__ double phi_at(const double* __restrict__ x, double sx, const CLay& C,
                                         const PBC& pbc, double h, int axis, int ci, int cj,
                                         int ck) {
  int c[3] = {ci, cj, ck};
  const int n = C.n(axis);
  if(c[axis] >= 0 && c[axis] < n) return x[C.idx(c[0], c[1], c[2])] - sx;
  const bool upper = c[axis] >= n;
  const int face = 2 * axis + (upper ? 1 : 0);
  const int type = pbc.type[face];
  if(type == kPPeriodic) {
    c[axis] = upper ? 0 : n - 1;
    return x[C.idx(c[0], c[1], c[2])] - sx;
  }
  c[axis] = upper ? n - 1 : 0;
  const double active = x[C.idx(c[0], c[1], c[2])] - sx;
  if(type == kPDirichlet) return 2.0 * pbc.value[face] - active;
  return upper ? active + pbc.gradient[face] * h : active - pbc.gradient[face] * h;
}

template <int Cc>
__global__ void __launch_bounds__(kTX* kTY)
    k_correct(Grid g, PBC pbc, const double* __restrict__ x, const SolveScalars* sc_in,
              const double* __restrict__ pred, double scale, double* __restrict__ out,
              const double* __restrict__ prev, SolveScalars* sc, int kchunk, RedBuf rb) {
  const Lay L = make_lay(g, kFaceX + Cc);
  const CLay C = make_clay(g.nx, g.ny, g.nz);
  const int i = blockIdx.x * kTX + threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  const bool valid = i < L.nx && j < L.ny;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, L.nz);
  const double sx = sc_in->sx;
  const double ih = 1.0 / g.h(Cc);
  double acc[2] = {0.0, 0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      // face (i, j, k) active -> storage (i+1, j+1, k+1); its cells are the
      // compact cells c and c - e_C
      int up[3] = {i, j, k};
      int lo[3] = {i, j, k};
      lo[Cc] -= 1;
      const double pu = phi_at(x, sx, C, pbc, g.h(Cc), Cc, up[0], up[1], up[2]);
      const double pl = phi_at(x, sx, C, pbc, g.h(Cc), Cc, lo[0], lo[1], lo[2]);
      const double grad = (pu - pl) * ih;
      const int q = L.idx(i + 1, j + 1, k + 1);
      const double v = pred[q] + scale * grad;
      out[q] = v;
      if(prev != nullptr) acc[0] = fmax(acc[0], fabs(v - prev[q]));
    }
  }
  const bool mx[2] = {true, false};
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    // max_velocity_change over the three components (solver/taylor_green.cpp:100-118)
    if(Cc == 0) sc->max_dv = s.v[0];
    else sc->max_dv = fmax(sc->max_dv, s.v[0]);
  });
}

__global__ void __launch_bounds__(kTX* kTY)
    k_cell_pass(CellPassArgs a, SolveScalars* sc, int kchunk, RedBuf rb) {
  const Grid& g = a.g;
  CELL_PROLOGUE(g)
  const Lay P = make_lay(g, kCell), U = make_lay(g, kFaceX), V = make_lay(g, kFaceY),
            W = make_lay(g, kFaceZ);
  const CLay C = make_clay(g.nx, g.ny, g.nz);
  const double idx = 1.0 / g.dx, idy = 1.0 / g.dy, idz = 1.0 / g.dz;
  const double sx = sc->sx;
  double acc[3] = {0.0, 0.0, 0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const int uq = U.idx(i + 1, j + 1, k + 1), vq = V.idx(i + 1, j + 1, k + 1),
                wq = W.idx(i + 1, j + 1, k + 1);
      const double u0 = a.u[uq], u1 = a.u[uq + 1];
      const double v0 = a.v[vq], v1 = a.v[vq + V.sx];
      const double w0 = a.w[wq], w1 = a.w[wq + W.sxy];
      const double div = (u1 - u0) * idx + (v1 - v0) * idy + (w1 - w0) * idz;
      acc[0] += div * div;
      const double phi = a.x[C.idx(i, j, k)] - sx;
      acc[1] += phi;
      const int pq = P.idx(i + 1, j + 1, k + 1);
      if(a.phi_padded != nullptr) a.phi_padded[pq] = phi;
      if(a.p_total != nullptr) {
        // p_total += phi; p_total += (-0.5 nu dt) rhs (solver/taylor_green.cpp:607-608)
        double pt = a.p_total[pq];
        pt += phi;
        pt += a.p_rhs_scale * a.rhs_padded[pq];
        a.p_total[pq] = pt;
      }
      if(a.dt > 0.0) {
        // compute_advective_cfl (solver/momentum_terms.cpp:327-355)
        const double uc = 0.5 * (u0 + u1), vc = 0.5 * (v0 + v1), wc = 0.5 * (w0 + w1);
        const double local = a.dt * (fabs(uc) * idx + fabs(vc) * idy + fabs(wc) * idz);
        acc[2] = fmax(acc[2], local);
      }
    }
  }
  const bool mx[3] = {false, false, true};
  const int n = C.count();
  reduce_finish<3>(acc, mx, rb, [=](const Sums<3>& s) {
    sc->div_after_l2 = sqrt(s.v[0] / n);
    sc->pressure_mean = s.v[1] / n;
    sc->max_cfl = s.v[2];
    sc->nonfinite = isfinite(sc->max_dv) && isfinite(sc->div_after_l2) ? 0 : 1;
  });
}

}  // namespace

void launch_divergence_rhs(const Grid& g, const PBC& pbc, const double* u, const double* v,
                           const double* w, double scale, double* rhs_padded, double* b,
                           SolveScalars* sc, RedBuf rb, cudaStream_t s) {
  int zm = 1, with_source = 0;
  for(int f = 0; f < 6; ++f) {
    if(pbc.type[f] == kPDirichlet) zm = 0;
    if((pbc.type[f] == kPDirichlet && pbc.value[f] != 0.0) ||
       (pbc.type[f] == kPNeumann && pbc.gradient[f] != 0.0))
      with_source = 1;
  }
  const Launch3 l = launch3(g.nx, g.ny, g.nz);
  ProfScope ps(kKDivergence, s);
  k_divergence_rhs<<<l.grid, l.block, 0, s>>>(g, pbc, u, v, w, scale, rhs_padded, b, sc, zm,
                                              with_source, l.kchunk, rb);
  OFB_LAUNCH_CHECK("k_divergence_rhs");
}

void launch_rhs_to_system(const Grid& g, const PBC& pbc, const double* rhs_padded, double* b,
                          SolveScalars* sc, RedBuf rb, cudaStream_t s) {
  int zm = 1;
  for(int f = 0; f < 6; ++f)
    if(pbc.type[f] == kPDirichlet) zm = 0;
  const Launch3 l = launch3(g.nx, g.ny, g.nz);
  ProfScope ps(kKOther, s);
  k_rhs_to_system<<<l.grid, l.block, 0, s>>>(g, pbc, rhs_padded, b, sc, zm, l.kchunk, rb);
  OFB_LAUNCH_CHECK("k_rhs_to_system");
}

void launch_pressure_to_compact(const Grid& g, const double* p_padded, double* x,
                                SolveScalars* sc, int zm, RedBuf rb, cudaStream_t s) {
  const Launch3 l = launch3(g.nx, g.ny, g.nz);
  ProfScope ps(kKOther, s);
  k_pressure_to_compact<<<l.grid, l.block, 0, s>>>(g, p_padded, x, sc, zm, l.kchunk, rb);
  OFB_LAUNCH_CHECK("k_pressure_to_compact");
}

void launch_correct_velocity(const Grid& g, const PBC& pbc, const double* x,
                             const SolveScalars* sc, const double* pu, const double* pv,
                             const double* pw, double scale, double* cu, double* cv, double* cw,
                             const double* prev_u, const double* prev_v, const double* prev_w,
                             SolveScalars* sc_out, RedBuf rb, cudaStream_t s) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  ProfScope ps(kKCorrect, s, 3);
  const Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  k_correct<0><<<l0.grid, l0.block, 0, s>>>(g, pbc, x, sc, pu, scale, cu, prev_u, sc_out,
                                            l0.kchunk, rb);
  const Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  k_correct<1><<<l1.grid, l1.block, 0, s>>>(g, pbc, x, sc, pv, scale, cv, prev_v, sc_out,
                                            l1.kchunk, rb);
  const Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_correct<2><<<l2.grid, l2.block, 0, s>>>(g, pbc, x, sc, pw, scale, cw, prev_w, sc_out,
                                            l2.kchunk, rb);
  OFB_LAUNCH_CHECK("k_correct");
}

void launch_cell_pass(const CellPassArgs& a, SolveScalars* sc, RedBuf rb, cudaStream_t s) {
  const Launch3 l = launch3(a.g.nx, a.g.ny, a.g.nz);
  ProfScope ps(kKCellPass, s);
  k_cell_pass<<<l.grid, l.block, 0, s>>>(a, sc, l.kchunk, rb);
  OFB_LAUNCH_CHECK("k_cell_pass");
}

}  // namespace ofb
