// Tangent-linear and adjoint kernels of the projection step on periodic grids.
//
// The step is linear in the state except for the TVD advection, so the
// tangent-linear step reuses the forward kernels with the advection replaced by
// its Jacobian-vector product about the base trajectory (limiter and upwind
// branches frozen at the base values).  The adjoint applies the exact
// transpose of every storage-level operation in reverse order: ghost fills and
// the duplicated periodic face averaging (solver/projection.cpp:207-300), the
// predictor's 27-point operator (solver/taylor_green.cpp:132-256), the ADI line
// solves (symmetric cyclic matrices, so the transposed sweep is the same solve,
// solver/projection.cpp:561-720), divergence and gradient
// (operators/discrete_operators.cpp:64-113) and the pressure solve (symmetric
// on the zero-mean subspace, linsolve/poisson_solver.cpp:678-809).  Edge and
// corner ghosts are constants of the step (never written), so their adjoints
// are dropped.
#include "kernels.hpp"

namespace ofb {

namespace {

constexpr double kSmallDen = 1.0e-14;  // solver/momentum_terms.cpp:14

// Value of one reconstruct_face call (solver/momentum_terms.cpp:42-151) and its
// partial derivatives with respect to (left, right, far_left, far_right) with
// the branches (upwind side, first-order fallback, limiter side) frozen.
// van Leer: phi(r) = (r + |r|) / (1 + |r|), phi'(r) = 2 / (1 + r)^2 for r > 0.
__device__ __forceinline__ double face_partials(double vel, double left, double right,
                                                double far_left, bool far_left_ok,
                                                double far_right, bool far_right_ok,
                                                double (&c)[4]) {
  const bool up = vel >= 0.0;
  const double delta = right - left;
  const double num = up ? left - far_left : far_right - right;
  const bool tiny = fabs(delta) < kSmallDen;
  const double r = tiny ? 0.0 : num / delta;
  // phi = (r + |r|) / (1 + |r|) is 0 for r <= 0 and 2 r s for r > 0, with
  // s = 1 / (1 + r), and phi' = 2 s^2: one division for both
  const bool positive = !tiny && r > 0.0;
  const double s = positive ? 1.0 / (1.0 + r) : 0.0;
  const double phi = 2.0 * r * s;
  const double dphi = 2.0 * s * s;
  const bool first = fabs(vel) < kSmallDen || (up ? !far_left_ok : !far_right_ok);
  if(first) {
    c[0] = up ? 1.0 : 0.0;
    c[1] = up ? 0.0 : 1.0;
    c[2] = 0.0;
    c[3] = 0.0;
    return up ? left : right;
  }
  // d phi = phi' (d num - r d delta) / delta, folded into the coefficients
  if(up) {
    c[0] = 1.0 + 0.5 * dphi * (1.0 + r) - 0.5 * phi;
    c[1] = -0.5 * dphi * r + 0.5 * phi;
    c[2] = -0.5 * dphi;
    c[3] = 0.0;
    return left + 0.5 * phi * delta;
  }
  c[0] = -0.5 * dphi * r + 0.5 * phi;
  c[1] = 1.0 + 0.5 * dphi * (1.0 + r) - 0.5 * phi;
  c[2] = 0.0;
  c[3] = -0.5 * dphi;
  return right - 0.5 * phi * delta;
}

// Storage positions and base values one axis of the advection stencil of
// component C at storage point (i, j, k) reads (solver/momentum_terms.cpp:153-266).
struct AxisStencil {
  int q_m2, q_m1, q_0, q_p1, q_p2;  // positions in vel[C]
  bool m2_ok, p2_ok, m1_ok, p1_ok;  // far-neighbour availability flags
  // face velocities: d == C -> from vel[C] at (q_m1, q_0) and (q_0, q_p1);
  // d != C -> from vel[d] at (lo0, lo1) and (hi0, hi1)
  int lo0, lo1, hi0, hi1;
};

template <int C>
__device__ __forceinline__ AxisStencil axis_stencil(const Grid& g, int d, int i, int j, int k) {
  const Lay L = make_lay(g, kFaceX + C);
  AxisStencil s;
  const int q = L.idx(i, j, k);
  const int pos[3] = {i, j, k};
  const int st = L.stride(d);
  const int smax = L.s(d) - 1;
  const int pd = pos[d];
  s.q_0 = q;
  s.q_m1 = q - st;
  s.q_p1 = q + st;
  s.q_m2 = pd - 2 >= 0 ? q - 2 * st : q - st;
  s.q_p2 = pd + 2 <= smax ? q + 2 * st : q + st;
  s.m2_ok = pd - 2 >= 0;
  s.p1_ok = pd + 1 <= smax;
  s.m1_ok = pd - 1 >= 0;
  s.p2_ok = pd + 2 <= smax;
  if(d == C) {
    s.lo0 = s.q_m1;
    s.lo1 = q;
    s.hi0 = q;
    s.hi1 = s.q_p1;
  } else {
    const Lay D = make_lay(g, kFaceX + d);
    int c0[3] = {i, j, k};
    c0[C] -= 1;
    const int qd = D.idx(i, j, k);
    const int qdm = D.idx(c0[0], c0[1], c0[2]);
    const int sd = D.stride(d);
    s.lo0 = qdm;
    s.lo1 = qd;
    s.hi0 = qdm + sd;
    s.hi1 = qd + sd;
  }
  return s;
}

// Jacobian-vector product of compute_{u,v,w}_advection at the active points
// of component C: out = A'(base) dir.
template <int C>
__global__ void __launch_bounds__(kTX* kTY)
    k_advect_jvp(Grid g, const double* __restrict__ bu, const double* __restrict__ bv,
                 const double* __restrict__ bw, const double* __restrict__ du,
                 const double* __restrict__ dv, const double* __restrict__ dw,
                 double* __restrict__ out, int kchunk) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > L.nx || j > L.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const double* base[3] = {bu, bv, bw};
  const double* dir[3] = {du, dv, dw};
  const double* f = base[C];
  const double* df = dir[C];
  for(int k = k0; k < k1; ++k) {
    double acc = 0.0;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
      const AxisStencil s = axis_stencil<C>(g, d, i, j, k);
      const double* fv = d == C ? f : base[d];
      const double* dfv = d == C ? df : dir[d];
      const double lv = 0.5 * (fv[s.lo0] + fv[s.lo1]);
      const double hv = 0.5 * (fv[s.hi0] + fv[s.hi1]);
      const double dlv = 0.5 * (dfv[s.lo0] + dfv[s.lo1]);
      const double dhv = 0.5 * (dfv[s.hi0] + dfv[s.hi1]);
      double cl[4], ch[4];
      const double lf = face_partials(lv, f[s.q_m1], f[s.q_0], f[s.q_m2], s.m2_ok, f[s.q_p1],
                                      s.p1_ok, cl);
      const double hf = face_partials(hv, f[s.q_0], f[s.q_p1], f[s.q_m1], s.m1_ok, f[s.q_p2],
                                      s.p2_ok, ch);
      const double dlf = cl[0] * df[s.q_m1] + cl[1] * df[s.q_0] + cl[2] * df[s.q_m2] + cl[3] * df[s.q_p1];
      const double dhf = ch[0] * df[s.q_0] + ch[1] * df[s.q_p1] + ch[2] * df[s.q_m1] + ch[3] * df[s.q_p2];
      acc += (dhv * hf + hv * dhf - dlv * lf - lv * dlf) / g.h(d);
    }
    out[L.idx(i, j, k)] = acc;
  }
}

// Vector-Jacobian product: lam_cur += A'(base)^T lam_adv, scattered with
// atomics into the padded velocity adjoints (ghost positions included).
template <int C>
__global__ void __launch_bounds__(kTX* kTY)
    k_advect_vjp(Grid g, const double* __restrict__ bu, const double* __restrict__ bv,
                 const double* __restrict__ bw, const double* __restrict__ lam_adv,
                 double* lu, double* lv_, double* lw, int kchunk) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > L.nx || j > L.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const double* base[3] = {bu, bv, bw};
  double* lam[3] = {lu, lv_, lw};
  const double* f = base[C];
  double* lf_out = lam[C];
  for(int k = k0; k < k1; ++k) {
    const double lam_q = lam_adv[L.idx(i, j, k)];
    if(lam_q == 0.0) continue;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
      const AxisStencil s = axis_stencil<C>(g, d, i, j, k);
      const double* fv = d == C ? f : base[d];
      double* lfv = d == C ? lf_out : lam[d];
      const double ih = 1.0 / g.h(d);
      const double lvel = 0.5 * (fv[s.lo0] + fv[s.lo1]);
      const double hvel = 0.5 * (fv[s.hi0] + fv[s.hi1]);
      double cl[4], ch[4];
      const double lface = face_partials(lvel, f[s.q_m1], f[s.q_0], f[s.q_m2], s.m2_ok, f[s.q_p1],
                                         s.p1_ok, cl);
      const double hface = face_partials(hvel, f[s.q_0], f[s.q_p1], f[s.q_m1], s.m1_ok, f[s.q_p2],
                                         s.p2_ok, ch);
      // flux = (hvel hface - lvel lface) / h
      const double g_hv = lam_q * hface * ih, g_lv = -lam_q * lface * ih;
      const double g_hf = lam_q * hvel * ih, g_lf = -lam_q * lvel * ih;
      atomicAdd(&lfv[s.hi0], 0.5 * g_hv);
      atomicAdd(&lfv[s.hi1], 0.5 * g_hv);
      atomicAdd(&lfv[s.lo0], 0.5 * g_lv);
      atomicAdd(&lfv[s.lo1], 0.5 * g_lv);
      atomicAdd(&lf_out[s.q_m1], g_lf * cl[0] + g_hf * ch[2]);
      atomicAdd(&lf_out[s.q_0], g_lf * cl[1] + g_hf * ch[0]);
      if(cl[2] != 0.0) atomicAdd(&lf_out[s.q_m2], g_lf * cl[2]);
      atomicAdd(&lf_out[s.q_p1], g_lf * cl[3] + g_hf * ch[1]);
      if(ch[3] != 0.0) atomicAdd(&lf_out[s.q_p2], g_hf * ch[3]);
    }
  }
}

// lam_cur[C] += W lam_rhs[C] over the whole padded storage: W is the
// predictor's symmetric 27-point operator (identity, 0.5 dt nu Laplacian and
// the factorisation correction), so its transpose is the same stencil read
// around each storage point.  lam_rhs is zero outside the active entries.
struct Stencil27 {
  double w[27];  // [dz+1][dy+1][dx+1]
};

template <int C>
__global__ void __launch_bounds__(kTX* kTY)
    k_stencil27_T(Grid g, Stencil27 st, const double* __restrict__ lam_rhs, double* lam_cur,
                  int kchunk) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  if(i >= L.sx || j >= L.sy) return;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, L.sz);
  for(int k = k0; k < k1; ++k) {
    double acc = 0.0;
    for(int dz = -1; dz <= 1; ++dz) {
      const int kk = k + dz;
      if(kk < 0 || kk >= L.sz) continue;
      for(int dy = -1; dy <= 1; ++dy) {
        const int jj = j + dy;
        if(jj < 0 || jj >= L.sy) continue;
        for(int dx = -1; dx <= 1; ++dx) {
          const int ii = i + dx;
          if(ii < 0 || ii >= L.sx) continue;
          const double w = st.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
          if(w != 0.0) acc += w * lam_rhs[L.idx(ii, jj, kk)];
        }
      }
    }
    lam_cur[L.idx(i, j, k)] += acc;
  }
}

// sum over active points of lam_rhs * (W_nu cur): the viscosity derivative of
// the predictor rhs; total added to *acc.
template <int C>
__global__ void __launch_bounds__(kTX* kTY)
    k_stencil27_dot(Grid g, Stencil27 st, const double* __restrict__ cur,
                    const double* __restrict__ lam_rhs, double* acc_out, int kchunk, RedBuf rb) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  const bool valid = i <= L.nx && j <= L.ny;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  double acc[1] = {0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      double v = 0.0;
      for(int dz = -1; dz <= 1; ++dz)
        for(int dy = -1; dy <= 1; ++dy)
          for(int dx = -1; dx <= 1; ++dx) {
            const double w = st.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
            if(w != 0.0) v += w * cur[L.idx(i + dx, j + dy, k + dz)];
          }
      acc[0] += lam_rhs[L.idx(i, j, k)] * v;
    }
  }
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { *acc_out += s.v[0]; });
}

// Pressure-gradient transpose of the predictor: lam_p[c] += s/h_C
// (lam_rhs_C[face c] - lam_rhs_C[face c + e_C]) for every cell storage point
// (the forward reads p at the face's cell and the one below, ghosts included).
__global__ void __launch_bounds__(kTX* kTY)
    k_grad_T(Grid g, double s, const double* __restrict__ lu, const double* __restrict__ lv,
             const double* __restrict__ lw, double* lam_p, int kchunk) {
  const Lay P = make_lay(g, kCell);
  const int i = blockIdx.x * kTX + threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  if(i >= P.sx || j >= P.sy) return;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, P.sz);
  const double* lam[3] = {lu, lv, lw};
  for(int k = k0; k < k1; ++k) {
    double acc = 0.0;
#pragma unroll
    for(int c = 0; c < 3; ++c) {
      const Lay F = make_lay(g, kFaceX + c);
      const int q = F.idx(i, j, k);
      acc += (lam[c][q] - lam[c][q + F.stride(c)]) / g.h(c);
    }
    lam_p[P.idx(i, j, k)] += s * acc;
  }
}

// out = a * x + b * y on the active entries of a padded field (other entries
// untouched); y may be null.
__global__ void k_axpby_active(Lay L, double a, const double* __restrict__ x, double b,
                               const double* __restrict__ y, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if(i > L.nx || j > L.ny || k > L.nz) return;
  const int q = L.idx(i, j, k);
  double v = a * x[q];
  if(y != nullptr) v += b * y[q];
  out[q] = v;
}

// Transposes of the periodic ghost fills of apply_velocity_component_boundaries
// (solver/projection.cpp:207-300) for one axis: the forward's elementary
// assignments undone in reverse order, per line.
__global__ void k_velocity_bc_axis_T(Grid g, int axis, int comp0, double* f0, double* f1,
                                     double* f2) {
  const int comp = comp0 + blockIdx.z;
  double* f = comp == 0 ? f0 : comp == 1 ? f1 : f2;
  if(f == nullptr) return;
  const Lay L = make_lay(g, kFaceX + comp);
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int t1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t2 = blockIdx.y * blockDim.y + threadIdx.y;
  if(t1 >= L.n(a1) || t2 >= L.n(a2)) return;
  int c[3] = {0, 0, 0};
  c[a1] = t1 + 1;
  c[a2] = t2 + 1;
  const int base = L.idx(c[0], c[1], c[2]);
  const int st = L.stride(axis);
  const int n = L.n(axis);
  auto at = [&](int q) -> double& { return f[base + q * st]; };
  if(comp == axis) {
    // forward: s = (x1 + xn)/2; x1 = s; xn = s; x0 = x_{n-1}; x_{n+1} = x2
    at(2) += at(n + 1);
    at(n + 1) = 0.0;
    at(n - 1) += at(0);
    at(0) = 0.0;
    const double t = 0.5 * (at(1) + at(n));
    at(1) = t;
    at(n) = t;
  } else {
    // forward: x0 = xn; x_{n+1} = x1
    at(1) += at(n + 1);
    at(n + 1) = 0.0;
    at(n) += at(0);
    at(0) = 0.0;
  }
}

// Transpose of the periodic total-pressure ghost fill for one axis.
__global__ void k_pressure_bc_axis_T(Grid g, int axis, double* p) {
  const Lay P = make_lay(g, kCell);
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int t1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t2 = blockIdx.y * blockDim.y + threadIdx.y;
  if(t1 >= P.n(a1) || t2 >= P.n(a2)) return;
  int c[3] = {0, 0, 0};
  c[a1] = t1 + 1;
  c[a2] = t2 + 1;
  const int base = P.idx(c[0], c[1], c[2]);
  const int st = P.stride(axis);
  const int n = P.n(axis);
  // forward: p0 = pn; p_{n+1} = p1
  p[base + st] += p[base + (n + 1) * st];
  p[base + (n + 1) * st] = 0.0;
  p[base + n * st] += p[base];
  p[base] = 0.0;
}

// Normal component along its periodic axis: the duplicated face.  fold: the
// first unknown takes the duplicate's adjoint (the forward copies the solved
// first unknown there); zero: clears the duplicate.
__global__ void k_duplicate(Grid g, int comp, int fold, double* f) {
  const Lay L = make_lay(g, kFaceX + comp);
  const int axis = comp;
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int t1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t2 = blockIdx.y * blockDim.y + threadIdx.y;
  if(t1 >= L.n(a1) || t2 >= L.n(a2)) return;
  int c[3] = {0, 0, 0};
  c[a1] = t1 + 1;
  c[a2] = t2 + 1;
  const int base = L.idx(c[0], c[1], c[2]);
  const int st = L.stride(axis);
  const int n = L.n(axis);
  if(fold) f[base + st] += f[base + n * st];
  f[base + n * st] = 0.0;
}

// Viscosity derivative of one periodic ADI sweep: sum over lines of
// mu . (D y) with D the cyclic second difference over the line's unknowns
// (the sweep solves (I - alpha D) y = x, so dy/dalpha = S D y).
__global__ void __launch_bounds__(256)
    k_adi_alpha_dot(Lay L, int axis, int begin, int n, double inv_h2, const double* __restrict__ mu,
                    const double* __restrict__ y, double* acc_out, RedBuf rb) {
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int lines = L.n(a1) * L.n(a2);
  double acc[1] = {0.0};
  for(int l = blockIdx.x * blockDim.x + threadIdx.x; l < lines; l += gridDim.x * blockDim.x) {
    int c[3] = {0, 0, 0};
    c[a1] = l % L.n(a1) + 1;
    c[a2] = l / L.n(a1) + 1;
    const int base = L.idx(c[0], c[1], c[2]) + begin * L.stride(axis);
    const int st = L.stride(axis);
    for(int q = 0; q < n; ++q) {
      const int qm = q == 0 ? n - 1 : q - 1;
      const int qp = q == n - 1 ? 0 : q + 1;
      const double dy = (y[base + qp * st] - 2.0 * y[base + q * st] + y[base + qm * st]) * inv_h2;
      acc[0] += mu[base + q * st] * dy;
    }
  }
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { *acc_out += s.v[0]; });
}

// Divergence transpose: lam_pred_a[f] += s/h_a (lam_q[f - e_a] - lam_q[f]) at
// face storage points (cells outside the storage or outside the active range
// carry zero adjoint).
template <int A>
__global__ void __launch_bounds__(kTX* kTY)
    k_div_T(Grid g, double s, const double* __restrict__ lam_q, double* lam_pred, int kchunk) {
  const Lay F = make_lay(g, kFaceX + A);
  const Lay P = make_lay(g, kCell);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > F.nx || j > F.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, F.nz + 1);
  for(int k = k0; k < k1; ++k) {
    int c[3] = {i, j, k};
    const int hi_ok = c[A] <= P.n(A);  // cell (c) active on the axis
    int cm[3] = {i, j, k};
    cm[A] -= 1;
    const int lo_ok = cm[A] >= 1;
    double v = 0.0;
    if(lo_ok) v += lam_q[P.idx(cm[0], cm[1], cm[2])];
    if(hi_ok) v -= lam_q[P.idx(c[0], c[1], c[2])];
    lam_pred[F.idx(i, j, k)] += s / g.h(A) * v;
  }
}

// Correction transpose (k_correct with periodic images): lam_phi[c] +=
// s/h (lam_corr[face c] + [c == 0] lam_corr[face n] - lam_corr[face c+1]
// - [c == n-1] lam_corr[face 0]) per component, at active cells of a padded
// cell field.
__global__ void __launch_bounds__(kTX* kTY)
    k_correct_T(Grid g, double s, const double* __restrict__ lu, const double* __restrict__ lv,
                const double* __restrict__ lw, double* lam_phi, int kchunk) {
  const Lay P = make_lay(g, kCell);
  const int i = blockIdx.x * kTX + threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  if(i >= g.nx || j >= g.ny) return;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.nz);
  const double* lam[3] = {lu, lv, lw};
  for(int k = k0; k < k1; ++k) {
    double acc = 0.0;
#pragma unroll
    for(int a = 0; a < 3; ++a) {
      const Lay F = make_lay(g, kFaceX + a);
      const int n = g.n(a);
      const int cc[3] = {i, j, k};
      auto face = [&](int fa) {
        int f[3] = {cc[0], cc[1], cc[2]};
        f[a] = fa;
        return lam[a][F.idx(f[0] + 1, f[1] + 1, f[2] + 1)];
      };
      double v = face(cc[a]) - face(cc[a] + 1);
      if(cc[a] == 0) v += face(n);
      if(cc[a] == n - 1) v -= face(0);
      acc += v / g.h(a);
    }
    lam_phi[P.idx(i + 1, j + 1, k + 1)] += s * acc;
  }
}

// Loss seed and value: lam = vel - target on the unique active entries
// (the duplicated periodic face excluded), zero elsewhere; *loss += 1/2 sum.
template <int C>
__global__ void __launch_bounds__(kTX* kTY)
    k_loss_seed(Grid g, const double* __restrict__ vel, const double* __restrict__ target,
                double* lam, double* loss, int periodic_normal, int kchunk, RedBuf rb) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  const bool valid = i <= L.nx && j <= L.ny;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  double acc[1] = {0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const int pos[3] = {i, j, k};
      const bool dup = periodic_normal && pos[C] == L.n(C);
      const int q = L.idx(i, j, k);
      const double d = dup ? 0.0 : vel[q] - target[q];
      lam[q] = d;
      acc[0] += 0.5 * d * d;
    }
  }
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { *loss += s.v[0]; });
}

// lam_q += x - sx on the active cells (the adjoint pressure solve's result).
__global__ void k_add_compact(Grid g, const double* __restrict__ x, const SolveScalars* sc,
                              double scale, double* lam_q) {
  const Lay P = make_lay(g, kCell);
  const CLay C = make_clay(g.nx, g.ny, g.nz);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if(i >= g.nx || j >= g.ny) return;
  lam_q[P.idx(i + 1, j + 1, k + 1)] += scale * (x[C.idx(i, j, k)] - sc->sx);
}

// sum over active cells of a * b (reduction into *acc).
__global__ void __launch_bounds__(kTX* kTY)
    k_dot_active(Lay L, const double* __restrict__ a, const double* __restrict__ b, double scale,
                 double* acc_out, int kchunk, RedBuf rb) {
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  const bool valid = i <= L.nx && j <= L.ny;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  double acc[1] = {0.0};
  if(valid)
    for(int k = k0; k < k1; ++k) acc[0] += a[L.idx(i, j, k)] * b[L.idx(i, j, k)];
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { *acc_out += scale * s.v[0]; });
}

dim3 line_grid(int d1, int d2, int comps, dim3& block) {
  block = dim3(32, 8, 1);
  return dim3((d1 + 31) / 32, (d2 + 7) / 8, comps);
}

}  // namespace

void launch_advection_jvp(const Grid& g, const double* const* base, const double* const* dir,
                          double* const* out, cudaStream_t s) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  ProfScope ps(kKAdvection, s, 3);
  const Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  const Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  const Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_advect_jvp<0><<<l0.grid, l0.block, 0, s>>>(g, base[0], base[1], base[2], dir[0], dir[1], dir[2],
                                                out[0], l0.kchunk);
  k_advect_jvp<1><<<l1.grid, l1.block, 0, s>>>(g, base[0], base[1], base[2], dir[0], dir[1], dir[2],
                                                out[1], l1.kchunk);
  k_advect_jvp<2><<<l2.grid, l2.block, 0, s>>>(g, base[0], base[1], base[2], dir[0], dir[1], dir[2],
                                                out[2], l2.kchunk);
  OFB_LAUNCH_CHECK("k_advect_jvp");
}

void launch_advection_vjp(const Grid& g, const double* const* base, const double* const* lam_adv,
                          double* const* lam_cur, cudaStream_t s) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  ProfScope ps(kKAdjoint, s, 3);
  const Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  const Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  const Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_advect_vjp<0><<<l0.grid, l0.block, 0, s>>>(g, base[0], base[1], base[2], lam_adv[0], lam_cur[0],
                                                lam_cur[1], lam_cur[2], l0.kchunk);
  k_advect_vjp<1><<<l1.grid, l1.block, 0, s>>>(g, base[0], base[1], base[2], lam_adv[1], lam_cur[0],
                                                lam_cur[1], lam_cur[2], l1.kchunk);
  k_advect_vjp<2><<<l2.grid, l2.block, 0, s>>>(g, base[0], base[1], base[2], lam_adv[2], lam_cur[0],
                                                lam_cur[1], lam_cur[2], l2.kchunk);
  OFB_LAUNCH_CHECK("k_advect_vjp");
}

namespace {

// 1-D second difference weights (1, -2, 1) / h^2 and the identity.
double s2(int d, double h) { return (d == 0 ? -2.0 : 1.0) / (h * h); }
double e1(int d) { return d == 0 ? 1.0 : 0.0; }

Stencil27 make_stencil(const Grid& g, double c_id, double c_lap, double c_d2, double c_d3) {
  Stencil27 st{};
  const bool three_d = g.nz != 1;
  for(int dz = -1; dz <= 1; ++dz)
    for(int dy = -1; dy <= 1; ++dy)
      for(int dx = -1; dx <= 1; ++dx) {
        const double X = s2(dx, g.dx), Y = s2(dy, g.dy), Z = s2(dz, g.dz);
        const double ex = e1(dx), ey = e1(dy), ez = e1(dz);
        const double lap = X * ey * ez + ex * Y * ez + ex * ey * Z;
        double d2 = X * Y * ez;
        double d3 = 0.0;
        if(three_d) {
          d2 += X * ey * Z + ex * Y * Z;
          d3 = X * Y * Z;
        }
        st.w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] =
            c_id * ex * ey * ez + c_lap * lap + c_d2 * d2 + c_d3 * d3;
      }
  return st;
}

}  // namespace

void launch_predictor_T(const Grid& g, double nu, double dt, double alpha, const double* const* lam_rhs,
                        double* const* lam_cur, double* lam_p, cudaStream_t s) {
  // rhs = cur + 0.5 dt nu Lap cur + alpha^2 (D2 - alpha D3) cur + ... (taylor_green.cpp:227-256)
  const Stencil27 st = make_stencil(g, 1.0, 0.5 * dt * nu, alpha * alpha, -alpha * alpha * alpha);
  ProfScope ps(kKAdjoint, s, 4);
  for(int c = 0; c < 3; ++c) {
    const Lay L = make_lay(g, kFaceX + c);
    const Launch3 l = launch3(L.sx, L.sy, L.sz);
    if(c == 0) k_stencil27_T<0><<<l.grid, l.block, 0, s>>>(g, st, lam_rhs[0], lam_cur[0], l.kchunk);
    if(c == 1) k_stencil27_T<1><<<l.grid, l.block, 0, s>>>(g, st, lam_rhs[1], lam_cur[1], l.kchunk);
    if(c == 2) k_stencil27_T<2><<<l.grid, l.block, 0, s>>>(g, st, lam_rhs[2], lam_cur[2], l.kchunk);
  }
  const Lay P = make_lay(g, kCell);
  const Launch3 lp = launch3(P.sx, P.sy, P.sz);
  k_grad_T<<<lp.grid, lp.block, 0, s>>>(g, -dt, lam_rhs[0], lam_rhs[1], lam_rhs[2], lam_p, lp.kchunk);
  OFB_LAUNCH_CHECK("predictor transpose");
}

void launch_predictor_nu_dot(const Grid& g, double dt, double alpha, const double* const* cur,
                             const double* const* lam_rhs, double* acc, RedBuf rb, cudaStream_t s) {
  // d rhs / d nu = 0.5 dt Lap cur + (d alpha / d nu)(2 alpha D2 - 3 alpha^2 D3) cur
  const double da = 0.5 * dt;
  const Stencil27 st = make_stencil(g, 0.0, 0.5 * dt, da * 2.0 * alpha, -da * 3.0 * alpha * alpha);
  ProfScope ps(kKAdjoint, s, 3);
  for(int c = 0; c < 3; ++c) {
    const Lay L = make_lay(g, kFaceX + c);
    const Launch3 l = launch3(L.nx, L.ny, L.nz);
    if(c == 0) k_stencil27_dot<0><<<l.grid, l.block, 0, s>>>(g, st, cur[0], lam_rhs[0], acc, l.kchunk, rb);
    if(c == 1) k_stencil27_dot<1><<<l.grid, l.block, 0, s>>>(g, st, cur[1], lam_rhs[1], acc, l.kchunk, rb);
    if(c == 2) k_stencil27_dot<2><<<l.grid, l.block, 0, s>>>(g, st, cur[2], lam_rhs[2], acc, l.kchunk, rb);
  }
  OFB_LAUNCH_CHECK("predictor nu derivative");
}

void launch_axpby_active(const Grid& g, int loc, double a, const double* x, double b,
                         const double* y, double* out, cudaStream_t s) {
  const Lay L = make_lay(g, loc);
  dim3 block(32, 8, 1);
  dim3 grid((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz);
  ProfScope ps(kKAdjoint, s);
  k_axpby_active<<<grid, block, 0, s>>>(L, a, x, b, y, out);
  OFB_LAUNCH_CHECK("k_axpby_active");
}

void launch_velocity_bc_T(const Grid& g, double* u, double* v, double* w, cudaStream_t s) {
  for(int axis = 2; axis >= 0; --axis) {
    const int d1 = (axis == 0 ? g.ny : g.nx) + 1;
    const int d2 = (axis == 2 ? g.ny : g.nz) + 1;
    dim3 block;
    const dim3 grid = line_grid(d1, d2, 3, block);
    ProfScope ps(kKAdjoint, s);
    k_velocity_bc_axis_T<<<grid, block, 0, s>>>(g, axis, 0, u, v, w);
    OFB_LAUNCH_CHECK("k_velocity_bc_axis_T");
  }
}

void launch_component_bc_T(const Grid& g, int comp, double* f, cudaStream_t s) {
  for(int axis = 2; axis >= 0; --axis) {
    const int d1 = (axis == 0 ? g.ny : g.nx) + 1;
    const int d2 = (axis == 2 ? g.ny : g.nz) + 1;
    dim3 block;
    const dim3 grid = line_grid(d1, d2, 1, block);
    double* fs[3] = {nullptr, nullptr, nullptr};
    fs[comp] = f;
    ProfScope ps(kKAdjoint, s);
    k_velocity_bc_axis_T<<<grid, block, 0, s>>>(g, axis, comp, fs[0], fs[1], fs[2]);
    OFB_LAUNCH_CHECK("k_velocity_bc_axis_T");
  }
}

void launch_pressure_bc_T(const Grid& g, double* p, cudaStream_t s) {
  for(int axis = 0; axis < 3; ++axis) {
    const int d1 = axis == 0 ? g.ny : g.nx;
    const int d2 = axis == 2 ? g.ny : g.nz;
    dim3 block;
    const dim3 grid = line_grid(d1, d2, 1, block);
    ProfScope ps(kKAdjoint, s);
    k_pressure_bc_axis_T<<<grid, block, 0, s>>>(g, axis, p);
    OFB_LAUNCH_CHECK("k_pressure_bc_axis_T");
  }
}

void launch_duplicate(const Grid& g, int comp, bool fold, double* f, cudaStream_t s) {
  const Lay L = make_lay(g, kFaceX + comp);
  const int a1 = comp == 0 ? 1 : 0;
  const int a2 = comp == 2 ? 1 : 2;
  dim3 block;
  const dim3 grid = line_grid(L.n(a1), L.n(a2), 1, block);
  ProfScope ps(kKAdjoint, s);
  k_duplicate<<<grid, block, 0, s>>>(g, comp, fold ? 1 : 0, f);
  OFB_LAUNCH_CHECK("k_duplicate");
}

void launch_adi_alpha_dot(const Grid& g, int comp, int axis, int begin, int n, const double* mu,
                          const double* y, double* acc, RedBuf rb, cudaStream_t s) {
  const Lay L = make_lay(g, kFaceX + comp);
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int lines = L.n(a1) * L.n(a2);
  int blocks = (lines + 255) / 256;
  if(blocks > kMaxBlocks) blocks = kMaxBlocks;
  const double h = g.h(axis);
  ProfScope ps(kKAdjoint, s);
  k_adi_alpha_dot<<<blocks, 256, 0, s>>>(L, axis, begin, n, 1.0 / (h * h), mu, y, acc, rb);
  OFB_LAUNCH_CHECK("k_adi_alpha_dot");
}

void launch_divergence_T(const Grid& g, double scale, const double* lam_q, double* const* lam_pred,
                         cudaStream_t s) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  const Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  const Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  const Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  ProfScope ps(kKAdjoint, s, 3);
  k_div_T<0><<<l0.grid, l0.block, 0, s>>>(g, scale, lam_q, lam_pred[0], l0.kchunk);
  k_div_T<1><<<l1.grid, l1.block, 0, s>>>(g, scale, lam_q, lam_pred[1], l1.kchunk);
  k_div_T<2><<<l2.grid, l2.block, 0, s>>>(g, scale, lam_q, lam_pred[2], l2.kchunk);
  OFB_LAUNCH_CHECK("k_div_T");
}

void launch_correct_T(const Grid& g, double scale, const double* const* lam_corr, double* lam_phi,
                      cudaStream_t s) {
  const Launch3 l = launch3(g.nx, g.ny, g.nz);
  ProfScope ps(kKAdjoint, s);
  k_correct_T<<<l.grid, l.block, 0, s>>>(g, scale, lam_corr[0], lam_corr[1], lam_corr[2], lam_phi,
                                         l.kchunk);
  OFB_LAUNCH_CHECK("k_correct_T");
}

void launch_loss_seed(const Grid& g, const VBC& bc, const double* const* vel,
                      const double* const* target, double* const* lam, double* loss, RedBuf rb,
                      cudaStream_t s) {
  ProfScope ps(kKAdjoint, s, 3);
  for(int c = 0; c < 3; ++c) {
    const Lay L = make_lay(g, kFaceX + c);
    const Launch3 l = launch3(L.nx, L.ny, L.nz);
    const int pn = bc.type[2 * c] == kPeriodic ? 1 : 0;
    if(c == 0) k_loss_seed<0><<<l.grid, l.block, 0, s>>>(g, vel[0], target[0], lam[0], loss, pn, l.kchunk, rb);
    if(c == 1) k_loss_seed<1><<<l.grid, l.block, 0, s>>>(g, vel[1], target[1], lam[1], loss, pn, l.kchunk, rb);
    if(c == 2) k_loss_seed<2><<<l.grid, l.block, 0, s>>>(g, vel[2], target[2], lam[2], loss, pn, l.kchunk, rb);
  }
  OFB_LAUNCH_CHECK("k_loss_seed");
}

void launch_add_compact(const Grid& g, const double* x, const SolveScalars* sc, double scale,
                        double* lam_q, cudaStream_t s) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
  ProfScope ps(kKAdjoint, s);
  k_add_compact<<<grid, block, 0, s>>>(g, x, sc, scale, lam_q);
  OFB_LAUNCH_CHECK("k_add_compact");
}

void launch_dot_active(const Grid& g, int loc, const double* a, const double* b, double scale,
                       double* acc, RedBuf rb, cudaStream_t s) {
  const Lay L = make_lay(g, loc);
  const Launch3 l = launch3(L.nx, L.ny, L.nz);
  ProfScope ps(kKAdjoint, s);
  k_dot_active<<<l.grid, l.block, 0, s>>>(L, a, b, scale, acc, l.kchunk, rb);
  OFB_LAUNCH_CHECK("k_dot_active");
}

}  // namespace ofb
