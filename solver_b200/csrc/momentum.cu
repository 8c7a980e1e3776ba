// Momentum-side stencils: the TVD/van Leer advection term (one launch per
// component), the rest of the predictor right-hand side (diffusion, pressure
// gradient, factorisation correction and the AB2 combination in one pass)
// and the Taylor-Green initial state.
#include "kernels.hpp"

namespace ofb {

namespace {

constexpr double kSmallDenominator = 1.0e-14;  // solver/momentum_terms.cpp:14

// Branch-free form of one reconstruct_face call: every candidate value is
// loaded before the velocity sign is known and the reference's three cases
// (first-order upwind for |u_f| < 1e-14 or near the storage bounds, van Leer
// MUSCL otherwise; solver/momentum_terms.cpp:42-151) are chosen by selects.
__device__ __forceinline__ double tvd_face(double vel, double left, double right, double far_left,
                                           bool far_left_ok, double far_right, bool far_right_ok) {
  const bool up = vel >= 0.0;
  const double delta = right - left;
  const double num = up ? left - far_left : far_right - right;
  // safe_ratio and limiter_value (solver/momentum_terms.cpp:26-40) enter as
  // 0.5 phi(r) delta with r = num / delta (0 when |delta| < 1e-14) and
  // phi = (r + |r|) / (1 + |r|): zero unless r > 0, and then equal to
  // num delta / (delta + num) -- one division instead of two; the value
  // differs from the two-division form by rounding only, the branches not
  // at all (the sign of r is the product of exact signs).
  const bool positive = fabs(delta) >= kSmallDenominator && num != 0.0 && ((num > 0.0) == (delta > 0.0));
  const double half_phi_delta = positive ? num * delta / (delta + num) : 0.0;
  const double muscl = up ? left + half_phi_delta : right - half_phi_delta;
  const bool first_order = fabs(vel) < kSmallDenominator || (up ? !far_left_ok : !far_right_ok);
  return first_order ? (up ? left : right) : muscl;
}

// compute_{u,v,w}_advection (solver/momentum_terms.cpp:153-266) at storage
// point (i, j, k) of component C, branch-free.
template <int C>
__device__ __forceinline__ double advection_bf(const Grid& g, const double* __restrict__ u,
                                               const double* __restrict__ v,
                                               const double* __restrict__ w, int i, int j, int k,
                                               const double (&inv_h)[3]) {
  const double* __restrict__ vel[3] = {u, v, w};
  const Lay L = make_lay(g, kFaceX + C);
  const double* __restrict__ f = vel[C];
  const int q = L.idx(i, j, k);
  const int pos[3] = {i, j, k};
  const double f0 = f[q];
  double flux_div = 0.0;
#pragma unroll
  for(int d = 0; d < 3; ++d) {
    const int st = L.stride(d);
    const int smax = L.s(d) - 1;
    const int pd = pos[d];
    const double fm1 = f[q - st];
    const double fp1 = f[q + st];
    const double fm2 = f[pd - 2 >= 0 ? q - 2 * st : q - st];
    const double fp2 = f[pd + 2 <= smax ? q + 2 * st : q + st];
    double lo_vel, hi_vel;
    if(d == C) {
      lo_vel = 0.5 * (fm1 + f0);
      hi_vel = 0.5 * (f0 + fp1);
    } else {
      const Lay D = make_lay(g, kFaceX + d);
      const double* __restrict__ fd = vel[d];
      int c0[3] = {i, j, k};
      c0[C] -= 1;
      const int qd = D.idx(i, j, k);
      const int qdm = D.idx(c0[0], c0[1], c0[2]);
      const int sd = D.stride(d);
      lo_vel = 0.5 * (fd[qdm] + fd[qd]);
      hi_vel = 0.5 * (fd[qdm + sd] + fd[qd + sd]);
    }
    const double lo_face = tvd_face(lo_vel, fm1, f0, fm2, pd - 2 >= 0, fp1, pd + 1 <= smax);
    const double hi_face = tvd_face(hi_vel, f0, fp1, fm1, pd - 1 >= 0, fp2, pd + 2 <= smax);
    flux_div += (hi_vel * hi_face - lo_vel * lo_face) * inv_h[d];
  }
  return flux_div;
}

// Advection term of component C at every active point, written to adv[C]
// (the first half of assemble_predictor_rhs, solver/taylor_green.cpp:238).
template <int C>
__global__ void __launch_bounds__(kTX* kTY)
    k_advect_bf(Grid g, const double* __restrict__ u, const double* __restrict__ v,
                const double* __restrict__ w, double* __restrict__ out, int kchunk) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > L.nx || j > L.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const double inv_h[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  for(int k = k0; k < k1; ++k) out[L.idx(i, j, k)] = advection_bf<C>(g, u, v, w, i, j, k, inv_h);
}

// The rest of assemble_predictor_rhs (solver/taylor_green.cpp:239-255):
// diffusion, total-pressure gradient, factorisation correction and the AB2
// combination with the advection term computed by k_advect_bf.  The 27-point
// correction is evaluated column by column (second z-differences first), so
// only 18 neighbourhood values are live at once.
template <int C>
__global__ void __launch_bounds__(kTX* kTY) k_predictor_rest(PredictorArgs a, int kchunk) {
  const Grid& g = a.g;
  const Lay L = make_lay(g, kFaceX + C);
  const Lay P = make_lay(g, kCell);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > L.nx || j > L.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const double ih = 1.0 / g.h(C);
  const double ix = 1.0 / (g.dx * g.dx), iy = 1.0 / (g.dy * g.dy), iz = 1.0 / (g.dz * g.dz);
  const double dy2 = g.dy * g.dy;
  const bool three_d = g.nz != 1;
  const double s_gp = -a.dt;
  const double s_dif = 0.5 * a.dt;
  const double s_adv = a.has_prev ? -1.5 * a.dt : -a.dt;
  const double s_prev = 0.5 * a.dt;
  const double s_corr = a.alpha * a.alpha;
  const double* __restrict__ f = a.cur[C];
  const int pstC = P.stride(C);
  for(int k = k0; k < k1; ++k) {
    const int q = L.idx(i, j, k);
    // in-plane values m[dy][dx] and second z-differences z2[dy][dx]
    double m[3][3], z2[3][3];
    double fzm = 0.0, fzp = 0.0;
#pragma unroll
    for(int b = 0; b < 3; ++b)
#pragma unroll
      for(int e = 0; e < 3; ++e) {
        const int qq = q + (e - 1) + (b - 1) * L.sx;
        const double lo = f[qq - L.sxy], mid = f[qq], hi = f[qq + L.sxy];
        m[b][e] = mid;
        z2[b][e] = (hi - 2.0 * mid + lo) * iz;
        if(b == 1 && e == 1) {
          fzm = lo;
          fzp = hi;
        }
      }
    const double c2 = 2.0 * m[1][1];
    const double lap = (m[1][2] - c2 + m[1][0]) * ix + (m[2][1] - c2 + m[0][1]) * iy +
                       (fzp - c2 + fzm) * iz;
    const double dif = lap * a.nu;
    const int pq = P.idx(i, j, k);
    const double gp = (a.p[pq] - a.p[pq - pstC]) * ih;
    double corr;
    if(a.variant == 1) {
      double dyy[3];
#pragma unroll
      for(int e = 0; e < 3; ++e) dyy[e] = (m[2][e] - 2.0 * m[1][e] + m[0][e]) / dy2;
      corr = (dyy[2] - 2.0 * dyy[1] + dyy[0]) * ix;
    } else {
      double d2y[3];
#pragma unroll
      for(int e = 0; e < 3; ++e) d2y[e] = (m[2][e] - 2.0 * m[1][e] + m[0][e]) * iy;
      corr = (d2y[2] - 2.0 * d2y[1] + d2y[0]) * ix;
      if(three_d) {
        const double mxz = (z2[1][2] - 2.0 * z2[1][1] + z2[1][0]) * ix;
        double myz[3];
#pragma unroll
        for(int e = 0; e < 3; ++e) myz[e] = (z2[2][e] - 2.0 * z2[1][e] + z2[0][e]) * iy;
        const double triple = (myz[2] - 2.0 * myz[1] + myz[0]) * ix;
        corr += mxz;
        corr += myz[1];
        corr -= a.alpha * triple;
      }
    }
    double r = m[1][1];
    r += s_gp * gp;
    r += s_dif * dif;
    r += s_adv * a.adv[C][q];
    if(a.has_prev) r += s_prev * a.prev[C][q];
    r += s_corr * corr;
    a.rhs[C][q] = r;
  }
}

// initialize_exact_state (solver/taylor_green.cpp:335-395), active entries.
__global__ void k_tg_init(Grid g, int mode, int loc, double* f) {
  const Lay L = make_lay(g, loc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if(i > L.nx || j > L.ny || k > L.nz) return;
  const bool three_d = g.nz > 1;
  // coordinate_for_storage_index (core/field_layout.hpp:226-238)
  const double x = (loc == kFaceX) ? (i - 1) * g.dx : (i - 1 + 0.5) * g.dx;
  const double y = (loc == kFaceY) ? (j - 1) * g.dy : (j - 1 + 0.5) * g.dy;
  const double z = (loc == kFaceZ) ? (k - 1) * g.dz : (k - 1 + 0.5) * g.dz;
  double val = 0.0;
  if(loc == kFaceX) {
    const double zf = three_d ? cos(z) : 1.0;
    val = mode == 0 ? -cos(x) * sin(y) * zf : sin(x) * cos(y) * zf;
  } else if(loc == kFaceY) {
    const double zf = three_d ? cos(z) : 1.0;
    val = mode == 0 ? sin(x) * cos(y) * zf : -cos(x) * sin(y) * zf;
  } else if(loc == kCell) {
    const double sign = mode == 0 ? 1.0 : -1.0;
    val = three_d ? sign * -0.0625 * (cos(2.0 * x) + cos(2.0 * y)) * (cos(2.0 * z) + 2.0)
                  : sign * -0.25 * (cos(2.0 * x) + cos(2.0 * y));
  }
  f[L.idx(i, j, k)] = val;
}

}  // namespace

void launch_predictor_rhs(const PredictorArgs& a, cudaStream_t s) {
  const Lay Lu = make_lay(a.g, kFaceX), Lv = make_lay(a.g, kFaceY), Lw = make_lay(a.g, kFaceZ);
  const Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  const Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  const Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  {
    ProfScope ps(kKAdvection, s, 3);
    k_advect_bf<0><<<l0.grid, l0.block, 0, s>>>(a.g, a.cur[0], a.cur[1], a.cur[2], a.adv[0], l0.kchunk);
    k_advect_bf<1><<<l1.grid, l1.block, 0, s>>>(a.g, a.cur[0], a.cur[1], a.cur[2], a.adv[1], l1.kchunk);
    k_advect_bf<2><<<l2.grid, l2.block, 0, s>>>(a.g, a.cur[0], a.cur[1], a.cur[2], a.adv[2], l2.kchunk);
    OFB_LAUNCH_CHECK("k_advect_bf");
  }
  launch_predictor_rest(a, s);
}

void launch_predictor_rest(const PredictorArgs& a, cudaStream_t s) {
  const Lay Lu = make_lay(a.g, kFaceX), Lv = make_lay(a.g, kFaceY), Lw = make_lay(a.g, kFaceZ);
  const Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  const Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  const Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  ProfScope ps(kKPredictor, s, 3);
  k_predictor_rest<0><<<l0.grid, l0.block, 0, s>>>(a, l0.kchunk);
  k_predictor_rest<1><<<l1.grid, l1.block, 0, s>>>(a, l1.kchunk);
  k_predictor_rest<2><<<l2.grid, l2.block, 0, s>>>(a, l2.kchunk);
  OFB_LAUNCH_CHECK("k_predictor_rest");
}

void launch_advection(const Grid& g, const double* u, const double* v, const double* w,
                      double* au, double* av, double* aw, cudaStream_t s) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  ProfScope ps(kKOther, s, 3);
  Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  k_advect_bf<0><<<l0.grid, l0.block, 0, s>>>(g, u, v, w, au, l0.kchunk);
  Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  k_advect_bf<1><<<l1.grid, l1.block, 0, s>>>(g, u, v, w, av, l1.kchunk);
  Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_advect_bf<2><<<l2.grid, l2.block, 0, s>>>(g, u, v, w, aw, l2.kchunk);
  OFB_LAUNCH_CHECK("k_advection");
}

void launch_tg_init(const Grid& g, int mode, double* u, double* v, double* w, double* p,
                    cudaStream_t s) {
  double* f[4] = {p, u, v, w};
  for(int loc = 0; loc < 4; ++loc) {
    if(loc == kFaceZ) continue;  // w = 0 (solver/taylor_green.cpp:368)
    const Lay L = make_lay(g, loc);
    dim3 block(32, 8, 1);
    dim3 grid((L.nx + 31) / 32, (L.ny + 7) / 8, L.nz);
    ProfScope ps(kKOther, s);
    k_tg_init<<<grid, block, 0, s>>>(g, mode, loc, f[loc]);
    OFB_LAUNCH_CHECK("k_tg_init");
  }
}

}  // namespace ofb
