// Momentum-side stencils: the fused predictor right-hand side (TVD/van Leer
// advection, diffusion, pressure gradient, factorisation correction and the
// AB2 combination in one pass), the stand-alone advection operator and the
// Taylor-Green initial state.
#include "kernels.hpp"

namespace ofb {

namespace {

constexpr double kSmallDenominator = 1.0e-14;  // solver/momentum_terms.cpp:14

__device__ __forceinline__ double van_leer(double r) {
  // limiter_value (solver/momentum_terms.cpp:26-33)
  const double a = fabs(r);
  return (r + a) / (1.0 + a);
}

__device__ __forceinline__ double safe_ratio(double num, double den) {
  // solver/momentum_terms.cpp:35-40
  return fabs(den) < kSmallDenominator ? 0.0 : num / den;
}

// reconstruct_face_{x,y,z} (solver/momentum_terms.cpp:42-151) for the face
// whose upper ("right") cell is q, along an axis with storage stride st;
// `ri` is the right cell's storage index on that axis and `smax` the last
// storage index.  Faces within two cells of the storage bounds fall back to
// first-order upwind, as in the reference.
__device__ __forceinline__ double reconstruct(const double* __restrict__ f, int q, int st, int ri,
                                              int smax, double vel) {
  const double left = f[q - st];
  const double right = f[q];
  if(fabs(vel) < kSmallDenominator) return vel >= 0.0 ? left : right;
  if(vel >= 0.0) {
    if(ri - 2 < 0) return left;
    const double delta_down = right - left;
    const double ratio = safe_ratio(left - f[q - 2 * st], delta_down);
    return left + 0.5 * van_leer(ratio) * delta_down;
  }
  if(ri + 1 > smax) return right;
  const double delta = right - left;
  const double ratio = safe_ratio(f[q + st] - right, delta);
  return right - 0.5 * van_leer(ratio) * delta;
}

// compute_{u,v,w}_advection (solver/momentum_terms.cpp:153-266) at storage
// point (i, j, k) of component C.
template <int C>
__device__ __forceinline__ double advection_at(const Grid& g, const double* __restrict__ const* vel,
                                               int i, int j, int k, const double (&inv_h)[3]) {
  const Lay L = make_lay(g, kFaceX + C);
  const double* __restrict__ f = vel[C];
  const int q = L.idx(i, j, k);
  const int pos[3] = {i, j, k};
  double flux_div = 0.0;
#pragma unroll
  for(int d = 0; d < 3; ++d) {
    double lo_vel, hi_vel;
    const int std_ = L.stride(d);
    if(d == C) {
      lo_vel = 0.5 * (f[q - std_] + f[q]);
      hi_vel = 0.5 * (f[q] + f[q + std_]);
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
    const int smax = L.s(d) - 1;
    const double lo_flux = lo_vel * reconstruct(f, q, std_, pos[d], smax, lo_vel);
    const double hi_flux = hi_vel * reconstruct(f, q + std_, std_, pos[d] + 1, smax, hi_vel);
    flux_div += (hi_flux - lo_flux) * inv_h[d];
  }
  return flux_div;
}

template <int C>
__global__ void __launch_bounds__(kTX* kTY) k_predictor_rhs(PredictorArgs a, int kchunk) {
  const Grid& g = a.g;
  const Lay L = make_lay(g, kFaceX + C);
  const Lay P = make_lay(g, kCell);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > L.nx || j > L.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const double inv_h[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  const double ix = 1.0 / (g.dx * g.dx), iy = 1.0 / (g.dy * g.dy), iz = 1.0 / (g.dz * g.dz);
  const double dy2 = g.dy * g.dy;
  const bool three_d = g.nz != 1;
  const double s_gp = -a.dt;
  const double s_dif = 0.5 * a.dt;
  const double s_adv = a.has_prev ? -1.5 * a.dt : -a.dt;
  const double s_prev = 0.5 * a.dt;
  const double s_corr = a.alpha * a.alpha;
  const double* __restrict__ f = a.cur[C];
  const int stC = L.stride(C);
  const int pstC = P.stride(C);
  for(int k = k0; k < k1; ++k) {
    const int q = L.idx(i, j, k);
    // 27-point neighbourhood v[dz][dy][dx]
    double v[3][3][3];
#pragma unroll
    for(int c = 0; c < 3; ++c)
#pragma unroll
      for(int b = 0; b < 3; ++b)
#pragma unroll
        for(int e = 0; e < 3; ++e) v[c][b][e] = f[q + (e - 1) + (b - 1) * L.sx + (c - 1) * L.sxy];

    const double adv = advection_at<C>(g, a.cur, i, j, k, inv_h);
    // compute_diffusion_term: (d2x + d2y + d2z) * nu
    const double c2 = 2.0 * v[1][1][1];
    const double lap = (v[1][1][2] - c2 + v[1][1][0]) * ix + (v[1][2][1] - c2 + v[1][0][1]) * iy +
                       (v[2][1][1] - c2 + v[0][1][1]) * iz;
    const double dif = lap * a.nu;
    // compute_gradient of the total pressure onto this face
    int pc[3] = {i, j, k};
    const int pq = P.idx(pc[0], pc[1], pc[2]);
    const double gp = (a.p[pq] - a.p[pq - pstC]) * inv_h[C];
    // factorisation correction (solver/taylor_green.cpp:196-225,
    // solver/lid_driven_cavity.cpp:219-252)
    double corr;
    if(a.variant == 1) {
      double dyy[3];
#pragma unroll
      for(int e = 0; e < 3; ++e) dyy[e] = (v[1][2][e] - 2.0 * v[1][1][e] + v[1][0][e]) / dy2;
      corr = (dyy[2] - 2.0 * dyy[1] + dyy[0]) * ix;
    } else {
      double d2y[3];
#pragma unroll
      for(int e = 0; e < 3; ++e) d2y[e] = (v[1][2][e] - 2.0 * v[1][1][e] + v[1][0][e]) * iy;
      corr = (d2y[2] - 2.0 * d2y[1] + d2y[0]) * ix;
      if(three_d) {
        double d2z[3][3];  // [dy][dx]
#pragma unroll
        for(int b = 0; b < 3; ++b)
#pragma unroll
          for(int e = 0; e < 3; ++e) d2z[b][e] = (v[2][b][e] - 2.0 * v[1][b][e] + v[0][b][e]) * iz;
        const double mxz = (d2z[1][2] - 2.0 * d2z[1][1] + d2z[1][0]) * ix;
        double myz[3];
#pragma unroll
        for(int e = 0; e < 3; ++e) myz[e] = (d2z[2][e] - 2.0 * d2z[1][e] + d2z[0][e]) * iy;
        const double triple = (myz[2] - 2.0 * myz[1] + myz[0]) * ix;
        corr += mxz;
        corr += myz[1];
        corr -= a.alpha * triple;
      }
    }
    // assemble_predictor_rhs (solver/taylor_green.cpp:244-255)
    double r = v[1][1][1];
    r += s_gp * gp;
    r += s_dif * dif;
    r += s_adv * adv;
    if(a.has_prev) r += s_prev * a.prev[C][q];
    r += s_corr * corr;
    a.adv[C][q] = adv;
    a.rhs[C][q] = r;
    (void)stC;
  }
}

template <int C>
__global__ void __launch_bounds__(kTX* kTY) k_advection(Grid g, const double* u, const double* v,
                                                        const double* w, double* out, int kchunk) {
  const Lay L = make_lay(g, kFaceX + C);
  const int i = blockIdx.x * kTX + threadIdx.x + 1;
  const int j = blockIdx.y * kTY + threadIdx.y + 1;
  if(i > L.nx || j > L.ny) return;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const double inv_h[3] = {1.0 / g.dx, 1.0 / g.dy, 1.0 / g.dz};
  const double* vel[3] = {u, v, w};
  for(int k = k0; k < k1; ++k) out[L.idx(i, j, k)] = advection_at<C>(g, vel, i, j, k, inv_h);
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
  ProfScope ps(kKPredictor, s, 3);
  Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  k_predictor_rhs<0><<<l0.grid, l0.block, 0, s>>>(a, l0.kchunk);
  OFB_LAUNCH_CHECK("k_predictor_rhs<0>");
  Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  k_predictor_rhs<1><<<l1.grid, l1.block, 0, s>>>(a, l1.kchunk);
  OFB_LAUNCH_CHECK("k_predictor_rhs<1>");
  Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_predictor_rhs<2><<<l2.grid, l2.block, 0, s>>>(a, l2.kchunk);
  OFB_LAUNCH_CHECK("k_predictor_rhs<2>");
}

void launch_advection(const Grid& g, const double* u, const double* v, const double* w,
                      double* au, double* av, double* aw, cudaStream_t s) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  ProfScope ps(kKOther, s, 3);
  Launch3 l0 = launch3(Lu.nx, Lu.ny, Lu.nz);
  k_advection<0><<<l0.grid, l0.block, 0, s>>>(g, u, v, w, au, l0.kchunk);
  Launch3 l1 = launch3(Lv.nx, Lv.ny, Lv.nz);
  k_advection<1><<<l1.grid, l1.block, 0, s>>>(g, u, v, w, av, l1.kchunk);
  Launch3 l2 = launch3(Lw.nx, Lw.ny, Lw.nz);
  k_advection<2><<<l2.grid, l2.block, 0, s>>>(g, u, v, w, aw, l2.kchunk);
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
