// Validation reductions of the case drivers: the Taylor-Green kinetic energy
// and velocity error against the analytic decay (solver/taylor_green.cpp:
// 263-333).  Both are deterministic two-stage reductions over the resident
// state; their totals land in a device array the caller reads back.
#include "kernels.hpp"

namespace ofb {

namespace {

// kinetic_energy (solver/taylor_green.cpp:269-289): the sum over cells of
// 1/2 |face-averaged velocity|^2.  out[0] = the sum (the caller divides by
// the cell count).
__global__ void k_kinetic_energy(Grid g, const double* u, const double* v, const double* w,
                                 RedBuf rb, double* out, int kchunk) {
  const Lay Lu = make_lay(g, kFaceX), Lv = make_lay(g, kFaceY), Lw = make_lay(g, kFaceZ);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, g.nz + 1);
  double acc = 0.0;
  if(i <= g.nx && j <= g.ny) {
    for(int k = k0; k < k1; ++k) {
      const double uc = 0.5 * (u[Lu.idx(i, j, k)] + u[Lu.idx(i + 1, j, k)]);
      const double vc = 0.5 * (v[Lv.idx(i, j, k)] + v[Lv.idx(i, j + 1, k)]);
      const double wc = 0.5 * (w[Lw.idx(i, j, k)] + w[Lw.idx(i, j, k + 1)]);
      acc += 0.5 * (uc * uc + vc * vc + wc * wc);
    }
  }
  double val[1] = {acc};
  const bool is_max[1] = {false};
  reduce_finish<1>(val, is_max, rb, [=](const Sums<1>& s) { out[0] = s.v[0]; });
}

// One component's share of velocity_relative_l2_error
// (solver/taylor_green.cpp:291-333): out[0] = sum (f - exact)^2,
// out[1] = sum exact^2 over the active entries, the exact field being the
// initial state (phase `mode`, as k_tg_init) times `decay`.
__global__ void k_tg_error(Grid g, int loc, int mode, double decay, const double* f, RedBuf rb,
                           double* out, int kchunk) {
  const Lay L = make_lay(g, loc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k0 = blockIdx.z * kchunk + 1;
  const int k1 = min(k0 + kchunk, L.nz + 1);
  const bool three_d = g.nz > 1;
  double num = 0.0, den = 0.0;
  if(i <= L.nx && j <= L.ny) {
    // coordinate_for_storage_index (core/field_layout.hpp:226-238)
    const double x = (loc == kFaceX) ? (i - 1) * g.dx : (i - 1 + 0.5) * g.dx;
    const double y = (loc == kFaceY) ? (j - 1) * g.dy : (j - 1 + 0.5) * g.dy;
    for(int k = k0; k < k1; ++k) {
      const double z = (loc == kFaceZ) ? (k - 1) * g.dz : (k - 1 + 0.5) * g.dz;
      const double zf = three_d ? cos(z) : 1.0;
      double ref = 0.0;
      if(loc == kFaceX)
        ref = (mode == 0 ? -cos(x) * sin(y) * zf : sin(x) * cos(y) * zf) * decay;
      else if(loc == kFaceY)
        ref = (mode == 0 ? sin(x) * cos(y) * zf : -cos(x) * sin(y) * zf) * decay;
      const double d = f[L.idx(i, j, k)] - ref;
      num += d * d;
      den += ref * ref;
    }
  }
  double val[2] = {num, den};
  const bool is_max[2] = {false, false};
  reduce_finish<2>(val, is_max, rb, [=](const Sums<2>& s) {
    out[0] = s.v[0];
    out[1] = s.v[1];
  });
}

}  // namespace

void launch_kinetic_energy(const Grid& g, const double* u, const double* v, const double* w,
                           RedBuf rb, double* out, cudaStream_t s) {
  const Launch3 l = launch3(g.nx, g.ny, g.nz);
  ProfScope ps(kKOther, s);
  k_kinetic_energy<<<l.grid, l.block, 0, s>>>(g, u, v, w, rb, out, l.kchunk);
  OFB_LAUNCH_CHECK("k_kinetic_energy");
}

void launch_tg_error(const Grid& g, int loc, int mode, double decay, const double* f, RedBuf rb,
                     double* out, cudaStream_t s) {
  const Lay L = make_lay(g, loc);
  const Launch3 l = launch3(L.nx, L.ny, L.nz);
  ProfScope ps(kKOther, s);
  k_tg_error<<<l.grid, l.block, 0, s>>>(g, loc, mode, decay, f, rb, out, l.kchunk);
  OFB_LAUNCH_CHECK("k_tg_error");
}

}  // namespace ofb
