// ADI predictor sweeps (solve_component_sweep / solve_component_sweep_periodic,
// solver/projection.cpp:619-866).  Every line of one (component, axis) sweep
// has the same constant-coefficient tridiagonal matrix -- Toeplitz with
// Dirichlet/ghost-relation end rows on walls, cyclic with Sherman-Morrison on
// periodic axes -- so the Thomas factors (modified upper diagonal and inverse
// pivots) and the Sherman-Morrison correction vector are computed once on the
// host in FP64 and shared.  On the device one thread solves one line: forward
// elimination, back substitution and the Sherman-Morrison update, in place in
// the output field.  Threads of a warp own adjacent lines, so y and z sweeps
// read and write unit-stride rows.
#include "kernels.hpp"

#include <cmath>
#include <vector>

namespace ofb {

struct AdiAxis {
  bool active = false;      // sweep runs (n > 0)
  bool periodic = false;
  bool copy_duplicate = false;
  int n = 0;                // unknowns per line
  int begin = 0;            // storage index of the first unknown
  int dup_index = 0;        // storage index of the duplicated periodic face
  int lines = 0;
  double lower = 0.0;       // sub-diagonal (rows 1..n-1)
  double rhs_first = 0.0;   // constants added to rhs[0], rhs[n-1] on walls
  double rhs_last = 0.0;
  double uc_over_gamma = 0.0;
  double inv_den = 0.0;
  size_t off = 0;           // offset of cu/ip/z in the coefficient buffer
};

struct AdiPlan {
  Grid g;
  AdiAxis ax[3][3];  // [component][axis]
  double* coef = nullptr;  // device: per (comp, axis): cu[n], ip[n], z[n]
};

namespace {

double tangential_coef(int type) {
  return (type == kNoSlip || type == kPrescribed) ? -1.0 : (type == kSymmetry || type == kFixedPressure) ? 1.0 : 0.0;
}

}  // namespace

AdiPlan* adi_plan_create(const Grid& g, const VBC& bc, double alpha) {
  AdiPlan* p = new AdiPlan();
  p->g = g;
  std::vector<double> host;
  for(int c = 0; c < 3; ++c) {
    const Lay L = make_lay(g, kFaceX + c);
    for(int a = 0; a < 3; ++a) {
      AdiAxis& A = p->ax[c][a];
      const double h = g.h(a);
      const double beta = alpha / (h * h);
      const bool periodic = bc.type[2 * a] == kPeriodic;
      int begin = 1, end = 1 + L.n(a);
      if(periodic) {
        if(c == a) end -= 1;
      } else if(c == a) {
        begin += is_dirichlet_velocity(bc.type[2 * a]) ? 1 : 0;
        end -= is_dirichlet_velocity(bc.type[2 * a + 1]) ? 1 : 0;
      }
      const int n = end - begin;
      int a1 = a == 0 ? 1 : 0, a2 = a == 2 ? 1 : 2;
      A.lines = L.n(a1) * L.n(a2);
      if(n <= 0) continue;
      A.active = true;
      A.periodic = periodic;
      A.n = n;
      A.begin = begin;
      A.copy_duplicate = periodic && c == a;
      A.dup_index = L.n(a);  // active_end - 1
      A.lower = -beta;
      std::vector<double> di(n, 1.0 + 2.0 * beta), up(n, -beta), lo(n, -beta);
      lo[0] = 0.0;
      up[n - 1] = 0.0;
      std::vector<double> cu(n), ip(n), z(n, 0.0);
      if(periodic) {
        const double lc = -beta, uc = -beta;
        if(n == 1) {
          // solve_cyclic_tridiagonal n == 1 (solver/projection.cpp:574-581)
          const double pivot = di[0] + lc + uc;
          if(std::fabs(pivot) < 1.0e-30) {
            delete p;
            throw std::runtime_error("cyclic tridiagonal solve encountered a zero pivot");
          }
          cu[0] = 0.0;
          ip[0] = 1.0 / pivot;
          A.uc_over_gamma = 0.0;
          A.inv_den = 0.0;
        } else {
          const double gamma = -di[0];
          std::vector<double> dm = di;
          dm[0] = di[0] - gamma;
          dm[n - 1] = di[n - 1] - lc * uc / gamma;
          // Thomas factors of the modified matrix
          double pivot = dm[0];
          cu[0] = n > 1 ? up[0] / pivot : 0.0;
          ip[0] = 1.0 / pivot;
          for(int q = 1; q < n; ++q) {
            pivot = dm[q] - lo[q] * cu[q - 1];
            if(std::fabs(pivot) < 1.0e-30) {
              delete p;
              throw std::runtime_error("tridiagonal solve encountered a zero pivot");
            }
            cu[q] = q + 1 < n ? up[q] / pivot : 0.0;
            ip[q] = 1.0 / pivot;
          }
          // z = M^-1 u with u = (gamma, 0, ..., 0, lower_corner), as the
          // reference's second Thomas solve (solver/projection.cpp:600-605)
          std::vector<double> mr(n), uvec(n, 0.0);
          uvec[0] = gamma;
          uvec[n - 1] = lc;
          double pv = dm[0];
          std::vector<double> mu(n);
          mu[0] = up[0] / pv;
          mr[0] = uvec[0] / pv;
          for(int q = 1; q < n; ++q) {
            pv = dm[q] - lo[q] * mu[q - 1];
            mu[q] = q + 1 < n ? up[q] / pv : 0.0;
            mr[q] = (uvec[q] - lo[q] * mr[q - 1]) / pv;
          }
          z[n - 1] = mr[n - 1];
          for(int q = n - 1; q-- > 0;) z[q] = mr[q] - mu[q] * z[q + 1];
          const double den = 1.0 + z[0] + uc * z[n - 1] / gamma;
          if(std::fabs(den) < 1.0e-30) {
            delete p;
            throw std::runtime_error(
                "cyclic tridiagonal solve encountered a singular Sherman-Morrison update");
          }
          A.uc_over_gamma = uc / gamma;
          A.inv_den = 1.0 / den;
        }
      } else {
        // wall rows (solver/projection.cpp:757-780)
        const int lo_t = bc.type[2 * a], hi_t = bc.type[2 * a + 1];
        double r0 = 0.0, rn = 0.0;
        if(c == a && is_dirichlet_velocity(lo_t)) {
          r0 += beta * bc.vel[2 * a][a];
        } else {
          di[0] -= beta * tangential_coef(lo_t);
          r0 += beta * ((lo_t == kNoSlip || lo_t == kPrescribed) ? 2.0 * bc.vel[2 * a][c] : 0.0);
        }
        if(c == a && is_dirichlet_velocity(hi_t)) {
          rn += beta * bc.vel[2 * a + 1][a];
        } else {
          di[n - 1] -= beta * tangential_coef(hi_t);
          rn += beta * ((hi_t == kNoSlip || hi_t == kPrescribed) ? 2.0 * bc.vel[2 * a + 1][c] : 0.0);
        }
        A.rhs_first = r0;
        A.rhs_last = rn;
        double pivot = di[0];
        if(std::fabs(pivot) < 1.0e-30) {
          delete p;
          throw std::runtime_error("tridiagonal solve encountered a zero pivot");
        }
        cu[0] = n > 1 ? up[0] / pivot : 0.0;
        ip[0] = 1.0 / pivot;
        for(int q = 1; q < n; ++q) {
          pivot = di[q] - lo[q] * cu[q - 1];
          if(std::fabs(pivot) < 1.0e-30) {
            delete p;
            throw std::runtime_error("tridiagonal solve encountered a zero pivot");
          }
          cu[q] = q + 1 < n ? up[q] / pivot : 0.0;
          ip[q] = 1.0 / pivot;
        }
      }
      A.off = host.size();
      host.insert(host.end(), cu.begin(), cu.end());
      host.insert(host.end(), ip.begin(), ip.end());
      host.insert(host.end(), z.begin(), z.end());
    }
  }
  if(!host.empty()) {
    OFB_CHECK(cudaMalloc(&p->coef, host.size() * sizeof(double)));
    OFB_CHECK(cudaMemcpy(p->coef, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  return p;
}

void adi_plan_destroy(AdiPlan* p) {
  if(p == nullptr) return;
  if(p->coef) cudaFree(p->coef);
  delete p;
}

int adi_line_count(const AdiPlan* p, int comp, int axis) {
  return p->ax[comp][axis].active ? p->ax[comp][axis].lines : 0;
}

bool adi_axis_active(const AdiPlan* p, int comp, int axis) { return p->ax[comp][axis].active; }

namespace {

struct SweepArgs {
  Lay L;
  int axis;
  int n, begin, dup_index, periodic, copy_duplicate;
  double lower, rhs_first, rhs_last, uc_over_gamma, inv_den;
  const double* cu;
  const double* ip;
  const double* z;
};

__global__ void __launch_bounds__(128) k_adi_sweep(SweepArgs a, const double* __restrict__ in,
                                                   double* __restrict__ out) {
  const Lay& L = a.L;
  const int axis = a.axis;
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int t1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t2 = blockIdx.y;
  if(t1 >= L.n(a1) || t2 >= L.n(a2)) return;
  int c[3] = {0, 0, 0};
  c[a1] = t1 + 1;
  c[a2] = t2 + 1;
  const int base = L.idx(c[0], c[1], c[2]);
  const int st = L.stride(axis);
  const int n = a.n;
  const double* __restrict__ src = in + base + a.begin * st;
  double* __restrict__ dst = out + base + a.begin * st;
  // forward elimination
  double r = src[0] + a.rhs_first;
  if(n == 1) r += a.rhs_last;
  double m = r * __ldg(&a.ip[0]);
  dst[0] = m;
  for(int q = 1; q < n; ++q) {
    double rq = src[q * st];
    if(q == n - 1) rq += a.rhs_last;
    m = (rq - a.lower * m) * __ldg(&a.ip[q]);
    dst[q * st] = m;
  }
  // back substitution
  const double x_last = m;
  double x = m;
  for(int q = n - 2; q >= 0; --q) {
    x = dst[q * st] - __ldg(&a.cu[q]) * x;
    dst[q * st] = x;
  }
  if(a.periodic && n > 1) {
    // Sherman-Morrison update (solver/projection.cpp:607-616)
    const double factor = (x + a.uc_over_gamma * x_last) * a.inv_den;
    for(int q = 0; q < n; ++q) dst[q * st] -= factor * __ldg(&a.z[q]);
  }
  if(a.copy_duplicate) out[base + a.dup_index * st] = dst[0];
}

}  // namespace

void launch_adi_sweep(const AdiPlan* p, int comp, int axis, const double* in, double* out,
                      cudaStream_t s) {
  const AdiAxis& A = p->ax[comp][axis];
  if(!A.active) return;
  SweepArgs a;
  a.L = make_lay(p->g, kFaceX + comp);
  a.axis = axis;
  a.n = A.n;
  a.begin = A.begin;
  a.dup_index = A.dup_index;
  a.periodic = A.periodic ? 1 : 0;
  a.copy_duplicate = A.copy_duplicate ? 1 : 0;
  a.lower = A.lower;
  a.rhs_first = A.rhs_first;
  a.rhs_last = A.rhs_last;
  a.uc_over_gamma = A.uc_over_gamma;
  a.inv_den = A.inv_den;
  a.cu = p->coef + A.off;
  a.ip = p->coef + A.off + A.n;
  a.z = p->coef + A.off + 2 * A.n;
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  dim3 block(128, 1, 1);
  dim3 grid((a.L.n(a1) + 127) / 128, a.L.n(a2), 1);
  ProfScope ps(kKAdi, s);
  k_adi_sweep<<<grid, block, 0, s>>>(a, in, out);
  OFB_LAUNCH_CHECK("k_adi_sweep");
}

}  // namespace ofb
