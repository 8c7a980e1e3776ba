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
  // partition (warp-scan) solver, used when 64 <= n <= 1024 (n a multiple of
  // 32 on periodic axes; wall lines are padded to a multiple of 32):
  // per-lane segment factors, spikes and the interface operator, all laid
  // out [element][lane] so that a warp reads them with one coalesced load
  bool partition = false;
  int seg = 0;              // K = ceil(n / 32)
  size_t poff = 0;          // offset: cu[K][32], ip[K][32], v[K][32], w[K][32], gl[64][32], gr[64][32]
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
      if(n >= 64 && (n + 31) / 32 <= 32 && (n % 32 == 0 || !periodic)) {
        // Warp-scan form of the two Thomas recurrences (lane p owns the
        // unknowns q = pK + j, j < K):
        //   forward  m_q = ip_q r_q + f_q m_{q-1},  f_q = -lower ip_q
        //   backward x_q = m_q + g_q x_{q+1},       g_q = -cu_q
        // Lane-local products of f (resp. g) and the per-step multipliers of
        // the Kogge-Stone scans are line-independent and stored here.  A line
        // whose n is not a multiple of 32 (walls) is padded to 32 K unknowns
        // with ip = cu = 0: the padding decouples (m = x = 0 there) and the
        // real unknowns are unchanged.  Periodic lines are not padded (the
        // Sherman-Morrison update reads the last unknown from lane 31).
        const int P = 32, K = (n + 31) / 32;
        std::vector<double> fB(K * P), gD(K * P), ipj(K * P), cuj(K * P), zj(K * P);
        std::vector<double> mf(5 * P, 0.0), mb(5 * P, 0.0);
        std::vector<double> lane_f(P), lane_g(P);
        for(int lane = 0; lane < P; ++lane) {
          double prod = 1.0;
          for(int j = 0; j < K; ++j) {
            const int q = lane * K + j;
            const double ipq = q < n ? ip[q] : 0.0;
            const double f = q == 0 ? 0.0 : -(-beta) * ipq;
            prod = j == 0 ? f : prod * f;
            fB[j * P + lane] = prod;
            ipj[j * P + lane] = ipq;
            cuj[j * P + lane] = q < n ? cu[q] : 0.0;
            zj[j * P + lane] = q < n ? z[q] : 0.0;
          }
          lane_f[lane] = prod;  // m_end = A + prod * m_in
          double dprod = 1.0;
          for(int j = K - 1; j >= 0; --j) {
            const int q = lane * K + j;
            const double g = q < n ? -cu[q] : 0.0;
            dprod = j == K - 1 ? g : dprod * g;
            gD[j * P + lane] = dprod;
          }
          lane_g[lane] = dprod;  // x_first = C + dprod * x_in
        }
        // Kogge-Stone multipliers: inclusive scan of (a, b) maps; step s
        // combines lane p with lane p - 2^s (forward) / p + 2^s (backward)
        std::vector<double> cf = lane_f, cb = lane_g;
        for(int st = 0; st < 5; ++st) {
          const int d = 1 << st;
          std::vector<double> nf = cf, nb = cb;
          for(int lane = 0; lane < P; ++lane) {
            mf[st * P + lane] = lane >= d ? cf[lane] : 0.0;
            if(lane >= d) nf[lane] = cf[lane] * cf[lane - d];
            mb[st * P + lane] = lane + d < P ? cb[lane] : 0.0;
            if(lane + d < P) nb[lane] = cb[lane] * cb[lane + d];
          }
          cf = nf;
          cb = nb;
        }
        A.partition = true;
        A.seg = K;
        A.poff = host.size();
        for(auto* v : {&ipj, &fB, &cuj, &gD, &zj}) host.insert(host.end(), v->begin(), v->end());
        host.insert(host.end(), mf.begin(), mf.end());
        host.insert(host.end(), mb.begin(), mb.end());
      }
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

void adi_axis_geometry(const AdiPlan* p, int comp, int axis, int* begin, int* n) {
  *begin = p->ax[comp][axis].begin;
  *n = p->ax[comp][axis].n;
}

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

// Shared-memory line solver: one warp stages `lines` whole lines in shared
// memory (coalesced: x-lines load row segments, y/z-lines load 32 adjacent
// i-lines so each warp load is one contiguous row), solves them there with
// the shared Thomas factors and the Sherman-Morrison update, and stores them
// back coalesced.  Lines of an x-sweep are stored [line][n + 1] (the pad
// spreads a warp's column accesses over the banks), lines of a y/z sweep
// [n][lines] (a warp reads one row).
template <bool XLINES>
__global__ void __launch_bounds__(32) k_adi_tile(SweepArgs a, const double* __restrict__ in,
                                                 double* __restrict__ out, int lines) {
  extern __shared__ double tile[];
  const Lay& L = a.L;
  const int axis = a.axis;
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int n = a.n;
  const int st = L.stride(axis);
  const int t = threadIdx.x;
  const int n1 = L.n(a1);
  const int n2 = L.n(a2);
  // line l of this block -> storage base of its position 0 along the axis
  auto line_base = [&](int l, bool& ok) {
    int c1, c2;
    if(XLINES) {
      const int flat = blockIdx.x * lines + l;
      c1 = flat % n1;
      c2 = flat / n1;
      ok = c2 < n2;
    } else {
      c1 = blockIdx.x * lines + l;
      c2 = blockIdx.y;
      ok = c1 < n1;
    }
    if(!ok) {
      c1 = 0;
      c2 = 0;
    }
    int c[3] = {0, 0, 0};
    c[a1] = c1 + 1;
    c[a2] = c2 + 1;
    return L.idx(c[0], c[1], c[2]) + a.begin * st;
  };
  auto at = [&](int l, int q) -> double& {
    return XLINES ? tile[l * (n + 1) + q] : tile[q * lines + l];
  };
  // load
  if(XLINES) {
    for(int l = 0; l < lines; ++l) {
      bool ok;
      const int base = line_base(l, ok);
      if(!ok) continue;
      for(int q = t; q < n; q += 32) at(l, q) = in[base + q];
    }
  } else {
    for(int q = 0; q < n; ++q) {
      for(int l = t; l < lines; l += 32) {
        bool ok;
        const int base = line_base(l, ok);
        if(ok) at(l, q) = in[base + q * st];
      }
    }
  }
  __syncwarp();
  // solve line t
  if(t < lines) {
    double r = at(t, 0) + a.rhs_first;
    if(n == 1) r += a.rhs_last;
    double m = r * __ldg(&a.ip[0]);
    at(t, 0) = m;
    for(int q = 1; q < n; ++q) {
      double rq = at(t, q);
      if(q == n - 1) rq += a.rhs_last;
      m = (rq - a.lower * m) * __ldg(&a.ip[q]);
      at(t, q) = m;
    }
    const double x_last = m;
    double x = m;
    for(int q = n - 2; q >= 0; --q) {
      x = at(t, q) - __ldg(&a.cu[q]) * x;
      at(t, q) = x;
    }
    if(a.periodic && n > 1) {
      const double factor = (x + a.uc_over_gamma * x_last) * a.inv_den;
      for(int q = 0; q < n; ++q) at(t, q) -= factor * __ldg(&a.z[q]);
    }
  }
  __syncwarp();
  // store (and the duplicated periodic face)
  if(XLINES) {
    for(int l = 0; l < lines; ++l) {
      bool ok;
      const int base = line_base(l, ok);
      if(!ok) continue;
      for(int q = t; q < n; q += 32) out[base + q] = at(l, q);
      if(a.copy_duplicate && t == 0) out[base - a.begin * st + a.dup_index * st] = at(l, 0);
    }
  } else {
    for(int q = 0; q < n; ++q) {
      for(int l = t; l < lines; l += 32) {
        bool ok;
        const int base = line_base(l, ok);
        if(ok) out[base + q * st] = at(l, q);
      }
    }
    if(a.copy_duplicate) {
      for(int l = t; l < lines; l += 32) {
        bool ok;
        const int base = line_base(l, ok);
        if(ok) out[base - a.begin * st + a.dup_index * st] = at(l, 0);
      }
    }
  }
}

constexpr size_t kAdiTileBytes = 64 * 1024;

struct ScanArgs {
  const double* ip;  // [K][32]
  const double* fB;  // lane-local forward products
  const double* cu;
  const double* gD;  // lane-local backward products
  const double* z;   // Sherman-Morrison vector
  const double* mf;  // [5][32] forward scan multipliers
  const double* mb;  // [5][32] backward scan multipliers
  int K;
};

// Warp-scan line solver: a block of LB warps stages LB lines in shared
// memory (element q = pK + j of a line at [j][p], so a warp's accesses are
// conflict-free); warp w solves line w.  Lane p evaluates its K forward
// elimination steps as an affine map of the unknown carried in from lane p-1,
// the 32 maps are composed by a Kogge-Stone scan over shuffles, and the same
// is done for back substitution; the periodic Sherman-Morrison update
// (solver/projection.cpp:607-616) follows.  Same Thomas factors as the
// reference's recurrences; the association of the products differs, so
// results agree to rounding.
template <bool XLINES, int LB>
__global__ void __launch_bounds__(32 * LB) k_adi_scan(SweepArgs a, ScanArgs sa,
                                                      const double* __restrict__ in,
                                                      double* __restrict__ out) {
  extern __shared__ double tile[];
  const Lay& L = a.L;
  const int axis = a.axis;
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const int n = a.n;
  const int K = sa.K;
  const int S = 32 * K + 1;  // per-line stride in the tile (n padded to 32 K)
  const int st = L.stride(axis);
  const int n1 = L.n(a1), n2 = L.n(a2);
  const int tid = threadIdx.x + 32 * threadIdx.y;
  const int lane = threadIdx.x, wl = threadIdx.y;
  auto line_base = [&](int l, bool& ok) {
    int c1, c2;
    if(XLINES) {
      const int flat = blockIdx.x * LB + l;
      c1 = flat % n1;
      c2 = flat / n1;
      ok = c2 < n2;
    } else {
      c1 = blockIdx.x * LB + l;
      c2 = blockIdx.y;
      ok = c1 < n1;
    }
    if(!ok) c1 = c2 = 0;
    int c[3] = {0, 0, 0};
    c[a1] = c1 + 1;
    c[a2] = c2 + 1;
    return L.idx(c[0], c[1], c[2]) + a.begin * st;
  };
  // element q = pK + j of a line sits at row j, column (p + rot j) mod 32 of
  // the line's tile.  On x lines a warp stages consecutive q (32 / K
  // consecutive p per j): the rotation spreads those accesses over all bank
  // groups and keeps the solve's row accesses (fixed j, lanes p = 0..31) a
  // permutation.  Other lines stage 16 lines x 2 elements per warp, already
  // spread by the odd line stride, so they keep rot = 0.
  const int rot = XLINES ? (K < 32 ? 32 / K : 1) : 0;
  auto col = [&](int j, int p) { return j * 32 + ((p + rot * j) & 31); };
  auto slot = [&](int l, int q) { return l * S + col(q % K, q / K); };
  // staged lines; the padding past n is zero
  if(XLINES) {
    bool ok;
    const int base = line_base(wl, ok);
    if(ok)
      for(int q = lane; q < 32 * K; q += 32) tile[slot(wl, q)] = q < n ? in[base + q] : 0.0;
  } else {
    const int l = tid % LB;
    bool ok;
    const int base = line_base(l, ok);
    if(ok)
      for(int q = tid / LB; q < 32 * K; q += 32) tile[slot(l, q)] = q < n ? in[base + q * st] : 0.0;
  }
  __syncthreads();
  {
    double* line = tile + wl * S;
    // forward elimination, lane-local part: m_{pK+j} = A_j + fB_j m_in
    double acc = 0.0;
    for(int j = 0; j < K; ++j) {
      const int q = lane * K + j;
      double r = line[col(j, lane)];
      if(q == 0) r += a.rhs_first;
      if(q == n - 1) r += a.rhs_last;
      const double ipq = __ldg(&sa.ip[j * 32 + lane]);
      // f_q = lower_coupling * ip_q with the coupling -(-beta) folded in
      const double f = q == 0 ? 0.0 : -a.lower * ipq;
      acc = j == 0 ? r * ipq : r * ipq + f * acc;
      line[col(j, lane)] = acc;  // A_j
    }
    // inclusive scan of lane maps: val = m at the lane's last unknown
    double val = acc;
#pragma unroll
    for(int s = 0; s < 5; ++s) {
      const double up = __shfl_up_sync(0xffffffffu, val, 1 << s);
      val += __ldg(&sa.mf[s * 32 + lane]) * up;
    }
    double m_in = __shfl_up_sync(0xffffffffu, val, 1);
    if(lane == 0) m_in = 0.0;
    for(int j = 0; j < K; ++j) {
      const double v = line[col(j, lane)] + __ldg(&sa.fB[j * 32 + lane]) * m_in;
      line[col(j, lane)] = v;  // m_q
    }
    // back substitution, lane-local: x_{pK+j} = C_j + gD_j x_in
    double cacc = 0.0;
    for(int j = K - 1; j >= 0; --j) {
      const double mq = line[col(j, lane)];
      cacc = j == K - 1 ? mq : mq - __ldg(&sa.cu[j * 32 + lane]) * cacc;
      line[col(j, lane)] = cacc;  // C_j
    }
    double bval = cacc;
#pragma unroll
    for(int s = 0; s < 5; ++s) {
      const double dn = __shfl_down_sync(0xffffffffu, bval, 1 << s);
      bval += __ldg(&sa.mb[s * 32 + lane]) * dn;
    }
    double x_in = __shfl_down_sync(0xffffffffu, bval, 1);
    if(lane == 31) x_in = 0.0;
    double x0 = 0.0, xl = 0.0;
    for(int j = 0; j < K; ++j) {
      const double x = line[col(j, lane)] + __ldg(&sa.gD[j * 32 + lane]) * x_in;
      line[col(j, lane)] = x;
      if(j == 0) x0 = x;
      if(j == K - 1) xl = x;
    }
    if(a.periodic) {
      const double first = __shfl_sync(0xffffffffu, x0, 0);
      const double last = __shfl_sync(0xffffffffu, xl, 31);
      const double factor = (first + a.uc_over_gamma * last) * a.inv_den;
      for(int j = 0; j < K; ++j) line[col(j, lane)] -= factor * __ldg(&sa.z[j * 32 + lane]);
    }
  }
  __syncthreads();
  if(XLINES) {
    bool ok;
    const int base = line_base(wl, ok);
    if(ok) {
      for(int q = lane; q < n; q += 32) out[base + q] = tile[slot(wl, q)];
      if(a.copy_duplicate && lane == 0) out[base - a.begin * st + a.dup_index * st] = tile[slot(wl, 0)];
    }
  } else {
    const int l = tid % LB;
    bool ok;
    const int base = line_base(l, ok);
    if(ok) {
      for(int q = tid / LB; q < n; q += 32) out[base + q * st] = tile[slot(l, q)];
      if(a.copy_duplicate && tid < LB) out[base - a.begin * st + a.dup_index * st] = tile[slot(l, 0)];
    }
  }
}

template <int LB>
void launch_scan(const SweepArgs& a, const ScanArgs& sa, int axis, int a1, int a2, const double* in,
                 double* out, cudaStream_t s) {
  const size_t smem = static_cast<size_t>(LB) * (32 * sa.K + 1) * sizeof(double);
  const dim3 block(32, LB, 1);
  if(axis == 0) {
    const long long nl = static_cast<long long>(a.L.n(a1)) * a.L.n(a2);
    const dim3 grid(static_cast<unsigned>((nl + LB - 1) / LB), 1, 1);
    OFB_CHECK(cudaFuncSetAttribute(k_adi_scan<true, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    k_adi_scan<true, LB><<<grid, block, smem, s>>>(a, sa, in, out);
  } else {
    const dim3 grid((a.L.n(a1) + LB - 1) / LB, a.L.n(a2), 1);
    OFB_CHECK(cudaFuncSetAttribute(k_adi_scan<false, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    k_adi_scan<false, LB><<<grid, block, smem, s>>>(a, sa, in, out);
  }
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
  ProfScope ps(kKAdi, s);
  if(A.partition) {
    ScanArgs sa;
    sa.K = A.seg;
    const int KP = A.seg * 32;
    const double* base = p->coef + A.poff;
    sa.ip = base;
    sa.fB = base + KP;
    sa.cu = base + 2 * KP;
    sa.gD = base + 3 * KP;
    sa.z = base + 4 * KP;
    sa.mf = base + 5 * KP;
    sa.mb = base + 5 * KP + 5 * 32;
    // 16 lines per block; 4 when that leaves fewer than two blocks per SM
    // (few long lines, e.g. a 2D sweep)
    const long long nl = static_cast<long long>(a.L.n(a1)) * a.L.n(a2);
    if((nl + 15) / 16 >= 2LL * 148)
      launch_scan<16>(a, sa, axis, a1, a2, in, out, s);
    else
      launch_scan<4>(a, sa, axis, a1, a2, in, out, s);
    OFB_LAUNCH_CHECK("k_adi_scan");
    return;
  }
  // lines per warp so that one tile fits kAdiTileBytes (32 when n <= 255)
  int lines = 32;
  while(lines > 1 && static_cast<size_t>(lines) * (a.n + 1) * sizeof(double) > kAdiTileBytes) lines /= 2;
  const size_t smem = static_cast<size_t>(lines) * (a.n + 1) * sizeof(double);
  if(axis == 0) {
    const long long nl = static_cast<long long>(a.L.n(a1)) * a.L.n(a2);
    dim3 grid(static_cast<unsigned>((nl + lines - 1) / lines), 1, 1);
    OFB_CHECK(cudaFuncSetAttribute(k_adi_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    k_adi_tile<true><<<grid, 32, smem, s>>>(a, in, out, lines);
  } else {
    dim3 grid((a.L.n(a1) + lines - 1) / lines, a.L.n(a2), 1);
    OFB_CHECK(cudaFuncSetAttribute(k_adi_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    k_adi_tile<false><<<grid, 32, smem, s>>>(a, in, out, lines);
  }
  OFB_LAUNCH_CHECK("k_adi_tile");
}

}  // namespace ofb
