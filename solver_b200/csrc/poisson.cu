// Multigrid-preconditioned CG for the pressure Poisson problem
// (linsolve/poisson_solver.cpp:678-809) on compact, ghost-free vectors.
//
// Algorithm: the reference's exactly -- PCG on A = -Lap_h with BC-aware
// neighbours (:195-269), one V(2,2) cycle per iteration with damped Jacobi
// (omega = 2/3), 2x2x2 cell-average restriction, piecewise-constant
// prolongation and a dense partially-pivoted Gaussian elimination on the
// coarsest grid, and the zero-mean projection on singular (periodic /
// all-Neumann) problems after every update.
//
// B200 form: each vector update is one kernel that also produces the sums the
// next step needs (deterministic two-stage reduction, common.cuh).  A mean
// removal is never a separate pass: the kernel that produces a vector records
// its mean as a pending shift, and every consumer subtracts the shift as it
// loads the vector -- the same arithmetic as the reference's
// subtract_active_mean, one kernel later.  The Jacobi diagonal is a 64-entry
// table per level (it only depends on whether a cell touches a boundary), the
// V-cycle's residual is restricted on the fly (never stored) and the
// prolongation is folded into the first post-smoothing sweep.  The V-cycle
// storage type T is double (OF_FP64) or float (OF_MIXED: FP32 storage and
// arithmetic inside the FP64 CG loop).
#include "kernels.hpp"
#include "vstencil.cuh"
#include "tma.cuh"

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <type_traits>
#include <vector>

namespace ofb {

namespace {

constexpr double kSmallNumber = 1.0e-30;
constexpr double kOmega = 2.0 / 3.0;
constexpr int kMaxCoarse = 1024;

struct OpInfo {
  CLay L;
  double inv2[3];  // 1 / h^2
  int periodic[3];
  int dir_lo[3], dir_hi[3];  // homogeneous Dirichlet (else Neumann) at each end
  const double* invd;        // 64-entry inverse-diagonal table
};

__device__ __forceinline__ int axis_class(int c, int n) {
  return n == 1 ? 3 : (c == 0 ? 1 : (c == n - 1 ? 2 : 0));
}

__device__ __forceinline__ double inv_diag(const OpInfo& o, int i, int j, int k) {
  const int t = axis_class(i, o.L.nx) + 4 * axis_class(j, o.L.ny) + 16 * axis_class(k, o.L.nz);
  return __ldg(&o.invd[t]);
}

// Neighbour coordinates along one axis, branch-free: the in-range neighbour,
// the periodic image, or the cell itself with sign +1 (homogeneous Neumann,
// ghost = centre) or -1 (homogeneous Dirichlet, ghost = -centre)
// (neighbor_value, linsolve/poisson_solver.cpp:195-242).  Every load is then
// unconditional and in bounds, so a thread can keep many loads in flight.
__device__ __forceinline__ void nb_lo(int c, int n, int per, int dir, int& cc, double& sg) {
  const bool in = c > 0;
  cc = in ? c - 1 : (per ? n - 1 : c);
  sg = (in || per || !dir) ? 1.0 : -1.0;
}

__device__ __forceinline__ void nb_hi(int c, int n, int per, int dir, int& cc, double& sg) {
  const bool in = c < n - 1;
  cc = in ? c + 1 : (per ? 0 : c);
  sg = (in || per || !dir) ? 1.0 : -1.0;
}

// In-plane neighbours of one (i, j) column; fixed while the thread marches in k.
struct ColNb {
  int xl, xr, yd, yu;
  double sxl, sxr, syd, syu;
};

__device__ __forceinline__ ColNb col_nb(const OpInfo& o, int i, int j) {
  ColNb c;
  nb_lo(i, o.L.nx, o.periodic[0], o.dir_lo[0], c.xl, c.sxl);
  nb_hi(i, o.L.nx, o.periodic[0], o.dir_hi[0], c.xr, c.sxr);
  nb_lo(j, o.L.ny, o.periodic[1], o.dir_lo[1], c.yd, c.syd);
  nb_hi(j, o.L.ny, o.periodic[1], o.dir_hi[1], c.yu, c.syu);
  return c;
}

// apply_poisson_operator at (i, j, k) (linsolve/poisson_solver.cpp:244-269):
// -(r - 2c + l)/dx^2 - (u - 2c + d)/dy^2 - (f - 2c + b)/dz^2 with the boundary
// rules above.  val(i, j, k) returns the operand at an in-range cell.
template <typename A, typename F>
__device__ __forceinline__ A apply_op(const OpInfo& o, const ColNb& nb, int i, int j, int k, F val,
                                      A& center) {
  int kb, kf;
  double sb, sf;
  nb_lo(k, o.L.nz, o.periodic[2], o.dir_lo[2], kb, sb);
  nb_hi(k, o.L.nz, o.periodic[2], o.dir_hi[2], kf, sf);
  const A c = val(i, j, k);
  const A l = A(nb.sxl) * val(nb.xl, j, k);
  const A r = A(nb.sxr) * val(nb.xr, j, k);
  const A d = A(nb.syd) * val(i, nb.yd, k);
  const A u = A(nb.syu) * val(i, nb.yu, k);
  const A b = A(sb) * val(i, j, kb);
  const A f = A(sf) * val(i, j, kf);
  center = c;
  const A two_c = A(2) * c;
  return -(r - two_c + l) * A(o.inv2[0]) - (u - two_c + d) * A(o.inv2[1]) -
         (f - two_c + b) * A(o.inv2[2]);
}

template <int K>
__device__ __forceinline__ void zero(double (&v)[K]) {
#pragma unroll
  for(int q = 0; q < K; ++q) v[q] = 0.0;
}

// Marches k in [k0, k1) in batches of KB planes: compute(k) holds only loads
// and arithmetic, commit(k, r) the stores and reductions, so the loads of a
// whole batch are independent and issued together.
constexpr int kBatch = 4;

template <int KB, typename Compute, typename Commit>
__device__ __forceinline__ void k_batched(int k0, int k1, Compute compute, Commit commit) {
  using R = decltype(compute(0));
  int k = k0;
  for(; k + KB <= k1; k += KB) {
    R r[KB];
#pragma unroll
    for(int t = 0; t < KB; ++t) r[t] = compute(k + t);
#pragma unroll
    for(int t = 0; t < KB; ++t) commit(k + t, r[t]);
  }
  for(; k < k1; ++k) commit(k, compute(k));
}

#define STENCIL_PROLOGUE(L)                                 \
  const int i = blockIdx.x * kTX + threadIdx.x;             \
  const int j = blockIdx.y * kTY + threadIdx.y;             \
  const bool valid = i < (L).nx && j < (L).ny;              \
  const int k0 = blockIdx.z * kchunk;                       \
  const int k1 = min(k0 + kchunk, (L).nz);

template <typename A>
struct Pair {
  A v;
  double w;
};

// ---------------------------------------------------------------------------
// V-cycle kernels.  Level vectors are T; shifts and scalars are double.
// ---------------------------------------------------------------------------

// Pre-smoothing sweep 1 from a zero correction: a = omega (b - sb) / D.
template <typename T, typename B>
__global__ void __launch_bounds__(kTX* kTY)
    k_smooth_first(OpInfo o, const B* __restrict__ b, const double* sb_ptr, T* __restrict__ a,
                   LevelScalars* ls, int zm, int kchunk, RedBuf rb) {
  pdl_enter();
  STENCIL_PROLOGUE(o.L)
  using A = T;
  const double sb = *sb_ptr;
  double acc[1];
  zero(acc);
  if(valid) {
    const A om = A(kOmega);
    k_batched<kBatch>(
        k0, k1,
        [&](int k) { return om * A(double(b[o.L.idx(i, j, k)]) - sb) * A(inv_diag(o, i, j, k)); },
        [&](int k, A v) {
          a[o.L.idx(i, j, k)] = T(v);
          acc[0] += double(v);
        });
  }
  const bool mx[1] = {false};
  const int n = o.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { ls->sa = zm ? s.v[0] / n : 0.0; });
}

// Jacobi sweep (smooth_jacobi, linsolve/poisson_solver.cpp:569-595):
// out = x + omega (b - sb - A x) / D with x = in - s_in; records mean(out).
// `which` selects the LevelScalars slot for the output mean (0: sa, 1: sx).
// On the finest level with sc != nullptr it also forms r.z for the CG.
template <typename T, typename B>
__global__ void __launch_bounds__(kTX* kTY)
    k_smooth(OpInfo o, const B* __restrict__ b, const double* sb_ptr, const T* __restrict__ in,
             const double* sin_ptr, T* __restrict__ out, LevelScalars* ls, int which, int zm,
             SolveScalars* sc, int kchunk, RedBuf rb) {
  pdl_enter();
  STENCIL_PROLOGUE(o.L)
  using A = T;
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  double acc[2];
  zero(acc);
  if(valid) {
    const ColNb nb = col_nb(o, i, j);
    const A om = A(kOmega);
    auto val = [&](int ii, int jj, int kk) { return A(in[o.L.idx(ii, jj, kk)]) - sin; };
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          A c;
          const A ax = apply_op<A>(o, nb, i, j, k, val, c);
          const double bq = double(b[o.L.idx(i, j, k)]) - sb;
          return Pair<A>{c + om * (A(bq) - ax) * A(inv_diag(o, i, j, k)), bq};
        },
        [&](int k, Pair<A> r) {
          out[o.L.idx(i, j, k)] = T(r.v);
          acc[0] += double(r.v);
          acc[1] += r.w * double(r.v);
        });
  }
  const bool mx[2] = {false, false};
  const int n = o.L.count();
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    const double mean = zm ? s.v[0] / n : 0.0;
    if(which == 0) ls->sa = mean;
    else {
      ls->sx = mean;
      ls->sum_x = s.v[0];
    }
    if(sc != nullptr) {
      // r.z with z = out - mean (linsolve/poisson_solver.cpp:749, :791)
      const double rz_new = s.v[1] - mean * (sc->sum_r - sc->n * sc->sr);
      if(sc->first) {
        sc->rz = rz_new;
      } else {
        sc->beta = rz_new / sc->rz;
        sc->rz = rz_new;
      }
    }
  });
}

// Residual + restriction (v_cycle :611-624 and restrict_full_weighting
// :397-424): coarse b = mean of the children's (b - sb - A x); x = in - s_in.
// RX, RY, RZ are the refinement ratios (1 or 2); children summed in the
// reference's dz, dy, dx order.
template <typename T, typename B, int RX, int RY, int RZ>
__global__ void __launch_bounds__(kTX* kTY)
    k_restrict_residual(OpInfo o, OpInfo oc, const B* __restrict__ b, const double* sb_ptr,
                        const T* __restrict__ in, const double* sin_ptr, T* __restrict__ bc,
                        LevelScalars* lsc, int zm, int kchunk, RedBuf rb) {
  pdl_enter();
  STENCIL_PROLOGUE(oc.L)
  using A = T;
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A inv_children = A(1.0 / double(RX * RY * RZ));
  double acc[1];
  zero(acc);
  if(valid) {
    ColNb nb[RY][RX];
#pragma unroll
    for(int dy = 0; dy < RY; ++dy)
#pragma unroll
      for(int dx = 0; dx < RX; ++dx) nb[dy][dx] = col_nb(o, i * RX + dx, j * RY + dy);
    auto val = [&](int ii, int jj, int kk) { return A(in[o.L.idx(ii, jj, kk)]) - sin; };
    k_batched<2>(
        k0, k1,
        [&](int kc) {
          A sum = A(0);
#pragma unroll
          for(int dz = 0; dz < RZ; ++dz)
#pragma unroll
            for(int dy = 0; dy < RY; ++dy)
#pragma unroll
              for(int dx = 0; dx < RX; ++dx) {
                const int fi = i * RX + dx, fj = j * RY + dy, fk = kc * RZ + dz;
                A c;
                const A ax = apply_op<A>(o, nb[dy][dx], fi, fj, fk, val, c);
                sum += A(double(b[o.L.idx(fi, fj, fk)]) - sb) - ax;
              }
          return inv_children * sum;
        },
        [&](int kc, A v) {
          bc[oc.L.idx(i, j, kc)] = T(v);
          acc[0] += double(v);
        });
  }
  const bool mx[1] = {false};
  const int n = oc.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { lsc->sb = zm ? s.v[0] / n : 0.0; });
}

// Prolongation + first post-smoothing sweep (prolongate_and_add :426-451,
// then smooth_jacobi): x3 = (in - s_in) + (e_parent - s_e); out = x3 +
// omega (b - sb - A x3) / D.  SX, SY, SZ are log2 of the refinement ratios.
template <typename T, typename B>
__global__ void __launch_bounds__(kTX* kTY)
    k_prolong_smooth(OpInfo o, CLay Lc, const B* __restrict__ b, const double* sb_ptr,
                     const T* __restrict__ in, const double* sin_ptr, const T* __restrict__ ec,
                     const double* sec_ptr, T* __restrict__ out, LevelScalars* ls, int sx, int sy,
                     int sz, int zm, int kchunk, RedBuf rb) {
  pdl_enter();
  STENCIL_PROLOGUE(o.L)
  using A = T;
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A sec = A(*sec_ptr);
  double acc[1];
  zero(acc);
  if(valid) {
    const ColNb nb = col_nb(o, i, j);
    const A om = A(kOmega);
    auto val = [&](int ii, int jj, int kk) {
      return (A(in[o.L.idx(ii, jj, kk)]) - sin) + (A(ec[Lc.idx(ii >> sx, jj >> sy, kk >> sz)]) - sec);
    };
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          A c;
          const A ax = apply_op<A>(o, nb, i, j, k, val, c);
          const A bq = A(double(b[o.L.idx(i, j, k)]) - sb);
          return c + om * (bq - ax) * A(inv_diag(o, i, j, k));
        },
        [&](int k, A v) {
          out[o.L.idx(i, j, k)] = T(v);
          acc[0] += double(v);
        });
  }
  const bool mx[1] = {false};
  const int n = o.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { ls->sa = zm ? s.v[0] / n : 0.0; });
}

// ---------------------------------------------------------------------------
// Row-vector kernels (vstencil.cuh) for levels whose rows split into 16-byte
// vectors; the column kernels above serve the rest.
// ---------------------------------------------------------------------------

template <typename T>
inline bool vfits(const CLay& L) {
  return vst::row_fits(L.nx, vst::Width<T>::W);
}

// Vector kernels can be switched off for comparisons: ORCHARD_B200_NO_VEC=1
// (all) or a comma list of smooth, pre, prolong, restrict, ap.  Read at each use so
// that a process can compare both forms.
bool vec_enabled(const char* which = "") {
  const char* e = std::getenv("ORCHARD_B200_NO_VEC");
  if(e == nullptr || e[0] == '\0' || e[0] == '0') return true;
  if(e[0] == '1') return false;
  return std::strstr(e, which) == nullptr || which[0] == '\0';
}

#define ROW_PROLOGUE(T)                                                          \
  constexpr int W = vst::Width<T>::W;                                             \
  const vst::RowGeom g = vst::row_geom<W>(o.L, o.periodic, o.dir_lo, o.dir_hi);   \
  const int k0 = blockIdx.z * kchunk;                                             \
  const int k1 = min(k0 + kchunk, o.L.nz);

// Jacobi sweep (smooth_jacobi); same contract as k_smooth with which = 1.
template <typename T, typename B>
__global__ void __launch_bounds__(256)
    k_vsmooth(OpInfo o, const B* __restrict__ b, const double* sb_ptr, const T* __restrict__ in,
              const double* sin_ptr, T* __restrict__ out, LevelScalars* ls, int zm,
              SolveScalars* sc, int kchunk, RedBuf rb) {
  pdl_enter();
  using A = T;
  ROW_PROLOGUE(T)
  using R = vst::Row<A, W>;
  using RB = vst::Row<double, W>;
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A om = A(kOmega);
  double acc[2] = {0.0, 0.0};
  vst::march<A, W, RB>(
      o, g, k0, k1,
      [&](int i0, int jj, int kk) {
        R r = vst::ld<A, W>(in + o.L.idx(i0, jj, kk));
#pragma unroll
        for(int t = 0; t < W; ++t) r.v[t] -= sin;
        return r;
      },
      [&](int ii, int jj, int kk) { return A(in[o.L.idx(ii, jj, kk)]) - sin; },
      [&](int i0, int jj, int kk) { return vst::ld<double, W>(b + o.L.idx(i0, jj, kk)); },
      [&](int k, const R& c, const R& ax, const RB& bb) {
        R v;
        double bq[W];
#pragma unroll
        for(int t = 0; t < W; ++t) {
          bq[t] = bb.v[t] - sb;
          v.v[t] = c.v[t] + om * (A(bq[t]) - ax.v[t]) * A(inv_diag(o, g.i0 + t, g.j, k));
        }
        if(g.act) {
          vst::st<T, W>(out + o.L.idx(g.i0, g.j, k), v);
#pragma unroll
          for(int t = 0; t < W; ++t) {
            acc[0] += double(v.v[t]);
            acc[1] += bq[t] * double(v.v[t]);
          }
        }
      });
  const bool mx[2] = {false, false};
  const int n = o.L.count();
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    const double mean = zm ? s.v[0] / n : 0.0;
    ls->sx = mean;
    ls->sum_x = s.v[0];
    if(sc != nullptr) {
      // r.z with z = out - mean (linsolve/poisson_solver.cpp:749, :791)
      const double rz_new = s.v[1] - mean * (sc->sum_r - sc->n * sc->sr);
      if(sc->first) {
        sc->rz = rz_new;
      } else {
        sc->beta = rz_new / sc->rz;
        sc->rz = rz_new;
      }
    }
  });
}

// Both pre-smoothing sweeps from a zero correction in one pass over b: the
// first sweep is pointwise, a = omega (b - sb) / D, so the second one,
// out = a + omega (b - sb - A a) / D, reads b alone (a is formed on load for
// every neighbour).  The reference removes mean(a) between the sweeps; A
// annihilates constants on the problems where it does that (periodic /
// all-Neumann), so the shift only moves out by a constant, which the mean
// recorded here (ls->sx) removes as before.
template <typename T, typename B>
__global__ void __launch_bounds__(256)
    k_vsmooth_pre(OpInfo o, const B* __restrict__ b, const double* sb_ptr, T* __restrict__ out,
                  LevelScalars* ls, int zm, int kchunk, RedBuf rb) {
  pdl_enter();
  using A = T;
  ROW_PROLOGUE(T)
  using R = vst::Row<A, W>;
  using RB = vst::Row<double, W>;
  const double sb = *sb_ptr;
  const A om = A(kOmega);
  auto a_at = [&](int ii, int jj, int kk, double bv) {
    return om * A(bv - sb) * A(inv_diag(o, ii, jj, kk));
  };
  double acc[1] = {0.0};
  vst::march<A, W, RB>(
      o, g, k0, k1,
      [&](int i0, int jj, int kk) {
        const RB bb = vst::ld<double, W>(b + o.L.idx(i0, jj, kk));
        R r;
#pragma unroll
        for(int t = 0; t < W; ++t) r.v[t] = a_at(i0 + t, jj, kk, bb.v[t]);
        return r;
      },
      [&](int ii, int jj, int kk) { return a_at(ii, jj, kk, double(b[o.L.idx(ii, jj, kk)])); },
      [&](int i0, int jj, int kk) { return vst::ld<double, W>(b + o.L.idx(i0, jj, kk)); },
      [&](int k, const R& c, const R& ax, const RB& bb) {
        R v;
#pragma unroll
        for(int t = 0; t < W; ++t)
          v.v[t] = c.v[t] + om * (A(bb.v[t] - sb) - ax.v[t]) * A(inv_diag(o, g.i0 + t, g.j, k));
        if(g.act) {
          vst::st<T, W>(out + o.L.idx(g.i0, g.j, k), v);
#pragma unroll
          for(int t = 0; t < W; ++t) acc[0] += double(v.v[t]);
        }
      });
  const bool mx[1] = {false};
  const int n = o.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) {
    ls->sx = zm ? s.v[0] / n : 0.0;
    ls->sum_x = s.v[0];
  });
}

// Prolongation + first post-smoothing sweep; same contract as k_prolong_smooth.
template <typename T, typename B>
__global__ void __launch_bounds__(256)
    k_vprolong_smooth(OpInfo o, CLay Lc, const B* __restrict__ b, const double* sb_ptr,
                      const T* __restrict__ in, const double* sin_ptr, const T* __restrict__ ec,
                      const double* sec_ptr, T* __restrict__ out, LevelScalars* ls, int sx, int sy,
                      int sz, int zm, int kchunk, RedBuf rb) {
  pdl_enter();
  using A = T;
  ROW_PROLOGUE(T)
  using R = vst::Row<A, W>;
  using RB = vst::Row<double, W>;
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A sec = A(*sec_ptr);
  const A om = A(kOmega);
  double acc[1] = {0.0};
  vst::march<A, W, RB>(
      o, g, k0, k1,
      [&](int i0, int jj, int kk) {
        R r = vst::ld<A, W>(in + o.L.idx(i0, jj, kk));
        const int pj = jj >> sy, pk = kk >> sz;
#pragma unroll
        for(int t = 0; t < W; ++t) r.v[t] = (r.v[t] - sin) + (A(ec[Lc.idx((i0 + t) >> sx, pj, pk)]) - sec);
        return r;
      },
      [&](int ii, int jj, int kk) {
        return (A(in[o.L.idx(ii, jj, kk)]) - sin) + (A(ec[Lc.idx(ii >> sx, jj >> sy, kk >> sz)]) - sec);
      },
      [&](int i0, int jj, int kk) { return vst::ld<double, W>(b + o.L.idx(i0, jj, kk)); },
      [&](int k, const R& c, const R& ax, const RB& bb) {
        R v;
#pragma unroll
        for(int t = 0; t < W; ++t)
          v.v[t] = c.v[t] + om * (A(bb.v[t] - sb) - ax.v[t]) * A(inv_diag(o, g.i0 + t, g.j, k));
        if(g.act) {
          vst::st<T, W>(out + o.L.idx(g.i0, g.j, k), v);
#pragma unroll
          for(int t = 0; t < W; ++t) acc[0] += double(v.v[t]);
        }
      });
  const bool mx[1] = {false};
  const int n = o.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { ls->sa = zm ? s.v[0] / n : 0.0; });
}

// A p; same contract as k_apply_ap.  V is the vector type (arithmetic FP64).
template <typename V>
__global__ void __launch_bounds__(256)
    k_vapply_ap(OpInfo o, const V* __restrict__ p, V* __restrict__ ap, SolveScalars* sc,
                int kchunk, RedBuf rb) {
  pdl_enter();
  ROW_PROLOGUE(V)
  using R = vst::Row<double, W>;
  const double sp = sc->sp;
  double acc[3] = {0.0, 0.0, 0.0};
  vst::march<double, W, int>(
      o, g, k0, k1,
      [&](int i0, int jj, int kk) {
        R r = vst::ld<double, W>(p + o.L.idx(i0, jj, kk));
#pragma unroll
        for(int t = 0; t < W; ++t) r.v[t] -= sp;
        return r;
      },
      [&](int ii, int jj, int kk) { return double(p[o.L.idx(ii, jj, kk)]) - sp; },
      [&](int, int, int) { return 0; },
      [&](int k, const R& c, const R& ax, int) {
        if(g.act) {
          vst::st<V, W>(ap + o.L.idx(g.i0, g.j, k), ax);
#pragma unroll
          for(int t = 0; t < W; ++t) {
            acc[0] += ax.v[t];
            acc[1] += c.v[t] * ax.v[t];
            acc[2] += c.v[t];
          }
        }
      });
  const bool mx[3] = {false, false, false};
  reduce_finish<3>(acc, mx, rb, [=](const Sums<3>& s) {
    const double sap = sc->zero_mean ? s.v[0] / sc->n : 0.0;
    sc->sap = sap;
    const double pap = s.v[1] - sap * s.v[2];
    sc->pap = pap;
    if(fabs(pap) < kSmallNumber) {
      sc->stop = 1;
    } else {
      sc->alpha = sc->rz / pap;
    }
  });
}

// Residual + 2x2x2 restriction on row vectors: a thread owns W fine cells of
// the two fine rows of a coarse row (W/2 coarse cells) and marches coarse
// planes (two fine planes each).
template <typename T, typename B>
__global__ void __launch_bounds__(256)
    k_vrestrict(OpInfo o, OpInfo oc, const B* __restrict__ b, const double* sb_ptr,
                const T* __restrict__ in, const double* sin_ptr, T* __restrict__ bc,
                LevelScalars* lsc, int zm, int kchunk, RedBuf rb) {
  pdl_enter();
  using A = T;
  constexpr int W = vst::Width<T>::W;
  using R = vst::Row<A, W>;
  const CLay& L = o.L;
  const int lane = threadIdx.x;
  int i0 = (blockIdx.x * 32 + lane) * W;
  const int jc = blockIdx.y * 8 + threadIdx.y;
  const bool act = i0 < L.nx && jc < oc.L.ny;
  if(i0 >= L.nx) i0 = L.nx - W;
  const int jcc = jc < oc.L.ny ? jc : oc.L.ny - 1;
  const int kc0 = blockIdx.z * kchunk;
  const int kc1 = min(kc0 + kchunk, oc.L.nz);
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  const int jr[2] = {2 * jcc, 2 * jcc + 1};
  int jdn, jup;
  double sdn, sup;
  nb_lo(jr[0], L.ny, o.periodic[1], o.dir_lo[1], jdn, sdn);
  nb_hi(jr[1], L.ny, o.periodic[1], o.dir_hi[1], jup, sup);
  const bool need_l = lane == 0 || i0 == 0;
  const bool need_r = lane == 31 || i0 + W >= L.nx;
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, L.nx, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + W - 1, L.nx, o.periodic[0], o.dir_hi[0], xr, sxr);
  auto rowv = [&](int jj, int kk) {
    R r = vst::ld<A, W>(in + L.idx(i0, jj, kk));
#pragma unroll
    for(int t = 0; t < W; ++t) r.v[t] -= sin;
    return r;
  };
  auto zrowv = [&](int jj, int kk) {
    double sg;
    const int kz = vst::zrow(kk, L.nz, o.periodic[2], o.dir_lo[2], o.dir_hi[2], sg);
    R r = rowv(jj, kz);
#pragma unroll
    for(int t = 0; t < W; ++t) r.v[t] *= A(sg);
    return r;
  };
  double acc[1] = {0.0};
  for(int kc = kc0; kc < kc1; ++kc) {
    const int kf = 2 * kc;
    // rows j0, j1 at planes kf-1 .. kf+2, neighbour rows at kf, kf+1
    R q[2][4];
#pragma unroll
    for(int r = 0; r < 2; ++r)
#pragma unroll
      for(int z = 0; z < 4; ++z) q[r][z] = zrowv(jr[r], kf - 1 + z);
    R dn[2], up[2];
    A hl[2][2], hr[2][2];
    vst::Row<double, W> bb[2][2];
#pragma unroll
    for(int z = 0; z < 2; ++z) {
      dn[z] = rowv(jdn, kf + z);
      up[z] = rowv(jup, kf + z);
#pragma unroll
      for(int t = 0; t < W; ++t) {
        dn[z].v[t] *= A(sdn);
        up[z].v[t] *= A(sup);
      }
#pragma unroll
      for(int r = 0; r < 2; ++r) {
        hl[r][z] = need_l ? A(sxl) * (A(in[L.idx(xl, jr[r], kf + z)]) - sin) : A(0);
        hr[r][z] = need_r ? A(sxr) * (A(in[L.idx(xr, jr[r], kf + z)]) - sin) : A(0);
        bb[r][z] = vst::ld<double, W>(b + L.idx(i0, jr[r], kf + z));
      }
    }
    A csum[W / 2];
#pragma unroll
    for(int c = 0; c < W / 2; ++c) csum[c] = A(0);
#pragma unroll
    for(int z = 0; z < 2; ++z)
#pragma unroll
      for(int r = 0; r < 2; ++r) {
        const R& cen = q[r][z + 1];
        const A from_l = __shfl_up_sync(0xffffffffu, cen.v[W - 1], 1);
        const A from_r = __shfl_down_sync(0xffffffffu, cen.v[0], 1);
        const A left = need_l ? hl[r][z] : from_l;
        const A right = need_r ? hr[r][z] : from_r;
        const R& d = r == 0 ? dn[z] : q[0][z + 1];
        const R& u = r == 0 ? q[1][z + 1] : up[z];
        const R ax = vst::row_ax<A, W>(cen, left, right, d, u, q[r][z], q[r][z + 2], ix, iy, iz);
#pragma unroll
        for(int t = 0; t < W; ++t) csum[t / 2] += A(bb[r][z].v[t] - sb) - ax.v[t];
      }
    if(act) {
#pragma unroll
      for(int c = 0; c < W / 2; ++c) {
        const A v = A(0.125) * csum[c];
        bc[oc.L.idx(i0 / 2 + c, jc, kc)] = T(v);
        acc[0] += double(v);
      }
    }
  }
  const bool mx[1] = {false};
  const int n = oc.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) { lsc->sb = zm ? s.v[0] / n : 0.0; });
}

// direct_coarse_solve (linsolve/poisson_solver.cpp:530-567) with the
// elimination precomputed on the host: row swaps, multipliers and the upper
// factor are applied to the right-hand side in the reference's order.
template <typename T, typename B>
__global__ void k_coarse_solve(int n, const int* __restrict__ swaps, const double* __restrict__ f,
                               const B* __restrict__ b, const double* sb_ptr, T* __restrict__ out,
                               LevelScalars* ls, int zm, SolveScalars* sc) {
  pdl_enter();
  __shared__ double y[kMaxCoarse];
  __shared__ double red[32];
  const int t = threadIdx.x;
  const double sb = *sb_ptr;
  for(int q = t; q < n; q += blockDim.x) y[q] = double(b[q]) - sb;
  __syncthreads();
  if(zm && t == 0) y[n - 1] = 0.0;
  __syncthreads();
  for(int p = 0; p < n; ++p) {
    if(t == 0 && swaps[p] != p) {
      const double tmp = y[p];
      y[p] = y[swaps[p]];
      y[swaps[p]] = tmp;
    }
    __syncthreads();
    const double yp = y[p];
    for(int r = p + 1 + t; r < n; r += blockDim.x) {
      const double factor = f[static_cast<size_t>(r) * n + p];
      if(factor != 0.0) y[r] -= factor * yp;
    }
    __syncthreads();
  }
  for(int row = n - 1; row >= 0; --row) {
    if(t == 0) y[row] = y[row] / f[static_cast<size_t>(row) * n + row];
    __syncthreads();
    const double yr = y[row];
    for(int r = t; r < row; r += blockDim.x) y[r] -= f[static_cast<size_t>(r) * n + row] * yr;
    __syncthreads();
  }
  // subtract_active_mean on the coarse correction
  double part = 0.0;
  for(int q = t; q < n; q += blockDim.x) part += y[q];
  part = warp_sum(part);
  if((t & 31) == 0) red[t >> 5] = part;
  __syncthreads();
  double mean = 0.0;
  if(zm) {
    double s = 0.0;
    for(int w = 0; w < (int(blockDim.x) + 31) / 32; ++w) s += red[w];
    mean = s / n;
  }
  double rzp = 0.0;
  for(int q = t; q < n; q += blockDim.x) {
    const double v = y[q] - mean;
    out[q] = T(v);
    rzp += (double(b[q]) - sb) * v;
  }
  __syncthreads();
  rzp = warp_sum(rzp);
  if((t & 31) == 0) red[t >> 5] = rzp;
  __syncthreads();
  if(t == 0) {
    ls->sx = 0.0;
    ls->sum_x = 0.0;
    if(sc != nullptr) {
      double s = 0.0;
      for(int w = 0; w < (int(blockDim.x) + 31) / 32; ++w) s += red[w];
      if(sc->first) {
        sc->rz = s;
      } else {
        sc->beta = s / sc->rz;
        sc->rz = s;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Plane-pipelined stencil kernels.  A block owns a tile of whole rows (all nx
// cells, TY = 1024 / nx rows) and a chunk of k planes.  One thread stages each
// plane of the operand -- the tile rows plus the two neighbour rows, fetched at
// their boundary images (periodic wrap or the mirrored row) -- and of the
// rhs into a ring of kTSlots shared-memory slots with TMA, kTSlots - 2 planes
// ahead of the compute; an mbarrier per slot carries the arrival.  Each
// thread owns four consecutive cells of one row: their z-neighbours come from
// a register queue, the in-plane neighbours from the staged plane.  Boundary
// signs (Dirichlet mirrors) and mean shifts are applied on read.  Used where
// nx is 64, 128 or 256 and TY divides ny.
// ---------------------------------------------------------------------------
constexpr int kTSlots = 5;

__host__ __device__ inline size_t tround(size_t b) { return (b + 127) / 128 * 128; }

template <typename T, typename B>
__host__ __device__ inline size_t tslot_bytes(int nx) {
  const int ty = 1024 / nx;
  return tround(static_cast<size_t>(ty + 2) * nx * sizeof(T)) + tround(static_cast<size_t>(ty) * nx * sizeof(B));
}

template <typename T, typename B>
__host__ __device__ inline size_t tprolong_bytes(int nx) {
  const int ty = 1024 / nx;
  return tround(static_cast<size_t>(ty + 2) * nx * sizeof(T)) + tround(static_cast<size_t>(ty) * nx * sizeof(B)) +
         tround(static_cast<size_t>(ty / 2 + 2) * (nx / 2) * sizeof(T));
}

// Four consecutive values from shared (or global) memory.  SWAP (FP64 only):
// lanes 32 bytes apart read their two 16-byte halves in an order that
// alternates with (lane ^ lane / 4), so that each quarter-warp phase of a
// 128-bit shared-memory load touches eight distinct 16-byte bank groups
// instead of four (no 2-way bank conflict); the same values either way, at
// the cost of a few registers for the lane-dependent select.
template <typename A, typename S, bool SWAP = false>
__device__ __forceinline__ void tload4(const S* p, A (&v)[4]) {
  if constexpr(std::is_same_v<S, double>) {
    double2 a, b;
    if constexpr(SWAP) {
      const int lane = threadIdx.x & 31;
      const int h = (lane ^ (lane >> 2)) & 1;
      const double2* q = reinterpret_cast<const double2*>(p);
      const double2 f = q[h];
      const double2 g = q[h ^ 1];
      a = h ? g : f;
      b = h ? f : g;
    } else {
      a = *reinterpret_cast<const double2*>(p);
      b = *reinterpret_cast<const double2*>(p + 2);
    }
    v[0] = A(a.x);
    v[1] = A(a.y);
    v[2] = A(b.x);
    v[3] = A(b.y);
  } else {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = A(a.x);
    v[1] = A(a.y);
    v[2] = A(a.z);
    v[3] = A(a.w);
  }
}

template <typename S, typename A>
__device__ __forceinline__ void tstore4(S* p, const A (&v)[4]) {
  if constexpr(std::is_same_v<S, double>) {
    *reinterpret_cast<double2*>(p) = make_double2(double(v[0]), double(v[1]));
    *reinterpret_cast<double2*>(p + 2) = make_double2(double(v[2]), double(v[3]));
  } else {
    *reinterpret_cast<float4*>(p) = make_float4(float(v[0]), float(v[1]), float(v[2]), float(v[3]));
  }
}

// Persistent schedule of the plane pipeline: the tile-planes (tile, k) of a
// level, k fastest, are split into gridDim.x contiguous ranges of equal length
// (within one); a block walks its range as segments (one per tile it touches)
// and streams each segment's planes k_begin - 1 .. k_end through one ring, so
// the pipeline is filled once per block and no block waits for a tail wave.
constexpr int kTMaxSeg = 8;

struct TSeg {
  int tile, kb, ke, lbase;  // planes [kb, ke) of `tile`; first load index
};

__device__ __forceinline__ int tsegments(int tiles, int nz, TSeg (&seg)[kTMaxSeg], int& nload) {
  if(gridDim.x % tiles == 0) {
    // z-aligned schedule (the host selects it by launching a multiple of the
    // tile count, tgrid_blocks): block b owns tile b % tiles and z chunk
    // b / tiles, so the blocks
    // of neighbouring tiles stream the same planes at the same time and a
    // tile's halo rows -- its neighbours' edge rows -- come from L2, not DRAM
    const int nzc = gridDim.x / tiles;
    const int tile = blockIdx.x % tiles, zc = blockIdx.x / tiles;
    const int kb = static_cast<int>(static_cast<long long>(nz) * zc / nzc);
    const int ke = static_cast<int>(static_cast<long long>(nz) * (zc + 1) / nzc);
    seg[0] = TSeg{tile, kb, ke, 0};
    nload = ke > kb ? ke - kb + 2 : 0;
    return ke > kb ? 1 : 0;
  }
  const long long total = static_cast<long long>(tiles) * nz;
  const long long f0 = total * blockIdx.x / gridDim.x;
  const long long f1 = total * (blockIdx.x + 1) / gridDim.x;
  int ns = 0;
  nload = 0;
  for(long long f = f0; f < f1 && ns < kTMaxSeg;) {
    const int tile = static_cast<int>(f / nz);
    const int kb = static_cast<int>(f % nz);
    const int ke = static_cast<int>(min(static_cast<long long>(nz), kb + (f1 - f)));
    seg[ns] = TSeg{tile, kb, ke, nload};
    nload += ke - kb + 2;
    f += ke - kb;
    ++ns;
  }
  return ns;
}

// Jacobi sweep (smooth_jacobi, linsolve/poisson_solver.cpp:569-595) on the
// plane pipeline: out = x + omega (b - sb - A x) / D with x = in - s_in;
// records mean(out) (ls->sx) and, on the finest level, r.z (sc).  Same
// contract as k_vsmooth.  CPT cells per thread (4 or 2), 1024 / CPT threads.
template <typename T, typename B, int CPT, bool PER>
__global__ void __launch_bounds__(1024 / CPT)
    k_tsmooth(OpInfo o, const __grid_constant__ CUtensorMap um, const __grid_constant__ CUtensorMap uh,
              const __grid_constant__ CUtensorMap bm, const double* sb_ptr, const double* sin_ptr,
              T* __restrict__ out, LevelScalars* ls, int zm, SolveScalars* sc, RedBuf rb, int* fault) {
  pdl_enter();
  using A = T;
  constexpr int D = kTSlots;
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ uint64_t bars[D];
  __shared__ double invd_s[64];
  const int NX = o.L.nx, NY = o.L.ny, NZ = o.L.nz;
  const int TY = 1024 / NX;
  const int tpr = NX / CPT;
  const int r = threadIdx.x / tpr;
  const int i0 = (threadIdx.x % tpr) * CPT;
  const size_t ubytes = tround(static_cast<size_t>(TY + 2) * NX * sizeof(T));
  const size_t sbytes = tslot_bytes<T, B>(NX);
  const uint32_t tx_bytes = static_cast<uint32_t>((TY + 2) * NX * sizeof(T) + TY * NX * sizeof(B));
  auto uslot = [&](int s) { return reinterpret_cast<T*>(tsm + s * sbytes); };
  auto bslot = [&](int s) { return reinterpret_cast<B*>(tsm + s * sbytes + ubytes); };
  TSeg seg[kTMaxSeg];
  int nload = 0;
  const int nseg = tsegments(NY / TY, NZ, seg, nload);
  // producer (thread 0): load l -> its segment's tile and plane image
  auto issue = [&](int l) {
    int q = 0;
    while(q + 1 < nseg && seg[q + 1].lbase <= l) ++q;
    const int j0 = seg[q].tile * TY;
    int jm, jp;
    double sg;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sg);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, sg);
    const int kz = vst::zrow(seg[q].kb - 1 + (l - seg[q].lbase), NZ, o.periodic[2], o.dir_lo[2],
                             o.dir_hi[2], sg);
    const int sl = l % D;
    tma::mbar_arrive_expect_tx(&bars[sl], tx_bytes);
    tma::load_3d(uslot(sl) + NX, &um, &bars[sl], 0, j0, kz);
    tma::load_3d(uslot(sl), &uh, &bars[sl], 0, jm, kz);
    tma::load_3d(uslot(sl) + (TY + 1) * NX, &uh, &bars[sl], 0, jp, kz);
    tma::load_3d(bslot(sl), &bm, &bars[sl], 0, j0, kz);
  };
  if(threadIdx.x == 0) {
    for(int sl = 0; sl < D; ++sl) tma::mbar_init(&bars[sl], 1);
    tma::fence_barrier_init();
  }
  if(threadIdx.x < 64) invd_s[threadIdx.x] = o.invd[threadIdx.x];
  __syncthreads();
  int next = 0;  // next load to issue (meaningful on thread 0)
  if(threadIdx.x == 0)
    while(next < nload && next < D) issue(next++);
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A om = A(kOmega);
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  auto ldrow = [&](const T* p, A (&v)[CPT]) {
    if constexpr(CPT == 4) {
      tload4<A>(p, v);
    } else if constexpr(std::is_same_v<T, double>) {
      const double2 a = *reinterpret_cast<const double2*>(p);
      v[0] = A(a.x);
      v[1] = A(a.y);
    } else {
      const float2 a = *reinterpret_cast<const float2*>(p);
      v[0] = A(a.x);
      v[1] = A(a.y);
    }
  };
  double acc[2] = {0.0, 0.0};
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, NX, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + CPT - 1, NX, o.periodic[0], o.dir_hi[0], xr, sxr);
  for(int q = 0; q < nseg; ++q) {
    const TSeg sg = seg[q];
    const int j0 = sg.tile * TY;
    const int j = j0 + r;
    int jm, jp;
    double sylo, syhi;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sylo);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, syhi);
    int cls[CPT];
#pragma unroll
    for(int t = 0; t < CPT; ++t) cls[t] = axis_class(i0 + t, NX) + 4 * axis_class(j, NY);
    auto own = [&](int l, A (&v)[CPT]) {
      tma::mbar_wait(&bars[l % D], (l / D) & 1, fault, 1);
      double zs;
      vst::zrow(sg.kb - 1 + (l - sg.lbase), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], zs);
      ldrow(uslot(l % D) + (r + 1) * NX + i0, v);
      if constexpr(!PER) {
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] = A(zs) * (v[t] - sin);
      }
    };
    // one output plane k from its staged slot and the z-queue (below, cen, above)
    auto plane = [&](int k, int c, const A (&below)[CPT], const A (&cen)[CPT], const A (&above)[CPT]) {
      const T* pk = uslot(c % D);
      const B* bk = bslot(c % D);
      A dn[CPT], up[CPT];
      ldrow(pk + r * NX + i0, dn);
      ldrow(pk + (r + 2) * NX + i0, up);
      A left = pk[(r + 1) * NX + xl], right = pk[(r + 1) * NX + xr];
      if constexpr(!PER) {
        // boundary signs and the mean shift (on a fully periodic grid the
        // operator annihilates the shift, so raw values are used there)
        const A sd = r == 0 ? A(sylo) : A(1), su = r == TY - 1 ? A(syhi) : A(1);
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] = sd * (dn[t] - sin);
          up[t] = su * (up[t] - sin);
        }
        left = A(sxl) * (left - sin);
        right = A(sxr) * (right - sin);
      }
      double bq[CPT];
      if constexpr(CPT == 4) {
        tload4<double>(bk + r * NX + i0, bq);
      } else {
#pragma unroll
        for(int t = 0; t < CPT; ++t) bq[t] = double(bk[r * NX + i0 + t]);
      }
      const int cz = 16 * axis_class(k, NZ);
      A v[CPT];
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        const double bd = bq[t] - sb;
        const A l = t > 0 ? cen[t - 1] : left;
        const A rr = t < CPT - 1 ? cen[t + 1] : right;
        const A two_c = A(2) * cen[t];
        const A ax = -(rr - two_c + l) * ix - (up[t] - two_c + dn[t]) * iy - (above[t] - two_c + below[t]) * iz;
        if constexpr(PER)
          v[t] = (cen[t] - sin) + om * (A(bd) - ax) * A(invd_s[0]);
        else
          v[t] = cen[t] + om * (A(bd) - ax) * A(invd_s[cls[t] + cz]);
        acc[0] += double(v[t]);
        acc[1] += bd * double(v[t]);
      }
      if constexpr(CPT == 4) {
        tstore4<T>(out + o.L.idx(i0, j, k), v);
      } else if constexpr(std::is_same_v<T, double>) {
        *reinterpret_cast<double2*>(out + o.L.idx(i0, j, k)) = make_double2(v[0], v[1]);
      } else {
        *reinterpret_cast<float2*>(out + o.L.idx(i0, j, k)) = make_float2(v[0], v[1]);
      }
    };
    A q0[CPT], q1[CPT], q2[CPT], q3[CPT];
    own(sg.lbase, q0);
    own(sg.lbase + 1, q1);
    __syncthreads();
    // two planes per step (one when a single plane is left)
    for(int k = sg.kb; k < sg.ke;) {
      const int c = sg.lbase + 1 + (k - sg.kb);  // load of plane k
      const bool two = k + 1 < sg.ke;
      if(threadIdx.x == 0) {
        tma::fence_proxy_async();
        while(next < nload && next <= c - 1 + D) issue(next++);
      }
      own(c + 1, q2);
      if(two) own(c + 2, q3);
      plane(k, c, q0, q1, q2);
      if(two) plane(k + 1, c + 1, q1, q2, q3);
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        q0[t] = two ? q2[t] : q1[t];
        q1[t] = two ? q3[t] : q2[t];
      }
      k += two ? 2 : 1;
      __syncthreads();
    }
  }
  const bool mx[2] = {false, false};
  const int n = o.L.count();
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& st) {
    const double mean = zm ? st.v[0] / n : 0.0;
    ls->sx = mean;
    ls->sum_x = st.v[0];
    if(sc != nullptr) {
      const double rz_new = st.v[1] - mean * (sc->sum_r - sc->n * sc->sr);
      if(sc->first) {
        sc->rz = rz_new;
      } else {
        sc->beta = rz_new / sc->rz;
        sc->rz = rz_new;
      }
    }
  });
}

// Both pre-smoothing sweeps from a zero correction on the plane pipeline
// (same contract as k_vsmooth_pre): the staged operand is b itself, and the
// first sweep's a = omega (b - sb) / D is formed on read for every stencil
// point, with the diagonal of the point's boundary image.  Warp-specialised:
// 1024 / CPT consumer threads and one producer warp that issues the TMA loads;
// each consumer warp releases a slot through an mbarrier when it has read it,
// so there is no block barrier per plane (at 256^3: 65.5 -> 60.7 us FP64,
// 45 -> 43 us FP32 per launch).
template <typename T, typename B, int CPT, bool PER>
__global__ void __launch_bounds__(1024 / CPT + 32)
    k_tsmooth_pre(OpInfo o, const __grid_constant__ CUtensorMap bm, const __grid_constant__ CUtensorMap bh,
                  const double* sb_ptr, T* __restrict__ out, LevelScalars* ls, int zm, RedBuf rb,
                  int* fault) {
  pdl_enter();
  using A = T;
  constexpr int D = kTSlots;
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ uint64_t bars[D], empt[D];  // slot loaded / slot released
  __shared__ A invd_s[64];
  using L = std::conditional_t<std::is_same_v<T, float>, float, double>;  // loaded rhs values
  const int NX = o.L.nx, NY = o.L.ny, NZ = o.L.nz;
  const int TY = 1024 / NX;
  const int tpr = NX / CPT;
  const int r = threadIdx.x / tpr;
  const int i0 = (threadIdx.x % tpr) * CPT;
  const size_t sbytes = tround(static_cast<size_t>(TY + 2) * NX * sizeof(B));
  const uint32_t tx_bytes = static_cast<uint32_t>((TY + 2) * NX * sizeof(B));
  auto slot = [&](int s) { return reinterpret_cast<B*>(tsm + s * sbytes); };
  TSeg seg[kTMaxSeg];
  int nload = 0;
  const int nseg = tsegments(NY / TY, NZ, seg, nload);
  auto issue = [&](int l) {
    int q = 0;
    while(q + 1 < nseg && seg[q + 1].lbase <= l) ++q;
    const int j0 = seg[q].tile * TY;
    int jm, jp;
    double sg;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sg);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, sg);
    const int kz = vst::zrow(seg[q].kb - 1 + (l - seg[q].lbase), NZ, o.periodic[2], o.dir_lo[2],
                             o.dir_hi[2], sg);
    const int sl = l % D;
    tma::mbar_arrive_expect_tx(&bars[sl], tx_bytes);
    tma::load_3d(slot(sl) + NX, &bm, &bars[sl], 0, j0, kz);
    tma::load_3d(slot(sl), &bh, &bars[sl], 0, jm, kz);
    tma::load_3d(slot(sl) + (TY + 1) * NX, &bh, &bars[sl], 0, jp, kz);
  };
  constexpr int NC = 1024 / CPT;  // consumer threads; the warp after them is the producer
  if(threadIdx.x == 0) {
    for(int sl = 0; sl < D; ++sl) {
      tma::mbar_init(&bars[sl], 1);
      tma::mbar_init(&empt[sl], NC / 32);
    }
    tma::fence_barrier_init();
  }
  if(threadIdx.x < 64) invd_s[threadIdx.x] = A(o.invd[threadIdx.x]);
  __syncthreads();
  const double sb = *sb_ptr;
  const A om = A(kOmega);
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  auto ldrow = [&](const B* p, L (&v)[CPT]) {
    if constexpr(CPT == 4) {
      tload4<L, B, std::is_same_v<B, double>>(p, v);
    } else {
#pragma unroll
      for(int t = 0; t < CPT; ++t) v[t] = L(p[t]);
    }
  };
  double acc[1] = {0.0};
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, NX, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + CPT - 1, NX, o.periodic[0], o.dir_hi[0], xr, sxr);
  // a consumer warp releases slot l once its lanes have read it
  auto release = [&](int l) {
    __syncwarp();
    if((threadIdx.x & 31) == 0) tma::mbar_arrive(&empt[l % D]);
  };
  if(threadIdx.x >= NC) {
    // producer: load l goes into slot l % D once every consumer warp has
    // released load l - D there (bounded waits, as for the loads)
    if(threadIdx.x == NC) {
      for(int l = 0; l < nload; ++l) {
        if(l >= D) tma::mbar_wait(&empt[l % D], ((l / D) - 1) & 1, fault, 1);
        issue(l);
      }
    }
  } else
  for(int q = 0; q < nseg; ++q) {
    const TSeg sg = seg[q];
    const int j0 = sg.tile * TY;
    const int j = j0 + r;
    int jm, jp;
    double sylo, syhi;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sylo);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, syhi);
    // boundary classes (x + 4 y) of the own cells and of their in-plane neighbours' images
    const int jd = r == 0 ? jm : j - 1, ju = r == TY - 1 ? jp : j + 1;
    const A sd = r == 0 ? A(sylo) : A(1), su = r == TY - 1 ? A(syhi) : A(1);
    int cown[CPT], cdn[CPT], cup[CPT];
#pragma unroll
    for(int t = 0; t < CPT; ++t) {
      const int cx = axis_class(i0 + t, NX);
      cown[t] = cx + 4 * axis_class(j, NY);
      cdn[t] = cx + 4 * axis_class(jd, NY);
      cup[t] = cx + 4 * axis_class(ju, NY);
    }
    const int cl = axis_class(xl, NX) + 4 * axis_class(j, NY);
    const int cr = axis_class(xr, NX) + 4 * axis_class(j, NY);
    // a of the own cells at load l (its plane's image and sign)
    auto own = [&](int l, A (&v)[CPT]) {
      tma::mbar_wait(&bars[l % D], (l / D) & 1, fault, 1);
      double zs;
      const int kz = vst::zrow(sg.kb - 1 + (l - sg.lbase), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], zs);
      const int cz = 16 * axis_class(kz, NZ);
      L b[CPT];
      ldrow(slot(l % D) + (r + 1) * NX + i0, b);
      if constexpr(PER) {
        // raw b: the operator annihilates the constant omega sb / D
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] = A(b[t]);
      } else {
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] = A(zs) * om * A(b[t] - L(sb)) * A(invd_s[cown[t] + cz]);
      }
    };
    A below[CPT], cen[CPT], above[CPT];
    own(sg.lbase, below);
    release(sg.lbase);
    own(sg.lbase + 1, cen);
    for(int k = sg.kb; k < sg.ke; ++k) {
      const int c = sg.lbase + 1 + (k - sg.kb);
      own(c + 1, above);
      const B* pk = slot(c % D);
      const int cz = 16 * axis_class(k, NZ);
      L bd[CPT], bu[CPT], bc[CPT];
      ldrow(pk + r * NX + i0, bd);
      ldrow(pk + (r + 2) * NX + i0, bu);
      ldrow(pk + (r + 1) * NX + i0, bc);
      A dn[CPT], up[CPT], left, right;
      if constexpr(PER) {
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] = A(bd[t]);
          up[t] = A(bu[t]);
        }
        left = A(pk[(r + 1) * NX + xl]);
        right = A(pk[(r + 1) * NX + xr]);
      } else {
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] = sd * om * A(bd[t] - L(sb)) * A(invd_s[cdn[t] + cz]);
          up[t] = su * om * A(bu[t] - L(sb)) * A(invd_s[cup[t] + cz]);
        }
        left = A(sxl) * om * A(L(pk[(r + 1) * NX + xl]) - L(sb)) * A(invd_s[cl + cz]);
        right = A(sxr) * om * A(L(pk[(r + 1) * NX + xr]) - L(sb)) * A(invd_s[cr + cz]);
      }
      A v[CPT];
      A ps0 = A(0);  // FP32: per-plane partial sum
      const A w0 = om * A(invd_s[0]);
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        const A l = t > 0 ? cen[t - 1] : left;
        const A rr = t < CPT - 1 ? cen[t + 1] : right;
        const A two_c = A(2) * cen[t];
        const A ax = -(rr - two_c + l) * ix - (up[t] - two_c + dn[t]) * iy - (above[t] - two_c + below[t]) * iz;
        if constexpr(PER) {
          // a = w (b - sb) on every point, so A a = w A b
          const A bcs = A(bc[t] - L(sb));
          v[t] = w0 * bcs + w0 * (bcs - w0 * ax);
        } else {
          v[t] = cen[t] + om * (A(bc[t] - L(sb)) - ax) * A(invd_s[cown[t] + cz]);
        }
        if constexpr(std::is_same_v<T, float>) ps0 += v[t];
        else acc[0] += double(v[t]);
      }
      if constexpr(std::is_same_v<T, float>) acc[0] += double(ps0);
      if constexpr(CPT == 4) {
        tstore4<T>(out + o.L.idx(i0, j, k), v);
      } else if constexpr(std::is_same_v<T, double>) {
        *reinterpret_cast<double2*>(out + o.L.idx(i0, j, k)) = make_double2(v[0], v[1]);
      } else {
        *reinterpret_cast<float2*>(out + o.L.idx(i0, j, k)) = make_float2(v[0], v[1]);
      }
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        below[t] = cen[t];
        cen[t] = above[t];
      }
      release(c);
    }
    release(sg.lbase + 1 + (sg.ke - sg.kb));
  }
  const bool mx[1] = {false};
  const int n = o.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& st) {
    ls->sx = zm ? st.v[0] / n : 0.0;
    ls->sum_x = st.v[0];
  });
}

// Prolongation + first post-smoothing sweep on the plane pipeline (same
// contract as k_vprolong_smooth, 2x2x2 coarsening): the staged operand is the
// level's correction x and the coarse correction ec (parent rows and the
// parents of the halo rows), combined on read as (x - sx) + (ec - sec).
template <typename T, typename B, int CPT, int D, bool PER>
__global__ void __launch_bounds__(1024 / CPT)
    k_tprolong(OpInfo o, const __grid_constant__ CUtensorMap xm, const __grid_constant__ CUtensorMap xh,
               const __grid_constant__ CUtensorMap bm, const __grid_constant__ CUtensorMap em,
               const __grid_constant__ CUtensorMap eh, const double* sb_ptr, const double* sin_ptr,
               const double* sec_ptr, T* __restrict__ out, LevelScalars* ls, int zm, RedBuf rb,
               int* fault) {
  pdl_enter();
  using A = T;
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ uint64_t bars[D];
  __shared__ A invd_s[64];
  using L = std::conditional_t<std::is_same_v<T, float>, float, double>;  // loaded rhs values
  const int NX = o.L.nx, NY = o.L.ny, NZ = o.L.nz;
  const int NXc = NX / 2, NZc = NZ / 2;
  const int TY = 1024 / NX;
  const int TYc = TY / 2;
  const int tpr = NX / CPT;
  const int r = threadIdx.x / tpr;
  const int i0 = (threadIdx.x % tpr) * CPT;
  const size_t xbytes = tround(static_cast<size_t>(TY + 2) * NX * sizeof(T));
  const size_t bbytes = tround(static_cast<size_t>(TY) * NX * sizeof(B));
  const size_t ebytes = tround(static_cast<size_t>(TYc + 2) * NXc * sizeof(T));
  const size_t sbytes = xbytes + bbytes + ebytes;
  const uint32_t tx_bytes = static_cast<uint32_t>((TY + 2) * NX * sizeof(T) + TY * NX * sizeof(B) +
                                                  (TYc + 2) * NXc * sizeof(T));
  auto xslot = [&](int s) { return reinterpret_cast<T*>(tsm + s * sbytes); };
  auto bslot = [&](int s) { return reinterpret_cast<B*>(tsm + s * sbytes + xbytes); };
  auto eslot = [&](int s) { return reinterpret_cast<T*>(tsm + s * sbytes + xbytes + bbytes); };
  TSeg seg[kTMaxSeg];
  int nload = 0;
  const int nseg = tsegments(NY / TY, NZ, seg, nload);
  auto issue = [&](int l) {
    int q = 0;
    while(q + 1 < nseg && seg[q + 1].lbase <= l) ++q;
    const int j0 = seg[q].tile * TY;
    int jm, jp;
    double sg;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sg);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, sg);
    const int kz = vst::zrow(seg[q].kb - 1 + (l - seg[q].lbase), NZ, o.periodic[2], o.dir_lo[2],
                             o.dir_hi[2], sg);
    const int sl = l % D;
    tma::mbar_arrive_expect_tx(&bars[sl], tx_bytes);
    tma::load_3d(xslot(sl) + NX, &xm, &bars[sl], 0, j0, kz);
    tma::load_3d(xslot(sl), &xh, &bars[sl], 0, jm, kz);
    tma::load_3d(xslot(sl) + (TY + 1) * NX, &xh, &bars[sl], 0, jp, kz);
    tma::load_3d(bslot(sl), &bm, &bars[sl], 0, j0, kz);
    tma::load_3d(eslot(sl) + NXc, &em, &bars[sl], 0, j0 >> 1, kz >> 1);
    tma::load_3d(eslot(sl), &eh, &bars[sl], 0, jm >> 1, kz >> 1);
    tma::load_3d(eslot(sl) + (TYc + 1) * NXc, &eh, &bars[sl], 0, jp >> 1, kz >> 1);
  };
  (void)NZc;
  if(threadIdx.x == 0) {
    for(int sl = 0; sl < D; ++sl) tma::mbar_init(&bars[sl], 1);
    tma::fence_barrier_init();
  }
  if(threadIdx.x < 64) invd_s[threadIdx.x] = A(o.invd[threadIdx.x]);
  __syncthreads();
  int next = 0;
  if(threadIdx.x == 0)
    while(next < nload && next < D) issue(next++);
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A sec = A(*sec_ptr);
  const A om = A(kOmega);
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  // fine slot row (0 .. TY+1) -> coarse slot row of its parent
  auto crow = [&](int fr) { return fr == 0 ? 0 : (fr == TY + 1 ? TYc + 1 : ((fr - 1) >> 1) + 1); };
  // combined operand of the CPT cells at fine slot row fr (shifted, unsigned)
  // (on a fully periodic grid the shifts are left out: the operator
  // annihilates constants, and only the centre value needs them)
  const A shx = PER ? A(0) : sin, she = PER ? A(0) : sec;
  auto operand = [&](const T* xs, const T* es, int fr, A (&v)[CPT]) {
    A xv[CPT];
    tload4<A>(xs + fr * NX + i0, xv);
    const T* erow = es + crow(fr) * NXc + (i0 >> 1);
    const A e0 = A(erow[0]) - she, e1 = A(erow[1]) - she;
    v[0] = (xv[0] - shx) + e0;
    v[1] = (xv[1] - shx) + e0;
    v[2] = (xv[2] - shx) + e1;
    v[3] = (xv[3] - shx) + e1;
  };
  double acc[1] = {0.0};
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, NX, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + CPT - 1, NX, o.periodic[0], o.dir_hi[0], xr, sxr);
  for(int q = 0; q < nseg; ++q) {
    const TSeg sg = seg[q];
    const int j0 = sg.tile * TY;
    const int j = j0 + r;
    int jm, jp;
    double sylo, syhi;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sylo);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, syhi);
    int cls[CPT];
#pragma unroll
    for(int t = 0; t < CPT; ++t) cls[t] = axis_class(i0 + t, NX) + 4 * axis_class(j, NY);
    auto own = [&](int l, A (&v)[CPT]) {
      tma::mbar_wait(&bars[l % D], (l / D) & 1, fault, 1);
      double zs;
      vst::zrow(sg.kb - 1 + (l - sg.lbase), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], zs);
      operand(xslot(l % D), eslot(l % D), r + 1, v);
      if constexpr(!PER) {
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] *= A(zs);
      }
    };
    A below[CPT], cen[CPT], above[CPT];
    own(sg.lbase, below);
    own(sg.lbase + 1, cen);
    __syncthreads();
    for(int k = sg.kb; k < sg.ke; ++k) {
      const int c = sg.lbase + 1 + (k - sg.kb);
      if(threadIdx.x == 0) {
        tma::fence_proxy_async();
        while(next < nload && next <= c - 1 + D) issue(next++);
      }
      own(c + 1, above);
      const T* xs = xslot(c % D);
      const T* es = eslot(c % D);
      const B* bk = bslot(c % D);
      A dn[CPT], up[CPT];
      operand(xs, es, r, dn);
      operand(xs, es, r + 2, up);
      if constexpr(!PER) {
        const A sd = r == 0 ? A(sylo) : A(1), su = r == TY - 1 ? A(syhi) : A(1);
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] *= sd;
          up[t] *= su;
        }
      }
      const T* erow = es + crow(r + 1) * NXc;
      A left = (A(xs[(r + 1) * NX + xl]) - shx) + (A(erow[xl >> 1]) - she);
      A right = (A(xs[(r + 1) * NX + xr]) - shx) + (A(erow[xr >> 1]) - she);
      if constexpr(!PER) {
        left *= A(sxl);
        right *= A(sxr);
      }
      L bq[CPT];
      tload4<L>(bk + r * NX + i0, bq);
      const int cz = 16 * axis_class(k, NZ);
      A v[CPT];
      A ps0 = A(0);  // FP32: per-plane partial sum
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        const A l = t > 0 ? cen[t - 1] : left;
        const A rr = t < CPT - 1 ? cen[t + 1] : right;
        const A two_c = A(2) * cen[t];
        const A ax = -(rr - two_c + l) * ix - (up[t] - two_c + dn[t]) * iy - (above[t] - two_c + below[t]) * iz;
        if constexpr(PER)
          v[t] = (cen[t] - sin - sec) + om * (A(bq[t] - L(sb)) - ax) * A(invd_s[0]);
        else
          v[t] = cen[t] + om * (A(bq[t] - L(sb)) - ax) * A(invd_s[cls[t] + cz]);
        if constexpr(std::is_same_v<T, float>) ps0 += v[t];
        else acc[0] += double(v[t]);
      }
      if constexpr(std::is_same_v<T, float>) acc[0] += double(ps0);
      tstore4<T>(out + o.L.idx(i0, j, k), v);
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        below[t] = cen[t];
        cen[t] = above[t];
      }
      __syncthreads();
    }
  }
  const bool mx[1] = {false};
  const int n = o.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& st) { ls->sa = zm ? st.v[0] / n : 0.0; });
}

// A p on the plane pipeline (same contract as k_vapply_ap).
template <typename V, int CPT, bool PER>
__global__ void __launch_bounds__(1024 / CPT)
    k_tap(OpInfo o, const __grid_constant__ CUtensorMap pm, const __grid_constant__ CUtensorMap ph,
          V* __restrict__ ap, SolveScalars* sc, RedBuf rb, int* fault) {
  pdl_enter();
  constexpr int D = kTSlots;
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ uint64_t bars[D];
  const int NX = o.L.nx, NY = o.L.ny, NZ = o.L.nz;
  const int TY = 1024 / NX;
  const int tpr = NX / CPT;
  const int r = threadIdx.x / tpr;
  const int i0 = (threadIdx.x % tpr) * CPT;
  const size_t sbytes = tround(static_cast<size_t>(TY + 2) * NX * sizeof(V));
  const uint32_t tx_bytes = static_cast<uint32_t>((TY + 2) * NX * sizeof(V));
  auto slot = [&](int s) { return reinterpret_cast<V*>(tsm + s * sbytes); };
  TSeg seg[kTMaxSeg];
  int nload = 0;
  const int nseg = tsegments(NY / TY, NZ, seg, nload);
  auto issue = [&](int l) {
    int q = 0;
    while(q + 1 < nseg && seg[q + 1].lbase <= l) ++q;
    const int j0 = seg[q].tile * TY;
    int jm, jp;
    double sg;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sg);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, sg);
    const int kz = vst::zrow(seg[q].kb - 1 + (l - seg[q].lbase), NZ, o.periodic[2], o.dir_lo[2],
                             o.dir_hi[2], sg);
    const int sl = l % D;
    tma::mbar_arrive_expect_tx(&bars[sl], tx_bytes);
    tma::load_3d(slot(sl) + NX, &pm, &bars[sl], 0, j0, kz);
    tma::load_3d(slot(sl), &ph, &bars[sl], 0, jm, kz);
    tma::load_3d(slot(sl) + (TY + 1) * NX, &ph, &bars[sl], 0, jp, kz);
  };
  if(threadIdx.x == 0) {
    for(int sl = 0; sl < D; ++sl) tma::mbar_init(&bars[sl], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  int next = 0;
  if(threadIdx.x == 0)
    while(next < nload && next < D) issue(next++);
  const double sp = sc->sp;
  const double ix = o.inv2[0], iy = o.inv2[1], iz = o.inv2[2];
  double acc[3] = {0.0, 0.0, 0.0};
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, NX, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + CPT - 1, NX, o.periodic[0], o.dir_hi[0], xr, sxr);
  for(int q = 0; q < nseg; ++q) {
    const TSeg sg = seg[q];
    const int j0 = sg.tile * TY;
    const int j = j0 + r;
    int jm, jp;
    double sylo, syhi;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sylo);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, syhi);
    auto own = [&](int l, double (&v)[CPT]) {
      tma::mbar_wait(&bars[l % D], (l / D) & 1, fault, 1);
      double zs;
      vst::zrow(sg.kb - 1 + (l - sg.lbase), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], zs);
      tload4<double>(slot(l % D) + (r + 1) * NX + i0, v);
      if constexpr(!PER) {
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] = zs * (v[t] - sp);
      }
    };
    double below[CPT], cen[CPT], above[CPT];
    own(sg.lbase, below);
    own(sg.lbase + 1, cen);
    __syncthreads();
    for(int k = sg.kb; k < sg.ke; ++k) {
      const int c = sg.lbase + 1 + (k - sg.kb);
      if(threadIdx.x == 0) {
        tma::fence_proxy_async();
        while(next < nload && next <= c - 1 + D) issue(next++);
      }
      own(c + 1, above);
      const V* pk = slot(c % D);
      double dn[CPT], up[CPT];
      tload4<double>(pk + r * NX + i0, dn);
      tload4<double>(pk + (r + 2) * NX + i0, up);
      double left = double(pk[(r + 1) * NX + xl]), right = double(pk[(r + 1) * NX + xr]);
      if constexpr(!PER) {
        const double sd = r == 0 ? sylo : 1.0, su = r == TY - 1 ? syhi : 1.0;
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] = sd * (dn[t] - sp);
          up[t] = su * (up[t] - sp);
        }
        left = sxl * (left - sp);
        right = sxr * (right - sp);
      }
      double v[CPT];
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        const double l = t > 0 ? cen[t - 1] : left;
        const double rr = t < CPT - 1 ? cen[t + 1] : right;
        const double two_c = 2.0 * cen[t];
        v[t] = -(rr - two_c + l) * ix - (up[t] - two_c + dn[t]) * iy - (above[t] - two_c + below[t]) * iz;
        const double cs = PER ? cen[t] - sp : cen[t];
        acc[0] += v[t];
        acc[1] += cs * v[t];
        acc[2] += cs;
      }
      tstore4<V>(ap + o.L.idx(i0, j, k), v);
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        below[t] = cen[t];
        cen[t] = above[t];
      }
      __syncthreads();
    }
  }
  const bool mx[3] = {false, false, false};
  reduce_finish<3>(acc, mx, rb, [=](const Sums<3>& st) {
    const double sap = sc->zero_mean ? st.v[0] / sc->n : 0.0;
    sc->sap = sap;
    const double pap = st.v[1] - sap * st.v[2];
    sc->pap = pap;
    if(fabs(pap) < kSmallNumber) {
      sc->stop = 1;
    } else {
      sc->alpha = sc->rz / pap;
    }
  });
}

// Fused CG step on the plane pipeline: p = (z - sz) + beta (p_old - sp_old)
// (p = z - sz on the first body), A p, and the previous iteration's deferred
// solution update x = (x - sx) + alpha_old (p_old - sp_old)
// (linsolve/poisson_solver.cpp:762-766, one body later).  The staged operand
// is z + beta p_old: the operator annihilates the mean shifts wherever they
// are nonzero (periodic / all-Neumann problems).  Records sp, sap, pap and
// alpha as k_update_p and k_apply_ap do, and mean(x).
// Ring depth of k_tpap: its registers allow two blocks per SM, so FP32
// planes (half the bytes) get twice the slots to keep as many bytes in flight.
template <typename V>
constexpr int tpap_slots() {
  return 4;
}

template <typename T, typename V, bool PER>
__global__ void __launch_bounds__(256)
    k_tpap(OpInfo o, const __grid_constant__ CUtensorMap zm_, const __grid_constant__ CUtensorMap zh,
           const __grid_constant__ CUtensorMap pm0, const __grid_constant__ CUtensorMap ph0,
           const __grid_constant__ CUtensorMap pm1, const __grid_constant__ CUtensorMap ph1,
           const LevelScalars* ls0, V* p0, V* p1, V* __restrict__ ap, V* __restrict__ x,
           SolveScalars* sc, RedBuf rb, int* fault) {
  pdl_enter();
  using A = V;  // arithmetic of the vector type: FP64, or FP32 on the mixed path's inner solve
  constexpr int CPT = 4;
  constexpr int D = tpap_slots<V>();
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ uint64_t bars[D];
  const int NX = o.L.nx, NY = o.L.ny, NZ = o.L.nz;
  const int TY = 1024 / NX;
  const int tpr = NX / CPT;
  const int r = threadIdx.x / tpr;
  const int i0 = (threadIdx.x % tpr) * CPT;
  const size_t zbytes = tround(static_cast<size_t>(TY + 2) * NX * sizeof(T));
  const size_t sbytes = zbytes + tround(static_cast<size_t>(TY + 2) * NX * sizeof(V));
  const uint32_t tx_bytes = static_cast<uint32_t>((TY + 2) * NX * (sizeof(T) + sizeof(V)));
  auto zslot = [&](int s) { return reinterpret_cast<T*>(tsm + s * sbytes); };
  auto pslot = [&](int s) { return reinterpret_cast<V*>(tsm + s * sbytes + zbytes); };
  // p ping-pongs between two buffers: body b reads p_old from buffer
  // (b + 1) & 1 and writes p to buffer b & 1 (other blocks still read p_old)
  const int par = sc->body_runs & 1;
  const CUtensorMap* pm = par ? &pm0 : &pm1;
  const CUtensorMap* ph = par ? &ph0 : &ph1;
  V* p_out = par ? p1 : p0;
  TSeg seg[kTMaxSeg];
  int nload = 0;
  const int nseg = tsegments(NY / TY, NZ, seg, nload);
  auto issue = [&](int l) {
    int q = 0;
    while(q + 1 < nseg && seg[q + 1].lbase <= l) ++q;
    const int j0 = seg[q].tile * TY;
    int jm, jp;
    double sg;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sg);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, sg);
    const int kz = vst::zrow(seg[q].kb - 1 + (l - seg[q].lbase), NZ, o.periodic[2], o.dir_lo[2],
                             o.dir_hi[2], sg);
    const int sl = l % D;
    tma::mbar_arrive_expect_tx(&bars[sl], tx_bytes);
    tma::load_3d(zslot(sl) + NX, &zm_, &bars[sl], 0, j0, kz);
    tma::load_3d(zslot(sl), &zh, &bars[sl], 0, jm, kz);
    tma::load_3d(zslot(sl) + (TY + 1) * NX, &zh, &bars[sl], 0, jp, kz);
    tma::load_3d(pslot(sl) + NX, pm, &bars[sl], 0, j0, kz);
    tma::load_3d(pslot(sl), ph, &bars[sl], 0, jm, kz);
    tma::load_3d(pslot(sl) + (TY + 1) * NX, ph, &bars[sl], 0, jp, kz);
  };
  if(threadIdx.x == 0) {
    for(int sl = 0; sl < D; ++sl) tma::mbar_init(&bars[sl], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  int next = 0;
  if(threadIdx.x == 0)
    while(next < nload && next < D) issue(next++);
  const int first = sc->first;
  const A beta = A(first ? 0.0 : sc->beta);
  const A sz = A(ls0->sx), spo = A(sc->sp);
  const A alpha_old = A(sc->alpha), sx = A(sc->sx);
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  // raw operand z + beta p_old of the 4 cells at slot row fr
  auto operand = [&](int sl, int fr, A (&v)[CPT]) {
    A zv[CPT], pv[CPT];
    tload4<A>(zslot(sl) + fr * NX + i0, zv);
    tload4<A>(pslot(sl) + fr * NX + i0, pv);
#pragma unroll
    for(int t = 0; t < CPT; ++t) v[t] = zv[t] + beta * pv[t];
  };
  auto point = [&](int sl, int fr, int ii) {
    return A(zslot(sl)[fr * NX + ii]) + beta * A(pslot(sl)[fr * NX + ii]);
  };
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, NX, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + CPT - 1, NX, o.periodic[0], o.dir_hi[0], xr, sxr);
  for(int q = 0; q < nseg; ++q) {
    const TSeg sg = seg[q];
    const int j0 = sg.tile * TY;
    const int j = j0 + r;
    int jm, jp;
    double sylo, syhi;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sylo);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, syhi);
    auto own = [&](int l, A (&v)[CPT]) {
      tma::mbar_wait(&bars[l % D], (l / D) & 1, fault, 1);
      operand(l % D, r + 1, v);
      if constexpr(!PER) {
        double zs;
        vst::zrow(sg.kb - 1 + (l - sg.lbase), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], zs);
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] *= A(zs);
      }
    };
    A below[CPT], cen[CPT], above[CPT];
    own(sg.lbase, below);
    own(sg.lbase + 1, cen);
    // x of the own cells one plane ahead (plain loads, prefetched a step early)
    A xn[CPT] = {A(0), A(0), A(0), A(0)};
    if(!first) tload4<A>(x + o.L.idx(i0, j, sg.kb), xn);
    __syncthreads();
    for(int k = sg.kb; k < sg.ke; ++k) {
      const int c = sg.lbase + 1 + (k - sg.kb);
      if(threadIdx.x == 0) {
        tma::fence_proxy_async();
        while(next < nload && next <= c - 1 + D) issue(next++);
      }
      own(c + 1, above);
      const int sl = c % D;
      A dn[CPT], up[CPT];
      operand(sl, r, dn);
      operand(sl, r + 2, up);
      A left = point(sl, r + 1, xl), right = point(sl, r + 1, xr);
      if constexpr(!PER) {
        const A sd = A(r == 0 ? sylo : 1.0), su = A(r == TY - 1 ? syhi : 1.0);
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] *= sd;
          up[t] *= su;
        }
        left *= A(sxl);
        right *= A(sxr);
      }
      // own cells: exact p (with shifts), the deferred x update
      A zc[CPT], pc[CPT];
      tload4<A>(zslot(sl) + (r + 1) * NX + i0, zc);
      tload4<A>(pslot(sl) + (r + 1) * NX + i0, pc);
      A pn[CPT], apv[CPT];
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        const A l = t > 0 ? cen[t - 1] : left;
        const A rr = t < CPT - 1 ? cen[t + 1] : right;
        const A two_c = A(2) * cen[t];
        apv[t] = -(rr - two_c + l) * ix - (up[t] - two_c + dn[t]) * iy - (above[t] - two_c + below[t]) * iz;
        pn[t] = first ? zc[t] - sz : (zc[t] - sz) + beta * (pc[t] - spo);
      }
      const size_t gq = o.L.idx(i0, j, k);
      tstore4<V>(p_out + gq, pn);
      tstore4<V>(ap + gq, apv);
      if(!first) {
        A xv[CPT];
#pragma unroll
        for(int t = 0; t < CPT; ++t) xv[t] = xn[t];
        if(k + 1 < sg.ke) tload4<A>(x + o.L.idx(i0, j, k + 1), xn);
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          xv[t] = (xv[t] - sx) + alpha_old * (pc[t] - spo);
          acc[3] += double(xv[t]);
        }
        tstore4<V>(x + gq, xv);
      }
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        acc[0] += double(pn[t]);
        acc[1] += double(apv[t]);
        acc[2] += double(pn[t]) * double(apv[t]);
        below[t] = cen[t];
        cen[t] = above[t];
      }
      __syncthreads();
    }
  }
  const bool mx[4] = {false, false, false, false};
  reduce_finish<4>(acc, mx, rb, [=](const Sums<4>& st) {
    const int n = sc->n;
    const int zmn = sc->zero_mean;
    const double sp = zmn ? st.v[0] / n : 0.0;
    const double sap = zmn ? st.v[1] / n : 0.0;
    sc->sp = sp;
    sc->sap = sap;
    if(!first) sc->sx = zmn ? st.v[3] / n : 0.0;
    sc->first = 0;
    const double pap = st.v[2] - sp * st.v[1] - sap * st.v[0] + n * sp * sap;
    sc->pap = pap;
    if(fabs(pap) < kSmallNumber) {
      sc->stop = 1;
    } else {
      sc->alpha = sc->rz / pap;
    }
  });
}

// r = (r - sr) - alpha (Ap - sap), its norm and the convergence test: the
// residual half of k_update_xr for the fused CG step (x is updated one body
// later by k_tpap, and after the loop by k_x_final).  The compact vector is
// one contiguous array, so it is swept flat, 16 bytes per load (float4 /
// double2) with kFlatUnroll loads of each operand in flight per thread.
constexpr int kFlatUnroll = 4;
constexpr int kFlatThreads = 256;

template <typename V>
struct Vec16;
template <>
struct Vec16<float> {
  using T = float4;
  static constexpr int W = 4;
};
template <>
struct Vec16<double> {
  using T = double2;
  static constexpr int W = 2;
};

template <typename V>
__global__ void __launch_bounds__(kFlatThreads)
    k_update_r_flat(int n, V* __restrict__ r, const V* __restrict__ ap, SolveScalars* sc, RedBuf rb,
                    cudaGraphConditionalHandle cond) {
  pdl_enter();
  using VT = typename Vec16<V>::T;
  constexpr int W = Vec16<V>::W;
  const int stop = sc->stop;
  const double alpha = sc->alpha, sr = sc->sr, sap = sc->sap;
  double acc[2];
  zero(acc);
  if(!stop) {
    const int nv = n / W;
    const int stride = gridDim.x * blockDim.x;
    VT* rv = reinterpret_cast<VT*>(r);
    const VT* av = reinterpret_cast<const VT*>(ap);
    for(int base = blockIdx.x * blockDim.x + threadIdx.x; base < nv; base += kFlatUnroll * stride) {
      VT rr[kFlatUnroll], aa[kFlatUnroll];
#pragma unroll
      for(int u = 0; u < kFlatUnroll; ++u) {
        const int q = base + u * stride;
        if(q < nv) {
          rr[u] = rv[q];
          aa[u] = av[q];
        }
      }
#pragma unroll
      for(int u = 0; u < kFlatUnroll; ++u) {
        const int q = base + u * stride;
        if(q < nv) {
          V* rs = reinterpret_cast<V*>(&rr[u]);
          const V* as = reinterpret_cast<const V*>(&aa[u]);
#pragma unroll
          for(int w = 0; w < W; ++w) {
            const double v = (double(rs[w]) - sr) - alpha * (double(as[w]) - sap);
            rs[w] = V(v);
            acc[0] += v;
            acc[1] += v * v;
          }
          rv[q] = rr[u];
        }
      }
    }
    // the n % W elements past the last full vector
    for(int q = nv * W + blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
      const double v = (double(r[q]) - sr) - alpha * (double(ap[q]) - sap);
      r[q] = V(v);
      acc[0] += v;
      acc[1] += v * v;
    }
  }
  const bool mx[2] = {false, false};
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    sc->body_runs += 1;
    if(sc->stop) {
      sc->cont = 0;
      if(cond) cudaGraphSetConditional(cond, 0);
      return;
    }
    const int nn = sc->n;
    const int zm = sc->zero_mean;
    const double srn = zm ? s.v[0] / nn : 0.0;
    sc->sr = srn;
    sc->sum_r = s.v[0];
    const double ss = fmax(s.v[1] - nn * srn * srn, 0.0);
    sc->rnorm = sqrt(ss / nn);
    sc->iterations += 1;
    sc->rel = sc->r0 > 0.0 ? sc->rnorm / sc->r0 : 0.0;
    if(sc->rel <= sc->tol) sc->converged = 1;
    if(sc->hist != nullptr && sc->iterations < sc->hist_cap) sc->hist[sc->iterations] = sc->rnorm;
    sc->cont = (sc->converged || sc->iterations >= sc->max_it) ? 0 : 1;
    if(cond) cudaGraphSetConditional(cond, sc->cont);
  });
}

// After a fused-step loop: the last deferred update x = (x - sx) + alpha (p - sp)
// unless the loop stopped on a vanishing p.Ap (then the reference skips it).
template <typename V>
__global__ void __launch_bounds__(kTX* kTY)
    k_x_final(CLay L, V* __restrict__ x, const V* p0, const V* p1, SolveScalars* sc, int kchunk, RedBuf rb) {
  STENCIL_PROLOGUE(L)
  const int skip = sc->stop || sc->body_runs == 0;
  const V* __restrict__ p = ((sc->body_runs - 1) & 1) ? p1 : p0;
  const double alpha = sc->alpha, sx = sc->sx, sp = sc->sp;
  double acc[1];
  zero(acc);
  if(valid && !skip) {
    for(int k = k0; k < k1; ++k) {
      const int q = L.idx(i, j, k);
      const double v = (double(x[q]) - sx) + alpha * (double(p[q]) - sp);
      x[q] = V(v);
      acc[0] += v;
    }
  }
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) {
    if(!skip) sc->sx = sc->zero_mean ? s.v[0] / sc->n : 0.0;
  });
}

// Residual + 2x2x2 restriction on the plane pipeline (same contract as
// k_vrestrict): each step forms the residual (b - sb) - A (x - sx) on the two
// fine planes of one coarse plane; a thread sums its cells pairwise in x and
// over the two planes, and the row pairs are combined through shared memory.
// The schedule runs over coarse planes, so each segment streams fine planes
// 2 kc_begin - 1 .. 2 kc_end.
template <typename T, typename B, int D, bool PER>
__global__ void __launch_bounds__(256)
    k_trestrict(OpInfo o, OpInfo oc, const __grid_constant__ CUtensorMap xm,
                const __grid_constant__ CUtensorMap xh, const __grid_constant__ CUtensorMap bm,
                const double* sb_ptr, const double* sin_ptr, T* __restrict__ bc, LevelScalars* lsc,
                int zm, RedBuf rb, int* fault) {
  pdl_enter();
  using A = T;
  constexpr int CPT = 4;
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ uint64_t bars[D];
  const int NX = o.L.nx, NY = o.L.ny, NZ = o.L.nz;
  const int TY = 1024 / NX;
  const int tpr = NX / CPT;
  const int r = threadIdx.x / tpr;
  const int i0 = (threadIdx.x % tpr) * CPT;
  const size_t ubytes = tround(static_cast<size_t>(TY + 2) * NX * sizeof(T));
  const size_t sbytes = tslot_bytes<T, B>(NX);
  const uint32_t tx_bytes = static_cast<uint32_t>((TY + 2) * NX * sizeof(T) + TY * NX * sizeof(B));
  auto uslot = [&](int s) { return reinterpret_cast<T*>(tsm + s * sbytes); };
  auto bslot = [&](int s) { return reinterpret_cast<B*>(tsm + s * sbytes + ubytes); };
  A* part = reinterpret_cast<A*>(tsm + D * sbytes);  // [TY][NX / 2] row partials
  // segments over coarse planes; loads count fine planes
  TSeg seg[kTMaxSeg];
  int nseg = 0, nload = 0;
  if(gridDim.x % (NY / TY) == 0) {
    // z-aligned schedule over coarse planes (as in tsegments)
    const int tiles = NY / TY, nzc = NZ / 2, nch = gridDim.x / tiles;
    const int tile = blockIdx.x % tiles, zc = blockIdx.x / tiles;
    const int kb = static_cast<int>(static_cast<long long>(nzc) * zc / nch);
    const int ke = static_cast<int>(static_cast<long long>(nzc) * (zc + 1) / nch);
    if(ke > kb) {
      seg[nseg++] = TSeg{tile, kb, ke, 0};
      nload = 2 * (ke - kb) + 2;
    }
  } else {
    const int nzc = NZ / 2;
    const long long total = static_cast<long long>(NY / TY) * nzc;
    const long long f0 = total * blockIdx.x / gridDim.x;
    const long long f1 = total * (blockIdx.x + 1) / gridDim.x;
    for(long long f = f0; f < f1 && nseg < kTMaxSeg;) {
      const int tile = static_cast<int>(f / nzc);
      const int kb = static_cast<int>(f % nzc);
      const int ke = static_cast<int>(min(static_cast<long long>(nzc), kb + (f1 - f)));
      seg[nseg++] = TSeg{tile, kb, ke, nload};
      nload += 2 * (ke - kb) + 2;
      f += ke - kb;
    }
  }
  auto fine_plane = [&](const TSeg& sg, int l) { return 2 * sg.kb - 1 + (l - sg.lbase); };
  auto issue = [&](int l) {
    int q = 0;
    while(q + 1 < nseg && seg[q + 1].lbase <= l) ++q;
    const int j0 = seg[q].tile * TY;
    int jm, jp;
    double sg;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sg);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, sg);
    const int kz = vst::zrow(fine_plane(seg[q], l), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], sg);
    const int sl = l % D;
    tma::mbar_arrive_expect_tx(&bars[sl], tx_bytes);
    tma::load_3d(uslot(sl) + NX, &xm, &bars[sl], 0, j0, kz);
    tma::load_3d(uslot(sl), &xh, &bars[sl], 0, jm, kz);
    tma::load_3d(uslot(sl) + (TY + 1) * NX, &xh, &bars[sl], 0, jp, kz);
    tma::load_3d(bslot(sl), &bm, &bars[sl], 0, j0, kz);
  };
  if(threadIdx.x == 0) {
    for(int sl = 0; sl < D; ++sl) tma::mbar_init(&bars[sl], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  int next = 0;
  if(threadIdx.x == 0)
    while(next < nload && next < D) issue(next++);
  const double sb = *sb_ptr;
  const A sin = A(*sin_ptr);
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  double acc[1] = {0.0};
  int xl, xr;
  double sxl, sxr;
  nb_lo(i0, NX, o.periodic[0], o.dir_lo[0], xl, sxl);
  nb_hi(i0 + CPT - 1, NX, o.periodic[0], o.dir_hi[0], xr, sxr);
  for(int q = 0; q < nseg; ++q) {
    const TSeg sg = seg[q];
    const int j0 = sg.tile * TY;
    const int j = j0 + r;
    int jm, jp;
    double sylo, syhi;
    nb_lo(j0, NY, o.periodic[1], o.dir_lo[1], jm, sylo);
    nb_hi(j0 + TY - 1, NY, o.periodic[1], o.dir_hi[1], jp, syhi);
    auto own = [&](int l, A (&v)[CPT]) {
      tma::mbar_wait(&bars[l % D], (l / D) & 1, fault, 1);
      double zs;
      vst::zrow(fine_plane(sg, l), NZ, o.periodic[2], o.dir_lo[2], o.dir_hi[2], zs);
      tload4<A>(uslot(l % D) + (r + 1) * NX + i0, v);
      if constexpr(!PER) {
#pragma unroll
        for(int t = 0; t < CPT; ++t) v[t] = A(zs) * (v[t] - sin);
      }
    };
    // residual of the CPT cells at the plane staged in load c
    auto residual = [&](int c, const A (&below)[CPT], const A (&cen)[CPT], const A (&above)[CPT],
                        A (&res)[CPT]) {
      const T* pk = uslot(c % D);
      const B* bk = bslot(c % D);
      A dn[CPT], up[CPT];
      tload4<A>(pk + r * NX + i0, dn);
      tload4<A>(pk + (r + 2) * NX + i0, up);
      A left = pk[(r + 1) * NX + xl], right = pk[(r + 1) * NX + xr];
      if constexpr(!PER) {
        const A sd = r == 0 ? A(sylo) : A(1), su = r == TY - 1 ? A(syhi) : A(1);
#pragma unroll
        for(int t = 0; t < CPT; ++t) {
          dn[t] = sd * (dn[t] - sin);
          up[t] = su * (up[t] - sin);
        }
        left = A(sxl) * (left - sin);
        right = A(sxr) * (right - sin);
      }
      double bq[CPT];
      tload4<double>(bk + r * NX + i0, bq);
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        const A l = t > 0 ? cen[t - 1] : left;
        const A rr = t < CPT - 1 ? cen[t + 1] : right;
        const A two_c = A(2) * cen[t];
        const A ax = -(rr - two_c + l) * ix - (up[t] - two_c + dn[t]) * iy - (above[t] - two_c + below[t]) * iz;
        res[t] = A(bq[t] - sb) - ax;
      }
    };
    A q0[CPT], q1[CPT], q2[CPT], q3[CPT];
    own(sg.lbase, q0);
    own(sg.lbase + 1, q1);
    __syncthreads();
    for(int kc = sg.kb; kc < sg.ke; ++kc) {
      const int c = sg.lbase + 1 + 2 * (kc - sg.kb);  // load of fine plane 2 kc
      if(threadIdx.x == 0) {
        tma::fence_proxy_async();
        while(next < nload && next <= c - 1 + D) issue(next++);
      }
      own(c + 1, q2);
      own(c + 2, q3);
      A r0[CPT], r1[CPT];
      residual(c, q0, q1, q2, r0);
      residual(c + 1, q1, q2, q3, r1);
      part[r * (NX / 2) + (i0 >> 1)] = (r0[0] + r0[1]) + (r1[0] + r1[1]);
      part[r * (NX / 2) + (i0 >> 1) + 1] = (r0[2] + r0[3]) + (r1[2] + r1[3]);
#pragma unroll
      for(int t = 0; t < CPT; ++t) {
        q0[t] = q2[t];
        q1[t] = q3[t];
      }
      __syncthreads();
      if((r & 1) == 0) {
        const int m = i0 >> 1;
        const A c0 = A(0.125) * (part[r * (NX / 2) + m] + part[(r + 1) * (NX / 2) + m]);
        const A c1 = A(0.125) * (part[r * (NX / 2) + m + 1] + part[(r + 1) * (NX / 2) + m + 1]);
        T* dst = bc + oc.L.idx(m, j >> 1, kc);
        if constexpr(std::is_same_v<T, double>) {
          *reinterpret_cast<double2*>(dst) = make_double2(c0, c1);
        } else {
          *reinterpret_cast<float2*>(dst) = make_float2(c0, c1);
        }
        acc[0] += double(c0) + double(c1);
      }
      __syncthreads();
    }
  }
  const bool mx[1] = {false};
  const int n = oc.L.count();
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& st) { lsc->sb = zm ? st.v[0] / n : 0.0; });
}

// ---------------------------------------------------------------------------
// The small end of the hierarchy in one block.  From the first level of at
// most kTailMaxCells cells down to the coarsest, v_cycle (:597-633) runs in
// one block with every level's rhs, correction and scratch in shared memory.
// Each phase ends with one barrier that also publishes the warp partials of
// the vector it produced; every thread then adds the partials itself (same
// order in every thread), so the mean of the reference's subtract_active_mean
// (after every sweep, on the residual, on the coarse rhs, after the
// prolongation) is known without a second barrier and is subtracted as the
// next phase loads the vector (a pending shift), as in the per-level kernels.
// The two pre-sweeps from zero are one phase (k_vsmooth_pre), the
// prolongation and the first post-sweep another (k_vprolong_smooth).
// ---------------------------------------------------------------------------
constexpr int kTailMaxCells = 4096;
constexpr int kTailMaxLevels = 12;
constexpr int kTailThreads = 512;

// Per tail level (all but the coarsest), built on the host when the plan is
// made and staged into shared memory by every tail launch:
//   nbr[6][n]   the six operand positions of each cell under the boundary
//               rules (nb_lo / nb_hi: neighbour, periodic image, or the cell
//               itself), as +-(index + 1), minus for a homogeneous-Dirichlet
//               image (ghost = -centre); order x-, x+, y-, y+, z-, z+
//   parent[n]   the cell's parent on the next coarser level
//   child[nc][nch]  each coarser cell's children in dz, dy, dx order
//   cls[n]      the cell's boundary class (x + 4 y + 16 z, each 0 interior,
//               1 first, 2 last, 3 both) and
//   itab[64]    the Jacobi inverse diagonal of each class (T)
// so a tail phase does no index arithmetic and reads no boundary flags.
struct TailLevel {
  OpInfo op;
  int sx, sy, sz;  // log2 of the refinement ratio to the next coarser level
  int off;         // offset of the level's b, x, s arrays in shared memory (elements)
  int tab;         // byte offset of the level's tables in the table region
  int nch;         // children per coarser cell
  double d0;       // the inverse diagonal, where every class has the same one
};

struct TailArgs {
  int count;  // levels in the tail; the last one is the coarsest
  TailLevel lv[kTailMaxLevels];
  int coarse_n;
  int coarse_off;  // offset (elements, 8-byte aligned) of the FP64 solve vector
  int fact_off;    // offset (8-byte aligned) of the staged factors (coarse_n <= 32)
  int tab_off;     // byte offset (16-aligned) of the table region in shared memory
  int tab_bytes;   // its size (a multiple of 16)
  const unsigned char* tabs;  // the tables in device memory
  const int* swaps;
  const double* factors;
  int zm;
  // every tail level fully periodic with power-of-two extents and one
  // inverse diagonal: neighbours, parents and children by bit arithmetic
  // (PerGeom), no tables staged
  int per;
};

// Byte layout of one tail level's tables (see TailLevel).
struct TailTabLayout {
  size_t nbr, parent, child, cls, itab, bytes;
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) / 16 * 16; }

__host__ __device__ inline TailTabLayout tail_tab_layout(int n, int nc, int nch, size_t tsz) {
  TailTabLayout t;
  t.nbr = 0;
  t.parent = 12 * static_cast<size_t>(n);
  t.child = t.parent + 2 * static_cast<size_t>(n);
  t.cls = t.child + 2 * static_cast<size_t>(nc) * nch;
  t.itab = align16(t.cls + static_cast<size_t>(n));
  t.bytes = align16(t.itab + 64 * tsz);
  return t;
}

// Block-wide sum; every thread gets the same total (fixed order).  red has
// 33 entries: the warp partials and the total.
__device__ __forceinline__ double tail_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if(lane == 0) red[warp] = v;
  __syncthreads();
  if(warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double x = lane < nw ? red[lane] : 0.0;
    x = warp_sum(x);
    if(lane == 0) red[32] = x;
  }
  __syncthreads();
  return red[32];
}

// Ends a tail phase: the block barrier, with the block-wide sum of v (warp
// partials alternate between two rows of red so that a fast thread's next
// phase never overwrites partials a slow thread is still adding).
__device__ __forceinline__ double tail_phase_sum(double v, double (*red)[32], int& par) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if(lane == 0) red[par][warp] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  double t = 0.0;
  for(int w = 0; w < nw; ++w) t += red[par][w];
  par ^= 1;
  return t;
}

// One operand value through a table entry e = +-(index + 1).
template <typename A, typename Op>
__device__ __forceinline__ A tab_nb(int e, Op op) {
  const A v = op(e < 0 ? -e - 1 : e - 1);
  return e < 0 ? -v : v;
}

// A u at cell q from the staged neighbour table; c gets u at q.
template <typename A, typename Op>
__device__ __forceinline__ A tab_apply(const short* nbr, int n, int q, A ix, A iy, A iz, Op op, A& c) {
  c = op(q);
  const A l = tab_nb<A>(nbr[q], op);
  const A r = tab_nb<A>(nbr[n + q], op);
  const A d = tab_nb<A>(nbr[2 * n + q], op);
  const A u = tab_nb<A>(nbr[3 * n + q], op);
  const A b = tab_nb<A>(nbr[4 * n + q], op);
  const A f = tab_nb<A>(nbr[5 * n + q], op);
  const A two_c = A(2) * c;
  return -(r - two_c + l) * ix - (u - two_c + d) * iy - (f - two_c + b) * iz;
}

// Index arithmetic of a periodic level with power-of-two extents: the same
// operand positions, parents and children (dz, dy, dx order) as the tables.
struct PerGeom {
  int lx, ly, mx, my, mz;  // log2 nx, log2 ny, nx - 1, ny - 1, nz - 1
};

__device__ __forceinline__ PerGeom per_geom(const CLay& L) {
  return PerGeom{__ffs(L.nx) - 1, __ffs(L.ny) - 1, L.nx - 1, L.ny - 1, L.nz - 1};
}

// A u at cell q (same operand order and arithmetic as tab_apply).
template <typename A, typename Op>
__device__ __forceinline__ A per_apply(const PerGeom& g, int q, A ix, A iy, A iz, Op op, A& c) {
  const int i = q & g.mx, j = (q >> g.lx) & g.my, sh = g.lx + g.ly, k = q >> sh;
  const int qi = q - i, qj = q - (j << g.lx), qk = q - (k << sh);
  c = op(q);
  const A l = op(qi + ((i - 1) & g.mx));
  const A r = op(qi + ((i + 1) & g.mx));
  const A d = op(qj + (((j - 1) & g.my) << g.lx));
  const A u = op(qj + (((j + 1) & g.my) << g.lx));
  const A b = op(qk + (((k - 1) & g.mz) << sh));
  const A f = op(qk + (((k + 1) & g.mz) << sh));
  const A two_c = A(2) * c;
  return -(r - two_c + l) * ix - (u - two_c + d) * iy - (f - two_c + b) * iz;
}

// The whole tail V-cycle in the calling block: b_in (shift sb) in, x_out
// (mean removed) out; sm is the tail's shared-memory layout (TailArgs).
template <typename T, bool PER>
__device__ void vcycle_tail_body(const TailArgs& a, const T* __restrict__ b_in, double sb,
                                 T* __restrict__ x_out, T* sm) {
  using A = T;
  __shared__ double red[2][32];
  int par = 0;
  const int tid = threadIdx.x, bd = blockDim.x;
  const int zm = a.zm;
  const A om = A(kOmega);
  auto B = [&](int l) { return sm + a.lv[l].off; };
  auto X = [&](int l) { return sm + a.lv[l].off + a.lv[l].op.L.count(); };
  auto S = [&](int l) { return sm + a.lv[l].off + 2 * a.lv[l].op.L.count(); };
  unsigned char* tabs = reinterpret_cast<unsigned char*>(sm) + a.tab_off;
  const int last = a.count - 1;
  const int nco = a.coarse_n;
  double* fact = reinterpret_cast<double*>(sm + a.fact_off);
  int* swp = reinterpret_cast<int*>(fact + (nco <= 32 ? nco * nco : 0));
  if(nco <= 32) {
    // the coarse factors, read by the one-warp elimination below
    for(int q = tid; q < nco * nco; q += bd) fact[q] = a.factors[q];
    for(int q = tid; q < nco; q += bd) swp[q] = a.swaps[q];
  }
  {
    if constexpr(!PER) {
      const uint4* src = reinterpret_cast<const uint4*>(a.tabs);
      uint4* dst = reinterpret_cast<uint4*>(tabs);
      for(int q = tid; q < a.tab_bytes / 16; q += bd) dst[q] = __ldg(&src[q]);
    }
    const int n0 = a.lv[0].op.L.count();
    for(int q = tid; q < n0; q += bd) B(0)[q] = A(double(b_in[q]) - sb);
  }
  __syncthreads();
  double sbs[kTailMaxLevels], sxs[kTailMaxLevels];
  sbs[0] = 0.0;
  // descent
  for(int l = 0; l < last; ++l) {
    const TailLevel& tl = a.lv[l];
    const int n = tl.op.L.count();
    const int nc = a.lv[l + 1].op.L.count();
    const TailTabLayout lay = tail_tab_layout(n, nc, tl.nch, sizeof(T));
    const short* nbr = reinterpret_cast<const short*>(tabs + tl.tab + lay.nbr);
    const short* child = reinterpret_cast<const short*>(tabs + tl.tab + lay.child);
    const unsigned char* cls = tabs + tl.tab + lay.cls;
    const A* itab = reinterpret_cast<const A*>(tabs + tl.tab + lay.itab);
    const A d0 = A(tl.d0);
    auto dinv = [&](int p) {
      if constexpr(PER) return d0;
      else return itab[cls[p]];
    };
    const PerGeom pg = per_geom(tl.op.L);
    const A ix = A(tl.op.inv2[0]), iy = A(tl.op.inv2[1]), iz = A(tl.op.inv2[2]);
    auto apply = [&](int q, auto op, A& c) {
      if constexpr(PER) return per_apply<A>(pg, q, ix, iy, iz, op, c);
      else return tab_apply<A>(nbr, n, q, ix, iy, iz, op, c);
    };
    const A* b = B(l);
    A* x = X(l);
    A* s = S(l);
    const A sbl = A(sbs[l]);
    // both pre-sweeps from a zero correction
    double part = 0.0;
    for(int q = tid; q < n; q += bd) {
      A c;
      const A ax = apply(q, [&](int p) { return om * (b[p] - sbl) * dinv(p); }, c);
      const A v = c + om * ((b[q] - sbl) - ax) * dinv(q);
      x[q] = v;
      part += double(v);
    }
    {
      const double t = tail_phase_sum(part, red, par);
      sxs[l] = zm ? t / n : 0.0;
    }
    // residual (b - sb) - A (x - sx)
    const A sxl = A(sxs[l]);
    for(int q = tid; q < n; q += bd) {
      A c;
      const A ax = apply(q, [&](int p) { return x[p] - sxl; }, c);
      s[q] = (b[q] - sbl) - ax;
    }
    __syncthreads();
    // restrict_full_weighting (:397-424), children in dz, dy, dx order
    const int nch = tl.nch;
    const A inv_children = A(1.0 / double(nch));
    A* bc = B(l + 1);
    part = 0.0;
    const PerGeom cg = per_geom(a.lv[l + 1].op.L);
    for(int Q = tid; Q < nc; Q += bd) {
      A sum = A(0);
      if constexpr(PER) {
        const int I = Q & cg.mx, J = (Q >> cg.lx) & cg.my, K = Q >> (cg.lx + cg.ly);
        for(int dz = 0; dz < (1 << tl.sz); ++dz)
          for(int dy = 0; dy < (1 << tl.sy); ++dy)
            for(int dx = 0; dx < (1 << tl.sx); ++dx)
              sum += s[((I << tl.sx) + dx) + (((J << tl.sy) + dy) << pg.lx) +
                       (((K << tl.sz) + dz) << (pg.lx + pg.ly))];
      } else {
        for(int t = 0; t < nch; ++t) sum += s[child[Q * nch + t]];
      }
      const A v = inv_children * sum;
      bc[Q] = v;
      part += double(v);
    }
    {
      const double t = tail_phase_sum(part, red, par);
      sbs[l + 1] = zm ? t / nc : 0.0;
    }
  }
  // direct_coarse_solve (:530-567): the host elimination replayed on the rhs
  // (its mean removed first, as the reference does before the solve).  Up to
  // 32 unknowns (every grid the hierarchy coarsens to 2 per axis) one warp
  // replays it with the rhs in registers and the factors in shared memory,
  // the same operations in the same order as the block-wide form below.
  if(nco <= 32) {
    const int n = nco;
    if(tid < 32) {
      constexpr unsigned kFull = 0xffffffffu;
      const int lane = tid;
      double yv = lane < n ? double(B(last)[lane]) - sbs[last] : 0.0;
      if(zm && lane == n - 1) yv = 0.0;
      for(int p = 0; p < n; ++p) {
        const int sp = swp[p];
        if(sp != p) {
          const double at_p = __shfl_sync(kFull, yv, p);
          const double at_s = __shfl_sync(kFull, yv, sp);
          if(lane == p) yv = at_s;
          else if(lane == sp) yv = at_p;
        }
        const double yp = __shfl_sync(kFull, yv, p);
        if(lane > p && lane < n) {
          const double factor = fact[lane * n + p];
          if(factor != 0.0) yv -= factor * yp;
        }
      }
      for(int row = n - 1; row >= 0; --row) {
        if(lane == row) yv = yv / fact[row * n + row];
        const double yr = __shfl_sync(kFull, yv, row);
        if(lane < row) yv -= fact[lane * n + row] * yr;
      }
      const double sum = __shfl_sync(kFull, warp_sum(lane < n ? yv : 0.0), 0);
      const double mean = zm ? sum / n : 0.0;
      if(lane < n) X(last)[lane] = A(yv - mean);
    }
    __syncthreads();
  } else {
    const int n = nco;
    __shared__ double cred[33];
    A* y = B(last);
    A* xc = X(last);
    double* yd = reinterpret_cast<double*>(sm + a.coarse_off);  // solve in FP64
    for(int q = tid; q < n; q += bd) yd[q] = double(y[q]) - sbs[last];
    __syncthreads();
    if(zm && tid == 0) yd[n - 1] = 0.0;
    __syncthreads();
    for(int p = 0; p < n; ++p) {
      if(tid == 0 && a.swaps[p] != p) {
        const double tmp = yd[p];
        yd[p] = yd[a.swaps[p]];
        yd[a.swaps[p]] = tmp;
      }
      __syncthreads();
      const double yp = yd[p];
      for(int r = p + 1 + tid; r < n; r += bd) {
        const double factor = a.factors[static_cast<size_t>(r) * n + p];
        if(factor != 0.0) yd[r] -= factor * yp;
      }
      __syncthreads();
    }
    for(int row = n - 1; row >= 0; --row) {
      if(tid == 0) yd[row] = yd[row] / a.factors[static_cast<size_t>(row) * n + row];
      __syncthreads();
      const double yr = yd[row];
      for(int r = tid; r < row; r += bd) yd[r] -= a.factors[static_cast<size_t>(r) * n + row] * yr;
      __syncthreads();
    }
    double part = 0.0;
    for(int q = tid; q < n; q += bd) part += yd[q];
    const double sum = tail_sum(part, cred);
    const double mean = zm ? sum / n : 0.0;
    for(int q = tid; q < n; q += bd) xc[q] = A(yd[q] - mean);
    __syncthreads();
  }
  // ascent: prolongate_and_add (:426-451) + first post-sweep, second post-sweep
  double sxc = 0.0;  // the coarse correction has its mean removed
  for(int l = last - 1; l >= 0; --l) {
    const TailLevel& tl = a.lv[l];
    const int n = tl.op.L.count();
    const int nc = a.lv[l + 1].op.L.count();
    const TailTabLayout lay = tail_tab_layout(n, nc, tl.nch, sizeof(T));
    const short* nbr = reinterpret_cast<const short*>(tabs + tl.tab + lay.nbr);
    const short* parent = reinterpret_cast<const short*>(tabs + tl.tab + lay.parent);
    const unsigned char* cls = tabs + tl.tab + lay.cls;
    const A* itab = reinterpret_cast<const A*>(tabs + tl.tab + lay.itab);
    const A d0 = A(tl.d0);
    auto dinv = [&](int p) {
      if constexpr(PER) return d0;
      else return itab[cls[p]];
    };
    const PerGeom pg = per_geom(tl.op.L);
    const PerGeom cg = per_geom(a.lv[l + 1].op.L);
    auto parent_of = [&](int p) {
      if constexpr(PER) {
        const int i = p & pg.mx, j = (p >> pg.lx) & pg.my, k = p >> (pg.lx + pg.ly);
        return (i >> tl.sx) + ((j >> tl.sy) << cg.lx) + ((k >> tl.sz) << (cg.lx + cg.ly));
      } else {
        return static_cast<int>(parent[p]);
      }
    };
    const A ix = A(tl.op.inv2[0]), iy = A(tl.op.inv2[1]), iz = A(tl.op.inv2[2]);
    auto apply = [&](int q, auto op, A& c) {
      if constexpr(PER) return per_apply<A>(pg, q, ix, iy, iz, op, c);
      else return tab_apply<A>(nbr, n, q, ix, iy, iz, op, c);
    };
    const A* b = B(l);
    A* x = X(l);
    A* s = S(l);
    const A* xc = X(l + 1);
    const A sbl = A(sbs[l]), sxl = A(sxs[l]), sec = A(sxc);
    double part = 0.0;
    for(int q = tid; q < n; q += bd) {
      A c;
      const A ax = apply(q, [&](int p) { return (x[p] - sxl) + (xc[parent_of(p)] - sec); }, c);
      const A v = c + om * ((b[q] - sbl) - ax) * dinv(q);
      s[q] = v;
      part += double(v);
    }
    double sa;
    {
      const double t = tail_phase_sum(part, red, par);
      sa = zm ? t / n : 0.0;
    }
    const A saa = A(sa);
    part = 0.0;
    for(int q = tid; q < n; q += bd) {
      A c;
      const A ax = apply(q, [&](int p) { return s[p] - saa; }, c);
      const A v = c + om * ((b[q] - sbl) - ax) * dinv(q);
      x[q] = v;
      part += double(v);
    }
    {
      const double t = tail_phase_sum(part, red, par);
      sxc = zm ? t / n : 0.0;
    }
  }
  const int n0 = a.lv[0].op.L.count();
  const A s0 = A(sxc);
  for(int q = tid; q < n0; q += bd) x_out[q] = X(0)[q] - s0;
}

template <typename T, bool PER>
__global__ void __launch_bounds__(kTailThreads)
    k_vcycle_tail(TailArgs a, const T* __restrict__ b_in, const double* sb_ptr, T* __restrict__ x_out,
                  LevelScalars* ls_out) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char tail_smem[];
  vcycle_tail_body<T, PER>(a, b_in, *sb_ptr, x_out, reinterpret_cast<T*>(tail_smem));
  if(threadIdx.x == 0) {
    ls_out->sx = 0.0;  // the mean is already removed
    ls_out->sum_x = 0.0;
  }
}

// ---------------------------------------------------------------------------
// CG kernels (FP64 vectors).
// ---------------------------------------------------------------------------

// r = (b - sb) - A (x - sx); initial residual (linsolve/poisson_solver.cpp:717-739).
template <typename V>
__global__ void __launch_bounds__(kTX* kTY)
    k_initial_residual(OpInfo o, const V* __restrict__ b, const V* __restrict__ x,
                       V* __restrict__ r, SolveScalars* sc, int kchunk, RedBuf rb,
                       cudaGraphConditionalHandle cond) {
  STENCIL_PROLOGUE(o.L)
  const double sb = sc->sb, sx = sc->sx;
  double acc[2];
  zero(acc);
  if(valid) {
    const ColNb nb = col_nb(o, i, j);
    auto val = [&](int ii, int jj, int kk) { return double(x[o.L.idx(ii, jj, kk)]) - sx; };
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          double c;
          const double ax = apply_op<double>(o, nb, i, j, k, val, c);
          return (double(b[o.L.idx(i, j, k)]) - sb) - ax;
        },
        [&](int k, double v) {
          r[o.L.idx(i, j, k)] = V(v);
          acc[0] += v;
          acc[1] += v * v;
        });
  }
  const bool mx[2] = {false, false};
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    const int n = sc->n;
    const double sr = sc->zero_mean ? s.v[0] / n : 0.0;
    sc->sr = sr;
    sc->sum_r = s.v[0];
    const double ss = fmax(s.v[1] - n * sr * sr, 0.0);
    const double r0 = sqrt(ss / n);
    sc->r0 = r0;
    sc->rnorm = r0;
    sc->rel = r0 > 0.0 ? 1.0 : 0.0;
    sc->iterations = 0;
    sc->stop = 0;
    sc->converged = r0 <= sc->tol ? 1 : 0;
    if(sc->converged) sc->rel = 0.0;
    sc->first = 1;
    sc->body_runs = 0;
    sc->cont = sc->converged ? 0 : 1;
    if(sc->hist != nullptr && sc->hist_cap > 0) sc->hist[0] = r0;
    if(cond) cudaGraphSetConditional(cond, sc->cont);
  });
}

// p = (z - sz) + beta (p - sp); first iteration p = z - sz.
template <typename T, typename V>
__global__ void __launch_bounds__(kTX* kTY)
    k_update_p(CLay L, const T* __restrict__ z, const LevelScalars* ls0, V* __restrict__ p,
               SolveScalars* sc, int kchunk, RedBuf rb) {
  pdl_enter();
  STENCIL_PROLOGUE(L)
  const int first = sc->first;
  const double sz = ls0->sx;
  const double beta = first ? 0.0 : sc->beta;
  const double sp = sc->sp;
  double acc[1];
  zero(acc);
  if(valid) {
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          const int q = L.idx(i, j, k);
          return first ? double(z[q]) - sz : (double(z[q]) - sz) + beta * (double(p[q]) - sp);
        },
        [&](int k, double v) {
          p[L.idx(i, j, k)] = V(v);
          acc[0] += v;
        });
  }
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) {
    sc->sp = sc->zero_mean ? s.v[0] / sc->n : 0.0;
    sc->first = 0;
  });
}

// Ap = A (p - sp); mean shift of Ap; p.Ap; alpha (linsolve/poisson_solver.cpp:751-761).
template <typename V>
__global__ void __launch_bounds__(kTX* kTY)
    k_apply_ap(OpInfo o, const V* __restrict__ p, V* __restrict__ ap, SolveScalars* sc,
               int kchunk, RedBuf rb) {
  pdl_enter();
  STENCIL_PROLOGUE(o.L)
  const double sp = sc->sp;
  double acc[3];
  zero(acc);
  if(valid) {
    const ColNb nb = col_nb(o, i, j);
    auto val = [&](int ii, int jj, int kk) { return double(p[o.L.idx(ii, jj, kk)]) - sp; };
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          double c;
          const double v = apply_op<double>(o, nb, i, j, k, val, c);
          return Pair<double>{v, c};
        },
        [&](int k, Pair<double> r) {
          ap[o.L.idx(i, j, k)] = V(r.v);
          acc[0] += r.v;
          acc[1] += r.w * r.v;
          acc[2] += r.w;
        });
  }
  const bool mx[3] = {false, false, false};
  reduce_finish<3>(acc, mx, rb, [=](const Sums<3>& s) {
    const double sap = sc->zero_mean ? s.v[0] / sc->n : 0.0;
    sc->sap = sap;
    const double pap = s.v[1] - sap * s.v[2];
    sc->pap = pap;
    if(fabs(pap) < kSmallNumber) {
      sc->stop = 1;
    } else {
      sc->alpha = sc->rz / pap;
    }
  });
}

// x = (x - sx) + alpha (p - sp); r = (r - sr) - alpha (Ap - sap); norms and
// the convergence test (linsolve/poisson_solver.cpp:762-782).
template <typename V>
__global__ void __launch_bounds__(kTX* kTY)
    k_update_xr(CLay L, V* __restrict__ x, V* __restrict__ r,
                const V* __restrict__ p, const V* __restrict__ ap, SolveScalars* sc,
                int kchunk, RedBuf rb, cudaGraphConditionalHandle cond) {
  pdl_enter();
  STENCIL_PROLOGUE(L)
  const int stop = sc->stop;
  const double alpha = sc->alpha, sx = sc->sx, sr = sc->sr, sp = sc->sp, sap = sc->sap;
  double acc[3];
  zero(acc);
  if(valid && !stop) {
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          const int q = L.idx(i, j, k);
          return Pair<double>{(double(x[q]) - sx) + alpha * (double(p[q]) - sp),
                              (double(r[q]) - sr) - alpha * (double(ap[q]) - sap)};
        },
        [&](int k, Pair<double> v) {
          const int q = L.idx(i, j, k);
          x[q] = V(v.v);
          r[q] = V(v.w);
          acc[0] += v.v;
          acc[1] += v.w;
          acc[2] += v.w * v.w;
        });
  }
  const bool mx[3] = {false, false, false};
  reduce_finish<3>(acc, mx, rb, [=](const Sums<3>& s) {
    sc->body_runs += 1;
    if(sc->stop) {
      sc->cont = 0;
      if(cond) cudaGraphSetConditional(cond, 0);
      return;
    }
    const int n = sc->n;
    const int zm = sc->zero_mean;
    sc->sx = zm ? s.v[0] / n : 0.0;
    const double srn = zm ? s.v[1] / n : 0.0;
    sc->sr = srn;
    sc->sum_r = s.v[1];
    const double ss = fmax(s.v[2] - n * srn * srn, 0.0);
    sc->rnorm = sqrt(ss / n);
    sc->iterations += 1;
    sc->rel = sc->r0 > 0.0 ? sc->rnorm / sc->r0 : 0.0;
    if(sc->rel <= sc->tol) sc->converged = 1;
    if(sc->hist != nullptr && sc->iterations < sc->hist_cap) sc->hist[sc->iterations] = sc->rnorm;
    // the reference's loop: at most max_iterations iterations, stop on convergence
    sc->cont = (sc->converged || sc->iterations >= sc->max_it) ? 0 : 1;
    if(cond) cudaGraphSetConditional(cond, sc->cont);
  });
}

// Mixed path: the FP64 residual scaled to unit RMS into the FP32 inner rhs,
// the inner correction cleared, and the inner loop's scalars initialised the
// way k_initial_residual does it for a zero initial guess.
__global__ void __launch_bounds__(kTX* kTY)
    k_dc_to_inner(CLay L, const double* __restrict__ r, const SolveScalars* sc,
                  float* __restrict__ r32, float* __restrict__ e32, SolveScalars* si, int kchunk,
                  RedBuf rb, cudaGraphConditionalHandle cond) {
  STENCIL_PROLOGUE(L)
  const double sr = sc->sr;
  const double inv = sc->rnorm > 0.0 ? 1.0 / sc->rnorm : 1.0;
  double acc[2];
  zero(acc);
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const int q = L.idx(i, j, k);
      const float v = float((r[q] - sr) * inv);
      r32[q] = v;
      e32[q] = 0.0f;
      acc[0] += double(v);
      acc[1] += double(v) * double(v);
    }
  }
  const bool mx[2] = {false, false};
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    const int n = si->n;
    const double srn = si->zero_mean ? s.v[0] / n : 0.0;
    si->sr = srn;
    si->sum_r = s.v[0];
    const double r0 = sqrt(fmax(s.v[1] - n * srn * srn, 0.0) / n);
    si->r0 = r0;
    si->rnorm = r0;
    si->rel = 1.0;
    si->iterations = 0;
    si->stop = 0;
    si->converged = 0;
    si->first = 1;
    si->body_runs = 0;
    si->sx = 0.0;
    si->sp = 0.0;
    si->hist = nullptr;
    si->hist_cap = 0;
    si->cont = r0 > 0.0 ? 1 : 0;
    if(cond) cudaGraphSetConditional(cond, si->cont);
  });
}

// Mixed path: x = (x - sx) + scale (e - sx_inner) with the scale the inner
// rhs was divided by; records mean(x).
__global__ void __launch_bounds__(kTX* kTY)
    k_dc_update_x(CLay L, double* __restrict__ x, const float* __restrict__ e32, SolveScalars* sc,
                  const SolveScalars* si, int kchunk, RedBuf rb) {
  STENCIL_PROLOGUE(L)
  const double scale = sc->rnorm > 0.0 ? sc->rnorm : 1.0;
  const double sx = sc->sx, sxi = si->sx;
  double acc[1];
  zero(acc);
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const int q = L.idx(i, j, k);
      const double v = (x[q] - sx) + scale * (double(e32[q]) - sxi);
      x[q] = v;
      acc[0] += v;
    }
  }
  const bool mx[1] = {false};
  reduce_finish<1>(acc, mx, rb, [=](const Sums<1>& s) {
    sc->sx = sc->zero_mean ? s.v[0] / sc->n : 0.0;
  });
}

// Mixed path: the FP64 residual r = (b - sb) - A (x - sx) after a correction,
// its norm, the convergence test against the reference's relative tolerance
// and the loop control (the total of inner iterations is the iteration count).
__global__ void __launch_bounds__(kTX* kTY)
    k_dc_residual(OpInfo o, const double* __restrict__ b, const double* __restrict__ x,
                  double* __restrict__ r, SolveScalars* sc, const SolveScalars* si, int kchunk,
                  RedBuf rb) {
  STENCIL_PROLOGUE(o.L)
  const double sb = sc->sb, sx = sc->sx;
  double acc[2];
  zero(acc);
  if(valid) {
    const ColNb nb = col_nb(o, i, j);
    auto val = [&](int ii, int jj, int kk) { return x[o.L.idx(ii, jj, kk)] - sx; };
    k_batched<kBatch>(
        k0, k1,
        [&](int k) {
          double c;
          const double ax = apply_op<double>(o, nb, i, j, k, val, c);
          return (b[o.L.idx(i, j, k)] - sb) - ax;
        },
        [&](int k, double v) {
          r[o.L.idx(i, j, k)] = v;
          acc[0] += v;
          acc[1] += v * v;
        });
  }
  const bool mx[2] = {false, false};
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    const int n = sc->n;
    const double srn = sc->zero_mean ? s.v[0] / n : 0.0;
    sc->sr = srn;
    sc->sum_r = s.v[0];
    const double rn = sqrt(fmax(s.v[1] - n * srn * srn, 0.0) / n);
    sc->rnorm = rn;
    sc->iterations += si->iterations;
    sc->body_runs += si->body_runs;
    sc->outer += 1;
    sc->rel = sc->r0 > 0.0 ? rn / sc->r0 : 0.0;
    if(sc->rel <= sc->tol) sc->converged = 1;
    if(sc->hist != nullptr && sc->outer < sc->hist_cap) sc->hist[sc->outer] = rn;
    const bool stalled = si->iterations == 0;
    sc->cont = (sc->converged || sc->iterations >= sc->max_it || sc->outer >= 100 || stalled) ? 0 : 1;
  });
}

__global__ void k_compact_to_pressure(Grid g, const double* __restrict__ x, const SolveScalars* sc,
                                      double* __restrict__ p) {
  const Lay P = make_lay(g, kCell);
  const CLay L = make_clay(g.nx, g.ny, g.nz);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if(i >= L.nx || j >= L.ny) return;
  p[P.idx(i + 1, j + 1, k + 1)] = x[L.idx(i, j, k)] - sc->sx;
}

}  // namespace

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------

struct Level {
  Grid g;
  CLay L;
  OpInfo op;
  void* a = nullptr;   // smoother output a
  void* x = nullptr;   // smoother output b (correction)
  void* b = nullptr;   // rhs (levels >= 1)
  double* invd = nullptr;
  int rx = 1, ry = 1, rz = 1;  // refinement ratio to the next coarser level
  // plane-pipeline (TMA) maps: a (main rows, one halo row) and the rhs
  bool tma = false;
  CUtensorMap tm_am, tm_ah, tm_bm, tm_bh;
  bool tma_prolong = false;  // 2x2x2 coarsening: correction x and the coarse result
  CUtensorMap tm_xm, tm_xh, tm_em, tm_eh;
};

struct PoissonPlan {
  Grid g;
  PBC pbc;
  int precision = 0;
  int zero_mean = 1;
  std::vector<Level> levels;
  int coarse_n = 0;
  int* swaps = nullptr;
  double* factors = nullptr;
  LevelScalars* ls = nullptr;  // device, one per level
  double *b = nullptr, *x = nullptr, *r = nullptr, *p = nullptr, *ap = nullptr;
  double* hist = nullptr;
  int hist_cap = 0;
  size_t bytes = 0;
  // the whole solve as one CUDA graph (built on first use)
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long pre_counts[kKernelCount] = {};
  long long body_counts[kKernelCount] = {};
  // mixed path: inner (FP32) CG vectors and scalars
  float *r32 = nullptr, *e32 = nullptr, *p32 = nullptr, *ap32 = nullptr;
  SolveScalars* sc_in = nullptr;
  int* fault = nullptr;  // device: a bounded wait in a plane-pipelined kernel gave up
  int sms = 148;         // streaming multiprocessors of the plan's device
  bool tma_ap = false;   // plane-pipelined A p on the finest level
  bool all_periodic = false;  // every face periodic: constant diagonal, no boundary signs
  CUtensorMap tm_pm, tm_ph, tm_pm2, tm_ph2;
  double* p2 = nullptr;     // second p buffer of the fused CG step
  float* p32b = nullptr;
  // levels tail_first.. run as one single-block launch (k_vcycle_tail)
  int tail_first = -1;
  TailArgs tail{};
  size_t tail_smem = 0;
  unsigned char* tail_tabs = nullptr;  // the tail's staged tables (TailLevel)
};

namespace {

bool can_coarsen_axis(int cells) { return cells > 1 && cells % 2 == 0 && cells > 2; }

OpInfo make_op(const Grid& g, const PBC& pbc) {
  OpInfo o;
  o.L = make_clay(g.nx, g.ny, g.nz);
  for(int a = 0; a < 3; ++a) {
    const double h = g.h(a);
    o.inv2[a] = 1.0 / (h * h);
    o.periodic[a] = pbc.type[2 * a] == kPPeriodic ? 1 : 0;
    o.dir_lo[a] = pbc.type[2 * a] == kPDirichlet ? 1 : 0;
    o.dir_hi[a] = pbc.type[2 * a + 1] == kPDirichlet ? 1 : 0;
  }
  o.invd = nullptr;
  return o;
}

// compute_operator_diagonal (linsolve/poisson_solver.cpp:271-314) by boundary class.
std::vector<double> inverse_diagonal_table(const Grid& g, const PBC& pbc) {
  std::vector<double> t(64, 0.0);
  for(int cz = 0; cz < 4; ++cz)
    for(int cy = 0; cy < 4; ++cy)
      for(int cx = 0; cx < 4; ++cx) {
        const int cls[3] = {cx, cy, cz};
        double value = 0.0;
        for(int a = 0; a < 3; ++a) {
          const double inv = 1.0 / std::pow(g.h(a), 2.0);
          double coefficient = 2.0 * inv;
          if(pbc.type[2 * a] == kPPeriodic) {
            value += coefficient;
            continue;
          }
          const bool first = cls[a] == 1 || cls[a] == 3;
          const bool last = cls[a] == 2 || cls[a] == 3;
          if(first) coefficient += pbc.type[2 * a] == kPDirichlet ? inv : -inv;
          if(last) coefficient += pbc.type[2 * a + 1] == kPDirichlet ? inv : -inv;
          value += coefficient;
        }
        t[cx + 4 * cy + 16 * cz] = value != 0.0 ? 1.0 / value : 0.0;
      }
  return t;
}

// Host copy of apply_poisson_operator with homogeneous rules, for assembling
// the coarse matrix column by column as direct_coarse_solve does.
void host_apply(const Grid& g, const PBC& pbc, const std::vector<double>& in,
                std::vector<double>& out) {
  const CLay L = make_clay(g.nx, g.ny, g.nz);
  auto val = [&](int i, int j, int k) { return in[L.idx(i, j, k)]; };
  for(int k = 0; k < L.nz; ++k)
    for(int j = 0; j < L.ny; ++j)
      for(int i = 0; i < L.nx; ++i) {
        const double c = val(i, j, k);
        const int pos[3] = {i, j, k};
        double nb[3][2];
        for(int a = 0; a < 3; ++a) {
          for(int s = 0; s < 2; ++s) {
            int q[3] = {i, j, k};
            const bool upper = s == 1;
            const int n = L.n(a);
            if((!upper && pos[a] > 0) || (upper && pos[a] < n - 1)) {
              q[a] += upper ? 1 : -1;
              nb[a][s] = val(q[0], q[1], q[2]);
              continue;
            }
            const int type = pbc.type[2 * a + s];
            if(type == kPPeriodic) {
              q[a] = upper ? 0 : n - 1;
              nb[a][s] = val(q[0], q[1], q[2]);
            } else if(type == kPNeumann) {
              nb[a][s] = c;
            } else {
              nb[a][s] = -c;
            }
          }
        }
        out[L.idx(i, j, k)] = -(nb[0][1] - 2.0 * c + nb[0][0]) / (g.dx * g.dx) -
                              (nb[1][1] - 2.0 * c + nb[1][0]) / (g.dy * g.dy) -
                              (nb[2][1] - 2.0 * c + nb[2][0]) / (g.dz * g.dz);
      }
}

}  // namespace

namespace {

// Chooses the first level (below the finest) whose cells fit the single-block
// tail and lays out its shared memory: per level b, x, s (T), then the
// coarsest solve's FP64 vector.  ORCHARD_B200_NO_TAIL=1 keeps every level on
// the per-level kernels (for comparisons).
// Whether the tail from level `first` can run on index arithmetic: every
// axis periodic, every extent a power of two, and one inverse diagonal for
// all 64 boundary classes of each level.
bool tail_periodic(const PoissonPlan* P, int first) {
  for(int l = first; l < static_cast<int>(P->levels.size()); ++l) {
    const Level& lv = P->levels[l];
    for(int a = 0; a < 3; ++a) {
      const int n = lv.L.n(a);
      if(!lv.op.periodic[a] || (n & (n - 1)) != 0) return false;
    }
    const std::vector<double> t = inverse_diagonal_table(lv.g, P->pbc);
    for(int c = 1; c < 64; ++c)
      if(t[c] != t[0]) return false;
  }
  return true;
}

void setup_tail(PoissonPlan* P, size_t tsz) {
  const char* e = std::getenv("ORCHARD_B200_NO_TAIL");
  if(e != nullptr && e[0] == '1') return;
  const int nl = static_cast<int>(P->levels.size());
  constexpr size_t kSmemLimit = 200 * 1024;
  for(int first = 1; first < nl; ++first) {
    if(P->levels[first].L.count() > kTailMaxCells || nl - first > kTailMaxLevels) continue;
    TailArgs t{};
    t.count = nl - first;
    size_t cursor = 0;  // elements of T
    const size_t align = 16 / tsz;
    for(int l = first; l < nl; ++l) {
      const Level& lv = P->levels[l];
      TailLevel& tl = t.lv[l - first];
      tl.op = lv.op;
      tl.sx = lv.rx == 2 ? 1 : 0;
      tl.sy = lv.ry == 2 ? 1 : 0;
      tl.sz = lv.rz == 2 ? 1 : 0;
      cursor = (cursor + align - 1) / align * align;
      tl.off = static_cast<int>(cursor);
      cursor += 3 * static_cast<size_t>(lv.L.count());
    }
    cursor = (cursor + align - 1) / align * align;
    t.coarse_off = static_cast<int>(cursor);
    t.coarse_n = P->coarse_n;
    cursor += static_cast<size_t>(P->coarse_n) * sizeof(double) / tsz;
    // staged factors (n^2 doubles) and swaps (n ints) of a coarse solve of
    // at most 32 unknowns
    cursor = (cursor + align - 1) / align * align;
    t.fact_off = static_cast<int>(cursor);
    if(P->coarse_n <= 32)
      cursor += (static_cast<size_t>(P->coarse_n) * P->coarse_n * sizeof(double) +
                 static_cast<size_t>(P->coarse_n) * sizeof(int) + tsz - 1) / tsz;
    // the staged tables of every level but the coarsest
    const size_t tab_off = align16(cursor * tsz);
    std::vector<unsigned char> blob;
    for(int l = first; l + 1 < nl; ++l) {
      const Level& lv = P->levels[l];
      const Level& cv = P->levels[l + 1];
      TailLevel& tl = t.lv[l - first];
      const int n = lv.L.count(), nc = cv.L.count();
      tl.nch = lv.rx * lv.ry * lv.rz;
      tl.tab = static_cast<int>(blob.size());
      const TailTabLayout lay = tail_tab_layout(n, nc, tl.nch, tsz);
      blob.resize(blob.size() + lay.bytes, 0);
      unsigned char* base = blob.data() + tl.tab;
      int16_t* nbr = reinterpret_cast<int16_t*>(base + lay.nbr);
      int16_t* parent = reinterpret_cast<int16_t*>(base + lay.parent);
      int16_t* child = reinterpret_cast<int16_t*>(base + lay.child);
      const std::vector<double> tinv = inverse_diagonal_table(lv.g, P->pbc);
      // nb_lo / nb_hi on the host: neighbour, periodic image or the cell itself,
      // with -1 for a homogeneous-Dirichlet image
      auto rule = [&](int a, int c, bool hi, int& cc) {
        const int N = lv.L.n(a);
        const bool per = lv.op.periodic[a] != 0;
        const bool dir = (hi ? lv.op.dir_hi[a] : lv.op.dir_lo[a]) != 0;
        const bool in = hi ? c < N - 1 : c > 0;
        cc = in ? (hi ? c + 1 : c - 1) : (per ? (hi ? 0 : N - 1) : c);
        return (in || per || !dir) ? 1 : -1;
      };
      auto cls = [](int c, int N) { return N == 1 ? 3 : (c == 0 ? 1 : (c == N - 1 ? 2 : 0)); };
      for(int k = 0; k < lv.L.nz; ++k)
        for(int j = 0; j < lv.L.ny; ++j)
          for(int i = 0; i < lv.L.nx; ++i) {
            const int q = lv.L.idx(i, j, k);
            int cc;
            int sg = rule(0, i, false, cc);
            nbr[q] = static_cast<int16_t>(sg * (lv.L.idx(cc, j, k) + 1));
            sg = rule(0, i, true, cc);
            nbr[n + q] = static_cast<int16_t>(sg * (lv.L.idx(cc, j, k) + 1));
            sg = rule(1, j, false, cc);
            nbr[2 * n + q] = static_cast<int16_t>(sg * (lv.L.idx(i, cc, k) + 1));
            sg = rule(1, j, true, cc);
            nbr[3 * n + q] = static_cast<int16_t>(sg * (lv.L.idx(i, cc, k) + 1));
            sg = rule(2, k, false, cc);
            nbr[4 * n + q] = static_cast<int16_t>(sg * (lv.L.idx(i, j, cc) + 1));
            sg = rule(2, k, true, cc);
            nbr[5 * n + q] = static_cast<int16_t>(sg * (lv.L.idx(i, j, cc) + 1));
            parent[q] = static_cast<int16_t>(cv.L.idx(i / lv.rx, j / lv.ry, k / lv.rz));
            base[lay.cls + q] =
                static_cast<unsigned char>(cls(i, lv.L.nx) + 4 * cls(j, lv.L.ny) + 16 * cls(k, lv.L.nz));
          }
      for(int c = 0; c < 64; ++c) {
        if(tsz == sizeof(float)) reinterpret_cast<float*>(base + lay.itab)[c] = static_cast<float>(tinv[c]);
        else reinterpret_cast<double*>(base + lay.itab)[c] = tinv[c];
      }
      for(int K = 0; K < cv.L.nz; ++K)
        for(int J = 0; J < cv.L.ny; ++J)
          for(int I = 0; I < cv.L.nx; ++I) {
            int c = 0;
            const int Q = cv.L.idx(I, J, K);
            for(int dz = 0; dz < lv.rz; ++dz)
              for(int dy = 0; dy < lv.ry; ++dy)
                for(int dx = 0; dx < lv.rx; ++dx)
                  child[Q * tl.nch + c++] =
                      static_cast<int16_t>(lv.L.idx(I * lv.rx + dx, J * lv.ry + dy, K * lv.rz + dz));
          }
    }
    t.tab_off = static_cast<int>(tab_off);
    t.tab_bytes = static_cast<int>(blob.size());
    const size_t bytes = tab_off + blob.size();
    if(bytes > kSmemLimit) continue;
    if(!blob.empty()) {
      OFB_CHECK(cudaMalloc(&P->tail_tabs, blob.size()));
      OFB_CHECK(cudaMemcpy(P->tail_tabs, blob.data(), blob.size(), cudaMemcpyHostToDevice));
    }
    t.tabs = P->tail_tabs;
    t.swaps = P->swaps;
    t.factors = P->factors;
    t.zm = P->zero_mean;
    t.per = tail_periodic(P, first) ? 1 : 0;
    for(int l = first; l < nl; ++l) t.lv[l - first].d0 = inverse_diagonal_table(P->levels[l].g, P->pbc)[0];
    auto smem_attr = [&](const void* k) {
      OFB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    };
    if(tsz == sizeof(float)) {
      smem_attr(reinterpret_cast<const void*>(k_vcycle_tail<float, false>));
      smem_attr(reinterpret_cast<const void*>(k_vcycle_tail<float, true>));
    } else {
      smem_attr(reinterpret_cast<const void*>(k_vcycle_tail<double, false>));
      smem_attr(reinterpret_cast<const void*>(k_vcycle_tail<double, true>));
    }
    P->tail = t;
    P->tail_first = first;
    P->tail_smem = bytes;
    return;
  }
}

// Tensor maps of the plane-pipelined kernels for every level above the
// single-block tail whose rows fit one TMA box (nx of 64, 128 or 256) and
// whose row tiles divide ny.  ORCHARD_B200_NO_TMA=1 keeps the row kernels.
bool tma_fits(const CLay& L) {
  if(L.nx != 64 && L.nx != 128 && L.nx != 256) return false;
  const int ty = 1024 / L.nx;
  return L.ny % ty == 0 && L.nz >= 1;
}

void setup_tma(PoissonPlan* P, size_t tsz) {
  const char* e = std::getenv("ORCHARD_B200_NO_TMA");
  if(e != nullptr && e[0] == '1') return;
  const int nl = static_cast<int>(P->levels.size());
  const int last = P->tail_first >= 0 ? P->tail_first : nl - 1;
  for(int l = 0; l < last; ++l) {
    Level& lv = P->levels[l];
    if(!tma_fits(lv.L)) continue;
    const int ty = 1024 / lv.L.nx;
    const int es = static_cast<int>(tsz);
    lv.tm_am = tma::make_map_3d(lv.a, es, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, ty);
    lv.tm_ah = tma::make_map_3d(lv.a, es, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, 1);
    // the finest level's rhs is the CG residual: FP64, or FP32 on the mixed path
    const void* bp = l > 0 ? lv.b : (P->precision == 1 ? static_cast<const void*>(P->r32) : P->r);
    const int bes = l > 0 ? es : (P->precision == 1 ? 4 : 8);
    lv.tm_bm = tma::make_map_3d(bp, bes, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, ty);
    lv.tm_bh = tma::make_map_3d(bp, bes, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, 1);
    lv.tma = true;
    if(lv.rx == 2 && lv.ry == 2 && lv.rz == 2 && l + 1 < nl) {
      const Level& cv = P->levels[l + 1];
      lv.tm_xm = tma::make_map_3d(lv.x, es, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, ty);
      lv.tm_xh = tma::make_map_3d(lv.x, es, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, 1);
      lv.tm_em = tma::make_map_3d(cv.x, es, cv.L.nx, cv.L.ny, cv.L.nz, cv.L.nx, ty / 2);
      lv.tm_eh = tma::make_map_3d(cv.x, es, cv.L.nx, cv.L.ny, cv.L.nz, cv.L.nx, 1);
      lv.tma_prolong = true;
    }
    if(l == 0) {
      const void* pp = P->precision == 1 ? static_cast<const void*>(P->p32) : P->p;
      const void* pp2 = P->precision == 1 ? static_cast<const void*>(P->p32b) : P->p2;
      const int pes = P->precision == 1 ? 4 : 8;
      P->tm_pm = tma::make_map_3d(pp, pes, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, ty);
      P->tm_ph = tma::make_map_3d(pp, pes, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, 1);
      P->tm_pm2 = tma::make_map_3d(pp2, pes, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, ty);
      P->tm_ph2 = tma::make_map_3d(pp2, pes, lv.L.nx, lv.L.ny, lv.L.nz, lv.L.nx, 1);
      P->tma_ap = true;
    }
  }
  auto attr = [](const void* fn, size_t bytes) {
    OFB_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
  };
  attr(reinterpret_cast<const void*>(k_tprolong<double, double, 4, 4, false>), tprolong_bytes<double, double>(256) * 4);
  attr(reinterpret_cast<const void*>(k_tprolong<double, double, 4, 4, true>), tprolong_bytes<double, double>(256) * 4);
  attr(reinterpret_cast<const void*>(k_tprolong<float, float, 4, 4, false>), tprolong_bytes<float, float>(256) * 4);
  attr(reinterpret_cast<const void*>(k_tprolong<float, float, 4, 4, true>), tprolong_bytes<float, float>(256) * 4);
  attr(reinterpret_cast<const void*>(k_tpap<double, double, false>), tround(6 * 256 * 8) * 2 * 4);
  attr(reinterpret_cast<const void*>(k_tpap<double, double, true>), tround(6 * 256 * 8) * 2 * 4);
  attr(reinterpret_cast<const void*>(k_tpap<float, float, false>), tround(6 * 256 * 4) * 2 * tpap_slots<float>());
  attr(reinterpret_cast<const void*>(k_tpap<float, float, true>), tround(6 * 256 * 4) * 2 * tpap_slots<float>());
  attr(reinterpret_cast<const void*>(k_tap<double, 4, false>), tround(static_cast<size_t>(6) * 256 * 8) * kTSlots);
  attr(reinterpret_cast<const void*>(k_tap<double, 4, true>), tround(static_cast<size_t>(6) * 256 * 8) * kTSlots);
  attr(reinterpret_cast<const void*>(k_tap<float, 4, false>), tround(static_cast<size_t>(6) * 256 * 4) * kTSlots);
  attr(reinterpret_cast<const void*>(k_tap<float, 4, true>), tround(static_cast<size_t>(6) * 256 * 4) * kTSlots);
  attr(reinterpret_cast<const void*>(k_trestrict<double, double, kTSlots, false>),
       tslot_bytes<double, double>(256) * kTSlots + 4 * 128 * 8);
  attr(reinterpret_cast<const void*>(k_trestrict<double, double, kTSlots, true>),
       tslot_bytes<double, double>(256) * kTSlots + 4 * 128 * 8);
  attr(reinterpret_cast<const void*>(k_trestrict<float, float, kTSlots, false>),
       tslot_bytes<float, float>(256) * kTSlots + 4 * 128 * 4);
  attr(reinterpret_cast<const void*>(k_trestrict<float, float, kTSlots, true>),
       tslot_bytes<float, float>(256) * kTSlots + 4 * 128 * 4);
  // the largest slot is that of nx = 256 (TY = 4): (TY + 2 + TY) rows of 256
  for(const void* fn : {reinterpret_cast<const void*>(k_tsmooth<double, double, 4, false>),
                         reinterpret_cast<const void*>(k_tsmooth<double, double, 4, true>)})
    attr(fn, tslot_bytes<double, double>(256) * kTSlots);
  for(const void* fn : {reinterpret_cast<const void*>(k_tsmooth<float, float, 4, false>),
                         reinterpret_cast<const void*>(k_tsmooth<float, float, 4, true>)})
    attr(fn, tslot_bytes<float, float>(256) * kTSlots);
  for(const void* fn : {reinterpret_cast<const void*>(k_tsmooth_pre<double, double, 4, false>),
                         reinterpret_cast<const void*>(k_tsmooth_pre<double, double, 4, true>)})
    attr(fn, tslot_bytes<double, double>(256) * kTSlots);
  for(const void* fn : {reinterpret_cast<const void*>(k_tsmooth_pre<float, float, 4, false>),
                         reinterpret_cast<const void*>(k_tsmooth_pre<float, float, 4, true>)})
    attr(fn, tslot_bytes<float, float>(256) * kTSlots);

}

}  // namespace

PoissonPlan* poisson_plan_create(const Grid& g, const PBC& pbc_in, int precision) {
  auto* P = new PoissonPlan();
  P->g = g;
  // homogeneous_boundary_conditions (linsolve/poisson_solver.cpp:164-173)
  P->pbc = pbc_in;
  for(int f = 0; f < 6; ++f) {
    P->pbc.value[f] = 0.0;
    P->pbc.gradient[f] = 0.0;
  }
  P->precision = precision;
  P->zero_mean = 1;
  for(int f = 0; f < 6; ++f)
    if(pbc_in.type[f] == kPDirichlet) P->zero_mean = 0;
  const size_t tsz = precision == 1 ? sizeof(float) : sizeof(double);

  // build_hierarchy (linsolve/poisson_solver.cpp:316-384)
  Grid cur = g;
  for(;;) {
    Level lv;
    lv.g = cur;
    lv.L = make_clay(cur.nx, cur.ny, cur.nz);
    lv.op = make_op(cur, P->pbc);
    P->levels.push_back(lv);
    if(!(can_coarsen_axis(cur.nx) || can_coarsen_axis(cur.ny) || can_coarsen_axis(cur.nz))) break;
    Grid c = cur;
    if(can_coarsen_axis(cur.nx)) { c.nx = cur.nx / 2; c.dx = 2.0 * cur.dx; }
    if(can_coarsen_axis(cur.ny)) { c.ny = cur.ny / 2; c.dy = 2.0 * cur.dy; }
    if(can_coarsen_axis(cur.nz)) { c.nz = cur.nz / 2; c.dz = 2.0 * cur.dz; }
    if(c.nx == cur.nx && c.ny == cur.ny && c.nz == cur.nz) break;
    Level& prev = P->levels.back();
    prev.rx = cur.nx == c.nx ? 1 : 2;
    prev.ry = cur.ny == c.ny ? 1 : 2;
    prev.rz = cur.nz == c.nz ? 1 : 2;
    cur = c;
  }
  const int nl = static_cast<int>(P->levels.size());
  for(int l = 0; l < nl; ++l) {
    Level& lv = P->levels[l];
    const size_t n = lv.L.count();
    OFB_CHECK(cudaMalloc(&lv.a, n * tsz));
    OFB_CHECK(cudaMalloc(&lv.x, n * tsz));
    P->bytes += 2 * n * tsz;
    if(l > 0) {
      OFB_CHECK(cudaMalloc(&lv.b, n * tsz));
      P->bytes += n * tsz;
    }
    std::vector<double> t = inverse_diagonal_table(lv.g, P->pbc);
    OFB_CHECK(cudaMalloc(&lv.invd, 64 * sizeof(double)));
    OFB_CHECK(cudaMemcpy(lv.invd, t.data(), 64 * sizeof(double), cudaMemcpyHostToDevice));
    lv.op.invd = lv.invd;
  }
  OFB_CHECK(cudaMalloc(&P->ls, nl * sizeof(LevelScalars)));
  OFB_CHECK(cudaMemset(P->ls, 0, nl * sizeof(LevelScalars)));

  // coarsest-grid elimination (direct_coarse_solve / gaussian_elimination,
  // linsolve/poisson_solver.cpp:482-567), done once on the host
  const Level& co = P->levels.back();
  const int n = co.L.count();
  if(n > kMaxCoarse) {
    poisson_plan_destroy(P);
    throw std::invalid_argument("coarsest multigrid level has " + std::to_string(n) +
                                " unknowns; at most " + std::to_string(kMaxCoarse) +
                                " are supported");
  }
  P->coarse_n = n;
  std::vector<double> m(static_cast<size_t>(n) * n, 0.0), e(n, 0.0), img(n, 0.0);
  for(int col = 0; col < n; ++col) {
    std::fill(e.begin(), e.end(), 0.0);
    e[col] = 1.0;
    host_apply(co.g, P->pbc, e, img);
    for(int row = 0; row < n; ++row) m[static_cast<size_t>(row) * n + col] = img[row];
  }
  if(P->zero_mean)
    for(int col = 0; col < n; ++col) m[static_cast<size_t>(n - 1) * n + col] = 1.0;
  std::vector<int> swaps(n);
  for(int piv = 0; piv < n; ++piv) {
    int best = piv;
    double best_abs = std::fabs(m[static_cast<size_t>(piv) * n + piv]);
    for(int row = piv + 1; row < n; ++row) {
      const double cand = std::fabs(m[static_cast<size_t>(row) * n + piv]);
      if(cand > best_abs) {
        best = row;
        best_abs = cand;
      }
    }
    if(best_abs < kSmallNumber) {
      poisson_plan_destroy(P);
      throw std::runtime_error("direct coarse solve encountered a singular matrix");
    }
    swaps[piv] = best;
    // Columns left of the pivot hold the multipliers of earlier steps; they
    // stay with their row position so the device replays the eliminations
    // on the right-hand side in the reference's order.
    if(best != piv)
      for(int c = piv; c < n; ++c)
        std::swap(m[static_cast<size_t>(piv) * n + c], m[static_cast<size_t>(best) * n + c]);
    const double inv = 1.0 / m[static_cast<size_t>(piv) * n + piv];
    for(int row = piv + 1; row < n; ++row) {
      const double factor = m[static_cast<size_t>(row) * n + piv] * inv;
      if(std::fabs(factor) < kSmallNumber) {
        m[static_cast<size_t>(row) * n + piv] = 0.0;
        continue;
      }
      for(int c = piv + 1; c < n; ++c)
        m[static_cast<size_t>(row) * n + c] -= factor * m[static_cast<size_t>(piv) * n + c];
      m[static_cast<size_t>(row) * n + piv] = factor;  // keep the multiplier
    }
  }
  OFB_CHECK(cudaMalloc(&P->swaps, n * sizeof(int)));
  OFB_CHECK(cudaMalloc(&P->factors, static_cast<size_t>(n) * n * sizeof(double)));
  OFB_CHECK(cudaMemcpy(P->swaps, swaps.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  OFB_CHECK(cudaMemcpy(P->factors, m.data(), static_cast<size_t>(n) * n * sizeof(double),
                       cudaMemcpyHostToDevice));

  setup_tail(P, tsz);

  const size_t nf = P->levels[0].L.count();
  OFB_CHECK(cudaMalloc(&P->b, nf * sizeof(double)));
  OFB_CHECK(cudaMalloc(&P->x, nf * sizeof(double)));
  OFB_CHECK(cudaMalloc(&P->r, nf * sizeof(double)));
  OFB_CHECK(cudaMalloc(&P->p, nf * sizeof(double)));
  OFB_CHECK(cudaMalloc(&P->ap, nf * sizeof(double)));
  OFB_CHECK(cudaMemset(P->p, 0, nf * sizeof(double)));
  OFB_CHECK(cudaMalloc(&P->p2, nf * sizeof(double)));
  OFB_CHECK(cudaMemset(P->p2, 0, nf * sizeof(double)));
  P->bytes += 6 * nf * sizeof(double);
  if(precision == 1) {
    for(float** v : {&P->r32, &P->e32, &P->p32, &P->ap32, &P->p32b}) {
      OFB_CHECK(cudaMalloc(v, nf * sizeof(float)));
      OFB_CHECK(cudaMemset(*v, 0, nf * sizeof(float)));
    }
    OFB_CHECK(cudaMalloc(&P->sc_in, sizeof(SolveScalars)));
    OFB_CHECK(cudaMemset(P->sc_in, 0, sizeof(SolveScalars)));
    P->bytes += 5 * nf * sizeof(float);
  }
  {
    int dev = 0;
    OFB_CHECK(cudaGetDevice(&dev));
    OFB_CHECK(cudaDeviceGetAttribute(&P->sms, cudaDevAttrMultiProcessorCount, dev));
  }
  OFB_CHECK(cudaMalloc(&P->fault, sizeof(int)));
  OFB_CHECK(cudaMemset(P->fault, 0, sizeof(int)));
  P->all_periodic = true;
  for(int f = 0; f < 6; ++f)
    if(P->pbc.type[f] != kPPeriodic) P->all_periodic = false;
  setup_tma(P, tsz);
  const char* no_graph = std::getenv("ORCHARD_B200_NO_GRAPH");
  P->use_graph = !(no_graph != nullptr && no_graph[0] == '1');
  return P;
}

void poisson_plan_destroy(PoissonPlan* P) {
  if(P == nullptr) return;
  for(Level& lv : P->levels) {
    cudaFree(lv.a);
    cudaFree(lv.x);
    cudaFree(lv.b);
    cudaFree(lv.invd);
  }
  if(P->exec) cudaGraphExecDestroy(P->exec);
  if(P->graph) cudaGraphDestroy(P->graph);
  cudaFree(P->hist);
  cudaFree(P->ls);
  cudaFree(P->swaps);
  cudaFree(P->factors);
  cudaFree(P->b);
  cudaFree(P->x);
  cudaFree(P->r);
  cudaFree(P->p);
  cudaFree(P->ap);
  cudaFree(P->r32);
  cudaFree(P->e32);
  cudaFree(P->p32);
  cudaFree(P->ap32);
  cudaFree(P->p2);
  cudaFree(P->p32b);
  cudaFree(P->sc_in);
  cudaFree(P->fault);
  cudaFree(P->tail_tabs);
  delete P;
}

int poisson_levels(const PoissonPlan* P) { return static_cast<int>(P->levels.size()); }
int poisson_coarse_unknowns(const PoissonPlan* P) { return P->coarse_n; }
size_t poisson_device_bytes(const PoissonPlan* P) { return P->bytes; }
double* poisson_b(PoissonPlan* P) { return P->b; }
double* poisson_x(PoissonPlan* P) { return P->x; }

namespace {

template <typename T, typename B, int RX, int RY, int RZ>
void launch_restrict_r(const Level& lv, const Level& cv, const B* b, const double* sb_ptr,
                       const T* x, const double* sx_ptr, T* bc, LevelScalars* lsc, int zm,
                       const Launch3& lc, RedBuf rb, cudaStream_t s) {
  launch_pdl(k_restrict_residual<T, B, RX, RY, RZ>, lc.grid, lc.block, 0, s, lv.op, cv.op, b, sb_ptr, x,
             sx_ptr, bc, lsc, zm, lc.kchunk, rb);
}

template <typename T, typename B>
void launch_restrict(const Level& lv, const Level& cv, const B* b, const double* sb_ptr, const T* x,
                     const double* sx_ptr, T* bc, LevelScalars* lsc, int zm, const Launch3& lc,
                     RedBuf rb, cudaStream_t s) {
  const int code = (lv.rx == 2 ? 4 : 0) + (lv.ry == 2 ? 2 : 0) + (lv.rz == 2 ? 1 : 0);
  switch(code) {
    case 7: launch_restrict_r<T, B, 2, 2, 2>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    case 6: launch_restrict_r<T, B, 2, 2, 1>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    case 5: launch_restrict_r<T, B, 2, 1, 2>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    case 4: launch_restrict_r<T, B, 2, 1, 1>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    case 3: launch_restrict_r<T, B, 1, 2, 2>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    case 2: launch_restrict_r<T, B, 1, 2, 1>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    case 1: launch_restrict_r<T, B, 1, 1, 2>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
    default: launch_restrict_r<T, B, 1, 1, 1>(lv, cv, b, sb_ptr, x, sx_ptr, bc, lsc, zm, lc, rb, s); break;
  }
}

// Grid of a persistent plane-pipelined launch on a level: at most two blocks
// per SM, each with a range of at least four tile-planes that fits kTMaxSeg
// segments.
struct TGrid {
  int grid, ty;
};

// Blocks per SM of the plane-pipeline kernels: four, or as many as fit (the
// rings of the FP64 kernels on a 256-wide level hold ~100 KB, so two of
// those; the lighter A p ring and the FP32 kernels, whose planes carry half
// the bytes, fit three or four and keep more bytes in flight per SM).
int tper_sm(size_t) { return 4; }

// Blocks of one plane-pipeline launch: tper_sm blocks per SM, no more than
// fit on an SM at once (the persistent schedule gives every block an equal
// share), at least 4 tile-planes per block.
int resident_blocks(const void* kernel, size_t smem, int threads = 256) {
  int n = 0;
  OFB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem));
  return std::max(1, n);
}

// Grid of a plane-pipeline launch over `tiles` row tiles and `nzu` planes (or
// coarse planes): a multiple of the tile count (the z-aligned schedule of
// tsegments) where the kernel gains from it (`aligned_always`: its halo rows
// come from L2) or where that keeps at least 95 % of the blocks that fit,
// else the contiguous ranges.  Measured at 256^3: the aligned schedule takes
// the FP64 k_tsmooth from 88 to 80 us and k_trestrict from 72 to 68 us
// although their 2 blocks per SM round down from 296 to 256; k_tprolong (both
// precisions), the FP32 k_tsmooth and k_tap (3 blocks per SM, 444 -> 384) lose
// more to the rounding down than they gain.
long long tgrid_blocks(const PoissonPlan* P, int tiles, int nzu, int per_sm, int min_units,
                       bool aligned_always) {
  const long long items = static_cast<long long>(tiles) * nzu;
  long long g = std::min<long long>(static_cast<long long>(per_sm) * P->sms, std::max(1LL, items / min_units));
  const long long aligned = tiles * std::min<long long>(nzu, g / tiles);
  if(aligned > 0 && (aligned_always || aligned * 20 >= g * 19)) return aligned;
  while((items / g + 1) / nzu + 2 > kTMaxSeg) ++g;
  if(g % tiles == 0) ++g;  // a multiple of the tile count would select the aligned schedule
  return g;
}

TGrid tgrid(const PoissonPlan* P, const CLay& L, size_t elem, const void* kernel, size_t smem,
            int threads = 256, bool aligned_always = false) {
  const int ty = 1024 / L.nx;
  const int per_sm = std::min(tper_sm(elem), resident_blocks(kernel, smem, threads));
  return TGrid{static_cast<int>(tgrid_blocks(P, L.ny / ty, L.nz, per_sm, 4, aligned_always)), ty};
}

// v_cycle (linsolve/poisson_solver.cpp:597-633) from level l; the finest
// level's rhs is the CG residual r0 (type V, shift sc->sr).
template <typename T, typename V>
void v_cycle(PoissonPlan* P, int l, const V* r0, SolveScalars* sc, RedBuf rb, cudaStream_t s) {
  Level& lv = P->levels[l];
  const int nl = static_cast<int>(P->levels.size());
  const int zm = P->zero_mean;
  LevelScalars* ls = P->ls + l;
  const double* sb_ptr = l == 0 ? &sc->sr : &ls->sb;
  SolveScalars* rz_sc = l == 0 ? sc : nullptr;
  T* a = static_cast<T*>(lv.a);
  T* x = static_cast<T*>(lv.x);
  if(l == P->tail_first) {
    ProfScope ps(kKCoarseLevels, s);
    launch_pdl(P->tail.per ? k_vcycle_tail<T, true> : k_vcycle_tail<T, false>, 1, kTailThreads, P->tail_smem,
               s, P->tail, static_cast<const T*>(lv.b), &ls->sb, x, ls);
    OFB_LAUNCH_CHECK("k_vcycle_tail");
    return;
  }
  if(l + 1 == nl) {
    ProfScope ps(kKCoarseSolve, s);
    if(l == 0)
      launch_pdl(k_coarse_solve<T, V>, 1, 256, 0, s, P->coarse_n, P->swaps, P->factors, r0, sb_ptr, x, ls, zm,
                 rz_sc);
    else
      launch_pdl(k_coarse_solve<T, T>, 1, 256, 0, s, P->coarse_n, P->swaps, P->factors,
                 static_cast<const T*>(lv.b), sb_ptr, x, ls, zm, rz_sc);
    OFB_LAUNCH_CHECK("k_coarse_solve");
    return;
  }
  const Launch3 ln = launch3(lv.L.nx, lv.L.ny, lv.L.nz);
  Level& cv = P->levels[l + 1];
  const Launch3 lc = launch3(cv.L.nx, cv.L.ny, cv.L.nz);
  LevelScalars* lsc = P->ls + (l + 1);
  auto smooth_chain = [&](auto* bptr) {
    using B = std::remove_cv_t<std::remove_pointer_t<decltype(bptr)>>;
    const bool fine = l == 0;
    const bool vec = vfits<T>(lv.L) && vec_enabled();
    const bool vsm = vec && vec_enabled("smooth");
    const bool vpr = vec && vec_enabled("prolong");
    const bool vre = vec && vec_enabled("restrict");
    const vst::RowLaunch lr = vst::row_launch(lv.L.nx, lv.L.ny, lv.L.nz, vst::Width<T>::W, 16);
    if(lv.tma && vec_enabled("tma")) {
      ProfScope ps(fine ? kKSmoothFirstFine : kKCoarseLevels, s);
      const size_t sm = tround(static_cast<size_t>(1024 / lv.L.nx + 2) * lv.L.nx * sizeof(B)) * kTSlots;
      const auto kern = P->all_periodic ? k_tsmooth_pre<T, B, 4, true> : k_tsmooth_pre<T, B, 4, false>;
      const TGrid tg = tgrid(P, lv.L, sizeof(T), reinterpret_cast<const void*>(kern), sm, 288);
      launch_pdl(kern, tg.grid, 288, sm, s, lv.op, lv.tm_bm, lv.tm_bh, sb_ptr, x, ls, zm, rb, P->fault);
    } else if(vsm && vec_enabled("pre")) {
      ProfScope ps(fine ? kKSmoothFirstFine : kKCoarseLevels, s);
      launch_pdl(k_vsmooth_pre<T, B>, lr.grid, lr.block, 0, s, lv.op, bptr, sb_ptr, x, ls, zm, lr.kchunk, rb);
    } else {
      {
        ProfScope ps(fine ? kKSmoothFirstFine : kKCoarseLevels, s);
        launch_pdl(k_smooth_first<T, B>, ln.grid, ln.block, 0, s, lv.op, bptr, sb_ptr, a, ls, zm, ln.kchunk,
                   rb);
      }
      ProfScope ps(fine ? kKSmoothFine : kKCoarseLevels, s);
      if(vsm)
        launch_pdl(k_vsmooth<T, B>, lr.grid, lr.block, 0, s, lv.op, bptr, sb_ptr, a, &ls->sa, x, ls, zm,
                   nullptr, lr.kchunk, rb);
      else
        launch_pdl(k_smooth<T, B>, ln.grid, ln.block, 0, s, lv.op, bptr, sb_ptr, a, &ls->sa, x, ls, 1, zm,
                   nullptr, ln.kchunk, rb);
    }
    if(lv.tma_prolong && vec_enabled("tma")) {
      ProfScope ps(fine ? kKRestrictFine : kKCoarseLevels, s);
      const int ty = 1024 / lv.L.nx;
      const size_t sm = tslot_bytes<T, B>(lv.L.nx) * kTSlots + static_cast<size_t>(ty) * (lv.L.nx / 2) * sizeof(T);
      const auto kern = P->all_periodic ? k_trestrict<T, B, kTSlots, true> : k_trestrict<T, B, kTSlots, false>;
      const int per_sm = std::min(tper_sm(sizeof(T)), resident_blocks(reinterpret_cast<const void*>(kern), sm));
      const long long g = tgrid_blocks(P, lv.L.ny / ty, lv.L.nz / 2, per_sm, 2, std::is_same_v<T, double>);
      launch_pdl(kern, static_cast<int>(g), 256, sm, s, lv.op, cv.op, lv.tm_xm, lv.tm_xh, lv.tm_bm, sb_ptr,
                 &ls->sx, static_cast<T*>(cv.b), lsc, zm, rb, P->fault);
    } else {
      ProfScope ps(fine ? kKRestrictFine : kKCoarseLevels, s);
      if(vre && lv.rx == 2 && lv.ry == 2 && lv.rz == 2) {
        const vst::RowLaunch lrc =
            vst::row_launch(lv.L.nx, cv.L.ny, cv.L.nz, vst::Width<T>::W, 8);
        launch_pdl(k_vrestrict<T, B>, lrc.grid, lrc.block, 0, s, lv.op, cv.op, bptr, sb_ptr, x, &ls->sx,
                   static_cast<T*>(cv.b), lsc, zm, lrc.kchunk, rb);
      } else
        launch_restrict<T, B>(lv, cv, bptr, sb_ptr, x, &ls->sx, static_cast<T*>(cv.b), lsc, zm,
                              lc, rb, s);
    }
    OFB_LAUNCH_CHECK("v_cycle descent");
    if(l == 0) {
      // the coarse levels are ~16 short dependent launches: time them as one
      // chain (one event pair per V-cycle, the coarse solve at the bottom
      // included) so that the measurement does not add an event pair's
      // overhead to each of them
      ProfSpan span(kKCoarseLevels, s);
      v_cycle<T, V>(P, l + 1, r0, sc, rb, s);
    } else {
      v_cycle<T, V>(P, l + 1, r0, sc, rb, s);
    }
    if(lv.tma_prolong && vec_enabled("tma")) {
      ProfScope ps(fine ? kKProlongFine : kKCoarseLevels, s);
      const size_t sm = tprolong_bytes<T, B>(lv.L.nx) * 4;
      const auto kern = P->all_periodic ? k_tprolong<T, B, 4, 4, true> : k_tprolong<T, B, 4, 4, false>;
      const TGrid tg = tgrid(P, lv.L, sizeof(T), reinterpret_cast<const void*>(kern), sm);
      launch_pdl(kern, tg.grid, 256, sm, s, lv.op, lv.tm_xm, lv.tm_xh, lv.tm_bm, lv.tm_em, lv.tm_eh, sb_ptr,
                 &ls->sx, &lsc->sx, a, ls, zm, rb, P->fault);
    } else {
      ProfScope ps(fine ? kKProlongFine : kKCoarseLevels, s);
      if(vpr)
        launch_pdl(k_vprolong_smooth<T, B>, lr.grid, lr.block, 0, s, lv.op, cv.L, bptr, sb_ptr, x, &ls->sx,
                   static_cast<const T*>(cv.x), &lsc->sx, a, ls, lv.rx == 2 ? 1 : 0, lv.ry == 2 ? 1 : 0,
                   lv.rz == 2 ? 1 : 0, zm, lr.kchunk, rb);
      else
        launch_pdl(k_prolong_smooth<T, B>, ln.grid, ln.block, 0, s, lv.op, cv.L, bptr, sb_ptr, x, &ls->sx,
                   static_cast<const T*>(cv.x), &lsc->sx, a, ls, lv.rx == 2 ? 1 : 0, lv.ry == 2 ? 1 : 0,
                   lv.rz == 2 ? 1 : 0, zm, ln.kchunk, rb);
    }
    if(lv.tma && vec_enabled("tma")) {
      ProfScope ps(fine ? kKSmoothFine : kKCoarseLevels, s);
      const size_t sm = tslot_bytes<T, B>(lv.L.nx) * kTSlots;
      const auto kern = P->all_periodic ? k_tsmooth<T, B, 4, true> : k_tsmooth<T, B, 4, false>;
      const TGrid tg =
          tgrid(P, lv.L, sizeof(T), reinterpret_cast<const void*>(kern), sm, 256, std::is_same_v<T, double>);
      launch_pdl(kern, tg.grid, 256, sm, s, lv.op, lv.tm_am, lv.tm_ah, lv.tm_bm, sb_ptr, &ls->sa, x, ls, zm,
                 rz_sc, rb, P->fault);
    } else {
      ProfScope ps(fine ? kKSmoothFine : kKCoarseLevels, s);
      if(vsm)
        launch_pdl(k_vsmooth<T, B>, lr.grid, lr.block, 0, s, lv.op, bptr, sb_ptr, a, &ls->sa, x, ls, zm,
                   rz_sc, lr.kchunk, rb);
      else
        launch_pdl(k_smooth<T, B>, ln.grid, ln.block, 0, s, lv.op, bptr, sb_ptr, a, &ls->sa, x, ls, 1, zm,
                   rz_sc, ln.kchunk, rb);
    }
    OFB_LAUNCH_CHECK("v_cycle ascent");
  };
  if(l == 0) smooth_chain(r0);
  else smooth_chain(static_cast<const T*>(lv.b));
}

// The vectors of one CG loop: FP64 for the reference's solve, FP32 for the
// inner solves of the mixed path's defect correction.
template <typename V>
struct CGVec {
  V *b, *x, *r, *p, *ap, *p2;  // p2: the fused step's second p buffer
};

CGVec<double> cg64(PoissonPlan* P) { return CGVec<double>{P->b, P->x, P->r, P->p, P->ap, P->p2}; }

// Initial residual and convergence test (linsolve/poisson_solver.cpp:717-739).
template <typename V>
void enqueue_pre(PoissonPlan* P, const CGVec<V>& v, SolveScalars* sc, RedBuf rb, cudaStream_t s,
                 cudaGraphConditionalHandle cond) {
  const Level& l0 = P->levels[0];
  const Launch3 ln = launch3(l0.L.nx, l0.L.ny, l0.L.nz);
  ProfScope ps(kKInitResidual, s);
  k_initial_residual<V><<<ln.grid, ln.block, 0, s>>>(l0.op, v.b, v.x, v.r, sc, ln.kchunk, rb, cond);
  OFB_LAUNCH_CHECK("k_initial_residual");
}

// The fused CG step needs the plane-pipeline maps of the finest level's
// correction (z) and of p.  It is used for the FP32 inner solves of the mixed
// path, where it is measurably faster; in FP64 the separate kernels are as
// fast.  ORCHARD_B200_NO_VEC containing "fuse" keeps the separate kernels.
bool fused_cg(const PoissonPlan* P) {
  const char* f64 = std::getenv("ORCHARD_B200_FUSE64");
  const bool fp64_fused = f64 != nullptr && f64[0] == '1';
  return (P->precision == 1 || fp64_fused) && P->tma_ap && P->levels[0].tma_prolong &&
         vec_enabled("tma") && vec_enabled("fuse");
}

// The last deferred x update of a fused-step loop.
template <typename V>
void enqueue_x_final(PoissonPlan* P, const CGVec<V>& v, SolveScalars* sc, RedBuf rb, cudaStream_t s) {
  if(!fused_cg(P)) return;
  const Level& l0 = P->levels[0];
  const Launch3 ln = launch3(l0.L.nx, l0.L.ny, l0.L.nz);
  ProfScope ps(kKUpdateXr, s);
  k_x_final<V><<<ln.grid, ln.block, 0, s>>>(l0.L, v.x, v.p, v.p2, sc, ln.kchunk, rb);
  OFB_LAUNCH_CHECK("k_x_final");
}

// One body of the rotated PCG loop: z = M r, p = z + beta p, A p, x/r update
// and the convergence test -- the reference's iteration (:750-806) with the
// preconditioner moved to the top; the body count is the reference's
// iteration count, and the first body forms p = z as the reference does
// before its loop (:741-749).
template <typename T, typename V>
void enqueue_body(PoissonPlan* P, const CGVec<V>& v, SolveScalars* sc, RedBuf rb, cudaStream_t s,
                  cudaGraphConditionalHandle cond) {
  const Level& l0 = P->levels[0];
  const Launch3 ln = launch3(l0.L.nx, l0.L.ny, l0.L.nz);
  v_cycle<T, V>(P, 0, v.r, sc, rb, s);
  if(fused_cg(P)) {
    // fused p update + A p + deferred x update, then the residual update
    {
      ProfScope ps(kKApplyAp, s);
      const int ty = 1024 / l0.L.nx;
      const size_t sm = (tround(static_cast<size_t>(ty + 2) * l0.L.nx * sizeof(T)) +
                         tround(static_cast<size_t>(ty + 2) * l0.L.nx * sizeof(V))) * tpap_slots<V>();
      const auto kern = P->all_periodic ? k_tpap<T, V, true> : k_tpap<T, V, false>;
      const TGrid tg = tgrid(P, l0.L, sizeof(V), reinterpret_cast<const void*>(kern), sm);
      launch_pdl(kern, tg.grid, 256, sm, s, l0.op, l0.tm_xm, l0.tm_xh, P->tm_pm, P->tm_ph, P->tm_pm2,
                 P->tm_ph2, P->ls, v.p, v.p2, v.ap, v.x, sc, rb, P->fault);
    }
    {
      ProfScope ps(kKUpdateXr, s);
      const int n = l0.L.count();
      const int blocks = static_cast<int>(std::min<long long>(
          kTargetBlocks, std::max(1LL, (static_cast<long long>(n) + kFlatThreads - 1) / kFlatThreads)));
      launch_pdl(k_update_r_flat<V>, blocks, kFlatThreads, 0, s, n, v.r, v.ap, sc, rb, cond);
    }
    OFB_LAUNCH_CHECK("fused pcg body");
    return;
  }
  {
    ProfScope ps(kKUpdateP, s);
    launch_pdl(k_update_p<T, V>, ln.grid, ln.block, 0, s, l0.L, static_cast<const T*>(l0.x), P->ls, v.p, sc,
               ln.kchunk, rb);
  }
  {
    ProfScope ps(kKApplyAp, s);
    if(P->tma_ap && vec_enabled("tma")) {
      const size_t sm = tround(static_cast<size_t>(1024 / l0.L.nx + 2) * l0.L.nx * sizeof(V)) * kTSlots;
      const auto kern = P->all_periodic ? k_tap<V, 4, true> : k_tap<V, 4, false>;
      const TGrid tg = tgrid(P, l0.L, sizeof(V), reinterpret_cast<const void*>(kern), sm);
      launch_pdl(kern, tg.grid, 256, sm, s, l0.op, P->tm_pm, P->tm_ph, v.ap, sc, rb, P->fault);
    } else if(vfits<V>(l0.L) && vec_enabled() && vec_enabled("ap")) {
      const vst::RowLaunch lr = vst::row_launch(l0.L.nx, l0.L.ny, l0.L.nz, vst::Width<V>::W, 16);
      launch_pdl(k_vapply_ap<V>, lr.grid, lr.block, 0, s, l0.op, v.p, v.ap, sc, lr.kchunk, rb);
    }
    else
      launch_pdl(k_apply_ap<V>, ln.grid, ln.block, 0, s, l0.op, v.p, v.ap, sc, ln.kchunk, rb);
  }
  {
    ProfScope ps(kKUpdateXr, s);
    launch_pdl(k_update_xr<V>, ln.grid, ln.block, 0, s, l0.L, v.x, v.r, v.p, v.ap, sc, ln.kchunk, rb, cond);
  }
  OFB_LAUNCH_CHECK("pcg body");
}

// A loop as one graph: pre -> WHILE(cont) { body }.  pre and body are
// enqueue callbacks taking the conditional handle; the loop is bounded by the
// iteration limit the body enforces (it clears the condition), so the graph
// always terminates.
template <typename Pre, typename Body>
cudaGraphExec_t build_loop_graph(PoissonPlan* P, cudaStream_t s, Pre pre, Body body,
                                 cudaGraph_t* graph_out) {
  cudaGraph_t g = nullptr;
  OFB_CHECK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle cond = 0;
  OFB_CHECK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
  for(int i = 0; i < kKernelCount; ++i) P->pre_counts[i] = P->body_counts[i] = 0;
  prof_capture_begin(P->pre_counts);
  OFB_CHECK(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  pre(cond);
  cudaStreamCaptureStatus status;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  OFB_CHECK(cudaStreamGetCaptureInfo(s, &status, nullptr, nullptr, &deps, &ndeps));
  std::vector<cudaGraphNode_t> leaf(deps, deps + ndeps);
  OFB_CHECK(cudaStreamEndCapture(s, &g));
  prof_capture_end();
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  OFB_CHECK(cudaGraphAddNode(&wnode, g, leaf.data(), leaf.size(), &cp));
  cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
  prof_capture_begin(P->body_counts);
  OFB_CHECK(cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
  body(cond);
  OFB_CHECK(cudaStreamEndCapture(s, &bodyg));
  prof_capture_end();
  cudaGraphExec_t exec = nullptr;
  OFB_CHECK(cudaGraphInstantiate(&exec, g, 0));
  *graph_out = g;
  return exec;
}

void ensure_history(PoissonPlan* P, int max_iterations) {
  if(P->hist_cap < max_iterations + 1) {
    if(P->hist) cudaFree(P->hist);
    P->hist = nullptr;
    OFB_CHECK(cudaMalloc(&P->hist, sizeof(double) * (max_iterations + 1)));
    P->hist_cap = max_iterations + 1;
  }
}

// Host-side initialisation of the solve scalars (b and x shifts were set by
// the kernels that filled them).
SolveScalars init_scalars(PoissonPlan* P, int max_iterations, double tolerance, SolveScalars* sc,
                          SolveScalars* host, cudaStream_t s) {
  OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
  OFB_CHECK(cudaStreamSynchronize(s));
  SolveScalars init = *host;
  init.zero_mean = P->zero_mean;
  init.n = P->levels[0].L.count();
  init.tol = tolerance;
  init.max_it = max_iterations;
  init.hist = P->hist;
  init.hist_cap = P->hist_cap;
  init.outer = 0;
  if(!P->zero_mean) {
    init.sb = 0.0;
    init.sx = 0.0;
    init.removed_rhs_mean = 0.0;
  }
  init.sp = 0.0;
  return init;
}

template <typename T>
void solve_impl(PoissonPlan* P, int max_iterations, double tolerance, SolveScalars* sc,
                SolveScalars* host, RedBuf rb, cudaStream_t s, double* history, int history_cap) {
  ensure_history(P, max_iterations);
  *host = init_scalars(P, max_iterations, tolerance, sc, host, s);
  OFB_CHECK(cudaMemcpyAsync(sc, host, sizeof(SolveScalars), cudaMemcpyHostToDevice, s));
  const CGVec<double> v = cg64(P);
  const bool use_graph = P->use_graph && !prof_enabled();
  if(use_graph) {
    if(P->exec == nullptr)
      P->exec = build_loop_graph(
          P, s, [&](cudaGraphConditionalHandle c) { enqueue_pre<double>(P, v, sc, rb, s, c); },
          [&](cudaGraphConditionalHandle c) { enqueue_body<T, double>(P, v, sc, rb, s, c); },
          &P->graph);
    OFB_CHECK(cudaGraphLaunch(P->exec, s));
    enqueue_x_final<double>(P, v, sc, rb, s);
    OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
    OFB_CHECK(cudaStreamSynchronize(s));
    prof_add_counts(P->pre_counts, 1);
    prof_add_counts(P->body_counts, host->body_runs);
  } else {
    enqueue_pre<double>(P, v, sc, rb, s, 0);
    OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
    OFB_CHECK(cudaStreamSynchronize(s));
    prof_collect();
    while(host->cont) {
      enqueue_body<T, double>(P, v, sc, rb, s, 0);
      OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
      OFB_CHECK(cudaStreamSynchronize(s));
      prof_collect();
    }
    enqueue_x_final<double>(P, v, sc, rb, s);
    OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
    OFB_CHECK(cudaStreamSynchronize(s));
    prof_collect();
  }
  if(history != nullptr && history_cap > 0) {
    const int n = std::min(history_cap, std::min(host->iterations + 1, P->hist_cap));
    OFB_CHECK(cudaMemcpy(history, P->hist, sizeof(double) * n, cudaMemcpyDeviceToHost));
  }
}

// ---------------------------------------------------------------------------
// Mixed path: defect correction.  The outer loop is FP64 -- residual
// r = b - A x, its norm and the convergence test against the reference's
// relative tolerance, the update x += e, the mean shifts -- and each inner
// solve A e = r runs the same MG-PCG entirely in FP32 storage and arithmetic
// (V-cycle and CG vectors; dot products and means accumulated in FP64) on the
// residual scaled to unit RMS, to a relative residual of kInnerTol.  The
// reported iteration count is the total number of inner iterations.
// ---------------------------------------------------------------------------
constexpr double kInnerTol = 1.0e-4;
constexpr int kInnerMaxIt = 60;

template <typename T>
void solve_dc(PoissonPlan* P, int max_iterations, double tolerance, SolveScalars* sc,
              SolveScalars* host, RedBuf rb, cudaStream_t s, double* history, int history_cap) {
  ensure_history(P, max_iterations);
  SolveScalars init = init_scalars(P, max_iterations, tolerance, sc, host, s);
  *host = init;
  OFB_CHECK(cudaMemcpyAsync(sc, host, sizeof(SolveScalars), cudaMemcpyHostToDevice, s));
  SolveScalars in{};
  in.zero_mean = P->zero_mean;
  in.n = init.n;
  in.tol = kInnerTol;
  in.max_it = kInnerMaxIt;
  OFB_CHECK(cudaMemcpyAsync(P->sc_in, &in, sizeof(SolveScalars), cudaMemcpyHostToDevice, s));
  const Level& l0 = P->levels[0];
  const Launch3 ln = launch3(l0.L.nx, l0.L.ny, l0.L.nz);
  // outer residual of the initial guess
  {
    ProfScope ps(kKInitResidual, s);
    k_initial_residual<double><<<ln.grid, ln.block, 0, s>>>(l0.op, P->b, P->x, P->r, sc, ln.kchunk,
                                                            rb, 0);
    OFB_LAUNCH_CHECK("k_initial_residual");
  }
  OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
  OFB_CHECK(cudaStreamSynchronize(s));
  const CGVec<float> v{nullptr, P->e32, P->r32, P->p32, P->ap32, P->p32b};
  SolveScalars* si = P->sc_in;
  auto pre = [&](cudaGraphConditionalHandle c) {
    ProfScope ps(kKDefectCorrection, s);
    k_dc_to_inner<<<ln.grid, ln.block, 0, s>>>(l0.L, P->r, sc, P->r32, P->e32, si, ln.kchunk, rb, c);
    OFB_LAUNCH_CHECK("k_dc_to_inner");
  };
  auto body = [&](cudaGraphConditionalHandle c) { enqueue_body<T, float>(P, v, si, rb, s, c); };
  auto post = [&]() {
    enqueue_x_final<float>(P, v, si, rb, s);
    ProfScope ps(kKDefectCorrection, s, 2);
    k_dc_update_x<<<ln.grid, ln.block, 0, s>>>(l0.L, P->x, P->e32, sc, si, ln.kchunk, rb);
    k_dc_residual<<<ln.grid, ln.block, 0, s>>>(l0.op, P->b, P->x, P->r, sc, si, ln.kchunk, rb);
    OFB_LAUNCH_CHECK("defect correction update");
  };
  const bool use_graph = P->use_graph && !prof_enabled();
  long long inner_runs = 0;
  while(host->cont) {
    if(use_graph) {
      if(P->exec == nullptr) P->exec = build_loop_graph(P, s, pre, body, &P->graph);
      OFB_CHECK(cudaGraphLaunch(P->exec, s));
      post();
    } else {
      pre(0);
      SolveScalars hi{};
      OFB_CHECK(cudaMemcpyAsync(&hi, si, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
      OFB_CHECK(cudaStreamSynchronize(s));
      prof_collect();
      while(hi.cont) {
        body(0);
        OFB_CHECK(cudaMemcpyAsync(&hi, si, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
        OFB_CHECK(cudaStreamSynchronize(s));
        prof_collect();
      }
      post();
    }
    OFB_CHECK(cudaMemcpyAsync(host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, s));
    OFB_CHECK(cudaStreamSynchronize(s));
    if(use_graph) {
      prof_add_counts(P->pre_counts, 1);
      prof_add_counts(P->body_counts, host->body_runs - inner_runs);
      inner_runs = host->body_runs;
    }
    prof_collect();
  }
  if(history != nullptr && history_cap > 0) {
    const int n = std::min(history_cap, std::min(host->outer + 1, P->hist_cap));
    OFB_CHECK(cudaMemcpy(history, P->hist, sizeof(double) * n, cudaMemcpyDeviceToHost));
  }
}

}  // namespace

void poisson_solve(PoissonPlan* P, int max_iterations, double tolerance, SolveScalars* sc_dev,
                   SolveScalars* sc_host, RedBuf rb, cudaStream_t s, double* history,
                   int history_cap) {
  // the fault word describes this solve only: a wait that gave up in an
  // earlier solve does not fail the next one
  OFB_CHECK(cudaMemsetAsync(P->fault, 0, sizeof(int), s));
  if(P->precision == 1)
    solve_dc<float>(P, max_iterations, tolerance, sc_dev, sc_host, rb, s, history, history_cap);
  else
    solve_impl<double>(P, max_iterations, tolerance, sc_dev, sc_host, rb, s, history, history_cap);
  int fault = 0;
  OFB_CHECK(cudaMemcpyAsync(&fault, P->fault, sizeof(int), cudaMemcpyDeviceToHost, s));
  OFB_CHECK(cudaStreamSynchronize(s));
  if(fault != 0)
    throw TimeoutError("a bounded wait for a TMA plane load gave up in the pressure solve (code " +
                       std::to_string(fault) + ")");
}

double poisson_time_coarse_chain(PoissonPlan* P, RedBuf rb, cudaStream_t s, int reps, int* launches) {
  *launches = 0;
  if(P->levels.size() < 2 || reps < 1) return 0.0;
  OFB_CHECK(cudaMemsetAsync(P->fault, 0, sizeof(int), s));
  long long counts[kKernelCount] = {};
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  prof_capture_begin(counts);
  OFB_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  // levels >= 1 read only their own level data and LevelScalars
  if(P->precision == 1)
    v_cycle<float, float>(P, 1, nullptr, nullptr, rb, s);
  else
    v_cycle<double, double>(P, 1, nullptr, nullptr, rb, s);
  OFB_CHECK(cudaStreamEndCapture(s, &g));
  prof_capture_end();
  for(int i = 0; i < kKernelCount; ++i) *launches += static_cast<int>(counts[i]);
  OFB_CHECK(cudaGraphInstantiate(&ge, g, 0));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  OFB_CHECK(cudaEventCreate(&e0));
  OFB_CHECK(cudaEventCreate(&e1));
  for(int i = 0; i < 3; ++i) OFB_CHECK(cudaGraphLaunch(ge, s));
  OFB_CHECK(cudaEventRecord(e0, s));
  for(int i = 0; i < reps; ++i) OFB_CHECK(cudaGraphLaunch(ge, s));
  OFB_CHECK(cudaEventRecord(e1, s));
  OFB_CHECK(cudaEventSynchronize(e1));
  float ms = 0.0f;
  OFB_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  int fault = 0;
  OFB_CHECK(cudaMemcpyAsync(&fault, P->fault, sizeof(int), cudaMemcpyDeviceToHost, s));
  OFB_CHECK(cudaStreamSynchronize(s));
  if(fault != 0)
    throw TimeoutError("a bounded wait for a TMA plane load gave up in the coarse-level chain (code " +
                       std::to_string(fault) + ")");
  return 1000.0 * ms / reps;
}

void launch_compact_to_pressure(const Grid& g, const double* x, const SolveScalars* sc,
                                double* p_padded, cudaStream_t s) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
  ProfScope ps(kKOther, s);
  k_compact_to_pressure<<<grid, block, 0, s>>>(g, x, sc, p_padded);
  OFB_LAUNCH_CHECK("k_compact_to_pressure");
}

}  // namespace ofb
