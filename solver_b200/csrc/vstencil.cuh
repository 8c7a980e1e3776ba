// Row-vector 7-point stencil engine for the pressure solve's large levels.
//
// A thread owns W consecutive cells of one (j, k) row (W = 16 bytes / value:
// 2 doubles or 4 floats) and marches k over its chunk.  Per plane it issues
// one 16-byte load for its row, two for the rows j-1 and j+1 and one for the
// epilogue's extra input, gets the x-neighbours of its end cells from the
// adjacent lanes by warp shuffle and the z-neighbours from a register queue;
// all loads for plane k+1 are issued while plane k is computed.  Boundary
// rules (periodic image, or +/- the boundary cell for homogeneous
// Neumann/Dirichlet, linsolve/poisson_solver.cpp:195-242) are applied to the
// loaded values, so the arithmetic has no branches.
#pragma once

#include <type_traits>

namespace ofb {
namespace vst {

template <typename T>
struct Width {
  static constexpr int W = 16 / sizeof(T);
};

template <typename A, int W>
struct Row {
  A v[W];
};

// Loads W values of type S starting at p (16-byte aligned when W * sizeof(S) >= 16)
// and converts them to A.
template <typename A, int W, typename S>
__device__ __forceinline__ Row<A, W> ld(const S* __restrict__ p) {
  Row<A, W> r;
  if constexpr(std::is_same_v<S, double> && W == 2) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    r.v[0] = A(t.x);
    r.v[1] = A(t.y);
  } else if constexpr(std::is_same_v<S, double> && W == 4) {
    const double2 t0 = *reinterpret_cast<const double2*>(p);
    const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
    r.v[0] = A(t0.x);
    r.v[1] = A(t0.y);
    r.v[2] = A(t1.x);
    r.v[3] = A(t1.y);
  } else if constexpr(std::is_same_v<S, float> && W == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    r.v[0] = A(t.x);
    r.v[1] = A(t.y);
    r.v[2] = A(t.z);
    r.v[3] = A(t.w);
  } else {
#pragma unroll
    for(int t = 0; t < W; ++t) r.v[t] = A(p[t]);
  }
  return r;
}

template <typename S, int W, typename A>
__device__ __forceinline__ void st(S* __restrict__ p, const Row<A, W>& r) {
  if constexpr(std::is_same_v<S, double> && W == 2) {
    *reinterpret_cast<double2*>(p) = make_double2(double(r.v[0]), double(r.v[1]));
  } else if constexpr(std::is_same_v<S, float> && W == 4) {
    *reinterpret_cast<float4*>(p) =
        make_float4(float(r.v[0]), float(r.v[1]), float(r.v[2]), float(r.v[3]));
  } else {
#pragma unroll
    for(int t = 0; t < W; ++t) p[t] = S(r.v[t]);
  }
}

template <typename A, int W>
__device__ __forceinline__ Row<A, W> scaled(const Row<A, W>& r, A s, A sh) {
  Row<A, W> o;
#pragma unroll
  for(int t = 0; t < W; ++t) o.v[t] = s * (r.v[t] - sh);
  return o;
}

// The launch shape: 32 x 8 threads, thread (tx, ty) -> cells i0 = (bx*32 + tx)*W
// .. i0+W-1 of row j = by*8 + ty; grid z = k chunks.
inline bool row_fits(int nx, int W) { return nx % W == 0 && nx >= W; }

struct RowLaunch {
  dim3 grid, block;
  int kchunk;
};

inline RowLaunch row_launch(int nx, int ny, int nz, int W, int min_chunk) {
  RowLaunch l;
  l.block = dim3(32, 8, 1);
  const int gx = (nx / W + 31) / 32;
  const int gy = (ny + 7) / 8;
  long long cols = static_cast<long long>(gx) * gy;
  int kchunk = min_chunk < nz ? min_chunk : nz;
  if(kchunk < 1) kchunk = 1;
  // Small levels: shorter chunks, so that enough blocks run at once to hide
  // the latency of each plane's loads (a long chunk on a few blocks is one
  // long chain of dependent plane loads).
  while(kchunk > 1 && cols * ((nz + kchunk - 1) / kchunk) < kTargetBlocks) kchunk /= 2;
  while(cols * ((nz + kchunk - 1) / kchunk) > kMaxBlocks) kchunk *= 2;
  l.kchunk = kchunk;
  l.grid = dim3(gx, gy, (nz + kchunk - 1) / kchunk);
  return l;
}

// Per-row geometry: neighbour rows, halo needs, signs (all branch-free).
struct RowGeom {
  int i0, j;
  bool act;          // the thread owns real cells
  int jd, ju;        // y-neighbour rows
  double syd, syu;   // their signs (rule rows repeat row j)
  bool need_l, need_r;
  int xl, xr;        // x-halo cells (loaded when need_*)
  double sxl, sxr;
};

template <int W>
__device__ __forceinline__ RowGeom row_geom(const CLay& L, const int (&per)[3], const int (&dlo)[3],
                                            const int (&dhi)[3]) {
  RowGeom g;
  const int lane = threadIdx.x;
  g.i0 = (blockIdx.x * 32 + lane) * W;
  g.j = blockIdx.y * 8 + threadIdx.y;
  g.act = g.i0 < L.nx && g.j < L.ny;
  // inactive threads work on a clamped row so that every load stays in bounds
  if(g.i0 >= L.nx) g.i0 = L.nx - W;
  if(g.j >= L.ny) g.j = L.ny - 1;
  // y neighbours (nb_lo / nb_hi rules)
  {
    const bool in = g.j > 0;
    g.jd = in ? g.j - 1 : (per[1] ? L.ny - 1 : g.j);
    g.syd = (in || per[1] || !dlo[1]) ? 1.0 : -1.0;
  }
  {
    const bool in = g.j < L.ny - 1;
    g.ju = in ? g.j + 1 : (per[1] ? 0 : g.j);
    g.syu = (in || per[1] || !dhi[1]) ? 1.0 : -1.0;
  }
  g.need_l = lane == 0 || g.i0 == 0;
  g.need_r = lane == 31 || g.i0 + W >= L.nx;
  {
    const bool in = g.i0 > 0;
    g.xl = in ? g.i0 - 1 : (per[0] ? L.nx - 1 : g.i0);
    g.sxl = (in || per[0] || !dlo[0]) ? 1.0 : -1.0;
  }
  {
    const int last = g.i0 + W - 1;
    const bool in = last < L.nx - 1;
    g.xr = in ? last + 1 : (per[0] ? 0 : last);
    g.sxr = (in || per[0] || !dhi[0]) ? 1.0 : -1.0;
  }
  return g;
}

// z-neighbour plane of kk (may be -1 or >= nz) with its sign.
__device__ __forceinline__ int zrow(int kk, int nz, int per, int dlo, int dhi, double& sg) {
  if(kk < 0) {
    sg = (per || !dlo) ? 1.0 : -1.0;
    return per ? nz - 1 : 0;
  }
  if(kk >= nz) {
    sg = (per || !dhi) ? 1.0 : -1.0;
    return per ? 0 : nz - 1;
  }
  sg = 1.0;
  return kk;
}

// A x on W cells of a row from the row, its x end-neighbours and the four
// neighbour rows: -(r - 2c + l)/dx^2 - (u - 2c + d)/dy^2 - (a - 2c + b)/dz^2.
template <typename A, int W>
__device__ __forceinline__ Row<A, W> row_ax(const Row<A, W>& c, A left, A right, const Row<A, W>& d,
                                            const Row<A, W>& u, const Row<A, W>& b,
                                            const Row<A, W>& a, A ix, A iy, A iz) {
  Row<A, W> o;
#pragma unroll
  for(int t = 0; t < W; ++t) {
    const A l = t > 0 ? c.v[t - 1] : left;
    const A r = t < W - 1 ? c.v[t + 1] : right;
    const A two_c = A(2) * c.v[t];
    o.v[t] = -(r - two_c + l) * ix - (u.v[t] - two_c + d.v[t]) * iy - (a.v[t] - two_c + b.v[t]) * iz;
  }
  return o;
}

// Everything one plane needs besides the register queue.
template <typename A, int W, typename X>
struct PlaneIn {
  Row<A, W> d, u;
  A hl, hr;
  X aux;
};

// Marches planes [k0, k1) of one row.  rowv(i0, j, k) returns the operand row
// (W values, shifts applied); cellv(i, j, k) one operand value; aux(i0, j, k)
// the epilogue's extra input; point(k, centre row, A x row, aux) consumes.
// All threads of a warp must call it (shuffles); inactive threads compute on
// clamped rows and their point() must not store.
template <typename A, int W, typename X, typename Op, typename RowV, typename CellV, typename Aux,
          typename Point>
__device__ __forceinline__ void march(const Op& o, const RowGeom& g, int k0, int k1, RowV rowv,
                                      CellV cellv, Aux aux, Point point) {
  const int nz = o.L.nz;
  const int pz = o.periodic[2], dlz = o.dir_lo[2], dhz = o.dir_hi[2];
  const A ix = A(o.inv2[0]), iy = A(o.inv2[1]), iz = A(o.inv2[2]);
  auto plane_in = [&](int k) {
    PlaneIn<A, W, X> p;
    p.d = rowv(g.i0, g.jd, k);
    p.u = rowv(g.i0, g.ju, k);
#pragma unroll
    for(int t = 0; t < W; ++t) {
      p.d.v[t] *= A(g.syd);
      p.u.v[t] *= A(g.syu);
    }
    p.hl = g.need_l ? A(g.sxl) * cellv(g.xl, g.j, k) : A(0);
    p.hr = g.need_r ? A(g.sxr) * cellv(g.xr, g.j, k) : A(0);
    p.aux = aux(g.i0, g.j, k);
    return p;
  };
  auto zq = [&](int kk) {
    double sg;
    const int kz = zrow(kk, nz, pz, dlz, dhz, sg);
    Row<A, W> r = rowv(g.i0, g.j, kz);
#pragma unroll
    for(int t = 0; t < W; ++t) r.v[t] *= A(sg);
    return r;
  };
  Row<A, W> below = zq(k0 - 1);
  Row<A, W> cen = zq(k0);
  Row<A, W> above = zq(k0 + 1);
  PlaneIn<A, W, X> cur = plane_in(k0);
  for(int k = k0; k < k1; ++k) {
    // prefetch plane k+1 (clamped; unused beyond k1)
    const int kn = k + 1 < nz ? k + 1 : nz - 1;
    const Row<A, W> above2 = zq(k + 2);
    const PlaneIn<A, W, X> nxt = plane_in(kn);
    const A from_l = __shfl_up_sync(0xffffffffu, cen.v[W - 1], 1);
    const A from_r = __shfl_down_sync(0xffffffffu, cen.v[0], 1);
    const A left = g.need_l ? cur.hl : from_l;
    const A right = g.need_r ? cur.hr : from_r;
    const Row<A, W> ax = row_ax<A, W>(cen, left, right, cur.d, cur.u, below, above, ix, iy, iz);
    point(k, cen, ax, cur.aux);
    below = cen;
    cen = above;
    above = above2;
    cur = nxt;
  }
}

}  // namespace vst
}  // namespace ofb
