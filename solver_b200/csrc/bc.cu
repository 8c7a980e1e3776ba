// Boundary-condition kernels: the reference's ghost fills restated as index
// rules over boundary planes.  One thread owns one line normal to the axis
// being filled and applies the lower face then the upper face, exactly in the
// reference's order, so faces that share a line (a two-face normal component)
// see each other's writes as they do on the CPU.  Edge and corner ghosts are
// never written, as in the reference (solver/projection.cpp:207-300 copies
// over the active range of the other axes only).
#include "kernels.hpp"

namespace ofb {

namespace {

__device__ __forceinline__ void other_axes(int axis, int& a1, int& a2) {
  a1 = axis == 0 ? 1 : 0;
  a2 = axis == 2 ? 1 : 2;
}

__device__ __forceinline__ int base_index(const Lay& L, int axis, int a1, int p1, int a2, int p2) {
  int c[3] = {0, 0, 0};
  c[a1] = p1;
  c[a2] = p2;
  (void)axis;
  return L.idx(c[0], c[1], c[2]);
}

// apply_velocity_component_boundaries for one axis (solver/projection.cpp:451-462):
// apply_periodic_pair (:207-300) or apply_face_field_boundary (:384-449).
__global__ void k_velocity_bc_axis(Grid g, VBC bc, int axis, int comp0, double* f0, double* f1,
                                   double* f2) {
  const int comp = comp0 + blockIdx.z;
  double* f = comp == 0 ? f0 : comp == 1 ? f1 : f2;
  if(f == nullptr) return;
  const Lay L = make_lay(g, kFaceX + comp);
  int a1, a2;
  other_axes(axis, a1, a2);
  const int t1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t2 = blockIdx.y * blockDim.y + threadIdx.y;
  if(t1 >= L.n(a1) || t2 >= L.n(a2)) return;
  const int base = base_index(L, axis, a1, t1 + 1, a2, t2 + 1);
  const int st = L.stride(axis);
  const int n = L.n(axis);
  auto at = [&](int q) -> double& { return f[base + q * st]; };

  if(bc.type[2 * axis] == kPeriodic) {
    if(comp == axis) {
      const double shared = 0.5 * (at(1) + at(n));
      at(1) = shared;
      at(n) = shared;
      at(0) = at(n - 1);
      at(n + 1) = at(2);
    } else {
      at(0) = at(n);
      at(n + 1) = at(1);
    }
    return;
  }
  for(int side = 0; side < 2; ++side) {
    const int face = 2 * axis + side;
    const int type = bc.type[face];
    if(type == kPeriodic) continue;
    const bool lower = side == 0;
    const int b = lower ? 1 : n;
    const int gq = lower ? 0 : n + 1;
    if(comp == axis) {
      const int ii = lower ? b + 1 : b - 1;
      if(type == kFixedPressure) {
        at(b) = at(ii);
        at(gq) = at(b);
        continue;
      }
      const double bv = type == kSymmetry ? 0.0 : bc.vel[face][comp];
      at(b) = bv;
      at(gq) = 2.0 * bv - at(ii);
      continue;
    }
    if(type == kNoSlip || type == kPrescribed) {
      at(gq) = 2.0 * bc.vel[face][comp] - at(b);
    } else if(type == kSymmetry || type == kFixedPressure) {
      at(gq) = at(b);
    }
  }
}

// nu * Laplacian of a face field at one point (compute_diffusion_term,
// solver/momentum_terms.cpp:316-325 via operators/discrete_operators.cpp:24-60).
__device__ __forceinline__ double diffusion_at(const Lay& L, const Grid& g, double nu,
                                               const double* f, int i, int j, int k) {
  const int q = L.idx(i, j, k);
  const double c2 = 2.0 * f[q];
  const double ix = 1.0 / (g.dx * g.dx), iy = 1.0 / (g.dy * g.dy), iz = 1.0 / (g.dz * g.dz);
  const double lap = (f[q + 1] - c2 + f[q - 1]) * ix + (f[q + L.sx] - c2 + f[q - L.sx]) * iy +
                     (f[q + L.sxy] - c2 + f[q - L.sxy]) * iz;
  return lap * nu;
}

// apply_total_pressure_boundary_conditions (solver/projection.cpp:986-1026):
// periodic pairs, wall-normal gradient ghosts (:339-382) and fixed-pressure
// Dirichlet ghosts (:302-337).  blockIdx.z selects the axis; axes are
// independent because every source is an active cell.
__global__ void k_total_pressure_bc(Grid g, VBC bc, double nu, const double* u, const double* v,
                                    const double* w, double* p) {
  const int axis = blockIdx.z;
  const Lay P = make_lay(g, kCell);
  int a1, a2;
  other_axes(axis, a1, a2);
  const int t1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int t2 = blockIdx.y * blockDim.y + threadIdx.y;
  if(t1 >= P.n(a1) || t2 >= P.n(a2)) return;
  const int base = base_index(P, axis, a1, t1 + 1, a2, t2 + 1);
  const int st = P.stride(axis);
  const int n = P.n(axis);
  if(bc.type[2 * axis] == kPeriodic) {
    p[base] = p[base + n * st];
    p[base + (n + 1) * st] = p[base + st];
    return;
  }
  const double spacing = g.h(axis);
  const double* src = axis == 0 ? u : axis == 1 ? v : w;
  const Lay S = make_lay(g, kFaceX + axis);
  for(int side = 0; side < 2; ++side) {
    const int face = 2 * axis + side;
    const int type = bc.type[face];
    const bool lower = side == 0;
    const int b = lower ? 1 : n;
    const int gq = lower ? 0 : n + 1;
    const double active = p[base + b * st];
    if(type == kNoSlip || type == kPrescribed || type == kSymmetry) {
      int c[3];
      c[a1] = t1 + 1;
      c[a2] = t2 + 1;
      c[axis] = lower ? 1 : S.n(axis);
      const double grad = diffusion_at(S, g, nu, src, c[0], c[1], c[2]);
      p[base + gq * st] = lower ? active - grad * spacing : active + grad * spacing;
    } else if(type == kFixedPressure) {
      p[base + gq * st] = 2.0 * bc.pressure[face] - active;
    }
  }
}

}  // namespace

void launch_component_bc(const Grid& g, const VBC& bc, int comp, double* f, cudaStream_t s) {
  for(int axis = 0; axis < 3; ++axis) {
    const int d1 = (axis == 0 ? g.ny : g.nx) + 1;
    const int d2 = (axis == 2 ? g.ny : g.nz) + 1;
    dim3 block(32, 8, 1);
    dim3 grid((d1 + 31) / 32, (d2 + 7) / 8, 1);
    double* fs[3] = {nullptr, nullptr, nullptr};
    fs[comp] = f;
    ProfScope ps(kKVelocityBc, s);
    k_velocity_bc_axis<<<grid, block, 0, s>>>(g, bc, axis, comp, fs[0], fs[1], fs[2]);
    OFB_LAUNCH_CHECK("k_velocity_bc_axis");
  }
}

void launch_velocity_bc(const Grid& g, const VBC& bc, double* u, double* v, double* w,
                        cudaStream_t s) {
  // One launch per axis covering the three components: the reference applies
  // x, then y, then z pairs per component, and later axes read active values
  // that earlier axes may have rewritten (duplicated faces, wall faces).
  for(int axis = 0; axis < 3; ++axis) {
    const int d1 = (axis == 0 ? g.ny : g.nx) + 1;
    const int d2 = (axis == 2 ? g.ny : g.nz) + 1;
    dim3 block(32, 8, 1);
    dim3 grid((d1 + 31) / 32, (d2 + 7) / 8, 3);
    ProfScope ps(kKVelocityBc, s);
    k_velocity_bc_axis<<<grid, block, 0, s>>>(g, bc, axis, 0, u, v, w);
    OFB_LAUNCH_CHECK("k_velocity_bc_axis");
  }
}

void launch_total_pressure_bc(const Grid& g, const VBC& bc, double nu, const double* u,
                              const double* v, const double* w, double* p, cudaStream_t s) {
  const int d1 = g.nx > g.ny ? g.nx : g.ny;
  const int d2 = g.ny > g.nz ? g.ny : g.nz;
  const int dm = d1 > d2 ? d1 : d2;
  dim3 block(32, 8, 1);
  dim3 grid((dm + 31) / 32, (dm + 7) / 8, 3);
  ProfScope ps(kKTotalPressureBc, s);
  k_total_pressure_bc<<<grid, block, 0, s>>>(g, bc, nu, u, v, w, p);
  OFB_LAUNCH_CHECK("k_total_pressure_bc");
}

}  // namespace ofb
