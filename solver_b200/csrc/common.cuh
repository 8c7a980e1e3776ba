// Shared device-side definitions of the B200 projection step: field layouts,
// boundary descriptors, launch shapes and the deterministic two-stage
// reduction used by every kernel that produces a norm, dot product or mean.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <utility>

namespace ofb {

// ---------------------------------------------------------------------------
// Field layouts.  Padded fields keep the reference's storage exactly
// (core/field_layout.hpp:69-290): one ghost layer, i unit-stride, so host and
// device copies are single contiguous transfers.  Poisson work vectors are
// compact (active cells only, no ghosts), i + nx*(j + ny*k).
// ---------------------------------------------------------------------------

enum Loc : int { kCell = 0, kFaceX = 1, kFaceY = 2, kFaceZ = 3 };

struct Lay {
  int nx, ny, nz;  // active extents
  int sx, sy, sz;  // storage extents
  int sxy;
  __host__ __device__ __forceinline__ int idx(int i, int j, int k) const {
    return i + sx * j + sxy * k;
  }
  __host__ __device__ __forceinline__ int n(int axis) const {
    return axis == 0 ? nx : axis == 1 ? ny : nz;
  }
  __host__ __device__ __forceinline__ int s(int axis) const {
    return axis == 0 ? sx : axis == 1 ? sy : sz;
  }
  __host__ __device__ __forceinline__ int stride(int axis) const {
    return axis == 0 ? 1 : axis == 1 ? sx : sxy;
  }
  __host__ __device__ __forceinline__ size_t size() const {
    return static_cast<size_t>(sxy) * static_cast<size_t>(sz);
  }
  __host__ __device__ __forceinline__ size_t active_count() const {
    return static_cast<size_t>(nx) * ny * nz;
  }
};

struct Grid {
  int nx, ny, nz;
  double dx, dy, dz;
  __host__ __device__ __forceinline__ double h(int axis) const {
    return axis == 0 ? dx : axis == 1 ? dy : dz;
  }
  __host__ __device__ __forceinline__ int n(int axis) const {
    return axis == 0 ? nx : axis == 1 ? ny : nz;
  }
};

__host__ __device__ __forceinline__ Lay make_lay(const Grid& g, int loc) {
  Lay L;
  L.nx = g.nx + (loc == kFaceX);
  L.ny = g.ny + (loc == kFaceY);
  L.nz = g.nz + (loc == kFaceZ);
  L.sx = L.nx + 2;
  L.sy = L.ny + 2;
  L.sz = L.nz + 2;
  L.sxy = L.sx * L.sy;
  return L;
}

// Compact (ghost-free) layout of a cell field, used by the pressure solve.
struct CLay {
  int nx, ny, nz, nxy;
  __host__ __device__ __forceinline__ int idx(int i, int j, int k) const {
    return i + nx * j + nxy * k;
  }
  __host__ __device__ __forceinline__ int n(int axis) const {
    return axis == 0 ? nx : axis == 1 ? ny : nz;
  }
  __host__ __device__ __forceinline__ int count() const { return nxy * nz; }
};

__host__ __device__ __forceinline__ CLay make_clay(int nx, int ny, int nz) {
  return CLay{nx, ny, nz, nx * ny};
}

// Boundary descriptors, faces x_min, x_max, y_min, y_max, z_min, z_max.
enum : int { kNoSlip = 0, kPrescribed = 1, kSymmetry = 2, kFixedPressure = 3, kPeriodic = 4 };
enum : int { kPNeumann = 0, kPDirichlet = 1, kPPeriodic = 2 };

struct VBC {
  int type[6];
  double vel[6][3];
  double pressure[6];
};

struct PBC {
  int type[6];
  double value[6];
  double gradient[6];
};

__host__ __device__ __forceinline__ bool is_dirichlet_velocity(int type) {
  return type == kNoSlip || type == kPrescribed || type == kSymmetry;
}

// ---------------------------------------------------------------------------
// Launch shapes.  Stencil kernels use 32x8 thread tiles over (i, j) and march
// a chunk of k planes per thread; the block count is kept at or below
// kMaxBlocks so that the second reduction stage fits one block.
// ---------------------------------------------------------------------------

constexpr int kTX = 32;
constexpr int kTY = 8;
constexpr int kMaxBlocks = 8192;
constexpr int kTargetBlocks = 8 * 148;  // eight blocks per SM of a B200
constexpr int kRedThreads = 256;

struct Launch3 {
  dim3 grid;
  dim3 block;
  int kchunk;
};

inline Launch3 launch3(int nx, int ny, int nz) {
  Launch3 l;
  l.block = dim3(kTX, kTY, 1);
  int gx = (nx + kTX - 1) / kTX;
  int gy = (ny + kTY - 1) / kTY;
  long long cols = static_cast<long long>(gx) * gy;
  if(cols > kMaxBlocks) {
    throw std::invalid_argument("grid cross-section too large: at most " +
                                std::to_string(kMaxBlocks * kTX * kTY) + " cells per k plane");
  }
  int kchunk = 1;
  while(cols * ((nz + kchunk - 1) / kchunk) > kMaxBlocks) kchunk *= 2;
  l.kchunk = kchunk;
  l.grid = dim3(gx, gy, (nz + kchunk - 1) / kchunk);
  return l;
}

inline int blocks_of(const Launch3& l) { return l.grid.x * l.grid.y * l.grid.z; }

// ---------------------------------------------------------------------------
// Deterministic reduction.  Each block reduces its threads' partial sums with
// warp shuffles and shared memory and stores them in `partials[k][block]`;
// the last block to finish (atomic ticket) sums the partials in a fixed order
// and runs an epilogue on thread 0 with the K totals.  The result does not
// depend on block scheduling, so runs are bitwise reproducible.  The ticket
// resets itself, so one (partials, ticket) pair serves all kernels of a stream.
// ---------------------------------------------------------------------------

struct RedBuf {
  double* partials;   // [kMaxRed][kMaxBlocks]
  unsigned int* ticket;
};
constexpr int kMaxRed = 6;

template <int K>
struct Sums {
  double v[K];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reduction of K values (sum, or max when is_max[k]); result valid
// on thread 0.  All threads of the block must call it.
template <int K>
__device__ __forceinline__ void block_reduce(double (&v)[K], const bool (&is_max)[K]) {
  __shared__ double sh[K][32];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nwarps = (nthreads + 31) >> 5;
#pragma unroll
  for(int k = 0; k < K; ++k) {
    double x = is_max[k] ? warp_max(v[k]) : warp_sum(v[k]);
    if(lane == 0) sh[k][warp] = x;
  }
  __syncthreads();
  if(warp == 0) {
#pragma unroll
    for(int k = 0; k < K; ++k) {
      double x = lane < nwarps ? sh[k][lane] : (is_max[k] ? -INFINITY : 0.0);
      v[k] = is_max[k] ? warp_max(x) : warp_sum(x);
    }
  }
  __syncthreads();
}

// Publishes the block's K partials; the last block combines all partials in
// fixed order and calls epi(totals) on its thread 0.
template <int K, typename Epi>
__device__ __forceinline__ void reduce_finish(double (&v)[K], const bool (&is_max)[K], RedBuf rb,
                                              Epi epi) {
  block_reduce<K>(v, is_max);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int nblocks = gridDim.x * gridDim.y * gridDim.z;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  __shared__ bool last;
  if(tid == 0) {
#pragma unroll
    for(int k = 0; k < K; ++k) rb.partials[k * kMaxBlocks + bid] = v[k];
    // one acquire-release ticket increment at GPU scope: it publishes this
    // block's partials and, in the last block, makes every other block's
    // visible (the CTA barrier below passes that on to the block's threads,
    // which read the partials from L2); cheaper than a full fence pair
    unsigned int t;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(t) : "l"(rb.ticket) : "memory");
    last = (t == static_cast<unsigned int>(nblocks - 1));
  }
  __syncthreads();
  if(!last) return;
  double w[K];
#pragma unroll
  for(int k = 0; k < K; ++k) {
    double acc = is_max[k] ? -INFINITY : 0.0;
    for(int b = tid; b < nblocks; b += nthreads) {
      const double x = __ldcg(&rb.partials[k * kMaxBlocks + b]);
      acc = is_max[k] ? fmax(acc, x) : acc + x;
    }
    w[k] = acc;
  }
  block_reduce<K>(w, is_max);
  if(tid == 0) {
    Sums<K> s;
#pragma unroll
    for(int k = 0; k < K; ++k) s.v[k] = w[k];
    epi(s);
    *rb.ticket = 0u;
  }
}

// ---------------------------------------------------------------------------
// Host-side error handling.
// ---------------------------------------------------------------------------

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// A bounded device-side wait gave up (reported as OF_TIMEOUT).
struct TimeoutError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void check_cuda(cudaError_t e, const char* what) {
  if(e != cudaSuccess) {
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
  }
}

#define OFB_CHECK(call) ::ofb::check_cuda((call), #call)
#define OFB_LAUNCH_CHECK(name) ::ofb::check_cuda(cudaGetLastError(), name)

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  A kernel launched with launch_pdl may begin
// launching before the kernel ahead of it in the stream has fully retired,
// which shortens the gap between the short dependent kernels of a V-cycle; in
// a CUDA graph the dependency becomes a programmatic edge.  Every kernel
// launched this way calls pdl_enter() before it touches global memory: it
// waits until the grids it depends on have completed and their writes are
// visible (a no-op under a plain launch).  No kernel triggers its dependents
// early (griddepcontrol.launch_dependents): at 256^3 that made the graph-run
// step 5 % slower, the resident waiting blocks of the next kernel getting in
// the way of the running one, while the implicit trigger at block exit gains
// 0.3 % in the graph and 16 % on the coarse levels of a host-driven loop.
// ORCHARD_B200_NO_PDL=1 makes every launch plain.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

inline bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("ORCHARD_B200_NO_PDL");
    return e == nullptr || e[0] != '1';
  }();
  return on;
}

template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                Args&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  OFB_CHECK(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

}  // namespace ofb
