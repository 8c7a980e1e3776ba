// Allocation-free pressure right-hand side pass for device-resident velocity:
// rhs = (density / dt) div(u) on the active cells (build_pressure_rhs,
// solver/projection.cpp:1049-1064) and the two norms project_velocity reports
// from it, divergence_l2_before and rhs_l2 (solver/projection.cpp:1110-1116,
// active_l2_norm at solver/projection.cpp:133-146).
//
// Who cannot allocate: a host framework that owns every byte of device memory
// through its own pool (PyTorch's caching allocator, a fixed per-run budget)
// and evaluates the pressure right-hand side of ITS velocity buffers inside
// its time-step loop.  A context (of_create) would allocate the whole per-grid
// working set, and cudaMalloc / cudaFree synchronise the device, which stalls
// every stream of the loop.  So this path takes the caller's device buffers
// and keeps the little scratch it needs -- the deterministic reduction's block
// partials, its last-block ticket and the two norms -- in one file-scope
// __device__ array; it calls no allocating API.
//
// The arithmetic, launch shape and reduction order are those of the context
// path's k_divergence_rhs, so both give bitwise the same rhs and norms.
#include "kernels.hpp"

#include <mutex>

namespace ofb {

namespace {

// Scratch layout (doubles): [0, 2*kMaxBlocks) block partials of the two sums
// (reduce_finish's [k][block] layout), then div_l2, rhs_l2, then one slot whose
// first 4 bytes are the ticket.  launch3 never launches more than kMaxBlocks
// blocks, so the partials always fit: 2 * 8192 + 4 doubles = 131,104 bytes.
constexpr int kNaResult = 2 * kMaxBlocks;
constexpr int kNaTicket = kNaResult + 2;
constexpr int kNaDoubles = kNaResult + 4;

__device__ __align__(256) double g_noalloc_scratch[kNaDoubles];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
double* g_na_ptr[kNaMaxDevices] = {};

__global__ void __launch_bounds__(kTX* kTY)
    k_pressure_rhs_noalloc(Grid g, const double* __restrict__ u, const double* __restrict__ v,
                           const double* __restrict__ w, double scale, double* __restrict__ rhs,
                           double* __restrict__ result, int kchunk, RedBuf rb) {
  const int i = blockIdx.x * kTX + threadIdx.x;
  const int j = blockIdx.y * kTY + threadIdx.y;
  const bool valid = i < g.nx && j < g.ny;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(k0 + kchunk, g.nz);
  const Lay P = make_lay(g, kCell), U = make_lay(g, kFaceX), V = make_lay(g, kFaceY),
            W = make_lay(g, kFaceZ);
  const double idx = 1.0 / g.dx, idy = 1.0 / g.dy, idz = 1.0 / g.dz;
  double acc[2] = {0.0, 0.0};
  if(valid) {
    for(int k = k0; k < k1; ++k) {
      const int uq = U.idx(i + 1, j + 1, k + 1), vq = V.idx(i + 1, j + 1, k + 1),
                wq = W.idx(i + 1, j + 1, k + 1);
      // compute_divergence (operators/discrete_operators.cpp:98-113)
      const double div = (u[uq + 1] - u[uq]) * idx + (v[vq + V.sx] - v[vq]) * idy +
                         (w[wq + W.sxy] - w[wq]) * idz;
      const double r = div * scale;
      rhs[P.idx(i + 1, j + 1, k + 1)] = r;
      acc[0] += div * div;
      acc[1] += r * r;
    }
  }
  const bool mx[2] = {false, false};
  const int n = g.nx * g.ny * g.nz;
  reduce_finish<2>(acc, mx, rb, [=](const Sums<2>& s) {
    result[0] = sqrt(s.v[0] / n);
    result[1] = sqrt(s.v[1] / n);
  });
}

}  // namespace

double* noalloc_scratch() {
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    throw CudaError("no CUDA device is available (the B200 path has no CPU fallback)");
  int dev = -1;
  OFB_CHECK(cudaGetDevice(&dev));
  if(dev < 0 || dev >= kNaMaxDevices)
    throw std::invalid_argument("of_pressure_rhs_noalloc supports CUDA devices 0.." +
                                std::to_string(kNaMaxDevices - 1));
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if(g_na_ptr[dev] == nullptr) {
    // First call on this device: the symbol lookup loads this module on the
    // device (if not loaded yet); later calls only read the cached address.
    // The address stays valid for the life of the process unless the device
    // is reset (cudaDeviceReset unloads the module), which callers of this
    // entry point must not do between calls.
    void* p = nullptr;
    OFB_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_na_ptr[dev] = static_cast<double*>(p);
  }
  return g_na_ptr[dev];
}

long long noalloc_max_plane_blocks() { return kMaxBlocks; }

void launch_pressure_rhs_noalloc(const Grid& g, const double* u, const double* v, const double* w,
                                 double scale, double* rhs, double* scratch, double* norms_host,
                                 cudaStream_t s) {
  const Launch3 l = launch3(g.nx, g.ny, g.nz);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kNaTicket);
  // the ticket must start at zero; it resets itself, but a launch that never
  // completed would leave it set
  OFB_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s));
  {
    ProfScope ps(kKDivergence, s);
    k_pressure_rhs_noalloc<<<l.grid, l.block, 0, s>>>(g, u, v, w, scale, rhs, scratch + kNaResult,
                                                      l.kchunk, RedBuf{scratch, ticket});
    OFB_LAUNCH_CHECK("k_pressure_rhs_noalloc");
  }
  if(norms_host) {
    OFB_CHECK(cudaMemcpyAsync(norms_host, scratch + kNaResult, 2 * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    OFB_CHECK(cudaStreamSynchronize(s));
  }
}

}  // namespace ofb
