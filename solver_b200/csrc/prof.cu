// Launch accounting and optional per-kernel CUDA-event timing.  Every launcher
// counts its launches (always on); when timing is enabled the launches of each
// kernel class are bracketed by event pairs on their stream and the elapsed
// times are collected at the next host synchronisation.  bench.py reads these
// to report the dominant kernel's achieved bandwidth from live launches.
#include "../../include/orchard_b200.h"
#include "prof.hpp"

#include <mutex>
#include <vector>

namespace ofb {

namespace {

struct Pending {
  int id;
  cudaEvent_t start;
  cudaEvent_t stop;
};

struct Profiler {
  std::mutex mu;
  bool enabled = false;
  long long launches[kKernelCount] = {};
  double total_ms[kKernelCount] = {};
  long long timed[kKernelCount] = {};
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t cur_start[kKernelCount] = {};
  long long* capture = nullptr;
  int mute = 0;  // inside a span: launches are counted, not timed one by one
  cudaEvent_t span_start[kKernelCount] = {};
};

Profiler& prof() {
  static Profiler p;
  return p;
}

cudaEvent_t take_event(Profiler& p) {
  if(!p.pool.empty()) {
    cudaEvent_t e = p.pool.back();
    p.pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

const char* kNames[kKernelCount] = {
    "predictor_rhs", "advection", "adi_sweep", "velocity_bc", "divergence_rhs", "pcg_initial_residual",
    "pcg_apply_ap", "pcg_update_xr", "pcg_update_p", "vcycle_smooth_first_fine",
    "vcycle_smooth_fine", "vcycle_restrict_fine", "vcycle_prolong_smooth_fine",
    "vcycle_coarse_levels", "vcycle_coarse_solve", "correct_velocity", "cell_pass",
    "total_pressure_bc", "adjoint", "defect_correction", "other"};

}  // namespace

void prof_launch(int id, cudaStream_t s, bool begin, int count) {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  if(p.capture != nullptr) {
    if(begin) p.capture[id] += count;
    return;
  }
  if(begin) {
    p.launches[id] += count;
    if(!p.enabled || p.mute > 0) return;
    cudaEvent_t e = take_event(p);
    cudaEventRecord(e, s);
    p.cur_start[id] = e;
    return;
  }
  if(!p.enabled || p.mute > 0 || p.cur_start[id] == nullptr) return;
  cudaEvent_t e = take_event(p);
  cudaEventRecord(e, s);
  p.pending.push_back(Pending{id, p.cur_start[id], e});
  p.cur_start[id] = nullptr;
}

void prof_span(int id, cudaStream_t s, bool begin) {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  if(p.capture != nullptr) return;
  if(begin) {
    if(p.enabled && p.mute == 0) {
      cudaEvent_t e = take_event(p);
      cudaEventRecord(e, s);
      p.span_start[id] = e;
    }
    ++p.mute;
    return;
  }
  --p.mute;
  if(p.mute > 0 || !p.enabled || p.span_start[id] == nullptr) return;
  cudaEvent_t e = take_event(p);
  cudaEventRecord(e, s);
  p.pending.push_back(Pending{id, p.span_start[id], e});
  p.span_start[id] = nullptr;
}

bool prof_enabled() {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  return p.enabled;
}

void prof_capture_begin(long long* counts) {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  p.capture = counts;
}

void prof_capture_end() {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  p.capture = nullptr;
}

void prof_add_counts(const long long* counts, long long times) {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  for(int i = 0; i < kKernelCount; ++i) p.launches[i] += counts[i] * times;
}

void prof_collect() {
  Profiler& p = prof();
  std::lock_guard<std::mutex> lock(p.mu);
  for(const Pending& q : p.pending) {
    float ms = 0.0f;
    if(cudaEventSynchronize(q.stop) == cudaSuccess && cudaEventElapsedTime(&ms, q.start, q.stop) == cudaSuccess) {
      p.total_ms[q.id] += ms;
      ++p.timed[q.id];
    }
    p.pool.push_back(q.start);
    p.pool.push_back(q.stop);
  }
  p.pending.clear();
}

}  // namespace ofb

extern "C" {

int of_kernel_class_count(void) { return ofb::kKernelCount; }

const char* of_kernel_class_name(int id) {
  return (id >= 0 && id < ofb::kKernelCount) ? ofb::kNames[id] : "";
}

of_status of_profile_enable(int enable) {
  ofb::prof_collect();
  ofb::Profiler& p = ofb::prof();
  std::lock_guard<std::mutex> lock(p.mu);
  p.enabled = enable != 0;
  return OF_OK;
}

of_status of_profile_reset(void) {
  ofb::prof_collect();
  ofb::Profiler& p = ofb::prof();
  std::lock_guard<std::mutex> lock(p.mu);
  for(int i = 0; i < ofb::kKernelCount; ++i) {
    p.launches[i] = 0;
    p.total_ms[i] = 0.0;
    p.timed[i] = 0;
  }
  return OF_OK;
}

of_status of_profile_read(int id, long long* launches, long long* timed, double* total_ms) {
  if(id < 0 || id >= ofb::kKernelCount) return OF_INVALID_ARGUMENT;
  ofb::prof_collect();
  ofb::Profiler& p = ofb::prof();
  std::lock_guard<std::mutex> lock(p.mu);
  if(launches) *launches = p.launches[id];
  if(timed) *timed = p.timed[id];
  if(total_ms) *total_ms = p.total_ms[id];
  return OF_OK;
}

}  // extern "C"
