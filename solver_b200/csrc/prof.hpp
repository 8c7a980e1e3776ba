// Kernel classes for launch accounting and event timing (prof.cu).
#pragma once

#include <cuda_runtime.h>

namespace ofb {

enum KernelClass : int {
  kKPredictor = 0,
  kKAdvection,
  kKAdi,
  kKVelocityBc,
  kKDivergence,
  kKInitResidual,
  kKApplyAp,
  kKUpdateXr,
  kKUpdateP,
  kKSmoothFirstFine,
  kKSmoothFine,
  kKRestrictFine,
  kKProlongFine,
  kKCoarseLevels,
  kKCoarseSolve,
  kKCorrect,
  kKCellPass,
  kKTotalPressureBc,
  kKAdjoint,
  kKDefectCorrection,
  kKOther,
  kKernelCount
};

void prof_launch(int id, cudaStream_t s, bool begin, int count = 1);
void prof_collect();
bool prof_enabled();
// While a graph is captured, launches are counted into `counts` (no events);
// prof_add_counts later credits the replays.
void prof_capture_begin(long long* counts);
void prof_capture_end();
void prof_add_counts(const long long* counts, long long times);

// Times a chain of launches with one event pair (class `id`) instead of one
// pair per launch; the launches inside are still counted by their scopes.
void prof_span(int id, cudaStream_t s, bool begin);

struct ProfSpan {
  int id;
  cudaStream_t s;
  ProfSpan(int id_, cudaStream_t s_) : id(id_), s(s_) { prof_span(id, s, true); }
  ~ProfSpan() { prof_span(id, s, false); }
};

// Brackets `count` kernel launches of one class: counts them and, when timing
// is on, records an event pair around them on their stream.
struct ProfScope {
  int id;
  cudaStream_t s;
  ProfScope(int id_, cudaStream_t s_, int count = 1) : id(id_), s(s_) {
    prof_launch(id, s, true, count);
  }
  ~ProfScope() { prof_launch(id, s, false); }
};

}  // namespace ofb
