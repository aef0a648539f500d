// Launch counting and optional per-pass MVP timing.
//
// When profiling is on, every block MVP records six events on its stream
// (before the first pass and after each of the five); bdda_profile_read
// synchronises them and returns the summed duration of each pass.  This is
// how a caller measures the product's kernels inside a full solve.
#include <atomic>
#include <mutex>
#include <vector>

#include "bdda_internal.h"

namespace bdda {

static std::atomic<unsigned long long> g_launches{0};
static std::atomic<bool> g_profiling{false};
static std::mutex g_mu;
static std::vector<cudaEvent_t> g_free;
static std::vector<cudaEvent_t> g_marks[6];
static std::vector<int> g_prec;   // precision of each recorded product

void count_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
bool profiling() { return g_profiling.load(std::memory_order_relaxed); }

void profile_mark(int pass, cudaStream_t st, int prec) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (pass == 0) g_prec.push_back(prec);
  cudaEvent_t e;
  if (!g_free.empty()) {
    e = g_free.back();
    g_free.pop_back();
  } else if (cudaEventCreate(&e) != cudaSuccess) {
    return;
  }
  cudaEventRecord(e, st);
  g_marks[pass].push_back(e);
}

}  // namespace bdda

using namespace bdda;

extern "C" {

unsigned long long bdda_launch_count(void) { return g_launches.load(); }

int bdda_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (int p = 0; p < 6; ++p) {
    for (cudaEvent_t e : g_marks[p]) g_free.push_back(e);
    g_marks[p].clear();
  }
  g_prec.clear();
  g_profiling.store(on != 0);
  return BDDA_OK;
}

int bdda_profile_read(int prec, double pass_ms[5], long long* n_mvp) {
  if (!pass_ms || !n_mvp) return BDDA_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_mu);
  const size_t n = g_marks[0].size();
  for (int p = 1; p < 6; ++p)
    if (g_marks[p].size() != n) return BDDA_BAD_ARG;
  if (g_prec.size() != n) return BDDA_BAD_ARG;
  for (int p = 0; p < 5; ++p) pass_ms[p] = 0.0;
  long long counted = 0;
  for (size_t i = 0; i < n; ++i) {
    if (prec >= 0 && g_prec[i] != prec) continue;
    ++counted;
    BDDA_CUDA_TRY(cudaEventSynchronize(g_marks[5][i]));
    for (int p = 0; p < 5; ++p) {
      float ms = 0.f;
      BDDA_CUDA_TRY(cudaEventElapsedTime(&ms, g_marks[p][i], g_marks[p + 1][i]));
      pass_ms[p] += ms;
    }
  }
  *n_mvp = counted;
  return BDDA_OK;
}

}  // extern "C"
