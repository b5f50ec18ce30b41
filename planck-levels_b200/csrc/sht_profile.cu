// Launch counting and optional per-kernel CUDA-event timing (see ProfScope in
// sht_device.h and sharp_b200_profile* in sharp_b200.h).
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "sht_device.h"

namespace sht {

namespace {
std::atomic<unsigned long long> g_launches{0};
std::atomic<bool> g_profile{false};
std::mutex g_prof_mutex;
struct Span {
  cudaEvent_t a, b;
};
std::map<std::string, std::vector<Span>> g_spans;
}  // namespace

ProfScope::ProfScope(const char *family, cudaStream_t st) : family_(family), st_(st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (g_profile.load(std::memory_order_relaxed)) {
    SHT_CUDA(cudaEventCreate(&start_));
    SHT_CUDA(cudaEventRecord(start_, st_));
  }
}

ProfScope::~ProfScope() {
  if (!start_) return;
  cudaEvent_t stop;
  if (cudaEventCreate(&stop) != cudaSuccess) return;
  cudaEventRecord(stop, st_);
  std::lock_guard<std::mutex> lk(g_prof_mutex);
  g_spans[family_].push_back({start_, stop});
}

}  // namespace sht

extern "C" {

unsigned long long sharp_b200_kernel_launches(void) { return sht::g_launches.load(); }

void sharp_b200_profile(int on) {
  std::lock_guard<std::mutex> lk(sht::g_prof_mutex);
  for (auto &kv : sht::g_spans)
    for (auto &s : kv.second) {
      cudaEventDestroy(s.a);
      cudaEventDestroy(s.b);
    }
  sht::g_spans.clear();
  sht::g_profile.store(on != 0);
}

double sharp_b200_profile_ms(const char *family, unsigned long long *launches) {
  std::lock_guard<std::mutex> lk(sht::g_prof_mutex);
  double ms = 0.0;
  unsigned long long n = 0;
  auto it = sht::g_spans.find(family ? family : "");
  if (it != sht::g_spans.end())
    for (auto &s : it->second) {
      float t = 0.f;
      if (cudaEventSynchronize(s.b) == cudaSuccess && cudaEventElapsedTime(&t, s.a, s.b) == cudaSuccess) {
        ms += t;
        ++n;
      }
    }
  if (launches) *launches = n;
  return ms;
}

}  // extern "C"
