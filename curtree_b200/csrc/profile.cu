// CUDA-event kernel timing behind crt_profile_* (see profile.h).
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"
#include "profile.h"

namespace crt {

namespace {
struct Rec {
  std::string name;
  cudaEvent_t a = nullptr, b = nullptr;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::map<std::string, std::pair<double, long long>> g_done;  // name -> (ms, launches)
}  // namespace

bool profiling() { return g_on; }

int prof_start(const char* name, cudaStream_t stream)
{
  if (!g_on) return -1;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return -1;
  Rec r;
  r.name = name;
  if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) return -1;
  cudaEventRecord(r.a, stream);
  std::lock_guard<std::mutex> lk(g_mu);
  g_recs.push_back(r);
  return (int)g_recs.size() - 1;
}

void prof_stop(int token, cudaStream_t stream)
{
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (token < (int)g_recs.size()) cudaEventRecord(g_recs[token].b, stream);
}

bool prof_register(const char* name, cudaEvent_t* a, cudaEvent_t* b)
{
  if (!g_on) return false;
  Rec r;
  r.name = name;
  if (cudaEventCreate(&r.a) != cudaSuccess) return false;
  if (cudaEventCreate(&r.b) != cudaSuccess) {
    cudaEventDestroy(r.a);
    return false;
  }
  *a = r.a;
  *b = r.b;
  std::lock_guard<std::mutex> lk(g_mu);
  g_recs.push_back(r);
  return true;
}

void prof_add(const char* name, double ms)
{
  std::lock_guard<std::mutex> lk(g_mu);
  auto& e = g_done[name];
  e.first += ms;
  e.second += 1;
}

static void drain_locked()
{
  for (auto& r : g_recs) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      auto& e = g_done[r.name];
      e.first += ms;
      e.second += 1;
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_recs.clear();
}

}  // namespace crt

using namespace crt;

extern "C" {

void crt_profile_enable(int on)
{
  std::lock_guard<std::mutex> lk(g_mu);
  if (!on) drain_locked();
  g_on = on != 0;
}

// Sums the recorded launches whose name equals `name` (all when name is
// NULL or empty) and forgets them.  Waits for the recorded events.
int crt_profile_collect(const char* name, double* total_ms, int64_t* launches)
{
  std::lock_guard<std::mutex> lk(g_mu);
  drain_locked();
  double ms = 0;
  long long n = 0;
  for (auto it = g_done.begin(); it != g_done.end();) {
    if (!name || !*name || it->first == name) {
      ms += it->second.first;
      n += it->second.second;
      it = g_done.erase(it);
    } else {
      ++it;
    }
  }
  if (total_ms) *total_ms = ms;
  if (launches) *launches = n;
  return CRT_OK;
}

}  // extern "C"
