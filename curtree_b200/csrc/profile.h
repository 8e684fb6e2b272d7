// Optional per-kernel CUDA-event timing.  Off by default; when enabled
// (crt_profile_enable), each major kernel launch is bracketed by an event pair
// on its own stream and crt_profile_collect sums the durations by name.  Used
// by the benchmark to time the dominant kernel inside its timed region.
#pragma once
#include <cuda_runtime.h>

namespace crt {

bool profiling();
// Records the start event of a launch named `name` on `stream` (no-op when
// profiling is off or the stream is capturing); returns a token for stop.
int prof_start(const char* name, cudaStream_t stream);
void prof_stop(int token, cudaStream_t stream);
// Adds an already measured duration (graph replays time themselves).
void prof_add(const char* name, double ms);

struct ProfScope {
  int tok;
  cudaStream_t s;
  ProfScope(const char* name, cudaStream_t stream) : tok(prof_start(name, stream)), s(stream) {}
  ~ProfScope() { prof_stop(tok, s); }
};

}  // namespace crt
