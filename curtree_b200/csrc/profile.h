// NVTX ranges around the library's calls and launches, and optional
// per-kernel CUDA-event timing.  Off by default; when enabled
// (crt_profile_enable), each major kernel launch is bracketed by an event pair
// on its own stream and crt_profile_collect sums the durations by name.  Used
// by the benchmark to time the dominant kernel inside its timed region.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace crt {

bool profiling();
// Records the start event of a launch named `name` on `stream` (no-op when
// profiling is off or the stream is capturing); returns a token for stop.
int prof_start(const char* name, cudaStream_t stream);
void prof_stop(int token, cudaStream_t stream);
// Adds an already measured duration (graph replays time themselves).
void prof_add(const char* name, double ms);
// Creates an event pair counted under `name` for a launch that records the
// events itself (the event-record nodes of a CUDA graph); false when
// profiling is off.  The pair is read and destroyed by crt_profile_collect.
bool prof_register(const char* name, cudaEvent_t* a, cudaEvent_t* b);

// Brackets one launch: an NVTX range on the host thread (seen by Nsight and
// other NVTX tools; a no-op without one attached) and, when kernel timing is
// on, an event pair on the launching stream.
struct ProfScope {
  int tok;
  cudaStream_t s;
  ProfScope(const char* name, cudaStream_t stream) : tok(prof_start(name, stream)), s(stream)
  {
    nvtxRangePushA(name);
  }
  ~ProfScope()
  {
    prof_stop(tok, s);
    nvtxRangePop();
  }
};

// An NVTX range over a whole library call (build, query, ingest).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

}  // namespace crt
