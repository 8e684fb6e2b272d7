// Minimal stand-in for rmm::exec_policy: a Thrust CUDA policy on the stream.
// Build-time shim for the reference runner only.
#pragma once
#include <thrust/execution_policy.h>
#include <thrust/system/cuda/execution_policy.h>
#include "cuda_stream_view.hpp"

namespace rmm {
inline auto exec_policy(cuda_stream_view s = cuda_stream_view{}) { return thrust::cuda::par.on(s.value()); }
}  // namespace rmm
