// Minimal stand-in for rmm::cuda_stream_view, enough for the reference's
// src/rtree_bfs_thrust.cuh to compile.  Build-time shim for the reference
// runner only (oracle/ref_gpu_thrust.cu); never part of the product library.
#pragma once
#include <cuda_runtime.h>

namespace rmm {
class cuda_stream_view {
 public:
  constexpr cuda_stream_view() = default;
  constexpr cuda_stream_view(cudaStream_t s) : s_(s) {}
  constexpr cudaStream_t value() const { return s_; }
  constexpr operator cudaStream_t() const { return s_; }

 private:
  cudaStream_t s_{nullptr};
};
static constexpr cuda_stream_view cuda_stream_default{};
}  // namespace rmm
