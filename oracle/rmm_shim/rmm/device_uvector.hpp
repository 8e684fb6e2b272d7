// Minimal stand-in for rmm::device_uvector backed by the stream-ordered CUDA
// allocator (cudaMallocAsync), which caches freed blocks the way the RMM pool
// of the reference's Thrust driver does (src/rtree_test_thrust.cu:48-61).
// Build-time shim for the reference runner only.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include "cuda_stream_view.hpp"

namespace rmm {
template <typename T>
class device_uvector {
 public:
  device_uvector(std::size_t n, cuda_stream_view s) : n_(n), s_(s)
  {
    if (n_ && cudaMallocAsync((void**)&p_, n_ * sizeof(T), s_.value()) != cudaSuccess) {
      std::fprintf(stderr, "rmm shim: cudaMallocAsync of %zu bytes failed\n", n_ * sizeof(T));
      std::exit(3);
    }
  }
  device_uvector(device_uvector&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; }
  device_uvector& operator=(device_uvector&& o) noexcept
  {
    if (this != &o) {
      release();
      p_ = o.p_; n_ = o.n_; s_ = o.s_;
      o.p_ = nullptr; o.n_ = 0;
    }
    return *this;
  }
  device_uvector(device_uvector const&)            = delete;
  device_uvector& operator=(device_uvector const&) = delete;
  ~device_uvector() { release(); }

  T* begin() { return p_; }
  T* end() { return p_ + n_; }
  T const* begin() const { return p_; }
  T const* end() const { return p_ + n_; }
  T* data() { return p_; }
  std::size_t size() const { return n_; }

  T back_element(cuda_stream_view s) const
  {
    T v{};
    cudaMemcpyAsync(&v, p_ + n_ - 1, sizeof(T), cudaMemcpyDeviceToHost, s.value());
    cudaStreamSynchronize(s.value());
    return v;
  }
  void set_element_to_zero_async(std::size_t i, cuda_stream_view s)
  {
    cudaMemsetAsync(p_ + i, 0, sizeof(T), s.value());
  }

 private:
  void release()
  {
    if (p_) cudaFreeAsync(p_, s_.value());
    p_ = nullptr;
    n_ = 0;
  }
  T* p_{nullptr};
  std::size_t n_{0};
  cuda_stream_view s_{};
};
}  // namespace rmm
