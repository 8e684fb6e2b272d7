// Shared device helpers of the crtree library: the reference's key and
// intersection arithmetic, warp utilities, bounded waits, error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "../../include/crtree.h"

namespace crt {

// ---------------------------------------------------------------------------
// Host-side error plumbing
// ---------------------------------------------------------------------------
void set_last_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
extern std::atomic<uint64_t> g_launches;

#define CRT_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return crt::cuda_fail(e_, #call); \
  } while (0)

#define CRT_LAUNCHED(k) (crt::g_launches.fetch_add((k), std::memory_order_relaxed))

inline int sm_count()
{
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// Reference arithmetic
// ---------------------------------------------------------------------------

// The reference's intersect (src/rtree_bfs_frontier.cuh:40-44,
// src/rtree_bfs_thrust.cuh:44-47, src/utility.h:16-20): closed intervals, and
// a NaN never excludes.  Argument order: window first, then box.
__device__ __forceinline__ bool intersects(float x1, float y1, float x2, float y2, float m1,
                                           float n1, float m2, float n2)
{
  return !(x1 > m2 || x2 < m1 || y1 > n2 || y2 < n1);
}

// Spread 16 bits over the even positions of a 32-bit word: the value of the
// reference's dilation-table lookup pair (src/z_order.cuh:63-65), computed
// with shifts and masks instead of a table.
__device__ __forceinline__ uint32_t dilate16(uint32_t x)
{
  x &= 0xFFFFu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// The reference's `(ushort)` cast of an fp32 centre
// (src/rtree_bulkload_thrust.cuh:55-56) as its device build performs it:
// truncate toward zero to an unsigned 32-bit integer (negative and NaN -> 0,
// >= 2^32 -> 2^32 - 1), then keep the low 16 bits.  Pinned against the
// reference's own build on centres outside [0, 65536).
__device__ __forceinline__ uint32_t f2u16(float v) { return __float2uint_rz(v) & 0xFFFFu; }

// mbr2key (src/rtree_bulkload_thrust.cuh:52-60) with bit 31 flipped, so that
// the reference's signed-int key order (src/rtree_bulkload_thrust.cuh:72,
// 83-86) becomes unsigned order for the radix sort.
__device__ __forceinline__ uint32_t sort_key(float xmin, float ymin, float xmax, float ymax)
{
  float cx = (xmin + xmax) / 2;
  float cy = (ymin + ymax) / 2;
  uint32_t z = (dilate16(f2u16(cy)) << 1) | dilate16(f2u16(cx));
  return z ^ 0x80000000u;
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt()
{
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p)
{
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v)
{
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_i32(const int* p)
{
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_ull(const unsigned long long* p)
{
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Upper bound on polls of any device-side wait before it gives up, records
// CRT_ERR_DEVICE_TIMEOUT and returns (about a second with the back-off).
constexpr uint32_t kSpinLimit = 1u << 22;

// Device error word: the first error raised wins.
__device__ __forceinline__ void raise_error(int* err, int code)
{
  if (err) atomicCAS(err, 0, code);
}

}  // namespace crt
