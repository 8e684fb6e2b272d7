// Canonical pair order on the GPU: (window, box id) ascending, the order the
// reference's drivers produce on the host with two stable sorts, first by box
// id and then by window (src/rtree_test_frontier.cu:102-105).  Two stable
// radix sorts do the same here: by box id carrying the window, then by window
// carrying the box id.  Both keys are compared as signed ints, as the
// reference's int ids are.
#include <cuda_runtime.h>

#include "internal.h"

namespace crt {

// keys = key_src ^ 0x80000000 (signed order as unsigned), vals = val_src, and
// the four digit histograms of the keys.
__global__ void canon_stage_kernel(const int32_t* __restrict__ key_src,
                                   const int32_t* __restrict__ val_src, int64_t n,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                   uint32_t* __restrict__ hist)
{
  __shared__ uint32_t sh[kDigits][kBins];
  for (int i = threadIdx.x; i < kDigits * kBins; i += blockDim.x) (&sh[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)key_src[i] ^ 0x80000000u;
    keys[i] = k;
    vals[i] = (uint32_t)val_src[i];
#pragma unroll
    for (int d = 0; d < kDigits; d++) atomicAdd(&sh[d][key_digit(k, d)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDigits * kBins; i += blockDim.x) {
    const uint32_t v = (&sh[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

// Writes the sorted (key, value) pairs back: key_dst = key ^ 0x80000000,
// val_dst = value, from the buffers the passes left them in.
__global__ void canon_unstage_kernel(SortBufs bufs, const SortCtrl* __restrict__ ctrl, int64_t n,
                                     int32_t* __restrict__ key_dst, int32_t* __restrict__ val_dst)
{
  const int p = ctrl->n_active & 1;
  const uint32_t* __restrict__ keys = bufs.keys[p];
  const uint32_t* __restrict__ vals = bufs.vals[p];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    key_dst[i] = (int32_t)(keys[i] ^ 0x80000000u);
    val_dst[i] = (int32_t)vals[i];
  }
}

int pairs_canonicalize(int32_t* fid, int32_t* tid, int64_t n, cudaStream_t stream)
{
  if (n < 0 || (n > 0 && (!fid || !tid))) return fail(CRT_ERR_INVALID_ARG, "canonicalize: bad arguments");
  if (n <= 1) return CRT_OK;
  if (n > INT32_MAX)
    return fail(CRT_ERR_NOT_SUPPORTED, "canonicalize: at most INT32_MAX pairs per call");
  const size_t zero = (sort_zero_bytes(n) + 255) / 256 * 256;
  const size_t kv = ((size_t)n * 4 + 255) / 256 * 256;
  char* scr = nullptr;
  if (cudaMallocAsync((void**)&scr, zero + 4 * kv, stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(CRT_ERR_OOM, "canonicalize: scratch allocation failed");
  }
  SortBufs bufs;
  bufs.keys[0] = (uint32_t*)(scr + zero);
  bufs.keys[1] = (uint32_t*)(scr + zero + kv);
  bufs.vals[0] = (uint32_t*)(scr + zero + 2 * kv);
  bufs.vals[1] = (uint32_t*)(scr + zero + 3 * kv);
  const int grid = (int)std::min<int64_t>(cdiv(n, 256), (int64_t)sm_count() * 8);
  // by box id (carrying the window), then stably by window (carrying the box id)
  for (int round = 0; round < 2; round++) {
    int32_t* key_src = round == 0 ? fid : tid;
    int32_t* val_src = round == 0 ? tid : fid;
    cudaMemsetAsync(scr, 0, sort_zero_bytes(n), stream);
    canon_stage_kernel<<<grid, 256, 0, stream>>>(key_src, val_src, n, bufs.keys[0], bufs.vals[0],
                                                 sort_hist(scr));
    sort_passes(bufs, n, scr, stream, kSortGivenValues | kSortKeepKeys);
    canon_unstage_kernel<<<grid, 256, 0, stream>>>(bufs, sort_ctrl(scr), n, key_src, val_src);
    CRT_LAUNCHED(2);
  }
  int dev_err = 0;
  cudaMemcpyAsync(&dev_err, &sort_ctrl(scr)->error, sizeof(int), cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(scr, stream);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "canonicalize");
  if (dev_err) return fail(dev_err, "canonicalize: device-side wait timed out in the radix sort");
  return CRT_OK;
}

// ---------------------------------------------------------------------------
// Per-window counts and order-independent digests of a pair list.  The
// reference's drivers check a result by sorting both pair vectors and
// comparing them (src/rtree_test_frontier.cu:102-123); at billions of pairs
// the same check is a per-window count plus a per-window sum (mod 2^64) of a
// 64-bit mix of each (window, box id) pair, which any pair order gives alike.
// The mix is the splitmix64 finaliser (Steele, Lea and Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long pair_mix(unsigned long long z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

constexpr int kDigestRun = 64;  // consecutive pairs per thread

// Each thread sums the pairs of its run window by window and adds each
// window's count and digest with one pair of atomics; when every lane of a
// warp saw one window only (the long runs of a batch query's output), the
// warp adds once.  Pairs are read through L2 only (ld.global.cg): they may
// come from a kernel still running on another stream, such as the serving
// loop, whose completed requests this checks.
__global__ void __launch_bounds__(256)
    digest_kernel(const int32_t* __restrict__ fid, const int32_t* __restrict__ tid, int64_t n,
                  int64_t base, int64_t nq, unsigned long long* __restrict__ counts,
                  unsigned long long* __restrict__ hashes, unsigned long long* __restrict__ bad)
{
  const int64_t nruns = (n + kDigestRun - 1) / kDigestRun;
  for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x; r0 < nruns;
       r0 += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = r0 + threadIdx.x;
    const int64_t i0 = r * kDigestRun;
    const int64_t i1 = min(n, i0 + kDigestRun);
    long long cur = -1;  // window of the open segment
    unsigned long long c = 0, h = 0, nbad = 0;
    bool single = true;  // the whole run is one window
    for (int64_t i = i0; i < i1; i++) {
      const long long w = (long long)__ldcg(tid + i) + base;
      if (w < 0 || w >= nq) {
        nbad++;
        single = false;
        continue;
      }
      if (w != cur) {
        if (cur >= 0) {
          atomicAdd(&counts[cur], c);
          atomicAdd(&hashes[cur], h);
          single = false;
        }
        cur = w;
        c = 0;
        h = 0;
      }
      c++;
      h += pair_mix(((unsigned long long)(uint32_t)w << 32) | (uint32_t)__ldcg(fid + i));
    }
    // warp aggregation: all lanes hold one segment of the same window
    const long long w0 = __shfl_sync(0xffffffffu, cur, 0);
    const bool same = __all_sync(0xffffffffu, single && cur == w0 && cur >= 0);
    if (same) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        h += __shfl_down_sync(0xffffffffu, h, o);
      }
      if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counts[w0], c);
        atomicAdd(&hashes[w0], h);
      }
    } else if (cur >= 0) {
      atomicAdd(&counts[cur], c);
      atomicAdd(&hashes[cur], h);
    }
    if (nbad && bad) atomicAdd(bad, nbad);
  }
}

int pairs_digest(const int32_t* fid, const int32_t* tid, int64_t n, int64_t window_base,
                 int64_t nq, int64_t* d_counts, uint64_t* d_hashes, int64_t* d_bad,
                 cudaStream_t stream)
{
  if (n < 0 || nq < 0 || (n > 0 && (!fid || !tid)) || (nq > 0 && (!d_counts || !d_hashes)))
    return fail(CRT_ERR_INVALID_ARG, "pairs_digest: bad arguments");
  if (n == 0) return CRT_OK;
  const int64_t nruns = cdiv(n, kDigestRun);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(nruns, 256), (int64_t)sm_count() * 8));
  digest_kernel<<<grid, 256, 0, stream>>>(fid, tid, n, window_base, nq,
                                          (unsigned long long*)d_counts,
                                          (unsigned long long*)d_hashes,
                                          (unsigned long long*)d_bad);
  CRT_LAUNCHED(1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "pairs_digest");
  return CRT_OK;
}

}  // namespace crt
