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
  __shared__ uint32_t sh[4][kBins];
  for (int i = threadIdx.x; i < 4 * kBins; i += blockDim.x) (&sh[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)key_src[i] ^ 0x80000000u;
    keys[i] = k;
    vals[i] = (uint32_t)val_src[i];
    atomicAdd(&sh[0][k & 0xFF], 1u);
    atomicAdd(&sh[1][(k >> 8) & 0xFF], 1u);
    atomicAdd(&sh[2][(k >> 16) & 0xFF], 1u);
    atomicAdd(&sh[3][k >> 24], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * kBins; i += blockDim.x) {
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

}  // namespace crt
