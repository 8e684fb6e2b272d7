// Z-order bulk load (replaces build_rtree, src/rtree_bulkload_thrust.cuh:62-213).
//
// Pipeline, all on one stream, no host synchronisation until the end:
//   1. encode      read the box SoA (float4 loads where aligned), write the
//                  flipped 32-bit Morton key and the slot of a 32-byte AoS
//                  record of each box (records of a 4096-box tile grouped by
//                  the key's top digit), and count all four 8-bit key digits.
//   2. plan        one CTA: which digit passes are non-uniform (a uniform digit
//                  leaves a stable order unchanged, so its pass is skipped) and
//                  the global bucket start of every digit value.
//   3. 4 x onesweep  stable LSD radix passes over (key, slot) with decoupled
//                  look-back across tiles: one read and one write of the pairs
//                  per pass.  The first active pass reads the encoder's slots,
//                  the last one writes only slots.
//   4. leaf level  gather each sorted box's record (runs of one top digit per
//                  tile, so lines are shared by neighbouring records), write the permuted
//                  SoA, and reduce every run of `fanout` boxes into its
//                  leaf-parent node.
//   5. upper levels  reduce runs of `fanout` nodes, level by level up to the root.
// Node order, pos and len follow the reference exactly (root at 0, levels
// downward, children contiguous, leaf-parent pos = R_sz + first slot).
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "internal.h"
#include "profile.h"

namespace crt {

struct alignas(32) Box32 {
  float4 mbr;  // xmin, ymin, xmax, ymax
  int4 idp;    // id, 0, 0, 0
};

constexpr int kSortThreads = 512;
constexpr int kSortIpt = kSortTile / kSortThreads;  // 16 keys per thread
constexpr int kSortWarps = kSortThreads / 32;
using BuildCtrl = SortCtrl;

constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagIncl = 2ull << 62;

// ---------------------------------------------------------------------------
// 1. encode
// ---------------------------------------------------------------------------
// Each CTA takes tiles of kEncTile boxes.  Per box it writes the key and, in
// input order, the slot of the box's 32-byte record; the records of a tile
// are placed in its own slot range grouped by the key's top digit.  The sort
// then carries those slots (its first pass reads them instead of making
// input indices), and the leaf level's gather in sorted order, which walks
// one top digit at a time, reads each tile's run for that digit (about
// kEncTile / 256 records, often several whole 128-byte lines) instead of
// single records scattered over the whole copy.  Order inside a run does not
// matter: ties in the sort keep input order because the (key, slot) pairs
// start in input order.
constexpr int kEncThreads = 256;
constexpr int kEncGroups = 4;                            // float4 groups per thread
constexpr int kEncTile = 4 * kEncGroups * kEncThreads;   // 4096 boxes
constexpr int kGroups = 256;                             // record runs: by the key's top byte
static_assert(kDigits * kDigitBits - kDigitBits >= 24, "the last digit lies in the top byte");
static_assert(kGroups <= kEncThreads, "one thread per run");

struct BoxIn {
  const float* __restrict__ xmin;
  const float* __restrict__ ymin;
  const float* __restrict__ xmax;
  const float* __restrict__ ymax;
  const int* __restrict__ id;
};

// Loads boxes j..j+3 (those below n); kVec: the arrays are 16-byte aligned.
template <bool kVec>
__device__ __forceinline__ void load4(const BoxIn& in, int64_t j, int64_t n, float4& a, float4& b,
                                      float4& c, float4& d, int4& e)
{
  if (kVec && j + 3 < n) {
    a = reinterpret_cast<const float4*>(in.xmin)[j >> 2];
    b = reinterpret_cast<const float4*>(in.ymin)[j >> 2];
    c = reinterpret_cast<const float4*>(in.xmax)[j >> 2];
    d = reinterpret_cast<const float4*>(in.ymax)[j >> 2];
    e = reinterpret_cast<const int4*>(in.id)[j >> 2];
    return;
  }
  float* pa = &a.x;
  float* pb = &b.x;
  float* pc = &c.x;
  float* pd = &d.x;
  int* pe = &e.x;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const bool v = j + k < n;
    pa[k] = v ? in.xmin[j + k] : 0.f;
    pb[k] = v ? in.ymin[j + k] : 0.f;
    pc[k] = v ? in.xmax[j + k] : 0.f;
    pd[k] = v ? in.ymax[j + k] : 0.f;
    pe[k] = v ? in.id[j + k] : 0;
  }
}

template <bool kVec>
__global__ void __launch_bounds__(kEncThreads) encode_kernel(BoxIn in, int64_t n,
                                                             uint32_t* __restrict__ keys,
                                                             uint32_t* __restrict__ slots,
                                                             Box32* __restrict__ aos,
                                                             uint32_t* __restrict__ hist)
{
  // digit histograms over all of this CTA's tiles (the last digit lies in
  // the top byte: it is added from the tile's top-byte counts)
  __shared__ uint32_t sh[kDigits][kBins];
  __shared__ uint32_t s_run[kGroups];  // this tile: count, then run start, per top byte
  __shared__ uint32_t s_wsum[kGroups / 32];
  __shared__ uint32_t s_dr[kEncTile];  // per box of the tile: top byte << 16 | rank in its run
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kDigits * kBins; i += kEncThreads) (&sh[0][0])[i] = 0;
  const int64_t ntiles = (n + kEncTile - 1) / kEncTile;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    if (tid < kGroups) s_run[tid] = 0;
    __syncthreads();
    const int64_t base = t * kEncTile;
#pragma unroll
    for (int g = 0; g < kEncGroups; g++) {
      const int i0 = 4 * (tid + g * kEncThreads);  // first box of the group in the tile
      const int64_t j = base + i0;
      float4 a, b, c, d;
      int4 e;
      load4<kVec>(in, j, n, a, b, c, d, e);
      const float* pa = &a.x;
      const float* pb = &b.x;
      const float* pc = &c.x;
      const float* pd = &d.x;
      uint32_t kk[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        kk[k] = sort_key(pa[k], pb[k], pc[k], pd[k]);
        if (j + k < n) {
          const uint32_t top = kk[k] >> 24;
          s_dr[i0 + k] = top << 16 | atomicAdd(&s_run[top], 1u);
#pragma unroll
          for (int dg = 0; dg < kDigits - 1; dg++) atomicAdd(&sh[dg][key_digit(kk[k], dg)], 1u);
        }
      }
      if (j + 3 < n) {
        *reinterpret_cast<uint4*>(keys + j) = make_uint4(kk[0], kk[1], kk[2], kk[3]);
      } else {
        for (int k = 0; k < 4; k++)
          if (j + k < n) keys[j + k] = kk[k];
      }
    }
    __syncthreads();
    // run starts: exclusive prefix of the tile's top-byte counts
    uint32_t cnt = 0, x = 0;
    if (tid < kGroups) {
      cnt = s_run[tid];
      if (cnt) atomicAdd(&sh[kDigits - 1][key_digit((uint32_t)tid << 24, kDigits - 1)], cnt);
      x = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) s_wsum[warp] = x;
    }
    __syncthreads();
    if (tid < kGroups) {
      uint32_t start = x - cnt;
      for (int w = 0; w < warp; w++) start += s_wsum[w];
      s_run[tid] = start;
    }
    __syncthreads();
    // records into their runs; slots in input order
#pragma unroll
    for (int g = 0; g < kEncGroups; g++) {
      const int i0 = 4 * (tid + g * kEncThreads);
      const int64_t j = base + i0;
      float4 a, b, c, d;
      int4 e;
      load4<kVec>(in, j, n, a, b, c, d, e);  // second read of the tile: from L2
      const float* pa = &a.x;
      const float* pb = &b.x;
      const float* pc = &c.x;
      const float* pd = &d.x;
      const int* pe = &e.x;
      uint32_t sl[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint32_t dr = j + k < n ? s_dr[i0 + k] : 0u;
        sl[k] = (uint32_t)base + s_run[dr >> 16] + (dr & 0xFFFFu);
        if (j + k < n) {
          Box32 bx;
          bx.mbr = make_float4(pa[k], pb[k], pc[k], pd[k]);
          bx.idp = make_int4(pe[k], 0, 0, 0);
          aos[sl[k]] = bx;
        }
      }
      if (j + 3 < n) {
        *reinterpret_cast<uint4*>(slots + j) = make_uint4(sl[0], sl[1], sl[2], sl[3]);
      } else {
        for (int k = 0; k < 4; k++)
          if (j + k < n) slots[j + k] = sl[k];
      }
    }
    __syncthreads();
  }
  for (int i = tid; i < kDigits * kBins; i += kEncThreads) {
    const uint32_t v = (&sh[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

// ---------------------------------------------------------------------------
// 2. plan
// ---------------------------------------------------------------------------
// One warp per digit: a digit whose histogram has one bin holding every key
// is uniform and its pass is skipped (a stable pass over a uniform digit
// leaves the order unchanged); the exclusive prefix of the bins is each
// bucket's global start.
__global__ void plan_kernel(const uint32_t* __restrict__ hist, int64_t n, BuildCtrl* ctrl)
{
  __shared__ int s_uniform[kDigits];
  if (threadIdx.x < kDigits) s_uniform[threadIdx.x] = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (w < kDigits) {
    const int nb = 1 << digit_bits(w);
    uint32_t carry = 0;
    for (int c = 0; c < nb; c += 32) {
      const bool in = c + l < nb;
      const uint32_t v = in ? hist[w * kBins + c + l] : 0u;
      if (in && (int64_t)v == n) s_uniform[w] = 1;
      uint32_t x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (l >= o) x += y;
      }
      if (in) ctrl->bucket_start[w * kBins + c + l] = (int)(carry + x - v);
      carry += __shfl_sync(0xffffffffu, x, 31);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int act = 0, na = 0;
    for (int d = 0; d < kDigits; d++)
      if (!s_uniform[d]) { act |= 1 << d; na++; }
    ctrl->active = act;
    ctrl->n_active = na;
  }
}

// ---------------------------------------------------------------------------
// 3. onesweep pass
// ---------------------------------------------------------------------------
// Lanes of the warp whose value equals this lane's (v < 2^kBits), from one
// ballot per bit; on this part it issues faster than __match_any_sync
// (measured over the four 8-bit passes of a 100M-key build: 3.7 ms against
// 4.3 ms).
template <int kBits>
__device__ __forceinline__ uint32_t peer_mask(uint32_t v)
{
  uint32_t peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < kBits; b++) {
    const bool bit = (v >> b) & 1u;
    const uint32_t bal = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? bal : ~bal;
  }
  return peers;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared memory of one pass over a kBits-bit digit: keys and values staged in
// destination order, the tile's incoming values prefetched while the tile is
// ranked (narrow digits only: with 1024 bins the per-warp counters take that
// room, and the values are copied straight to their staged slots instead),
// the per-warp digit counters (16-bit: at most 8192 per tile), the bins'
// global offsets and the warp sums of the bin scan.
template <int kBits>
struct SweepSmem {
  static constexpr int kB = 1 << kBits;
  static constexpr bool kPrefetch = kBits <= 8;
  static constexpr size_t kKeys = 0;
  static constexpr size_t kVals = kKeys + 4 * (size_t)kSortTile;
  static constexpr size_t kVin = kVals + 4 * (size_t)kSortTile;
  static constexpr size_t kHist = kVin + (kPrefetch ? 4 * (size_t)kSortTile : 0);
  static constexpr size_t kGbase = kHist + 2 * (size_t)kSortWarps * (kB < 2 ? 2 : kB);
  static constexpr size_t kWsum = kGbase + 4 * (size_t)kB;
  static constexpr size_t kBytes = kWsum + 4 * 32;
};
static_assert(2 * (SweepSmem<10>::kBytes + 1024) <= 227 * 1024, "two 10-bit CTAs per SM");
static_assert(2 * (SweepSmem<8>::kBytes + 1024) <= 227 * 1024, "two 8-bit CTAs per SM");

// Ranks this thread's keys inside its warp, stably (rounds in order, lanes in
// order).  kFull: every item of the tile is valid (no bounds checks, and the
// digit fits kBits bits); otherwise invalid items take digit 2^kBits.
template <bool kFull, int kBits>
__device__ __forceinline__ void rank_keys(const uint32_t (&key)[kSortIpt], uint32_t (&rank)[kSortIpt],
                                          uint16_t* wh, int wbase, int tile_n, int shift)
{
  constexpr uint32_t kMask = (1u << kBits) - 1u;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kSortIpt; i++) {
    const bool v = kFull || wbase + 32 * i < tile_n;
    const uint32_t dig = v ? (key[i] >> shift) & kMask : kMask + 1u;
    const uint32_t peers = kFull ? peer_mask<kBits>(dig) : peer_mask<kBits + 1>(dig);
    const uint32_t old = v ? wh[dig] : 0u;
    __syncwarp();
    if (v && (peers & lt) == 0) wh[dig] = (uint16_t)(old + __popc(peers));
    __syncwarp();
    rank[i] = old + __popc(peers & lt);
  }
}

// One stable LSD pass over (key, value) pairs for the kBits-bit digit at
// `digit` (bits digit * kDigitBits ...), with decoupled look-back across
// tiles.  Indices are 32-bit: the key count is below 2^31 (the C ABI's int
// sizes).
template <int kBits>
__global__ void __launch_bounds__(kSortThreads, 2)
    onesweep_kernel(int digit, SortBufs bufs, int64_t n64, uint64_t* __restrict__ status,
                    BuildCtrl* __restrict__ ctrl, int flags)
{
  using L = SweepSmem<kBits>;
  constexpr int kB = L::kB;
  constexpr uint32_t kMask = (uint32_t)kB - 1u;
  constexpr int kBPT = (kB + kSortThreads - 1) / kSortThreads;  // bins per thread
  extern __shared__ __align__(16) unsigned char sweep_smem[];
  uint32_t* s_key = (uint32_t*)(sweep_smem + L::kKeys);
  uint32_t* s_val = (uint32_t*)(sweep_smem + L::kVals);
  uint32_t* s_vin = (uint32_t*)(sweep_smem + L::kVin);
  uint16_t* s_whist = (uint16_t*)(sweep_smem + L::kHist);
  int* s_gbase = (int*)(sweep_smem + L::kGbase);
  int* s_wsum = (int*)(sweep_smem + L::kWsum);
  __shared__ int s_tile;

  const int active = ctrl->active;
  if (!((active >> digit) & 1)) return;
  const int before = active & ((1 << digit) - 1);
  const int parity = __popc(before) & 1;
  const bool first = before == 0 && !(flags & kSortGivenValues);
  const bool last = (active >> (digit + 1)) == 0 && !(flags & kSortKeepKeys);
  const int shift = digit * kDigitBits;
  const int n = (int)n64;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(&ctrl->tile_ctr[digit], 1);
  for (int i = tid; i < kSortWarps * kB / 2; i += kSortThreads) ((uint32_t*)s_whist)[i] = 0;
  if (kB < 2 && tid < kSortWarps) s_whist[tid] = 0;
  __syncthreads();
  const int tile = s_tile;
  const int base = tile * kSortTile;
  const int tile_n = min(kSortTile, n - base);
  const uint32_t* __restrict__ src_k = bufs.keys[parity] + base;
  const uint32_t* __restrict__ src_v = bufs.vals[parity] + base;
  uint32_t* __restrict__ dst_k = bufs.keys[parity ^ 1];
  uint32_t* __restrict__ dst_v = bufs.vals[parity ^ 1];
  const int wbase = warp * 32 * kSortIpt + lane;  // this lane's first item in the tile

  // the tile's incoming values land in shared memory while the keys are
  // ranked (16-byte async copies; the tile start is 32 KiB-aligned)
  if (L::kPrefetch && !first) {
#pragma unroll
    for (int c = tid; c < kSortTile / 4; c += kSortThreads) {
      const int left = tile_n - 4 * c;
      if (left > 0) {
        const int bytes = min(left, 4) * 4;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(s_vin + 4 * c)),
                     "l"(src_v + 4 * c), "r"(bytes)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }

  // load keys (warp-striped: item i of a lane is wbase + 32 i)
  uint32_t key[kSortIpt];
  uint32_t rank[kSortIpt];
  uint16_t* wh = s_whist + warp * kB;
  if (tile_n == kSortTile) {
#pragma unroll
    for (int i = 0; i < kSortIpt; i++) key[i] = src_k[wbase + 32 * i];
    rank_keys<true, kBits>(key, rank, wh, wbase, tile_n, shift);
  } else {
#pragma unroll
    for (int i = 0; i < kSortIpt; i++) {
      const int j = wbase + 32 * i;
      key[i] = j < tile_n ? src_k[j] : 0u;
    }
    rank_keys<false, kBits>(key, rank, wh, wbase, tile_n, shift);
  }
  __syncthreads();
  // per owned bin: exclusive prefix over warps and the tile count
  int cnt[kBPT];
  int tsum = 0;
#pragma unroll
  for (int j = 0; j < kBPT; j++) {
    const int b = tid * kBPT + j;
    int run = 0;
    if (b < kB) {
#pragma unroll
      for (int w = 0; w < kSortWarps; w++) {
        const int c = (int)s_whist[w * kB + b];
        s_whist[w * kB + b] = (uint16_t)run;
        run += c;
      }
    }
    cnt[j] = run;
    tsum += run;
  }
  // exclusive scan of the per-thread bin sums over the CTA (bins in order)
  int x = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_wsum[warp] = x;
  // publish this tile's aggregate of every owned bin before waiting on
  // predecessors (tile 0 publishes its inclusive count at once)
#pragma unroll
  for (int j = 0; j < kBPT; j++) {
    const int b = tid * kBPT + j;
    if (b < kB)
      st_relaxed_u64(&status[(int64_t)tile * kB + b],
                     (tile == 0 ? kFlagIncl : kFlagAgg) | (uint32_t)cnt[j]);
  }
  __syncthreads();
  int binstart = x - tsum;
  for (int w = 0; w < warp; w++) binstart += s_wsum[w];
#pragma unroll
  for (int j = 0; j < kBPT; j++) {
    const int b = tid * kBPT + j;
    if (b < kB) {
      // fold the bin start into every warp's offset: one lookup per key later
#pragma unroll
      for (int w = 0; w < kSortWarps; w++)
        s_whist[w * kB + b] = (uint16_t)(s_whist[w * kB + b] + binstart);
      // decoupled look-back for bin b
      int excl = 0;
      if (tile > 0) {
        int t = tile - 1;
        uint32_t spins = 0;
        while (true) {
          const uint64_t v = ld_relaxed_u64(&status[(int64_t)t * kB + b]);
          const uint64_t flag = v & (3ull << 62);
          if (flag == 0) {
            if (++spins > kSpinLimit || ld_relaxed_i32(&ctrl->error) != 0) {
              raise_error(&ctrl->error, CRT_ERR_DEVICE_TIMEOUT);
              break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
          }
          excl += (int)(uint32_t)v;
          if (flag == kFlagIncl) break;
          --t;
        }
        st_relaxed_u64(&status[(int64_t)tile * kB + b], kFlagIncl | (uint32_t)(excl + cnt[j]));
      }
      s_gbase[b] = ctrl->bucket_start[digit * kBins + b] + excl - binstart;
    }
    binstart += cnt[j];
  }
  if (L::kPrefetch && !first) asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();

  // stage (key, value) pairs in the order of their destination
#pragma unroll
  for (int i = 0; i < kSortIpt; i++) {
    const int j = wbase + 32 * i;
    const int pos = (int)(wh[(key[i] >> shift) & kMask] + rank[i]);
    if (j < tile_n && (unsigned)pos < (unsigned)kSortTile) {  // pos < tile_n by construction
      s_key[pos] = key[i];
      if (first) {
        s_val[pos] = (uint32_t)(base + j);
      } else if (L::kPrefetch) {
        s_val[pos] = s_vin[j];
      } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(s_val + pos)),
                     "l"(src_v + j)
                     : "memory");
      }
    }
  }
  if (!L::kPrefetch && !first) {
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_all;" ::: "memory");
  }
  __syncthreads();
  for (int j = tid; j < tile_n; j += kSortThreads) {
    const uint32_t k = s_key[j];
    const int dst = s_gbase[(k >> shift) & kMask] + j;
    if ((uint32_t)dst < (uint32_t)n) {
      // evict-first: a pass's output is read once, by the next pass, and
      // the look-back status words and the next tiles' runs want L2
      if (!last) __stcs(dst_k + dst, k);
      __stcs(dst_v + dst, s_val[j]);
    }
  }
}

// ---------------------------------------------------------------------------
// 4./5. level reductions
// ---------------------------------------------------------------------------
constexpr int kLevelThreads = 256;
constexpr int kLevelChunk = 2048;  // children staged per round

// Reduces runs of `fanout` consecutive children into parent nodes
// (reduce_op, src/rtree_bulkload_thrust.cuh:38-50: min, min, max, max of the
// MBR, first child index, child count).  kLeaf: children are the sorted boxes,
// gathered from the AoS copy through the sorted slot order, and the permuted
// SoA is written on the way; otherwise children are nodes at child_start.
template <bool kLeaf>
__global__ void __launch_bounds__(kLevelThreads, 3)  // 80 registers: three CTAs per SM
    level_kernel(int nodes_per_cta, int fanout, int64_t nchild, int64_t nparent,
                 int64_t parent_start, int64_t pos_base,
                 // leaf inputs/outputs
                 const uint32_t* __restrict__ vals0, const uint32_t* __restrict__ vals1,
                 const BuildCtrl* __restrict__ ctrl, const Box32* __restrict__ aos,
                 float* __restrict__ oxmin, float* __restrict__ oymin,
                 float* __restrict__ oxmax, float* __restrict__ oymax, int* __restrict__ oid,
                 // node arrays
                 float* __restrict__ nxmin, float* __restrict__ nymin,
                 float* __restrict__ nxmax, float* __restrict__ nymax, int* __restrict__ npos,
                 int* __restrict__ nlen, int64_t child_start)
{
  __shared__ float4 s_mbr[kLevelChunk];
  const int64_t p0 = (int64_t)blockIdx.x * nodes_per_cta;
  const int64_t p1 = min(nparent, p0 + nodes_per_cta);
  if (p0 >= p1) return;
  const int64_t c0 = p0 * fanout;
  const int64_t c1 = min(nchild, p1 * fanout);
  const uint32_t* sorted = nullptr;
  if (kLeaf) {
    // record slots in sorted order (the encoder's slots when no pass ran)
    int na = ctrl->n_active;
    sorted = (na & 1) ? vals1 : vals0;
  }
  // this thread's parent (if any) and its child range
  const int64_t my = p0 + threadIdx.x;
  const bool have = my < p1;
  const int64_t my_c0 = my * fanout;
  const int64_t my_c1 = min(nchild, my_c0 + fanout);
  float a = 0.f, b = 0.f, c = 0.f, d = 0.f;
  bool init = false;
  for (int64_t cb = c0; cb < c1; cb += kLevelChunk) {
    const int64_t ce = min(c1, cb + (int64_t)kLevelChunk);
    if (kLeaf) {
      // all slot loads, then all 32-byte record loads, then the stores: each
      // thread keeps kGather record reads in flight
      constexpr int kGather = kLevelChunk / kLevelThreads;
      uint32_t src[kGather];
#pragma unroll
      for (int u = 0; u < kGather; u++) {
        const int64_t s = cb + threadIdx.x + u * kLevelThreads;
        src[u] = s < ce ? sorted[s] : 0u;
        if ((int64_t)src[u] >= nchild) src[u] = s < ce ? (uint32_t)s : 0u;  // only after a sort error (reported)
      }
      Box32 bx[kGather];
#pragma unroll
      for (int u = 0; u < kGather; u++)
        if (cb + threadIdx.x + u * kLevelThreads < ce) bx[u] = aos[src[u]];
#pragma unroll
      for (int u = 0; u < kGather; u++) {
        const int64_t s = cb + threadIdx.x + u * kLevelThreads;
        if (s < ce) {
          const float4 m = bx[u].mbr;
          __stcs(oxmin + s, m.x);
          __stcs(oymin + s, m.y);
          __stcs(oxmax + s, m.z);
          __stcs(oymax + s, m.w);
          __stcs(oid + s, bx[u].idp.x);
          s_mbr[s - cb] = m;
        }
      }
    } else {
      for (int64_t s = cb + threadIdx.x; s < ce; s += kLevelThreads) {
        const int64_t i = child_start + s;
        s_mbr[s - cb] = make_float4(nxmin[i], nymin[i], nxmax[i], nymax[i]);
      }
    }
    __syncthreads();
    if (have) {
      const int64_t lo = max(my_c0, cb), hi = min(my_c1, ce);
      for (int64_t s = lo; s < hi; s++) {
        float4 m = s_mbr[s - cb];
        if (!init) {
          a = m.x; b = m.y; c = m.z; d = m.w;
          init = true;
        } else {
          a = fminf(a, m.x);
          b = fminf(b, m.y);
          c = fmaxf(c, m.z);
          d = fmaxf(d, m.w);
        }
      }
    }
    __syncthreads();
  }
  if (have) {
    const int64_t o = parent_start + my;
    nxmin[o] = a;
    nymin[o] = b;
    nxmax[o] = c;
    nymax[o] = d;
    npos[o] = (int)(pos_base + my_c0);
    nlen[o] = (int)(my_c1 - my_c0);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int tree_levels(int64_t n, int fanout, std::vector<int64_t>& lv)
{
  lv.clear();
  if (n < 1 || fanout < 2) return -1;
  int64_t len = n;
  while (len != 1) {
    len = (len + fanout - 1) / fanout;
    lv.push_back(len);
  }
  return (int)lv.size();
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

static int64_t sort_tiles(int64_t n) { return std::max<int64_t>(1, cdiv(n, kSortTile)); }

// Look-back status words: one per (tile, bin) of every digit.
static int64_t status_words_before(int digit, int64_t tiles)
{
  int64_t w = 0;
  for (int d = 0; d < digit; d++) w += tiles << digit_bits(d);
  return w;
}

size_t sort_zero_bytes(int64_t n)
{
  return sizeof(SortCtrl) + (size_t)kDigits * kBins * sizeof(uint32_t) +
         (size_t)status_words_before(kDigits, sort_tiles(n)) * sizeof(uint64_t);
}
SortCtrl* sort_ctrl(void* zero_block) { return (SortCtrl*)zero_block; }
uint32_t* sort_hist(void* zero_block) { return (uint32_t*)((char*)zero_block + sizeof(SortCtrl)); }
static uint64_t* sort_status(void* zero_block)
{
  return (uint64_t*)((char*)zero_block + sizeof(SortCtrl) + (size_t)kDigits * kBins * sizeof(uint32_t));
}

template <int kBits>
static void launch_pass(int d, SortBufs bufs, int64_t n, uint64_t* status, SortCtrl* ctrl,
                        int flags, cudaStream_t stream)
{
  const size_t smem = SweepSmem<kBits>::kBytes;
  cudaFuncSetAttribute(onesweep_kernel<kBits>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  onesweep_kernel<kBits><<<(unsigned)sort_tiles(n), kSortThreads, smem, stream>>>(d, bufs, n, status,
                                                                                  ctrl, flags);
}

void sort_passes(SortBufs bufs, int64_t n, void* zero_block, cudaStream_t stream, int flags)
{
  const int64_t ntiles = sort_tiles(n);
  SortCtrl* ctrl = sort_ctrl(zero_block);
  plan_kernel<<<1, 32 * kDigits, 0, stream>>>(sort_hist(zero_block), n, ctrl);
  for (int d = 0; d < kDigits; d++) {
    ProfScope ps("sort_pass", stream);
    uint64_t* status = sort_status(zero_block) + status_words_before(d, ntiles);
    switch (digit_bits(d)) {
      case 10: launch_pass<10>(d, bufs, n, status, ctrl, flags, stream); break;
      case 8: launch_pass<8>(d, bufs, n, status, ctrl, flags, stream); break;
      case 2: launch_pass<2>(d, bufs, n, status, ctrl, flags, stream); break;
      default: launch_pass<kDigitBits>(d, bufs, n, status, ctrl, flags, stream); break;
    }
  }
  CRT_LAUNCHED(1 + kDigits);
}

// Builds the tree of `n` boxes.  in_* may alias out_* (in-place build).
// Node arrays must hold R_sz entries.  Synchronises `stream` at the end and
// reports device-side errors.
int build_tree(const float* in_xmin, const float* in_ymin, const float* in_xmax,
               const float* in_ymax, const int* in_id, int64_t n, int fanout, float* out_xmin,
               float* out_ymin, float* out_xmax, float* out_ymax, int* out_id, float* nxmin,
               float* nymin, float* nxmax, float* nymax, int* npos, int* nlen,
               cudaStream_t stream)
{
  NvtxRange range("crt_build");
  std::vector<int64_t> lv;
  if (tree_levels(n, fanout, lv) < 0)
    return fail(CRT_ERR_INVALID_ARG, "build: need n >= 1 and fanout >= 2");
  int64_t rsz = 0;
  for (auto x : lv) rsz += x;
  if (n + rsz > INT32_MAX)
    return fail(CRT_ERR_INVALID_ARG, "build: n + R_sz exceeds the int32 pos range of RTREE");

  // scratch: [ctrl | hist | status] (zeroed) then keys/vals/aos
  const size_t zero_bytes = sort_zero_bytes(n);
  const size_t kv_bytes = ((size_t)n * 4 + 255) / 256 * 256;
  const size_t aos_bytes = (size_t)n * sizeof(Box32);
  const size_t total = (zero_bytes + 255) / 256 * 256 + 4 * kv_bytes + aos_bytes + 256;
  char* scratch = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&scratch, total, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CRT_ERR_OOM, "build: scratch allocation failed");
  }
  size_t off = (zero_bytes + 255) / 256 * 256;
  BuildCtrl* ctrl = sort_ctrl(scratch);
  uint32_t* hist = sort_hist(scratch);
  SortBufs bufs;
  bufs.keys[0] = (uint32_t*)(scratch + off); off += kv_bytes;
  bufs.keys[1] = (uint32_t*)(scratch + off); off += kv_bytes;
  bufs.vals[0] = (uint32_t*)(scratch + off); off += kv_bytes;
  bufs.vals[1] = (uint32_t*)(scratch + off); off += kv_bytes;
  Box32* aos = (Box32*)(scratch + off);

  int rc = CRT_OK;
  do {
    if ((e = cudaMemsetAsync(scratch, 0, zero_bytes, stream)) != cudaSuccess) break;
    const int sms = sm_count();
    const bool vec = aligned16(in_xmin) && aligned16(in_ymin) && aligned16(in_xmax) &&
                     aligned16(in_ymax) && aligned16(in_id);
    int grid = (int)std::min<int64_t>(cdiv(n, kEncTile), (int64_t)sms * 3);
    if (grid < 1) grid = 1;
    const BoxIn bin{in_xmin, in_ymin, in_xmax, in_ymax, in_id};
    {
    ProfScope ps("encode", stream);
    if (vec)
      encode_kernel<true><<<grid, kEncThreads, 0, stream>>>(bin, n, bufs.keys[0], bufs.vals[0],
                                                            aos, hist);
    else
      encode_kernel<false><<<grid, kEncThreads, 0, stream>>>(bin, n, bufs.keys[0], bufs.vals[0],
                                                             aos, hist);
    }
    CRT_LAUNCHED(1);
    sort_passes(bufs, n, scratch, stream, kSortGivenValues);

    // leaf-parent level
    int64_t parent_start = rsz;
    int64_t child_start = 0, nchild = n;
    for (size_t l = 0; l < lv.size(); l++) {
      const int64_t np = lv[l];
      parent_start -= np;
      int npc = (int)std::max<int64_t>(1, std::min<int64_t>(kLevelThreads, kLevelChunk / fanout));
      unsigned g = (unsigned)cdiv(np, npc);
      ProfScope ps("level", stream);
      if (l == 0)
        level_kernel<true><<<g, kLevelThreads, 0, stream>>>(
            npc, fanout, nchild, np, parent_start, rsz, bufs.vals[0], bufs.vals[1], ctrl, aos,
            out_xmin, out_ymin, out_xmax, out_ymax, out_id, nxmin, nymin, nxmax, nymax, npos,
            nlen, 0);
      else
        level_kernel<false><<<g, kLevelThreads, 0, stream>>>(
            npc, fanout, nchild, np, parent_start, child_start, nullptr, nullptr, ctrl, nullptr,
            nullptr, nullptr, nullptr, nullptr, nullptr, nxmin, nymin, nxmax, nymax, npos, nlen,
            child_start);
      CRT_LAUNCHED(1);
      child_start = parent_start;
      nchild = np;
    }
    if (lv.empty()) {
      // one box, no nodes: the sorted box set is the input itself
      if (out_xmin != in_xmin) {
        cudaMemcpyAsync(out_xmin, in_xmin, 4, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(out_ymin, in_ymin, 4, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(out_xmax, in_xmax, 4, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(out_ymax, in_ymax, 4, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(out_id, in_id, 4, cudaMemcpyDeviceToDevice, stream);
      }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    int dev_err = 0;
    if ((e = cudaMemcpyAsync(&dev_err, &ctrl->error, sizeof(int), cudaMemcpyDeviceToHost,
                             stream)) != cudaSuccess)
      break;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) break;
    if (dev_err) rc = fail(dev_err, "build: device-side wait timed out in the radix sort");
  } while (0);
  cudaFreeAsync(scratch, stream);
  if (e != cudaSuccess) return cuda_fail(e, "build");
  return rc;
}

}  // namespace crt
