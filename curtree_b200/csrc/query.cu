// Batched window query (replaces bfs_frontier, src/rtree_bfs_frontier.cuh:292-529,
// and bfs_thrust, src/rtree_bfs_thrust.cuh:59-256).
//
// Semantics kept from the reference: the root is never tested; a node whose
// children are nodes passes on the children whose MBR intersects the window
// (src/rtree_bfs_frontier.cuh:110-124); a leaf-parent (pos >= R_sz) tests its
// boxes at slots [pos - R_sz, pos - R_sz + len) (count_hit/write_hit,
// :191-289); a hit emits (fid = sorted box's id, tid = window index).
//
// Traversal: one warp per window.  The warp keeps its frontier in shared
// memory as a stack of node indices.  Each step pops up to K = 32 / fanout
// nodes (one child per lane, children read in SoA layout, coalesced), tests
// the children, compacts the intersecting inner children back onto the stack
// with a ballot/popc prefix, and emits leaf hits warp-collectively.  Popping
// the top K entries and pushing shallower parents' children first keeps the
// stack ordered by depth, so it never holds more than K*fanout entries per
// level: (levels - 1) * K * fanout + 1 in total, which the host sizes exactly.
//
// Two forms:
//   plain       one warp per window in input order, a count pass, an int64
//               exclusive scan and a write pass: output grouped by window.
//   persistent  #SM x occupancy CTAs; warps take windows from an atomic ticket
//               in Morton order of the window centres (neighbouring windows
//               share tree paths, so the tree stays in L2); the top tree levels
//               are staged in shared memory with bulk async copies; hits go to
//               4096-slot chunks a warp reserves with one atomic, and a
//               compaction pass moves the tail of the array into the unused
//               ends of each warp's last chunk so the output is dense.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.h"
#include "profile.h"
#include "traverse.cuh"

namespace crt {

// Device-side counters of one query (int64 words; zeroed before a launch).
struct QueryCounters {
  unsigned long long ticket;  // next window (persistent)
  unsigned long long next;    // next unreserved output slot
  unsigned long long hits;    // exact pair count
  unsigned long long nholes;  // unused chunk ends recorded
  int error;
  int pad;
  unsigned long long nq;      // window count (read by graph replays)
};

// query_stats and the allocation-free entry point keep the counters in the
// first 256 bytes of their scratch.
static_assert(sizeof(QueryCounters) <= 256, "counters fit their scratch slot");

struct Hole {
  long long start;
  long long len;
};

// ---------------------------------------------------------------------------
// Emitters: warp-collective; `hit` and `id` are per lane.
// ---------------------------------------------------------------------------
struct CountEmit {
  static constexpr bool kCountsTests = false;
  long long hits = 0;
  __device__ __forceinline__ void begin(int) {}
  __device__ __forceinline__ void operator()(bool hit, int) { hits += __popc(__ballot_sync(0xffffffffu, hit)); }
  __device__ __forceinline__ void range(const int*, long long, long long count) { hits += count; }
  __device__ __forceinline__ void small_ranges(const int*, bool mine, long long, int count)
  {
    hits += __reduce_add_sync(0xffffffffu, mine ? (unsigned)count : 0u);
  }
  __device__ __forceinline__ void big_ranges(const int* bid, bool mine, long long first, long long count)
  {
    emit_ranges_each(*this, bid, mine, first, count);
  }
};

// Counts hits and the leaf boxes tested (workload statistics).
struct StatEmit {
  static constexpr bool kCountsTests = true;
  long long hits = 0;
  long long tested = 0;
  __device__ __forceinline__ void begin(int) {}
  __device__ __forceinline__ void operator()(bool hit, int) { hits += __popc(__ballot_sync(0xffffffffu, hit)); }
  long long range_hits = 0;
  __device__ __forceinline__ void leaf_tests(int n) { tested += n; }
  __device__ __forceinline__ void range(const int*, long long, long long count)
  {
    hits += count;
    range_hits += count;
  }
  __device__ __forceinline__ void small_ranges(const int*, bool mine, long long, int count)
  {
    const unsigned n = __reduce_add_sync(0xffffffffu, mine ? (unsigned)count : 0u);
    hits += n;
    range_hits += n;
  }
  __device__ __forceinline__ void big_ranges(const int* bid, bool mine, long long first, long long count)
  {
    emit_ranges_each(*this, bid, mine, first, count);
  }
};

// Writes at precomputed per-window offsets (plain write pass).
struct OffsetEmit {
  static constexpr bool kCountsTests = false;
  int32_t* fid;
  int32_t* tid;
  long long base;
  long long cap;
  int q;
  __device__ __forceinline__ void begin(int qq) { q = qq; }
  __device__ __forceinline__ void operator()(bool hit, int id)
  {
    uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (!m) return;
    long long slot = base + __popc(m & lanemask_lt());
    if (hit && slot < cap) {
      __stcs(fid + slot, id);
      if (tid) __stcs(tid + slot, q);  // no window column: CSR output
    }
    base += __popc(m);
  }
  __device__ __forceinline__ void range(const int* bid, long long first, long long count)
  {
    copy_range(bid, first, count, fid, tid, base, cap, q);
    base += count;
  }
  __device__ __forceinline__ void small_ranges(const int* bid, bool mine, long long first, int count)
  {
    emit_small_ranges(*this, bid, mine, first, count);
  }
  __device__ __forceinline__ void big_ranges(const int* bid, bool mine, long long first, long long count)
  {
    emit_ranges_each(*this, bid, mine, first, count);
  }
};

// ---------------------------------------------------------------------------
// Range sharing (persistent form).  One window can own a contained subtree of
// millions of boxes; copied by one warp it leaves the rest of the GPU idle at
// the end of a batch.  The warp that finds such a range reserves its output,
// cuts it into kPiece-id pieces, publishes them in a job queue and goes on
// with its window.  Warps that find no window left claim queue indices with
// one fetch-and-add each and copy the pieces as they are published, so the
// tail of a batch runs on every warp of the GPU.  A claimed index that no
// window will ever fill ends the claimer's wait once every window is done.
// ---------------------------------------------------------------------------
struct RangeJob {
  long long first;  // first sorted slot
  long long slot;   // first output slot
  int count;
  int q;
  unsigned ready;   // 1 once published; the taker clears it
  int pad;
};
// The queue's counters, each on its own 128-byte line: waiting warps poll
// them, and they must not share a line with the ticket and output counters
// every busy warp updates.
struct JobQueue {
  unsigned long long tail;  // pieces reserved
  unsigned long long pad0[15];
  unsigned long long head;  // queue indices claimed
  unsigned long long pad1[15];
  unsigned long long active;  // warps not yet past their ticket loop
  unsigned long long pad2[15];
  RangeJob entries[1];  // kJobs
};
constexpr int kJobs = 1 << 18;         // queue entries per launch (8 MiB)
constexpr int kPiece = 16384;          // ids per piece
constexpr int kShareMin = 2 * kPiece;  // ranges shorter than this stay with their finder
constexpr size_t kJobQueueBytes = offsetof(JobQueue, entries) + sizeof(RangeJob) * kJobs;

__device__ __forceinline__ void fence_sc_gpu() { asm volatile("fence.sc.gpu;" ::: "memory"); }

// Waits (lane 0) until queue index h is published, and takes the piece; 0 when
// h will never be published (every ticket is taken, no warp still works on
// one, and h was not reserved) or the bounded wait ran out (an error is
// recorded).  ntickets: the ticket count of the launch.
__device__ __forceinline__ int wait_piece(JobQueue* Q, const QueryCounters* ctr,
                                          unsigned long long ntickets, long long h, RangeJob& out,
                                          int* err)
{
  RangeJob* J = Q->entries + h;
  uint32_t nap = 64;
  for (uint32_t spin = 0; spin < kSpinLimit / 16; spin++) {
    if (ld_acquire_u32(&J->ready)) {
      out.first = J->first;
      out.slot = J->slot;
      out.count = J->count;
      out.q = J->q;
      J->ready = 0;
      return 1;
    }
    if (ld_relaxed_ull(&Q->tail) <= (unsigned long long)h) {
      // not reserved yet: can any window still reserve it?
      fence_sc_gpu();
      const unsigned long long t = ld_relaxed_ull(&ctr->ticket);
      fence_sc_gpu();
      const unsigned long long a = ld_relaxed_ull(&Q->active);
      if (t >= ntickets && a == 0) {
        fence_sc_gpu();
        if (ld_relaxed_ull(&Q->tail) <= (unsigned long long)h) return 0;
      }
    }
    __nanosleep(nap);
    nap = min(2u * nap, 8192u);
  }
  raise_error(err, CRT_ERR_DEVICE_TIMEOUT);
  return 0;
}

// Warp-reserved output chunks (persistent form).
struct ChunkEmit {
  static constexpr bool kCountsTests = false;
  int32_t* fid;
  int32_t* tid;
  long long cap;
  unsigned long long* next;
  long long cur = 0, end = 0;
  long long hits = 0;
  int chunk;
  int q;
  JobQueue* jobs = nullptr;  // null: no range sharing
  __device__ __forceinline__ void begin(int qq) { q = qq; }
  __device__ __forceinline__ void operator()(bool hit, int id)
  {
    uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (!m) return;
    const int nh = __popc(m);
    const int r = __popc(m & lanemask_lt());
    hits += nh;
    long long slot;
    if (cur + nh <= end) {
      slot = cur + r;
      cur += nh;
    } else {
      const long long left = end - cur;
      unsigned long long nb = 0;
      if (lane_id() == 0) nb = atomicAdd(next, (unsigned long long)chunk);
      nb = __shfl_sync(0xffffffffu, nb, 0);
      slot = r < left ? cur + r : (long long)nb + (r - left);
      cur = (long long)nb + (nh - left);
      end = (long long)nb + chunk;
    }
    if (hit && slot < cap) {
      __stcs(fid + slot, id);
      __stcs(tid + slot, q);
    }
  }
  __device__ __forceinline__ void small_ranges(const int* bid, bool mine, long long first, int count)
  {
    emit_small_ranges(*this, bid, mine, first, count);
  }
  // Large contained subtrees go to an exact reservation (no unused chunk
  // end), all of one step's in one: each lane's range at its prefix offset.
  // One atomic per step instead of one per range keeps the shared output
  // counter from becoming the bottleneck when every warp meets large
  // subtrees at once (10M boxes x 250k windows of side 1e-2..1e-1: 21 ms
  // with one atomic per range, 12.4 ms with one per step).
  __device__ __forceinline__ void big_ranges(const int* bid, bool mine, long long first, long long count)
  {
    const int lane = (int)lane_id();
    const long long c = mine ? count : 0;
    long long x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const long long total = __shfl_sync(0xffffffffu, x, 31);
    unsigned long long nb = 0;
    if (lane == 0) nb = atomicAdd(next, (unsigned long long)total);
    nb = __shfl_sync(0xffffffffu, nb, 0);
    const long long excl = x - c;
    uint32_t im = __ballot_sync(0xffffffffu, mine);
    while (im) {
      const int src = __ffs(im) - 1;
      im &= im - 1;
      place(bid, __shfl_sync(0xffffffffu, first, src), __shfl_sync(0xffffffffu, count, src),
            (long long)nb + __shfl_sync(0xffffffffu, excl, src));
    }
  }
  // Copies a contained subtree's ids to its reservation at output slot nb
  // (large ones cut into pieces that idle warps copy).
  __device__ __forceinline__ void place(const int* bid, long long first, long long count,
                                        long long nb)
  {
    hits += count;
    if (!jobs || count < kShareMin) {
      copy_range_realign(bid, first, count, fid, tid, nb, cap, q);
      return;
    }
    // publish the pieces; the ones the queue has no room for are copied here
    const long long np = (count + kPiece - 1) / kPiece;
    unsigned long long j0 = 0;
    if (lane_id() == 0) j0 = atomicAdd(&jobs->tail, (unsigned long long)np);
    j0 = __shfl_sync(0xffffffffu, j0, 0);
    const long long own = max(0ll, min(np, (long long)kJobs - (long long)j0));
    for (long long p = lane_id(); p < own; p += 32) {
      RangeJob& J = jobs->entries[(long long)j0 + p];
      const long long off = p * kPiece;
      J.first = first + off;
      J.slot = (long long)nb + off;
      J.count = (int)min((long long)kPiece, count - off);
      J.q = q;
      st_release_u32(&J.ready, 1u);
    }
    if (own < np)
      copy_range(bid, first + own * kPiece, count - own * kPiece, fid, tid,
                 (long long)nb + own * kPiece, cap, q);
  }
};

// ---------------------------------------------------------------------------
// Plain form: count pass / write pass, one warp per window in input order
// ---------------------------------------------------------------------------
constexpr int kPlainWarps = 8;

__global__ void __launch_bounds__(kPlainWarps * 32)
    plain_count_kernel(TreeView T, WindowView W, int K, int stack_cap,
                       long long* __restrict__ counts, QueryCounters* ctr)
{
  extern __shared__ FrontierEntry s_stack[];
  const int warp = threadIdx.x >> 5;
  const long long q = (long long)blockIdx.x * kPlainWarps + warp;
  if (q >= W.n) return;
  int lg, lc;
  lane_map(T.fanout, lg, lc);
  NodeCache C{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
  CountEmit emit;
  traverse(T, C, K, lg, lc, W.xmin[q], W.ymin[q], W.xmax[q], W.ymax[q],
           s_stack + warp * stack_cap, stack_cap, emit, &ctr->error);
  if (lane_id() == 0) counts[q] = emit.hits;
}

__global__ void __launch_bounds__(kPlainWarps * 32)
    plain_write_kernel(TreeView T, WindowView W, int K, int stack_cap,
                       const long long* __restrict__ offsets, int32_t* fid, int32_t* tid,
                       long long cap, QueryCounters* ctr)
{
  extern __shared__ FrontierEntry s_stack[];
  const int warp = threadIdx.x >> 5;
  const long long q = (long long)blockIdx.x * kPlainWarps + warp;
  if (q >= W.n) return;
  if (offsets[W.n] > cap) return;  // overflow: the host reports the required size
  int lg, lc;
  lane_map(T.fanout, lg, lc);
  NodeCache C{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
  OffsetEmit emit{fid, tid, offsets[q], cap, (int)q};
  traverse(T, C, K, lg, lc, W.xmin[q], W.ymin[q], W.xmax[q], W.ymax[q],
           s_stack + warp * stack_cap, stack_cap, emit, &ctr->error);
}

template <bool kContain>
__global__ void __launch_bounds__(kPlainWarps * 32)
    stats_kernel(TreeView T, WindowView W, int K, int stack_cap, long long* __restrict__ hits,
                 long long* __restrict__ tested, unsigned long long* __restrict__ totals,
                 QueryCounters* ctr)
{
  extern __shared__ FrontierEntry s_stack[];
  const int warp = threadIdx.x >> 5;
  const long long q = (long long)blockIdx.x * kPlainWarps + warp;
  if (q >= W.n) return;
  int lg, lc;
  lane_map(T.fanout, lg, lc);
  NodeCache C{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
  StatEmit emit;
  traverse<StatEmit, kContain>(T, C, K, lg, lc, W.xmin[q], W.ymin[q], W.xmax[q], W.ymax[q],
                               s_stack + warp * stack_cap, stack_cap, emit, &ctr->error);
  if (lane_id() == 0) {
    if (hits) hits[q] = emit.hits;
    if (tested) tested[q] = emit.tested;
    atomicAdd(&totals[0], (unsigned long long)emit.hits);
    atomicAdd(&totals[1], (unsigned long long)emit.tested);
    atomicAdd(&totals[2], (unsigned long long)emit.range_hits);
  }
}

// int64 exclusive scan (counts -> offsets[0..n]), three kernels
constexpr int kScanThreads = 1024;

__device__ __forceinline__ long long block_incl_scan(long long v, long long* s_warp)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += s_warp[warp - 1];
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_block_sums(const long long* __restrict__ in, long long n, long long* __restrict__ sums)
{
  __shared__ long long s_warp[32];
  long long i = (long long)blockIdx.x * kScanThreads + threadIdx.x;
  long long v = i < n ? in[i] : 0;
  v = block_incl_scan(v, s_warp);
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_sums_kernel(long long* __restrict__ sums, long long nb)
{
  __shared__ long long s_warp[32];
  __shared__ long long s_tot;
  long long carry = 0;
  for (long long b0 = 0; b0 < nb; b0 += kScanThreads) {
    long long i = b0 + threadIdx.x;
    long long v = i < nb ? sums[i] : 0;
    long long x = block_incl_scan(v, s_warp);
    if (i < nb) sums[i] = carry + x - v;  // exclusive
    if (threadIdx.x == kScanThreads - 1) s_tot = x;
    __syncthreads();
    carry += s_tot;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads)
    scan_apply_kernel(const long long* __restrict__ in, long long n,
                      const long long* __restrict__ sums, long long* __restrict__ out)
{
  __shared__ long long s_warp[32];
  long long i = (long long)blockIdx.x * kScanThreads + threadIdx.x;
  long long v = i < n ? in[i] : 0;
  long long x = block_incl_scan(v, s_warp);
  long long base = sums[blockIdx.x];
  if (i < n) out[i] = base + x - v;
  if (i == n - 1) out[n] = base + x;
}

// Writes the result block of a plain query.
__global__ void plain_result_kernel(const long long* __restrict__ offsets, long long n,
                                    long long cap, QueryCounters* ctr, crt_query_result* res)
{
  long long total = n > 0 ? offsets[n] : 0;
  res->required = total;
  res->overflow = total > cap ? 1 : 0;
  res->count = total > cap ? 0 : total;
  res->error = ctr->error;
}

// ---------------------------------------------------------------------------
// Persistent form
// ---------------------------------------------------------------------------
struct PersistParams {
  TreeView T;
  WindowView W;
  const uint32_t* order0;  // sorted window order candidates (vals[0], vals[1])
  const uint32_t* order1;
  const SortCtrl* sort_ctrl;  // n_active picks the buffer; null: input order
  int K;
  int stack_cap;
  int stage_n;  // nodes staged in shared memory (multiple of 4), 0 = none
  int parts;    // warps sharing one window (shares of the root's children)
  int chunk;
  int32_t* fid;
  int32_t* tid;
  long long cap;
  QueryCounters* ctr;
  Hole* holes;
  long long max_holes;
  JobQueue* jobs;  // counters and kJobs entries, zeroed before the launch
};

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// One bulk async copy global -> shared (16-byte aligned, size a multiple of
// 16), completing on the mbarrier at `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// kShare: range sharing (the job queue).  Its code needs registers the
// tighter CTA shapes do not have, so only the 8-warp shape (64 registers)
// shares ranges; the autotuner weighs the shapes against each other.
template <int kThreads, int kMinBlocks, bool kShare>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    persistent_kernel(PersistParams P)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long s_mbar;
  __shared__ int s_stage_ok;
  const int warps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5;
  // layout: [staged nodes: 6 arrays x stage_n x 4 B][stacks: warps x stack_cap x 4 B]
  float* c_xmin = (float*)smem_raw;
  float* c_ymin = c_xmin + P.stage_n;
  float* c_xmax = c_ymin + P.stage_n;
  float* c_ymax = c_xmax + P.stage_n;
  int* c_pos = (int*)(c_ymax + P.stage_n);
  int* c_len = c_pos + P.stage_n;
  FrontierEntry* stacks = (FrontierEntry*)(c_len + P.stage_n);
  NodeCache C{c_xmin, c_ymin, c_xmax, c_ymax, c_pos, c_len, 0};

  if (P.stage_n > 0) {
    // bulk async copies of the top levels into shared memory, one mbarrier
    const uint32_t bar = smem_addr(&s_mbar);
    const uint32_t bytes = (uint32_t)P.stage_n * 4u;
    if (threadIdx.x == 0) {
      s_stage_ok = 1;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                   "r"(6u * bytes)
                   : "memory");
      bulk_load(c_xmin, P.T.nxmin, bytes, bar);
      bulk_load(c_ymin, P.T.nymin, bytes, bar);
      bulk_load(c_xmax, P.T.nxmax, bytes, bar);
      bulk_load(c_ymax, P.T.nymax, bytes, bar);
      bulk_load(c_pos, P.T.npos, bytes, bar);
      bulk_load(c_len, P.T.nlen, bytes, bar);
    }
    // bounded wait for phase 0 (twice the usual limit: after a timeout the
    // copies must not still be landing when the CTA leaves)
    uint32_t done = 0;
    for (uint32_t spin = 0; spin < 2 * kSpinLimit; spin++) {
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
          : "=r"(done)
          : "r"(bar)
          : "memory");
      if (done) break;
    }
    if (!done) {
      if (threadIdx.x == 0) s_stage_ok = 0;
      raise_error(&P.ctr->error, CRT_ERR_DEVICE_TIMEOUT);
    }
    __syncthreads();
    if (!s_stage_ok) return;
    C.n = P.stage_n;
  }

  FrontierEntry* stack = stacks + warp * P.stack_cap;
  int lg, lc;
  lane_map(P.T.fanout, lg, lc);
  const uint32_t* order = nullptr;
  if (P.sort_ctrl) {
    const int na = P.sort_ctrl->n_active;
    order = na == 0 ? nullptr : ((na & 1) ? P.order1 : P.order0);
  }
  const long long nq = (long long)P.ctr->nq;
  const int parts = P.parts;
  const long long ntickets = nq * parts;  // one ticket per (window, share)
  ChunkEmit emit;
  emit.fid = P.fid;
  emit.tid = P.tid;
  emit.cap = P.cap;
  emit.next = &P.ctr->next;
  emit.chunk = P.chunk;
  emit.jobs = kShare ? P.jobs : nullptr;
  JobQueue* Q = kShare ? P.jobs : nullptr;
  (void)warps;
  // a warp counts as active from before its first ticket until it has left
  // the ticket loop, so a waiting warp that sees the tickets gone and no
  // warp active knows no window can publish any more
  if (Q && lane_id() == 0) {
    atomicAdd(&Q->active, 1ull);
    fence_sc_gpu();
  }
  while (true) {
    unsigned long long t = 0;
    if (lane_id() == 0) t = atomicAdd(&P.ctr->ticket, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if ((long long)t >= ntickets) break;
    const long long qi = parts == 1 ? (long long)t : (long long)t / parts;
    const int part = parts == 1 ? 0 : (int)((long long)t - qi * parts);
    int q = order ? (int)order[qi] : (int)qi;
    if (q < 0 || (long long)q >= nq) q = (int)qi;  // only after a sort error (reported)
    emit.begin(q);
    traverse(P.T, C, P.K, lg, lc, P.W.xmin[q], P.W.ymin[q], P.W.xmax[q], P.W.ymax[q], stack,
             P.stack_cap, emit, &P.ctr->error, part, parts);
  }
  if (Q) {
    __syncwarp();
    if (lane_id() == 0) {
      fence_sc_gpu();  // this warp's reservations before it stops counting
      atomicAdd(&Q->active, ~0ull);  // -1
    }
  }
  // No window left: copy published pieces until no window can publish more.
  if (Q) {
    while (true) {
      long long h = 0;
      if (lane_id() == 0) h = (long long)atomicAdd(&Q->head, 1ull);
      h = __shfl_sync(0xffffffffu, h, 0);
      if (h >= kJobs) break;  // past the queue: never published
      RangeJob J{};
      int got = 0;
      if (lane_id() == 0) got = wait_piece(Q, P.ctr, (unsigned long long)ntickets, h, J, &P.ctr->error);
      if (!__shfl_sync(0xffffffffu, got, 0)) break;
      const long long first = __shfl_sync(0xffffffffu, J.first, 0);
      const long long slot = __shfl_sync(0xffffffffu, J.slot, 0);
      const int count = __shfl_sync(0xffffffffu, J.count, 0);
      const int jq = __shfl_sync(0xffffffffu, J.q, 0);
      copy_range(P.T.bid, first, count, P.fid, P.tid, slot, P.cap, jq);
    }
  }
  if (lane_id() == 0) {
    if (emit.hits) atomicAdd(&P.ctr->hits, (unsigned long long)emit.hits);
    if (emit.end > emit.cur) {
      unsigned long long h = atomicAdd(&P.ctr->nholes, 1ull);
      if ((long long)h < P.max_holes) {
        P.holes[h].start = emit.cur;
        P.holes[h].len = emit.end - emit.cur;
      } else {
        raise_error(&P.ctr->error, CRT_ERR_NOT_SUPPORTED);
      }
    }
  }
}

// Sorts the recorded holes by start: rank by counting (starts are distinct:
// holes do not overlap), one hole per thread, all starts streamed through
// shared memory in tiles.
constexpr int kHoleTile = 2048;

__global__ void __launch_bounds__(256)
    hole_sort_kernel(const Hole* __restrict__ holes, Hole* __restrict__ sorted,
                     const QueryCounters* __restrict__ ctr, long long max_holes)
{
  __shared__ long long s_start[kHoleTile];
  const long long nh = min((long long)ctr->nholes, max_holes);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if ((long long)blockIdx.x * blockDim.x >= nh) return;  // whole CTA idle
  const long long my = i < nh ? holes[i].start : 0;
  long long r = 0;
  for (long long t0 = 0; t0 < nh; t0 += kHoleTile) {
    const int m = (int)min((long long)kHoleTile, nh - t0);
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += blockDim.x) s_start[k] = holes[t0 + k].start;
    __syncthreads();
    for (int k = 0; k < m; k++) r += s_start[k] < my;
  }
  if (i < nh) sorted[r] = holes[i];
}

// Exclusive prefix of the sorted hole lengths (one CTA).
__global__ void __launch_bounds__(kScanThreads)
    hole_prefix_kernel(const Hole* __restrict__ sorted, long long* __restrict__ cum,
                       const QueryCounters* __restrict__ ctr, long long max_holes)
{
  __shared__ long long s_warp[32];
  __shared__ long long s_tot;
  const long long nh = min((long long)ctr->nholes, max_holes);
  long long carry = 0;
  for (long long b0 = 0; b0 < nh; b0 += kScanThreads) {
    long long i = b0 + threadIdx.x;
    long long v = i < nh ? sorted[i].len : 0;
    long long x = block_incl_scan(v, s_warp);
    if (i < nh) cum[i] = carry + x - v;
    if (threadIdx.x == kScanThreads - 1) s_tot = x;
    __syncthreads();
    carry += s_tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) cum[nh] = carry;
}

// Hole slots in [0, x): cum[i] + min(x - st[i], len[i]) for the last hole
// starting before x.
__device__ __forceinline__ long long holes_below(const Hole* h, const long long* cum, long long nh,
                                                 long long x)
{
  long long lo = 0, hi = nh;  // first hole with start >= x
  while (lo < hi) {
    long long m = (lo + hi) >> 1;
    if (h[m].start < x) lo = m + 1; else hi = m;
  }
  if (lo == 0) return 0;
  const long long i = lo - 1;
  return cum[i] + min(x - h[i].start, h[i].len);
}

// First hole (sorted by start) whose start is >= x.
__device__ __forceinline__ long long hole_at_or_after(const Hole* h, long long nh, long long x)
{
  long long lo = 0, hi = nh;
  while (lo < hi) {
    long long m = (lo + hi) >> 1;
    if (h[m].start < x) lo = m + 1; else hi = m;
  }
  return lo;
}

// Moves every pair stored at or above `hits` (T) into the holes below it, so
// the output is dense [0, T); then writes the result block.  The B pairs to
// move are the data slots of [T, next) in order, and their destinations the
// hole slots below T in order: both are runs, so each CTA takes a piece of
// kMovePiece consecutive moves, finds where its sources and destinations
// start with binary searches, and then copies run by run with coalesced
// accesses.
constexpr long long kMovePiece = 8192;

__global__ void __launch_bounds__(256)
    compact_kernel(const Hole* __restrict__ h, const long long* __restrict__ cum,
                   QueryCounters* __restrict__ ctr, long long max_holes, int32_t* fid,
                   int32_t* tid, long long cap, crt_query_result* __restrict__ res)
{
  const long long nh = min((long long)ctr->nholes, max_holes);
  const long long T = (long long)ctr->hits;
  const long long R = (long long)ctr->next;
  const bool overflow = R > cap;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    res->required = T;
    res->overflow = overflow ? 1 : 0;
    res->count = overflow ? 0 : T;
    res->error = ctr->error;
  }
  if (overflow || ctr->error || nh == 0) return;
  const long long B = holes_below(h, cum, nh, T);  // pairs to move
  for (long long r0 = (long long)blockIdx.x * kMovePiece; r0 < B;
       r0 += (long long)gridDim.x * kMovePiece) {
    long long rem = min(kMovePiece, B - r0);
    // destination of move r0: the r0-th hole slot below T
    long long a = 0;
    {
      long long lo = 0, hi = nh;  // last hole with cum <= r0
      while (hi - lo > 1) {
        const long long m = (lo + hi) >> 1;
        if (cum[m] <= r0) lo = m; else hi = m;
      }
      a = lo;
    }
    long long d = h[a].start + (r0 - cum[a]);
    // source of move r0: the smallest x >= T with r0 + 1 data slots in [T, x]
    long long s = T;
    {
      long long lo = T, hi = R - 1;
      while (lo < hi) {
        const long long m = (lo + hi) >> 1;
        const long long data = (m + 1 - T) - (holes_below(h, cum, nh, m + 1) - B);
        if (data >= r0 + 1) hi = m; else lo = m + 1;
      }
      s = lo;
    }
    long long jn = hole_at_or_after(h, nh, s + 1);  // next hole above the source
    while (rem > 0) {
      const long long src_end = jn < nh ? h[jn].start : R;
      const long long dst_end = min(h[a].start + h[a].len, T);
      const long long n = min(rem, min(src_end - s, dst_end - d));
      if (n <= 0 || d < 0 || s + n > R || d + n > T) {  // inconsistent holes: report, stop
        if (threadIdx.x == 0) raise_error(&res->error, CRT_ERR_CUDA);
        break;
      }
      for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        fid[d + i] = fid[s + i];
        tid[d + i] = tid[s + i];
      }
      s += n;
      d += n;
      rem -= n;
      while (jn < nh && s == h[jn].start) {  // skip the hole(s) above the source
        s = h[jn].start + h[jn].len;
        jn++;
      }
      if (rem > 0 && d == dst_end) {
        if (++a >= nh) {
          if (threadIdx.x == 0) raise_error(&res->error, CRT_ERR_CUDA);
          break;
        }
        d = h[a].start;
      }
    }
  }
}

// Window keys (same Morton key as the boxes) and digit histograms.
__global__ void window_key_kernel(WindowView W, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ hist)
{
  __shared__ uint32_t sh[kDigits][kBins];
  for (int i = threadIdx.x; i < kDigits * kBins; i += blockDim.x) (&sh[0][0])[i] = 0;
  __syncthreads();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < W.n;
       i += (long long)gridDim.x * blockDim.x) {
    uint32_t k = sort_key(W.xmin[i], W.ymin[i], W.xmax[i], W.ymax[i]);
    keys[i] = k;
#pragma unroll
    for (int d = 0; d < kDigits; d++) atomicAdd(&sh[d][key_digit(k, d)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDigits * kBins; i += blockDim.x) {
    uint32_t v = (&sh[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

__global__ void set_nq_kernel(QueryCounters* ctr, long long nq) { ctr->nq = (unsigned long long)nq; }

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static TreeView make_view(const crt_rtree_f32& rt, const crt_bbox_f32& rb)
{
  TreeView T;
  T.nxmin = rt.xmin; T.nymin = rt.ymin; T.nxmax = rt.xmax; T.nymax = rt.ymax;
  T.npos = rt.pos; T.nlen = rt.len; T.rsz = rt.sz; T.fanout = rt.fanout;
  T.bxmin = rb.xmin; T.bymin = rb.ymin; T.bxmax = rb.xmax; T.bymax = rb.ymax; T.bid = rb.id;
  T.nbox = rb.sz;
  T.nlev = 0;
  T.lvl_first = nullptr;
  T.lvl_span = nullptr;
  T.lvl_odd = nullptr;
  return T;
}

// The tables hold only for the reference's packed layout, which a tree has
// exactly when its node count is the packed count for its box count.
LevelTables level_tables(const crt_rtree_f32& rt, int64_t nbox)
{
  LevelTables t;
  if (rt.sz <= 0 || rt.fanout < 2 || rt.fanout > kLenMask) return t;
  std::vector<int64_t> lv;
  const int L = tree_levels(nbox, rt.fanout, lv);
  if (L <= 0 || L > kMaxLevels) return t;
  int64_t rsz = 0;
  for (auto x : lv) rsz += x;
  if (rsz != rt.sz) return t;
  int64_t start = rsz;
  long long sp = rt.fanout;
  for (int h = 0; h < L; h++) {
    start -= lv[h];
    t.first[h] = (int)start;
    t.span[h] = sp;
    sp = sp > (1ll << 40) ? sp : sp * rt.fanout;
  }
  t.nlev = L;
  return t;
}

// Writes the tables (passed by value) to device memory: a one-thread kernel
// instead of a copy from host memory, so the caller's host thread never waits
// on a pageable transfer and the write can be recorded in a CUDA graph.
__global__ void write_levels_kernel(LevelTables t, int* __restrict__ first,
                                    long long* __restrict__ span)
{
  for (int h = threadIdx.x; h < kMaxLevels; h += blockDim.x) {
    first[h] = t.first[h];
    span[h] = t.span[h];
  }
}

// *odd = 1 when some box is not ordinary (*odd was zeroed before).  Every
// thread that sees one stores the same value.
__global__ void __launch_bounds__(256)
    odd_boxes_kernel(const float* __restrict__ xmin, const float* __restrict__ ymin,
                     const float* __restrict__ xmax, const float* __restrict__ ymax, int64_t n,
                     int* __restrict__ odd)
{
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    bad |= !(xmin[i] <= xmax[i] && ymin[i] <= ymax[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) *odd = 1;
}

void launch_odd_boxes(const float* xmin, const float* ymin, const float* xmax, const float* ymax,
                      int64_t n, int* odd, cudaStream_t stream)
{
  cudaMemsetAsync(odd, 0, sizeof(int), stream);
  if (n <= 0) return;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, 256), (int64_t)sm_count() * 8));
  odd_boxes_kernel<<<grid, 256, 0, stream>>>(xmin, ymin, xmax, ymax, n, odd);
  CRT_LAUNCHED(1);
}

// Puts the tables at `dev` (kLevelTableBytes, 8-byte aligned), checks the
// view's boxes for the shortcut and points the view at both.
static void attach_levels(TreeView& T, const LevelTables& t, void* dev, cudaStream_t stream)
{
  if (t.nlev == 0) return;
  int* first = (int*)dev;
  long long* span = (long long*)((char*)dev + sizeof(int) * kMaxLevels);
  int* odd = (int*)((char*)dev + kLevelOddOffset);
  write_levels_kernel<<<1, 64, 0, stream>>>(t, first, span);
  CRT_LAUNCHED(1);
  launch_odd_boxes(T.bxmin, T.bymin, T.bxmax, T.bymax, T.nbox, odd, stream);
  T.nlev = t.nlev;
  T.lvl_first = first;
  T.lvl_span = span;
  T.lvl_odd = odd;
}

// Number of levels of a tree with R_sz nodes over nbox boxes at this fanout
// (1 when the root is the only level).
static int levels_of(int64_t nbox, int fanout)
{
  std::vector<int64_t> lv;
  int L = tree_levels(std::max<int64_t>(nbox, 1), std::max(fanout, 2), lv);
  return std::max(L, 1);
}

struct TraversalShape {
  int K;
  int stack_cap;
};

static TraversalShape traversal_shape(int64_t nbox, int fanout)
{
  const int L = levels_of(nbox, fanout);
  TraversalShape s;
  s.K = fanout <= 32 ? std::max(1, 32 / fanout) : 1;
  // at most K*fanout entries per pushed level (levels 1 .. L-1), plus the root
  s.stack_cap = (L - 1) * s.K * fanout + 1;
  s.stack_cap = (s.stack_cap + 31) / 32 * 32;
  return s;
}

constexpr int kDefaultChunk = 4096;

// Persistent traversal variants: CTA width and CTAs per SM, which fix the
// register budget (65536 / (threads x CTAs)).  Wider CTAs share one staged
// copy of the top levels among more warps; narrower ones get more registers.
struct PersistVariant {
  int threads;
  int min_blocks;
  const void* fn;
};

static const PersistVariant kVariants[] = {
    {1024, 2, (const void*)persistent_kernel<1024, 2, false>},  // 64 warps/SM, 32 registers
    {512, 3, (const void*)persistent_kernel<512, 3, false>},    // 48 warps/SM, 40 registers
    {256, 4, (const void*)persistent_kernel<256, 4, true>},     // 32 warps/SM, 64 registers
};

static const PersistVariant& variant_for(int warps_per_cta)
{
  for (const auto& v : kVariants)
    if (v.threads / 32 == warps_per_cta) return v;
  return kVariants[2];  // default: 8 warps per CTA
}

static int persistent_grid(const PersistVariant& v, size_t smem)
{
  int per_sm = 0;
  cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.threads, smem);
  if (per_sm < 1) per_sm = 1;
  return per_sm * sm_count();
}

// Shared memory of the persistent traversal: the staged top levels (6 arrays)
// and one frontier stack per warp.  When that does not let the variant's CTAs
// share an SM, staging is dropped; a stack too deep for one CTA per SM is an
// error.
struct PersistShape {
  const PersistVariant* v;
  int stage_n;
  size_t smem;
};

static PersistShape persist_shape(int stack_cap, int stage_n, int warps_per_cta)
{
  const PersistVariant& v = variant_for(warps_per_cta);
  const size_t per_sm = 227 * 1024;
  for (int pass = 0; pass < 3; pass++) {
    const int sn = pass == 0 ? stage_n : 0;
    const size_t smem = (size_t)sn * 24 + (size_t)(v.threads / 32) * stack_cap * sizeof(FrontierEntry);
    const size_t limit = pass < 2 ? per_sm / v.min_blocks - 1024 : 220 * 1024;
    if (smem <= limit) return PersistShape{&v, sn, smem};
  }
  return PersistShape{nullptr, 0, 0};
}

int64_t query_capacity(int64_t pairs, const crt_query_opts& o)
{
  if (o.mode == CRT_QUERY_PLAIN) return pairs;
  const int chunk = o.chunk > 0 ? o.chunk : kDefaultChunk;
  // every resident warp may leave one partly used chunk
  const int64_t warps = (int64_t)sm_count() * 64;  // resident warps per SM at most
  return pairs + warps * chunk;
}

struct PersistScratch {
  QueryCounters* ctr;
  Hole* holes;
  Hole* sorted;
  long long* cum;
  void* sort_zero;
  SortBufs bufs;
  long long max_holes;
  JobQueue* jobs;
  size_t bytes;
};

static size_t persist_scratch_bytes(int64_t max_nq, long long max_holes, bool sort)
{
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  size_t b = al(sizeof(QueryCounters)) + 2 * al(sizeof(Hole) * max_holes) +
             al(sizeof(long long) * (max_holes + 1)) + al(kJobQueueBytes);
  if (sort) b += al(sort_zero_bytes(max_nq)) + 4 * al(4 * (size_t)std::max<int64_t>(max_nq, 1));
  return b;
}

static void persist_scratch_carve(char* base, int64_t max_nq, long long max_holes, bool sort,
                                  PersistScratch& S)
{
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  size_t off = 0;
  S.ctr = (QueryCounters*)(base + off); off += al(sizeof(QueryCounters));
  S.holes = (Hole*)(base + off); off += al(sizeof(Hole) * max_holes);
  S.sorted = (Hole*)(base + off); off += al(sizeof(Hole) * max_holes);
  S.cum = (long long*)(base + off); off += al(sizeof(long long) * (max_holes + 1));
  S.jobs = (JobQueue*)(base + off); off += al(kJobQueueBytes);
  S.sort_zero = nullptr;
  if (sort) {
    S.sort_zero = base + off; off += al(sort_zero_bytes(max_nq));
    size_t kv = al(4 * (size_t)std::max<int64_t>(max_nq, 1));
    S.bufs.keys[0] = (uint32_t*)(base + off); off += kv;
    S.bufs.keys[1] = (uint32_t*)(base + off); off += kv;
    S.bufs.vals[0] = (uint32_t*)(base + off); off += kv;
    S.bufs.vals[1] = (uint32_t*)(base + off); off += kv;
  }
  S.max_holes = max_holes;
  S.bytes = off;
}

// A persistent query is three stages on one stream, none synchronising the
// host: `pre` (reset the counters, order the windows), the traversal kernel,
// and `post` (sort the unused chunk ends, compact, write the result block).
// A plan records all three as one CUDA graph.
static void enqueue_pre(const WindowView& W, int64_t max_nq, const PersistScratch& S, bool sort,
                        cudaStream_t stream)
{
  // counters (keep nq), the job queue's ready flags and the sort's zeroed block
  cudaMemsetAsync(S.ctr, 0, offsetof(QueryCounters, nq), stream);
  cudaMemsetAsync(S.jobs, 0, kJobQueueBytes, stream);
  if (sort && max_nq > 0) {
    const int sms = sm_count();
    cudaMemsetAsync(S.sort_zero, 0, sort_zero_bytes(max_nq), stream);
    int g = (int)std::min<int64_t>(cdiv(max_nq, 256), (int64_t)sms * 4);
    window_key_kernel<<<std::max(g, 1), 256, 0, stream>>>(W, S.bufs.keys[0], sort_hist(S.sort_zero));
    sort_passes(S.bufs, W.n, S.sort_zero, stream);
    CRT_LAUNCHED(1);
  }
}

struct TraverseLaunch {
  PersistParams P;
  size_t smem;
  int grid;
  int threads;
  const void* fn;
};

static TraverseLaunch make_traverse(const TreeView& T, const WindowView& W,
                                    const PersistScratch& S, bool sort, int stage_n,
                                    int32_t* fid, int32_t* tid, long long cap, int chunk,
                                    int warps_per_cta, int parts)
{
  const TraversalShape sh = traversal_shape(T.nbox, T.fanout);
  const PersistShape ps = persist_shape(sh.stack_cap, stage_n, warps_per_cta);
  TraverseLaunch L;
  PersistParams& P = L.P;
  P.T = T;
  P.W = W;
  P.order0 = S.bufs.vals[0];
  P.order1 = S.bufs.vals[1];
  P.sort_ctrl = sort ? sort_ctrl(S.sort_zero) : nullptr;
  P.K = sh.K;
  P.stack_cap = sh.stack_cap;
  P.stage_n = ps.stage_n;
  P.parts = parts;
  P.chunk = chunk;
  P.fid = fid;
  P.tid = tid;
  P.cap = cap;
  P.ctr = S.ctr;
  P.holes = S.holes;
  P.max_holes = S.max_holes;
  P.jobs = S.jobs;
  L.smem = ps.smem;
  L.threads = ps.v->threads;
  L.fn = ps.v->fn;
  L.grid = persistent_grid(*ps.v, L.smem);
  return L;
}

static cudaError_t launch_traverse(const TraverseLaunch& L, cudaStream_t stream)
{
  ProfScope ps("traverse_persistent", stream);
  void* args[] = {(void*)&L.P};
  cudaError_t e = cudaLaunchKernel(L.fn, dim3(L.grid), dim3(L.threads), args, L.smem, stream);
  CRT_LAUNCHED(1);
  return e;
}

static void enqueue_post(const PersistScratch& S, int32_t* fid, int32_t* tid, long long cap,
                         crt_query_result* res, cudaStream_t stream)
{
  const int sms = sm_count();
  hole_sort_kernel<<<std::max(1, (int)cdiv(S.max_holes, 256)), 256, 0, stream>>>(
      S.holes, S.sorted, S.ctr, S.max_holes);
  hole_prefix_kernel<<<1, kScanThreads, 0, stream>>>(S.sorted, S.cum, S.ctr, S.max_holes);
  compact_kernel<<<sms * 4, 256, 0, stream>>>(S.sorted, S.cum, S.ctr, S.max_holes, fid, tid,
                                              cap, res);
  CRT_LAUNCHED(3);
}

// Nodes of the root and the `levels` whole tree levels below it, rounded up
// to a multiple of 4 (16-byte bulk copies; the extra nodes are staged too)
// and at most R_sz rounded down to one; 0 when staging is off or the node
// arrays are not 16-byte aligned.
static int stage_nodes_for(const crt_rtree_f32& rt, int64_t nbox, int levels)
{
  if (levels <= 0 || rt.sz <= 0) return 0;
  const void* arrs[6] = {rt.xmin, rt.ymin, rt.xmax, rt.ymax, rt.pos, rt.len};
  for (auto p : arrs)
    if (((uintptr_t)p & 15u) != 0) return 0;
  std::vector<int64_t> lv;  // leaf-parent level first, root last
  const int L = tree_levels(std::max<int64_t>(nbox, 1), std::max(rt.fanout, 2), lv);
  int64_t n = 0;
  for (int i = 0; i <= levels && i < L; i++) n += lv[L - 1 - i];
  n = std::min<int64_t>((int64_t)rt.sz & ~(int64_t)3, (n + 3) & ~(int64_t)3);
  return (int)n;
}

// The deepest staging (at most `levels` levels) whose nodes fit beside the
// warps' stacks at the variant's full occupancy.
static int fit_stage_nodes(const crt_rtree_f32& rt, int64_t nbox, int levels, int stack_cap,
                           int warps_per_cta)
{
  for (int k = levels; k > 0; k--) {
    const int sn = stage_nodes_for(rt, nbox, k);
    if (sn > 0 && persist_shape(stack_cap, sn, warps_per_cta).stage_n == sn) return sn;
  }
  return 0;
}

static long long max_holes_for(int stack_cap, int stage_n, int warps_per_cta)
{
  const PersistShape ps = persist_shape(stack_cap, stage_n, warps_per_cta);
  return (long long)persistent_grid(*ps.v, ps.smem) * (ps.v->threads / 32);
}

// Warps per window of the persistent form (0 = 1); -1 for an unsupported value.
static int window_parts(const crt_query_opts& o)
{
  const int w = o.warps_per_window <= 0 ? 1 : o.warps_per_window;
  return (w == 1 || w == 2 || w == 4) ? w : -1;
}

int query_into(const crt_rtree_f32& rt, const crt_bbox_f32& rbox, const crt_bbox_f32& qbox,
               int32_t* fid, int32_t* tid, int64_t capacity, crt_query_result* d_result,
               int64_t* d_offsets, const crt_query_opts& opts, cudaStream_t stream)
{
  NvtxRange range(opts.mode == CRT_QUERY_PLAIN ? "crt_query_plain" : "crt_query_persistent");
  if (!d_result) return fail(CRT_ERR_INVALID_ARG, "query: result block is required");
  if (qbox.sz < 0 || rbox.sz < 0 || rt.sz < 0)
    return fail(CRT_ERR_INVALID_ARG, "query: negative size");
  if (rt.sz > 0 && rt.fanout < 2) return fail(CRT_ERR_INVALID_ARG, "query: fanout < 2");
  if (capacity > 0 && !fid) return fail(CRT_ERR_INVALID_ARG, "query: null output");
  // without a window column the output is CSR: only the plain form with offsets
  if (capacity > 0 && !tid && (opts.mode != CRT_QUERY_PLAIN || !d_offsets))
    return fail(CRT_ERR_INVALID_ARG, "query: null window column outside PLAIN with offsets");
  TreeView T = make_view(rt, rbox);
  const LevelTables lt = opts.no_contain ? LevelTables() : level_tables(rt, rbox.sz);
  WindowView W{qbox.xmin, qbox.ymin, qbox.xmax, qbox.ymax, qbox.sz};
  const int64_t nq = qbox.sz;
  const TraversalShape sh = traversal_shape(rbox.sz, rt.fanout);
  const int sms = sm_count();

  if (opts.mode == CRT_QUERY_PLAIN) {
    // scratch: counters, counts, block sums (+ offsets when the caller gave none)
    const int64_t nb = std::max<int64_t>(1, cdiv(nq, kScanThreads));
    size_t bytes = 256 + 8 * (size_t)std::max<int64_t>(nq, 1) + 8 * (size_t)nb + 256 +
                   (d_offsets ? 0 : 8 * (size_t)(nq + 1) + 256) + kLevelTableBytes + 256;
    char* scr = nullptr;
    if (cudaMallocAsync((void**)&scr, bytes, stream) != cudaSuccess) {
      cudaGetLastError();
      return fail(CRT_ERR_OOM, "query: scratch allocation failed");
    }
    QueryCounters* ctr = (QueryCounters*)scr;
    long long* counts = (long long*)(scr + 256);
    long long* sums = counts + std::max<int64_t>(nq, 1);
    long long* offsets = d_offsets ? (long long*)d_offsets : sums + nb + 32;
    char* tables = (char*)(((uintptr_t)(scr + bytes - kLevelTableBytes - 256) + 255) & ~(uintptr_t)255);
    attach_levels(T, lt, tables, stream);
    cudaMemsetAsync(ctr, 0, sizeof(QueryCounters), stream);
    cudaMemsetAsync(offsets, 0, 8, stream);
    const size_t smem = (size_t)kPlainWarps * sh.stack_cap * sizeof(FrontierEntry);
    cudaFuncSetAttribute(plain_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(plain_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (nq > 0) {
      const unsigned g = (unsigned)cdiv(nq, kPlainWarps);
      {
        ProfScope ps("traverse_plain", stream);
        plain_count_kernel<<<g, kPlainWarps * 32, smem, stream>>>(T, W, sh.K, sh.stack_cap, counts,
                                                                  ctr);
      }
      scan_block_sums<<<(unsigned)nb, kScanThreads, 0, stream>>>(counts, nq, sums);
      scan_sums_kernel<<<1, kScanThreads, 0, stream>>>(sums, nb);
      scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, stream>>>(counts, nq, sums, offsets);
      {
        ProfScope ps("traverse_plain", stream);
        plain_write_kernel<<<g, kPlainWarps * 32, smem, stream>>>(T, W, sh.K, sh.stack_cap,
                                                                  offsets, fid, tid, capacity, ctr);
      }
      CRT_LAUNCHED(5);
    }
    plain_result_kernel<<<1, 1, 0, stream>>>(offsets, nq, capacity, ctr, d_result);
    CRT_LAUNCHED(1);
    cudaFreeAsync(scr, stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "query (plain)");
    return CRT_OK;
  }

  // persistent
  const bool sort = opts.sort_windows != 0 && nq > 1;
  const int stage_n = fit_stage_nodes(rt, rbox.sz, opts.stage_levels, sh.stack_cap,
                                      opts.warps_per_cta);
  const int chunk = opts.chunk >= 64 ? opts.chunk : kDefaultChunk;
  const int parts = window_parts(opts);
  if (parts < 0) return fail(CRT_ERR_INVALID_ARG, "query: warps_per_window must be 1, 2 or 4");
  if (!persist_shape(sh.stack_cap, stage_n, opts.warps_per_cta).v)
    return fail(CRT_ERR_NOT_SUPPORTED, "query: traversal stack too large");
  const long long max_holes = max_holes_for(sh.stack_cap, stage_n, opts.warps_per_cta);
  const size_t bytes = persist_scratch_bytes(nq, max_holes, sort) + kLevelTableBytes;
  char* scr = nullptr;
  if (cudaMallocAsync((void**)&scr, bytes, stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(CRT_ERR_OOM, "query: scratch allocation failed");
  }
  PersistScratch S;
  persist_scratch_carve(scr, nq, max_holes, sort, S);
  attach_levels(T, lt, scr + S.bytes, stream);
  set_nq_kernel<<<1, 1, 0, stream>>>(S.ctr, nq);
  CRT_LAUNCHED(1);
  enqueue_pre(W, nq, S, sort, stream);
  cudaError_t e = launch_traverse(make_traverse(T, W, S, sort, stage_n, fid, tid, capacity, chunk,
                                                opts.warps_per_cta, parts),
                                  stream);
  enqueue_post(S, fid, tid, capacity, d_result, stream);
  cudaFreeAsync(scr, stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  else cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "query (persistent)");
  (void)sms;
  return CRT_OK;
}

// ---------------------------------------------------------------------------
// Plain query without allocation
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory while they run: a process whose
// device memory is owned by another allocator (an engine that reserves the
// GPU's memory up front and must account for every byte), or a
// latency-critical loop that cannot afford cudaMalloc's implicit device
// synchronisation.  For them the plain query has a variant whose scratch --
// counters, per-window counts, scan partials, offsets and containment tables
// -- lives in this fixed device array instead of the stream-ordered pool.
//
// The array is a module global: every GPU that loads the library holds its
// 1 MiB until the process exits.  In host code `g_noalloc_scratch` is only a
// host-side stand-in; the device address comes from cudaGetSymbolAddress,
// looked up once per device (the first call on a device does it, with that
// device current).  All calls share the array and it keeps the last call's
// contents, so the counters are cleared on every call; calls whose work
// overlaps on the GPU (different streams, or another thread) race on it and
// must be serialised by the caller.
constexpr int64_t kNoAllocMaxWindows = 1 << 16;
constexpr size_t kNoAllocCountsOff = 256;
constexpr size_t kNoAllocSumsOff = kNoAllocCountsOff + 8 * (size_t)kNoAllocMaxWindows;
constexpr size_t kNoAllocOffsetsOff = kNoAllocSumsOff + 8 * 256;
constexpr size_t kNoAllocTablesOff =
    (kNoAllocOffsetsOff + 8 * (size_t)(kNoAllocMaxWindows + 1) + 255) / 256 * 256;
constexpr size_t kNoAllocBytes = kNoAllocTablesOff + (kLevelTableBytes + 255) / 256 * 256;
static_assert(kNoAllocBytes <= (1u << 20) + 4096, "no-alloc scratch stays near 1 MiB");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

static int noalloc_scratch_address(char** out)
{
  static std::mutex mu;
  static std::vector<std::pair<int, char*>> addr;  // device -> device address of the array
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "query_plain_noalloc: cudaGetDevice");
  std::lock_guard<std::mutex> lk(mu);
  for (auto& a : addr)
    if (a.first == dev) {
      *out = a.second;
      return CRT_OK;
    }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "query_plain_noalloc: cudaGetSymbolAddress");
  addr.emplace_back(dev, (char*)p);
  *out = (char*)p;
  return CRT_OK;
}

int query_plain_noalloc(const crt_rtree_f32& rt, const crt_bbox_f32& rbox,
                        const crt_bbox_f32& qbox, int32_t* fid, int32_t* tid, int64_t capacity,
                        crt_query_result* d_result, cudaStream_t stream)
{
  if (!d_result) return fail(CRT_ERR_INVALID_ARG, "query_plain_noalloc: result block is required");
  if (qbox.sz < 0 || rbox.sz < 0 || rt.sz < 0 || capacity < 0)
    return fail(CRT_ERR_INVALID_ARG, "query_plain_noalloc: negative size");
  if (qbox.sz > kNoAllocMaxWindows)
    return fail(CRT_ERR_INVALID_ARG,
                "query_plain_noalloc: at most 65536 windows per call (fixed scratch); "
                "split the batch or use crt_query_into_f32");
  if (rt.sz > 0 && rt.fanout < 2) return fail(CRT_ERR_INVALID_ARG, "query_plain_noalloc: fanout < 2");
  if (capacity > 0 && (!fid || !tid))
    return fail(CRT_ERR_INVALID_ARG, "query_plain_noalloc: null output");
  char* scr = nullptr;
  int rc = noalloc_scratch_address(&scr);
  if (rc != CRT_OK) return rc;
  TreeView T = make_view(rt, rbox);
  attach_levels(T, level_tables(rt, rbox.sz), scr + kNoAllocTablesOff, stream);
  WindowView W{qbox.xmin, qbox.ymin, qbox.xmax, qbox.ymax, qbox.sz};
  const int64_t nq = qbox.sz;
  const TraversalShape sh = traversal_shape(rbox.sz, rt.fanout);
  QueryCounters* ctr = (QueryCounters*)scr;
  long long* counts = (long long*)(scr + kNoAllocCountsOff);
  long long* sums = (long long*)(scr + kNoAllocSumsOff);
  long long* offsets = (long long*)(scr + kNoAllocOffsetsOff);
  const int64_t nb = std::max<int64_t>(1, cdiv(nq, kScanThreads));
  cudaMemsetAsync(ctr, 0, sizeof(QueryCounters), stream);
  cudaMemsetAsync(offsets, 0, 8, stream);
  const size_t smem = (size_t)kPlainWarps * sh.stack_cap * sizeof(FrontierEntry);
  cudaFuncSetAttribute(plain_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(plain_write_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (nq > 0) {
    const unsigned g = (unsigned)cdiv(nq, kPlainWarps);
    plain_count_kernel<<<g, kPlainWarps * 32, smem, stream>>>(T, W, sh.K, sh.stack_cap, counts, ctr);
    scan_block_sums<<<(unsigned)nb, kScanThreads, 0, stream>>>(counts, nq, sums);
    scan_sums_kernel<<<1, kScanThreads, 0, stream>>>(sums, nb);
    scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, stream>>>(counts, nq, sums, offsets);
    plain_write_kernel<<<g, kPlainWarps * 32, smem, stream>>>(T, W, sh.K, sh.stack_cap, offsets,
                                                              fid, tid, capacity, ctr);
    CRT_LAUNCHED(5);
  }
  plain_result_kernel<<<1, 1, 0, stream>>>(offsets, nq, capacity, ctr, d_result);
  CRT_LAUNCHED(1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "query_plain_noalloc");
  return CRT_OK;
}

int query_stats(const crt_rtree_f32& rt, const crt_bbox_f32& rbox, const crt_bbox_f32& qbox,
                int64_t* d_hits, int64_t* d_tested, int64_t* h_totals, cudaStream_t stream)
{
  TreeView T = make_view(rt, rbox);
  WindowView W{qbox.xmin, qbox.ymin, qbox.xmax, qbox.ymax, qbox.sz};
  const TraversalShape sh = traversal_shape(rbox.sz, rt.fanout);
  char* scr = nullptr;
  if (cudaMallocAsync((void**)&scr, 1024 + kLevelTableBytes, stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(CRT_ERR_OOM, "query_stats: scratch allocation failed");
  }
  QueryCounters* ctr = (QueryCounters*)scr;
  unsigned long long* tot = (unsigned long long*)(scr + 256);  // [3] box-by-box, [3] containment
  cudaMemsetAsync(scr, 0, 1024, stream);
  const size_t smem = (size_t)kPlainWarps * sh.stack_cap * sizeof(FrontierEntry);
  cudaFuncSetAttribute(stats_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(stats_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (qbox.sz > 0) {
    const unsigned g = (unsigned)cdiv(qbox.sz, kPlainWarps);
    // the reference algorithm: every leaf box under an intersecting node is tested
    stats_kernel<false><<<g, kPlainWarps * 32, smem, stream>>>(
        T, W, sh.K, sh.stack_cap, (long long*)d_hits, (long long*)d_tested, tot, ctr);
    // this library's: contained subtrees are emitted by slot range
    TreeView Tc = T;
    attach_levels(Tc, level_tables(rt, rbox.sz), scr + 1024, stream);
    stats_kernel<true><<<g, kPlainWarps * 32, smem, stream>>>(Tc, W, sh.K, sh.stack_cap, nullptr,
                                                              nullptr, tot + 3, ctr);
    CRT_LAUNCHED(2);
  }
  unsigned long long h[6] = {0, 0, 0, 0, 0, 0};
  int err = 0;
  cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(&err, &ctr->error, sizeof(int), cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(scr, stream);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "query_stats");
  if (err) return fail(err, "query_stats: device-side error");
  if (h[0] != h[3]) return fail(CRT_ERR_CUDA, "query_stats: the two traversals disagree on the pair count");
  if (h_totals) {
    h_totals[0] = (int64_t)h[0];  // hits
    h_totals[1] = (int64_t)h[1];  // leaf boxes tested box by box
    h_totals[2] = (int64_t)h[4];  // leaf boxes tested with containment
    h_totals[3] = (int64_t)h[5];  // hits emitted by contained slot ranges
  }
  return CRT_OK;
}

// ---------------------------------------------------------------------------
// Persistent plan captured in a CUDA graph
// ---------------------------------------------------------------------------
// The whole query -- counter reset, window ordering, the persistent traversal
// and the output compaction -- is one graph, replayed with one
// cudaGraphLaunch.  Two event-record nodes bracket the traversal: they record
// the plan's own events, or, while kernel timing is on, a fresh event pair
// per launch (set into the instantiated graph before the launch), so the
// traversal's duration is measured inside the replay.
struct Plan {
  TreeView T;
  WindowView W;
  int64_t max_nq;
  PersistScratch S;
  char* scratch = nullptr;
  bool sort;
  int stage_n;
  int chunk;
  int32_t* fid;
  int32_t* tid;
  long long cap;
  crt_query_result* res;
  TraverseLaunch traverse;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t own[2] = {nullptr, nullptr};         // recorded when timing is off
  cudaGraphNode_t ev_node[2] = {nullptr, nullptr};  // the event-record nodes
};

int plan_destroy(void* hp);

// The event-record node of `graph` that records `ev`.
static cudaGraphNode_t find_event_node(cudaGraph_t graph, cudaEvent_t ev)
{
  size_t n = 0;
  if (cudaGraphGetNodes(graph, nullptr, &n) != cudaSuccess || n == 0) return nullptr;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) return nullptr;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    cudaEvent_t e = nullptr;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeEventRecord &&
        cudaGraphEventRecordNodeGetEvent(nd, &e) == cudaSuccess && e == ev)
      return nd;
  }
  return nullptr;
}

int plan_create(const crt_rtree_f32& rt, const crt_bbox_f32& rbox, const crt_bbox_f32& qbox,
                int64_t max_nq, int32_t* fid, int32_t* tid, int64_t capacity,
                crt_query_result* res, const crt_query_opts& opts, cudaStream_t stream,
                void** out)
{
  if (!res || max_nq < 0) return fail(CRT_ERR_INVALID_ARG, "plan: bad arguments");
  Plan* p = new Plan();
  p->T = make_view(rt, rbox);
  p->W = WindowView{qbox.xmin, qbox.ymin, qbox.xmax, qbox.ymax, max_nq};
  p->max_nq = max_nq;
  p->sort = opts.sort_windows != 0 && max_nq > 1;
  p->chunk = opts.chunk >= 64 ? opts.chunk : kDefaultChunk;
  const int parts = window_parts(opts);
  if (parts < 0) {
    delete p;
    return fail(CRT_ERR_INVALID_ARG, "plan: warps_per_window must be 1, 2 or 4");
  }
  p->fid = fid;
  p->tid = tid;
  p->cap = capacity;
  p->res = res;
  const TraversalShape sh = traversal_shape(rbox.sz, rt.fanout);
  p->stage_n = fit_stage_nodes(rt, rbox.sz, opts.stage_levels, sh.stack_cap, opts.warps_per_cta);
  if (!persist_shape(sh.stack_cap, p->stage_n, opts.warps_per_cta).v) {
    delete p;
    return fail(CRT_ERR_NOT_SUPPORTED, "plan: traversal stack too large");
  }
  const long long max_holes = max_holes_for(sh.stack_cap, p->stage_n, opts.warps_per_cta);
  const size_t bytes = persist_scratch_bytes(max_nq, max_holes, p->sort) + kLevelTableBytes;
  if (cudaMalloc((void**)&p->scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    delete p;
    return fail(CRT_ERR_OOM, "plan: scratch allocation failed");
  }
  persist_scratch_carve(p->scratch, max_nq, max_holes, p->sort, p->S);
  if (!opts.no_contain) attach_levels(p->T, level_tables(rt, rbox.sz), p->scratch + p->S.bytes, stream);
  cudaMemsetAsync(p->S.ctr, 0, sizeof(QueryCounters), stream);
  set_nq_kernel<<<1, 1, 0, stream>>>(p->S.ctr, max_nq);
  CRT_LAUNCHED(1);
  p->traverse = make_traverse(p->T, p->W, p->S, p->sort, p->stage_n, fid, tid, capacity, p->chunk,
                              opts.warps_per_cta, parts);
  // capture the whole query on a private stream; a window-sorting plan
  // orders exactly max_nq windows, so it only runs with nq == max_nq
  // (plan_set_nq enforces it); without sorting the kernel reads the live
  // count from ctr->nq
  cudaStream_t cs = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&p->own[0]);
  if (e == cudaSuccess) e = cudaEventCreate(&p->own[1]);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue_pre(p->W, max_nq, p->S, p->sort, cs);
    cudaError_t le = cudaEventRecordWithFlags(p->own[0], cs, cudaEventRecordExternal);
    if (le == cudaSuccess) le = launch_traverse(p->traverse, cs);
    if (le == cudaSuccess) le = cudaEventRecordWithFlags(p->own[1], cs, cudaEventRecordExternal);
    enqueue_post(p->S, fid, tid, capacity, res, cs);
    e = cudaStreamEndCapture(cs, &p->graph);
    if (e == cudaSuccess && le != cudaSuccess) e = le;
  }
  if (e == cudaSuccess) {
    p->ev_node[0] = find_event_node(p->graph, p->own[0]);
    p->ev_node[1] = find_event_node(p->graph, p->own[1]);
    if (!p->ev_node[0] || !p->ev_node[1]) e = cudaErrorInvalidValue;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
  cudaStreamSynchronize(stream);
  if (cs) cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    cudaGetLastError();
    plan_destroy(p);
    return cuda_fail(e, "plan: graph capture");
  }
  *out = p;
  return CRT_OK;
}

int plan_set_nq(void* hp, int64_t nq, cudaStream_t stream)
{
  Plan* p = (Plan*)hp;
  if (nq < 0 || nq > p->max_nq) return fail(CRT_ERR_INVALID_ARG, "plan: nq out of range");
  if (p->sort && nq != p->max_nq)
    return fail(CRT_ERR_NOT_SUPPORTED, "plan: a window-sorting plan runs exactly max_nq windows");
  set_nq_kernel<<<1, 1, 0, stream>>>(p->S.ctr, nq);
  CRT_LAUNCHED(1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CRT_OK : cuda_fail(e, "plan_set_nq");
}

int plan_launch(void* hp, cudaStream_t stream)
{
  NvtxRange range("crt_plan_launch");
  Plan* p = (Plan*)hp;
  cudaEvent_t a = p->own[0], b = p->own[1];
  cudaError_t e = cudaSuccess;
  if (prof_register("traverse_persistent", &a, &b)) {
    // this launch records a fresh pair (read and destroyed when the timings
    // are collected); the nodes go back to the plan's own events right after,
    // so the instantiated graph never refers to a destroyed event
    e = cudaGraphExecEventRecordNodeSetEvent(p->exec, p->ev_node[0], a);
    if (e == cudaSuccess) e = cudaGraphExecEventRecordNodeSetEvent(p->exec, p->ev_node[1], b);
    if (e == cudaSuccess) e = cudaGraphLaunch(p->exec, stream);
    cudaError_t r = cudaGraphExecEventRecordNodeSetEvent(p->exec, p->ev_node[0], p->own[0]);
    if (r == cudaSuccess) r = cudaGraphExecEventRecordNodeSetEvent(p->exec, p->ev_node[1], p->own[1]);
    if (e == cudaSuccess) e = r;
  } else {
    e = cudaGraphLaunch(p->exec, stream);
  }
  if (e != cudaSuccess) return cuda_fail(e, "plan_launch");
  // window keys, sort plan, four sort passes; the traversal; hole sort,
  // prefix and compaction
  CRT_LAUNCHED((p->sort ? 6 : 0) + 1 + 3);
  return CRT_OK;
}

int plan_destroy(void* hp)
{
  Plan* p = (Plan*)hp;
  if (!p) return CRT_OK;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  for (auto ev : p->own)
    if (ev) cudaEventDestroy(ev);
  if (p->scratch) cudaFree(p->scratch);
  delete p;
  return CRT_OK;
}

}  // namespace crt
