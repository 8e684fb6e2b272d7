// Serving loop: continuous batching of window-query requests against several
// device-resident trees.  No reference counterpart (the reference answers one
// batch per call, src/rtree_bfs_frontier.cuh:292); the per-window traversal is
// the same as the batch query's.
//
// Device side: one persistent kernel.  Every admitted request owns a
// contiguous range of window tickets; warps take tickets from one atomic
// counter, bounded by the `published` count the host raises as it admits
// requests.  A warp finds its ticket's request through the descriptor ring
// (request r lives in slot r % slots, tagged with its sequence number r),
// traverses that request's tree for that window, stages the hits in shared
// memory and flushes them with one atomicAdd per 256 pairs into the request's
// own output range, so each request's output is dense.  The warp that
// finishes a request's last window writes its pair count and sequence number
// to pinned host memory, which the host polls: no stream synchronisation per
// request.  Every wait is bounded: an idle warp gives up after
// `device_wait_us`, records CRT_ERR_DEVICE_TIMEOUT and returns.
//
// Host side: submit() checks the request's HBM footprint (windows + output
// estimate) against a fixed device arena and copies its windows in, or
// answers CRT_ERR_BUSY.  A dispatcher thread publishes admitted requests in
// batches (descriptors, counters, then the new ticket limit), keeps the
// kernel running while there is work, stops it after `idle_ms` without work,
// collects completions, and re-runs a request whose output estimate was too
// small with its exact size (overflow-and-retry).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.h"
#include "traverse.cuh"

namespace crt {

// ---------------------------------------------------------------------------
// Device structures
// ---------------------------------------------------------------------------
struct SrvTree {
  const float* nxmin;
  const float* nymin;
  const float* nxmax;
  const float* nymax;
  const int* npos;
  const int* nlen;
  const float* bxmin;
  const float* bymin;
  const float* bxmax;
  const float* bymax;
  const int* bid;
  int rsz;
  int fanout;
  int nbox;
  int K;
  int nlev;  // containment tables (nlev == 0: off)
  const int* lvl_first;
  const long long* lvl_span;
  const int* lvl_odd;  // set: some box is not ordinary (shortcut off)
};

struct SrvDesc {
  long long seq;  // request sequence number r (slot r % slots)
  long long base; // first ticket
  long long nq;
  const float* x0;
  const float* y0;
  const float* x1;
  const float* y1;
  int32_t* fid;
  int32_t* tid;
  long long cap;
  int tree;
  int pad;
};

struct SrvCtr {
  unsigned long long next;  // output slots reserved (= pairs found)
  unsigned long long done;  // windows finished
};

struct SrvDone {  // pinned host memory, written by the device
  volatile long long seq;
  volatile long long count;
};

struct SrvState {
  unsigned long long next_ticket;
  unsigned long long published;
  long long r_start;  // oldest request a fresh warp may meet
  int shutdown;
  int error;
  unsigned long long reserved;
};

// Control words in mapped (zero-copy) host memory: the host stops the loop
// and reads its error status with plain loads and stores, no CUDA call, so
// neither waits behind other work queued on the device.
struct SrvCtl {
  int shutdown;
  int error;
};

constexpr int kSrvThreads = 256;
constexpr int kSrvWarps = kSrvThreads / 32;
constexpr int kStage = 256;  // staged pairs per warp

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p)
{
  return *(const volatile unsigned long long*)p;
}

struct StagedEmit {
  static constexpr bool kCountsTests = false;
  int32_t* s_fid;  // this warp's staging, kStage entries
  int32_t* s_tid;
  int n = 0;
  int q = 0;
  SrvCtr* ctr;
  int32_t* fid;
  int32_t* tid;
  long long cap;
  __device__ __forceinline__ void flush()
  {
    const int lane = (int)lane_id();
    __syncwarp();
    if (n > 0) {
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(&ctr->next, (unsigned long long)n);
      b = __shfl_sync(0xffffffffu, b, 0);
      for (int i = lane; i < n; i += 32) {
        const long long slot = (long long)b + i;
        if (slot < cap) {
          fid[slot] = s_fid[i];
          tid[slot] = s_tid[i];
        }
      }
      n = 0;
    }
    __syncwarp();
  }
  __device__ __forceinline__ void begin(int qq) { q = qq; }
  __device__ __forceinline__ void small_ranges(const int* bid, bool mine, long long first, int count)
  {
    emit_small_ranges(*this, bid, mine, first, count);
  }
  __device__ __forceinline__ void big_ranges(const int* bid, bool mine, long long first, long long count)
  {
    emit_ranges_each(*this, bid, mine, first, count);
  }
  // A contained subtree's ids go straight to an exact reservation.
  __device__ __forceinline__ void range(const int* bid, long long first, long long count)
  {
    if (count < kStage) {
      emit_range_default(*this, bid, first, count);
      return;
    }
    unsigned long long b = 0;
    if (lane_id() == 0) b = atomicAdd(&ctr->next, (unsigned long long)count);
    b = __shfl_sync(0xffffffffu, b, 0);
    copy_range(bid, first, count, fid, tid, (long long)b, cap, q);
  }
  __device__ __forceinline__ void operator()(bool hit, int id)
  {
    const uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (!m) return;
    const int c = __popc(m);
    if (n + c > kStage) flush();
    if (hit) {
      const int i = n + __popc(m & lanemask_lt());
      s_fid[i] = id;
      s_tid[i] = q;
    }
    n += c;
  }
};

// Descriptors and windows are rewritten between requests (slots and arena
// space are reused), so they are read through L2 only, never a stale L1 line.
__device__ __forceinline__ void load_desc(const SrvDesc* p, SrvDesc& d)
{
  const long long* src = (const long long*)p;
  long long* dst = (long long*)&d;
#pragma unroll
  for (int i = 0; i < (int)(sizeof(SrvDesc) / 8); i++) dst[i] = __ldcg(src + i);
}

// Three CTAs per SM (at most 85 registers): at two the loop has a third
// fewer warps to hide the traversal's memory latency with.
__global__ void __launch_bounds__(kSrvThreads, 3)
    serve_kernel(SrvState* st, SrvCtl* ctl, const SrvTree* __restrict__ trees,
                 const SrvDesc* descs, SrvCtr* ctrs, SrvDone* done_host, int slots, int stack_cap,
                 unsigned long long wait_ns)
{
  extern __shared__ int smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = (int)lane_id();
  FrontierEntry* stack = (FrontierEntry*)smem + warp * stack_cap;
  int32_t* stage = (int32_t*)((FrontierEntry*)smem + kSrvWarps * stack_cap) + warp * 2 * kStage;
  long long r = st->r_start;
  while (true) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&st->next_ticket, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    // wait (bounded) until ticket t is published
    int state = 0;  // 0 work, 1 shutdown, 2 timeout
    if (lane == 0) {
      unsigned long long t0 = 0;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
      unsigned sleep = 32;
      while (t >= ld_volatile_u64(&st->published)) {
        if (*(volatile int*)&st->shutdown) { state = 1; break; }
        // one warp polls the host's mapped stop flag (a read across the
        // host link) and relays it to the device word the others poll
        if (blockIdx.x == 0 && warp == 0 && *(volatile int*)&ctl->shutdown) {
          *(volatile int*)&st->shutdown = 1;
          __threadfence();
          state = 1;
          break;
        }
        unsigned long long now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if (now - t0 > wait_ns) { state = 2; break; }
        __nanosleep(sleep);
        sleep = min(sleep * 2, 4096u);
      }
      __threadfence();
    }
    state = __shfl_sync(0xffffffffu, state, 0);
    if (state == 1) break;
    if (state == 2) {
      raise_error(&st->error, CRT_ERR_DEVICE_TIMEOUT);
      break;
    }
    // locate the request holding ticket t (requests are published in ticket
    // order; a slot tagged with a later sequence number belongs to a request
    // that reused the slot after request r completed)
    SrvDesc d;
    bool found = false;
    for (int hops = 0; hops <= 2 * slots; hops++) {
      load_desc(&descs[r % slots], d);
      if (d.seq == r && (long long)t < d.base + d.nq) { found = true; break; }
      if (d.seq < r) break;  // unpublished: cannot happen for t < published
      ++r;
    }
    if (!found) {
      raise_error(&st->error, CRT_ERR_NOT_SUPPORTED);
      break;
    }
    const long long w = (long long)t - d.base;
    const SrvTree& tr = trees[d.tree];
    TreeView T;
    T.nxmin = tr.nxmin; T.nymin = tr.nymin; T.nxmax = tr.nxmax; T.nymax = tr.nymax;
    T.npos = tr.npos; T.nlen = tr.nlen; T.rsz = tr.rsz; T.fanout = tr.fanout;
    T.bxmin = tr.bxmin; T.bymin = tr.bymin; T.bxmax = tr.bxmax; T.bymax = tr.bymax;
    T.bid = tr.bid; T.nbox = tr.nbox;
    T.nlev = tr.nlev; T.lvl_first = tr.lvl_first; T.lvl_span = tr.lvl_span;
    T.lvl_odd = tr.lvl_odd;
    int lg, lc;
    lane_map(T.fanout, lg, lc);
    SrvCtr* ctr = &ctrs[r % slots];
    StagedEmit emit;
    emit.s_fid = stage;
    emit.s_tid = stage + kStage;
    emit.ctr = ctr;
    emit.fid = d.fid;
    emit.tid = d.tid;
    emit.cap = d.cap;
    emit.begin((int)w);
    NodeCache C{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
    traverse(T, C, tr.K, lg, lc, __ldcg(d.x0 + w), __ldcg(d.y0 + w), __ldcg(d.x1 + w),
             __ldcg(d.y1 + w), stack, stack_cap, emit, &st->error);
    emit.flush();
    if (lane == 0) {
      __threadfence();
      const unsigned long long fin = atomicAdd(&ctr->done, 1ull) + 1;
      if ((long long)fin == d.nq) {
        __threadfence();
        const unsigned long long count = ld_volatile_u64(&ctr->next);
        done_host[r % slots].count = (long long)count;
        __threadfence_system();
        done_host[r % slots].seq = r;
        __threadfence_system();
      }
    }
    __syncwarp();
  }
  // a warp that leaves on an error reports it to the host's mapped word
  if (lane == 0) {
    const int e = *(volatile int*)&st->error;
    if (e) {
      *(volatile int*)&ctl->error = e;
      __threadfence_system();
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator over a device arena (offsets, 256-byte granules).
class Arena {
 public:
  void init(size_t bytes) { free_[0] = bytes; }
  bool alloc(size_t bytes, size_t& off)
  {
    bytes = (bytes + 255) / 256 * 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        off = it->first;
        size_t rest = it->second - bytes;
        size_t at = it->first + bytes;
        free_.erase(it);
        if (rest) free_[at] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes)
  {
    if (bytes == 0) return;
    bytes = (bytes + 255) / 256 * 256;
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t used_ = 0;
};

struct Request {
  long long id;
  int tree;
  long long nq;
  size_t win_off = 0, win_bytes = 0;
  size_t out_off = 0, out_bytes = 0;
  long long cap = 0;
  long long seq = -1;  // sequence number while published
  double t_submit = 0;
  int retries = 0;
  double predicted = 0;  // area-based pair estimate (0: none)
  // a re-run's windows, held on the host while it waits for arena space
  std::shared_ptr<std::vector<float>> host_windows;
};

size_t granules(size_t bytes) { return (bytes + 255) / 256 * 256; }

// Host-side statistics of a tree for output estimates.
struct TreeStats {
  double rx1 = 0, ry1 = 0, rx2 = 0, ry2 = 0;  // root MBR
  double density = 0;                          // boxes per unit area
  double mbw = 0, mbh = 0;                     // mean box extents (sample)
  double corr = 1.0;                           // EMA of actual / predicted pairs
};

}  // namespace

struct Server {
  crt_server_opts opts{};
  int device = 0;
  cudaStream_t compute = nullptr, copy = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  Arena alloc;
  // device tables
  SrvTree* d_trees = nullptr;
  std::vector<SrvTree> trees;
  std::vector<char*> tables;  // containment tables, one allocation per tree
  std::vector<double> tree_ppw;  // pairs per window estimate per tree
  std::vector<TreeStats> tree_stats;
  std::deque<Request> retry_wait;  // re-runs waiting for arena space
  SrvDesc* d_descs = nullptr;
  SrvCtr* d_ctrs = nullptr;
  SrvState* d_state = nullptr;
  SrvDone* h_done = nullptr;  // pinned, mapped
  SrvDone* d_done = nullptr;
  SrvDesc* h_desc_stage = nullptr;  // pinned staging for descriptor uploads
  // Copies made while the device loop may run go through pinned host memory
  // (asynchronous on their stream; a pageable copy is staged by the host
  // thread and returns only when it is done).  The loop's stop flag and error
  // status are mapped words (SrvCtl) that need no copy at all: any stream
  // operation can wait behind other work queued on the device (a client's
  // kernel queued behind the loop, in a hardware queue the streams share),
  // and the dispatcher must still be able to stop the loop then.
  struct Mailbox {
    SrvState launch;
    unsigned long long published;
  };
  Mailbox* h_box = nullptr;             // pinned: the dispatcher's words
  SrvCtl* h_ctl = nullptr;              // mapped: stop flag and error status
  SrvCtl* d_ctl = nullptr;
  static constexpr size_t kBounce = 8u << 20;
  char* h_bounce = nullptr;             // pinned bounce buffer: the dispatcher
  char* h_bounce_submit = nullptr;      // pinned bounce buffer: submitters
  std::mutex submit_mu;                 // guards h_bounce_submit and `upload`
  cudaStream_t upload = nullptr;        // submitters' window copies
  int slots = 0;
  int stack_cap = 32;
  // bookkeeping
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request> pending;                    // admitted, not yet published
  std::unordered_map<long long, Request> flight;  // published, by seq
  std::deque<crt_server_completion> completed;
  std::unordered_map<long long, Request> finished;  // by request id, until release
  long long next_id = 1;
  long long next_seq = 0;
  unsigned long long published = 0;
  long long oldest_seq = 0;
  bool kernel_running = false;
  bool stop = false;
  int device_error = 0;
  std::thread worker;
  std::atomic<long long> n_submitted{0}, n_completed{0}, n_retried{0};
  double last_work = 0;
  double last_err_check = 0;

  size_t smem() const
  {
    return (size_t)kSrvWarps * stack_cap * sizeof(FrontierEntry) + (size_t)kSrvWarps * 2 * kStage * 4;
  }
  // All CTA slots but one SM's worth: a loop that held every slot would keep
  // any other kernel of the process from starting until it stops.  The block
  // scheduler spreads the CTAs, so a few SMs keep a free slot, on which a
  // kernel of another stream runs -- when that stream has a hardware queue of
  // its own (CUDA_DEVICE_MAX_CONNECTIONS); one that shares the loop's queue
  // waits for the loop to stop, idle_ms after its last request.
  int grid() const
  {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel, kSrvThreads, smem());
    per_sm = std::max(1, per_sm);
    return std::max(1, per_sm * sm_count() - per_sm);
  }

  // Copies `bytes` between pageable host memory and the device in kBounce
  // pieces through the pinned buffer `buf`, on stream `st`.
  static cudaError_t bounce_copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                                 char* buf, cudaStream_t st)
  {
    for (size_t off = 0; off < bytes; off += kBounce) {
      const size_t n = std::min(kBounce, bytes - off);
      cudaError_t e;
      if (kind == cudaMemcpyHostToDevice) {
        std::memcpy(buf, (const char*)src + off, n);
        e = cudaMemcpyAsync((char*)dst + off, buf, n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      } else {
        e = cudaMemcpyAsync(buf, (const char*)src + off, n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) std::memcpy((char*)dst + off, buf, n);
      }
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  // The device loop's last error status (the mapped word).
  int read_device_error()
  {
    std::atomic_thread_fence(std::memory_order_acquire);
    return *(volatile int*)&h_ctl->error;
  }

  void launch_kernel()
  {
    // reset the ticket counter to the published count: tickets taken past it
    // by the previous instance carried no work
    SrvState& s = h_box->launch;
    s = SrvState{};
    s.next_ticket = published;
    s.published = published;
    s.r_start = oldest_seq;
    cudaMemcpyAsync(d_state, &s, sizeof(s), cudaMemcpyHostToDevice, copy);
    cudaStreamSynchronize(copy);
    *(volatile int*)&h_ctl->shutdown = 0;
    *(volatile int*)&h_ctl->error = 0;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    cudaFuncSetAttribute(serve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
    serve_kernel<<<grid(), kSrvThreads, smem(), compute>>>(
        d_state, d_ctl, d_trees, d_descs, d_ctrs, d_done, slots, stack_cap,
        (unsigned long long)opts.device_wait_us * 1000ull);
    CRT_LAUNCHED(1);
    kernel_running = true;
  }

  void stop_kernel()
  {
    *(volatile int*)&h_ctl->shutdown = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    cudaStreamSynchronize(compute);
    const int err = read_device_error();
    if (err) device_error = err;
    kernel_running = false;
  }

  // Publish every pending request (lock held by the caller).
  void publish_locked()
  {
    if (pending.empty()) return;
    std::vector<Request> batch(pending.begin(), pending.end());
    pending.clear();
    for (size_t i = 0; i < batch.size(); i++) {
      Request& q = batch[i];
      q.seq = next_seq++;
      SrvDesc& d = h_desc_stage[i];
      d.seq = q.seq;
      d.base = (long long)published;
      d.nq = q.nq;
      const float* w = (const float*)(arena + q.win_off);
      d.x0 = w;
      d.y0 = w + q.nq;
      d.x1 = w + 2 * q.nq;
      d.y1 = w + 3 * q.nq;
      d.fid = (int32_t*)(arena + q.out_off);
      d.tid = d.fid + q.cap;
      d.cap = q.cap;
      d.tree = q.tree;
      d.pad = 0;
      published += (unsigned long long)q.nq;
      const int slot = (int)(q.seq % slots);
      cudaMemcpyAsync(d_descs + slot, &d, sizeof(SrvDesc), cudaMemcpyHostToDevice, copy);
      cudaMemsetAsync(d_ctrs + slot, 0, sizeof(SrvCtr), copy);
      h_done[slot].seq = -1;
      flight.emplace(q.seq, q);
    }
    cudaStreamSynchronize(copy);  // descriptors and counters are in device memory
    h_box->published = published;
    cudaMemcpyAsync(&d_state->published, &h_box->published, sizeof(published),
                    cudaMemcpyHostToDevice, copy);
    cudaStreamSynchronize(copy);
  }

  // Expected pairs of a window batch against a tree: windows clipped to the
  // tree's root MBR and grown by the mean box extents, times the box density,
  // times the tree's learned correction.
  double predict_locked(int tree, const float* x1, const float* y1, const float* x2,
                        const float* y2, long long nq) const
  {
    const TreeStats& t = tree_stats[tree];
    if (t.density <= 0) return 0;
    double sum = 0;
    for (long long i = 0; i < nq; i++) {
      const double w = std::min<double>(x2[i] + t.mbw, t.rx2) - std::max<double>(x1[i] - t.mbw, t.rx1);
      const double h = std::min<double>(y2[i] + t.mbh, t.ry2) - std::max<double>(y1[i] - t.mbh, t.ry1);
      if (w > 0 && h > 0) sum += w * h;
    }
    return sum * t.density;
  }

  void learn_locked(const Request& q, long long count)
  {
    tree_ppw[q.tree] = 0.8 * tree_ppw[q.tree] + 0.2 * ((double)count / std::max(1LL, q.nq));
    if (q.predicted > 0) {
      TreeStats& t = tree_stats[q.tree];
      const double r = std::min(16.0, std::max(1.0 / 16, (double)count / q.predicted));
      t.corr = 0.7 * t.corr + 0.3 * r;
    }
  }

  void finish_locked(Request& q, long long count, int status)
  {
    crt_server_completion c{};
    c.request_id = q.id;
    c.tree_id = q.tree;
    c.status = status;
    c.nq = q.nq;
    c.count = count;
    c.d_fid = q.out_bytes ? (int32_t*)(arena + q.out_off) : nullptr;
    c.d_tid = q.out_bytes ? c.d_fid + q.cap : nullptr;
    c.submit_time_s = q.t_submit;
    c.complete_time_s = now_s();
    c.retries = q.retries;
    completed.push_back(c);
    finished.emplace(q.id, q);
    n_completed++;
  }

  void loop()
  {
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
      // collect completions
      bool progressed = false;
      for (auto it = flight.begin(); it != flight.end();) {
        Request& q = it->second;
        const int slot = (int)(q.seq % slots);
        if (h_done[slot].seq == q.seq) {
          const long long count = h_done[slot].count;
          progressed = true;
          learn_locked(q, count);
          if (count > q.cap) {
            // overflow-and-retry: re-run with the exact size.  The windows
            // move to the host and both of the request's blocks are freed,
            // so the re-run needs one block (windows + exact output) that
            // fits as soon as the arena drains: waiting for an output block
            // beside a window block left in the middle of the arena could
            // wait forever.
            n_retried++;
            Request rq = q;
            rq.host_windows = std::make_shared<std::vector<float>>((size_t)q.nq * 4);
            cudaError_t ce = bounce_copy(rq.host_windows->data(), arena + q.win_off,
                                         (size_t)q.nq * 16, cudaMemcpyDeviceToHost, h_bounce, copy);
            alloc.release(q.out_off, q.out_bytes);
            alloc.release(q.win_off, q.win_bytes);
            rq.cap = count;
            rq.out_bytes = (size_t)count * 8;
            rq.win_off = rq.out_off = 0;
            rq.retries++;
            rq.seq = -1;
            if (ce != cudaSuccess || granules(rq.win_bytes) + granules(rq.out_bytes) > arena_bytes) {
              // never fits (or the windows could not be saved): fail it
              if (ce != cudaSuccess) cudaGetLastError();
              rq.win_bytes = rq.out_bytes = 0;
              rq.cap = 0;
              rq.host_windows.reset();
              finish_locked(rq, count, ce != cudaSuccess ? CRT_ERR_CUDA : CRT_ERR_OOM);
            } else {
              retry_wait.push_back(rq);
            }
          } else {
            finish_locked(q, count, CRT_OK);
          }
          it = flight.erase(it);
        } else {
          ++it;
        }
      }
      if (!flight.empty()) {
        long long m = flight.begin()->first;
        for (auto& kv : flight) m = std::min(m, kv.first);
        oldest_seq = m;
      } else {
        oldest_seq = next_seq;
      }
      // re-runs waiting for arena space, oldest first: one block holds the
      // windows (copied back in) and the exact output
      while (!retry_wait.empty()) {
        Request& f = retry_wait.front();
        size_t off;
        if (!alloc.alloc(granules(f.win_bytes) + granules(f.out_bytes), off)) break;
        Request rq = f;
        retry_wait.pop_front();
        rq.win_off = off;
        rq.out_off = off + granules(rq.win_bytes);
        cudaError_t ce = bounce_copy(arena + rq.win_off, rq.host_windows->data(),
                                     (size_t)rq.nq * 16, cudaMemcpyHostToDevice, h_bounce, copy);
        rq.host_windows.reset();
        if (ce != cudaSuccess) {
          cudaGetLastError();
          finish_locked(rq, 0, CRT_ERR_CUDA);
          progressed = true;
          continue;
        }
        pending.push_back(rq);
      }
      if (progressed) cv.notify_all();
      if (!pending.empty()) {
        if (!kernel_running) launch_kernel();
        publish_locked();
        last_work = now_s();
      }
      if (!flight.empty()) last_work = now_s();
      // re-runs waiting for space do not keep the device loop running: their
      // space comes from requests the client releases, not from the device
      if (kernel_running && flight.empty() && pending.empty() &&
          now_s() - last_work > opts.idle_ms * 1e-3) {
        lk.unlock();
        stop_kernel();
        lk.lock();
      }
      if (kernel_running && now_s() - last_err_check > 1e-3) {
        last_err_check = now_s();
        // a timed-out device loop: report it on every request in flight
        const int err = read_device_error();
        if (err) {
          // some warps gave up waiting (the host stalled past device_wait_us)
          // and may have dropped tickets: stop the loop, then re-run every
          // request that had not completed, from scratch, in a fresh loop
          device_error = err;
          lk.unlock();
          stop_kernel();
          lk.lock();
          std::vector<Request> rerun;
          for (auto& kv : flight) {
            Request& q = kv.second;
            const int slot = (int)(q.seq % slots);
            if (h_done[slot].seq == q.seq && h_done[slot].count <= q.cap) {
              finish_locked(q, h_done[slot].count, CRT_OK);
            } else {
              q.seq = -1;
              rerun.push_back(q);
            }
          }
          flight.clear();
          for (auto it = rerun.rbegin(); it != rerun.rend(); ++it) pending.push_front(*it);
          oldest_seq = next_seq;
          cv.notify_all();
        }
      }
      cv.wait_for(lk, std::chrono::microseconds(flight.empty() && pending.empty() ? 2000 : 50));
    }
    if (kernel_running) {
      lk.unlock();
      stop_kernel();
      lk.lock();
    }
  }
};

}  // namespace crt

using namespace crt;

extern "C" {

void crt_server_opts_default(crt_server_opts* o)
{
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->arena_bytes = 8ll << 30;
  o->max_requests = 4096;
  o->max_trees = 16;
  o->pairs_per_window = 64.0;
  o->idle_ms = 20;
  o->device_wait_us = 2000000;
  o->output_slack = 1.5;
}

int crt_server_create(const crt_server_opts* opts, crt_server* out)
{
  if (!out) return fail(CRT_ERR_INVALID_ARG, "server_create: null out");
  Server* s = new Server();
  crt_server_opts_default(&s->opts);
  if (opts) s->opts = *opts;
  auto& o = s->opts;
  if (o.arena_bytes <= 0 || o.max_requests <= 0 || o.max_trees <= 0 || o.idle_ms < 0 ||
      o.device_wait_us <= 0) {
    delete s;
    return fail(CRT_ERR_INVALID_ARG, "server_create: bad options");
  }
  if (!(o.output_slack > 0)) o.output_slack = 1.5;
  cudaGetDevice(&s->device);
  s->slots = o.max_requests;
  s->arena_bytes = (size_t)o.arena_bytes;
  cudaError_t e = cudaSuccess;
  do {
    if ((e = cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking)) != cudaSuccess) break;
    if ((e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking)) != cudaSuccess) break;
    if ((e = cudaMalloc((void**)&s->arena, s->arena_bytes)) != cudaSuccess) break;
    if ((e = cudaMalloc((void**)&s->d_trees, sizeof(SrvTree) * o.max_trees)) != cudaSuccess) break;
    if ((e = cudaMalloc((void**)&s->d_descs, sizeof(SrvDesc) * s->slots)) != cudaSuccess) break;
    if ((e = cudaMalloc((void**)&s->d_ctrs, sizeof(SrvCtr) * s->slots)) != cudaSuccess) break;
    if ((e = cudaMalloc((void**)&s->d_state, sizeof(SrvState))) != cudaSuccess) break;
    if ((e = cudaHostAlloc((void**)&s->h_done, sizeof(SrvDone) * s->slots, cudaHostAllocMapped)) !=
        cudaSuccess)
      break;
    if ((e = cudaHostGetDevicePointer((void**)&s->d_done, s->h_done, 0)) != cudaSuccess) break;
    if ((e = cudaHostAlloc((void**)&s->h_desc_stage, sizeof(SrvDesc) * s->slots,
                           cudaHostAllocDefault)) != cudaSuccess)
      break;
    if ((e = cudaHostAlloc((void**)&s->h_box, sizeof(Server::Mailbox), cudaHostAllocDefault)) !=
        cudaSuccess)
      break;
    if ((e = cudaHostAlloc((void**)&s->h_ctl, sizeof(SrvCtl), cudaHostAllocMapped)) != cudaSuccess)
      break;
    if ((e = cudaHostGetDevicePointer((void**)&s->d_ctl, s->h_ctl, 0)) != cudaSuccess) break;
    s->h_ctl->shutdown = 0;
    s->h_ctl->error = 0;
    if ((e = cudaHostAlloc((void**)&s->h_bounce, Server::kBounce, cudaHostAllocDefault)) != cudaSuccess)
      break;
    if ((e = cudaHostAlloc((void**)&s->h_bounce_submit, Server::kBounce, cudaHostAllocDefault)) !=
        cudaSuccess)
      break;
    if ((e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking)) != cudaSuccess) break;
  } while (0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    crt_server_destroy((crt_server)s);
    return cuda_fail(e, "server_create");
  }
  // seq -1 marks an unused descriptor slot
  std::vector<SrvDesc> init(s->slots);
  for (auto& d : init) {
    std::memset(&d, 0, sizeof(d));
    d.seq = -1;
  }
  cudaMemcpy(s->d_descs, init.data(), sizeof(SrvDesc) * s->slots, cudaMemcpyHostToDevice);
  for (int i = 0; i < s->slots; i++) s->h_done[i].seq = -1;
  cudaMemset(s->d_state, 0, sizeof(SrvState));
  s->alloc.init(s->arena_bytes);
  s->last_work = now_s();
  s->worker = std::thread([s] { s->loop(); });
  *out = (crt_server)s;
  return CRT_OK;
}

int crt_server_add_tree(crt_server h, const crt_rtree_f32* rt, const crt_bbox_f32* rbox,
                        int* tree_id)
{
  Server* s = (Server*)h;
  if (!s || !rt || !rbox || !tree_id || rbox->sz < 0 || rt->sz < 0 ||
      (rt->sz > 0 && rt->fanout < 2))
    return fail(CRT_ERR_INVALID_ARG, "server_add_tree: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  if ((int)s->trees.size() >= s->opts.max_trees)
    return fail(CRT_ERR_BUSY, "server_add_tree: tree table full");
  if (s->kernel_running)
    return fail(CRT_ERR_BUSY, "server_add_tree: add trees before submitting requests");
  SrvTree t{};
  t.nxmin = rt->xmin; t.nymin = rt->ymin; t.nxmax = rt->xmax; t.nymax = rt->ymax;
  t.npos = rt->pos; t.nlen = rt->len; t.rsz = rt->sz; t.fanout = rt->fanout;
  t.bxmin = rbox->xmin; t.bymin = rbox->ymin; t.bxmax = rbox->xmax; t.bymax = rbox->ymax;
  t.bid = rbox->id; t.nbox = rbox->sz;
  std::vector<int64_t> lv;
  int L = std::max(1, tree_levels(std::max(1, rbox->sz), std::max(2, rt->fanout), lv));
  t.K = rt->fanout <= 32 ? std::max(1, 32 / std::max(2, rt->fanout)) : 1;
  int cap = ((L - 1) * t.K * std::max(2, rt->fanout) + 1 + 31) / 32 * 32;
  s->stack_cap = std::max(s->stack_cap, cap);
  if (s->smem() > 200 * 1024) return fail(CRT_ERR_NOT_SUPPORTED, "server_add_tree: tree too deep");
  const LevelTables lt = level_tables(*rt, rbox->sz);
  t.nlev = 0;
  if (lt.nlev > 0) {
    char* dev = nullptr;
    if (cudaMalloc((void**)&dev, kLevelTableBytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(CRT_ERR_OOM, "server_add_tree: table allocation failed");
    }
    cudaMemcpy(dev, lt.first, sizeof(int) * kMaxLevels, cudaMemcpyHostToDevice);
    cudaMemcpy(dev + sizeof(int) * kMaxLevels, lt.span, sizeof(long long) * kMaxLevels,
               cudaMemcpyHostToDevice);
    s->tables.push_back(dev);
    launch_odd_boxes(rbox->xmin, rbox->ymin, rbox->xmax, rbox->ymax, rbox->sz,
                     (int*)(dev + kLevelOddOffset), 0);
    const cudaError_t e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) return cuda_fail(e, "server_add_tree");
    t.nlev = lt.nlev;
    t.lvl_first = (const int*)dev;
    t.lvl_span = (const long long*)(dev + sizeof(int) * kMaxLevels);
    t.lvl_odd = (const int*)(dev + kLevelOddOffset);
  }
  TreeStats ts;
  if (rt->sz > 0 && rbox->sz > 0) {
    // root MBR and a sample of box extents
    float root[4];
    const float* src[4] = {rt->xmin, rt->ymin, rt->xmax, rt->ymax};
    for (int a = 0; a < 4; a++) cudaMemcpy(&root[a], src[a], sizeof(float), cudaMemcpyDeviceToHost);
    const int m = std::min(rbox->sz, 4096);
    std::vector<float> bx[4];
    const float* bs[4] = {rbox->xmin, rbox->ymin, rbox->xmax, rbox->ymax};
    for (int a = 0; a < 4; a++) {
      bx[a].resize(m);
      cudaMemcpy(bx[a].data(), bs[a], sizeof(float) * m, cudaMemcpyDeviceToHost);
    }
    double sw = 0, sh = 0;
    for (int i = 0; i < m; i++) {
      if (bx[2][i] >= bx[0][i]) sw += bx[2][i] - bx[0][i];
      if (bx[3][i] >= bx[1][i]) sh += bx[3][i] - bx[1][i];
    }
    ts.rx1 = root[0]; ts.ry1 = root[1]; ts.rx2 = root[2]; ts.ry2 = root[3];
    const double area = (ts.rx2 - ts.rx1) * (ts.ry2 - ts.ry1);
    ts.density = area > 0 && std::isfinite(area) ? rbox->sz / area : 0;
    ts.mbw = sw / m;
    ts.mbh = sh / m;
  }
  const int id = (int)s->trees.size();
  s->trees.push_back(t);
  s->tree_stats.push_back(ts);
  s->tree_ppw.push_back(s->opts.pairs_per_window);
  cudaError_t e = cudaMemcpy(s->d_trees + id, &t, sizeof(t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "server_add_tree");
  *tree_id = id;
  return CRT_OK;
}

int crt_server_submit(crt_server h, int tree_id, const float* xmin, const float* ymin,
                      const float* xmax, const float* ymax, int64_t nq, int64_t* request_id)
{
  Server* s = (Server*)h;
  if (!s || nq < 1 || !xmin || !ymin || !xmax || !ymax)
    return fail(CRT_ERR_INVALID_ARG, "server_submit: bad arguments");
  Request q;
  bool pageable = false;  // the windows are in pageable host memory
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (tree_id < 0 || tree_id >= (int)s->trees.size())
      return fail(CRT_ERR_INVALID_ARG, "server_submit: unknown tree");
    if ((long long)(s->flight.size() + s->pending.size()) >= s->slots)
      return fail(CRT_ERR_BUSY, "server_submit: all request slots in use");
    // a re-run waiting for arena space goes first: new requests would take
    // the space it waits for
    if (!s->retry_wait.empty())
      return fail(CRT_ERR_BUSY, "server_submit: a re-run is waiting for arena space");
    q.id = s->next_id++;
    q.tree = tree_id;
    q.nq = nq;
    q.win_bytes = (size_t)nq * 16;
    cudaPointerAttributes pa{};
    const bool host_windows = cudaPointerGetAttributes(&pa, xmin) == cudaSuccess &&
                              pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged;
    cudaGetLastError();
    pageable = host_windows && pa.type == cudaMemoryTypeUnregistered;
    if (host_windows) {
      q.predicted = s->predict_locked(tree_id, xmin, ymin, xmax, ymax, nq);
    } else {
      // device-resident windows: the same area estimate from a host copy
      // (16 B per window); a running pairs-per-window average is no guide
      // when window sizes span orders of magnitude
      std::vector<float> hw((size_t)nq * 4);
      const float* src[4] = {xmin, ymin, xmax, ymax};
      cudaError_t ce = cudaSuccess;
      {
        std::lock_guard<std::mutex> ul(s->submit_mu);
        for (int a = 0; a < 4 && ce == cudaSuccess; a++)
          ce = Server::bounce_copy(hw.data() + (size_t)a * nq, src[a], sizeof(float) * (size_t)nq,
                                   cudaMemcpyDeviceToHost, s->h_bounce_submit, s->upload);
      }
      if (ce == cudaSuccess)
        q.predicted = s->predict_locked(tree_id, hw.data(), hw.data() + nq, hw.data() + 2 * nq,
                                        hw.data() + 3 * nq, nq);
      else
        cudaGetLastError();
    }
    double est = q.predicted > 0
                     ? s->tree_stats[tree_id].corr * q.predicted * s->opts.output_slack + 256.0
                     : s->tree_ppw[tree_id] * (double)nq * s->opts.output_slack + 256.0;
    // no single estimate may hold more than a quarter of the arena: an
    // estimate past the arena would never be admitted, and a request that
    // needs more re-runs at its exact size (overflow-and-retry)
    est = std::min(est, (double)s->arena_bytes / 4.0 / 8.0);
    q.cap = (long long)std::max(256.0, std::min(est, 4.0e12));
    q.out_bytes = (size_t)q.cap * 8;
    if (!s->alloc.alloc(q.win_bytes, q.win_off))
      return fail(CRT_ERR_BUSY, "server_submit: arena full (windows)");
    if (!s->alloc.alloc(q.out_bytes, q.out_off)) {
      s->alloc.release(q.win_off, q.win_bytes);
      return fail(CRT_ERR_BUSY, "server_submit: arena full (output)");
    }
  }
  // copy the windows in (the caller's buffers are free again on return)
  float* w = (float*)(s->arena + q.win_off);
  cudaError_t e = cudaSuccess;
  const float* src[4] = {xmin, ymin, xmax, ymax};
  {
    std::lock_guard<std::mutex> ul(s->submit_mu);
    for (int a = 0; a < 4 && e == cudaSuccess; a++)
      e = pageable ? Server::bounce_copy(w + a * nq, src[a], sizeof(float) * (size_t)nq,
                                         cudaMemcpyHostToDevice, s->h_bounce_submit, s->upload)
                   : cudaMemcpyAsync(w + a * nq, src[a], sizeof(float) * (size_t)nq,
                                     cudaMemcpyDefault, s->upload);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->upload);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (e != cudaSuccess) {
    s->alloc.release(q.win_off, q.win_bytes);
    s->alloc.release(q.out_off, q.out_bytes);
    return cuda_fail(e, "server_submit: window copy");
  }
  q.t_submit = now_s();
  s->pending.push_back(q);
  s->n_submitted++;
  s->cv.notify_all();
  if (request_id) *request_id = q.id;
  return CRT_OK;
}

int crt_server_poll(crt_server h, crt_server_completion* out, int max_out, int* n_out, int wait_ms)
{
  Server* s = (Server*)h;
  if (!s || (!out && max_out > 0) || !n_out) return fail(CRT_ERR_INVALID_ARG, "server_poll");
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->completed.empty() && wait_ms > 0)
    s->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] { return !s->completed.empty(); });
  int n = 0;
  while (n < max_out && !s->completed.empty()) {
    out[n++] = s->completed.front();
    s->completed.pop_front();
  }
  *n_out = n;
  return CRT_OK;
}

int crt_server_release(crt_server h, int64_t request_id)
{
  Server* s = (Server*)h;
  if (!s) return fail(CRT_ERR_INVALID_ARG, "server_release");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->finished.find(request_id);
  if (it == s->finished.end()) return fail(CRT_ERR_INVALID_ARG, "server_release: unknown request");
  if (it->second.win_bytes) s->alloc.release(it->second.win_off, it->second.win_bytes);
  if (it->second.out_bytes) s->alloc.release(it->second.out_off, it->second.out_bytes);
  s->finished.erase(it);
  return CRT_OK;
}

int crt_server_stats(crt_server h, int64_t* submitted, int64_t* completed, int64_t* retried,
                     int64_t* arena_used)
{
  Server* s = (Server*)h;
  if (!s) return fail(CRT_ERR_INVALID_ARG, "server_stats");
  std::lock_guard<std::mutex> lk(s->mu);
  if (submitted) *submitted = s->n_submitted;
  if (completed) *completed = s->n_completed;
  if (retried) *retried = s->n_retried;
  if (arena_used) *arena_used = (int64_t)s->alloc.used();
  return s->device_error ? s->device_error : CRT_OK;
}

int crt_server_destroy(crt_server h)
{
  Server* s = (Server*)h;
  if (!s) return CRT_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  if (s->compute) cudaStreamSynchronize(s->compute);
  cudaFree(s->arena);
  for (char* t : s->tables) cudaFree(t);
  cudaFree(s->d_trees);
  cudaFree(s->d_descs);
  cudaFree(s->d_ctrs);
  cudaFree(s->d_state);
  if (s->h_done) cudaFreeHost(s->h_done);
  if (s->h_desc_stage) cudaFreeHost(s->h_desc_stage);
  if (s->h_box) cudaFreeHost(s->h_box);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_bounce) cudaFreeHost(s->h_bounce);
  if (s->h_bounce_submit) cudaFreeHost(s->h_bounce_submit);
  if (s->upload) cudaStreamDestroy(s->upload);
  if (s->compute) cudaStreamDestroy(s->compute);
  if (s->copy) cudaStreamDestroy(s->copy);
  const int err = s->device_error;
  delete s;
  return err ? fail(err, "server_destroy: the device loop reported an error") : CRT_OK;
}

}  // extern "C"
