// The C ABI of include/crtree.h: argument checks, ownership of the arrays the
// drop-in entry points allocate, status codes, and the glue to the build and
// query pipelines.
#include <cuda_runtime.h>

#include <algorithm>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace crt {

std::atomic<uint64_t> g_launches{0};
static thread_local std::string t_last_error;

void set_last_error(const std::string& msg) { t_last_error = msg; }
int fail(int status, const std::string& msg)
{
  t_last_error = msg;
  return status;
}
int cuda_fail(cudaError_t e, const char* what)
{
  t_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? CRT_ERR_OOM : CRT_ERR_CUDA;
}

// Keep freed stream-ordered blocks in the device pool between calls, so the
// scratch of repeated builds and queries does not go back to the driver.
static void init_device()
{
  static std::mutex mu;
  static std::vector<int> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(mu);
  for (int d : done)
    if (d == dev) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done.push_back(dev);
}

int plan_create(const crt_rtree_f32& rt, const crt_bbox_f32& rbox, const crt_bbox_f32& qbox,
                int64_t max_nq, int32_t* fid, int32_t* tid, int64_t capacity,
                crt_query_result* res, const crt_query_opts& opts, cudaStream_t stream,
                void** out);
int plan_set_nq(void* p, int64_t nq, cudaStream_t stream);
int query_stats(const crt_rtree_f32& rt, const crt_bbox_f32& rbox, const crt_bbox_f32& qbox,
                int64_t* d_hits, int64_t* d_tested, int64_t* h_totals, cudaStream_t stream);
int query_plain_noalloc(const crt_rtree_f32& rt, const crt_bbox_f32& rbox,
                        const crt_bbox_f32& qbox, int32_t* fid, int32_t* tid, int64_t capacity,
                        crt_query_result* d_result, cudaStream_t stream);
int plan_launch(void* p, cudaStream_t stream);
int plan_destroy(void* p);

static bool box_ok(const crt_bbox_f32* b)
{
  return b && b->sz >= 0 &&
         (b->sz == 0 || (b->xmin && b->ymin && b->xmax && b->ymax && b->id));
}
static bool tree_ok(const crt_rtree_f32* t)
{
  return t && t->sz >= 0 &&
         (t->sz == 0 || (t->xmin && t->ymin && t->xmax && t->ymax && t->pos && t->len &&
                         t->fanout >= 2));
}

// Pairs-per-window estimate of the last drop-in query, used to size the next
// one's output before its exact count is known.
static std::atomic<double> g_pairs_per_window{64.0};

// The drop-in query runs into a working buffer from the stream-ordered pool
// (sized from the last call's pairs per window, re-run once at the exact size
// if that was too small), then copies the pairs into two exact-size arrays
// from the same pool, which the caller frees with cudaFree as the reference's
// idpair_d_free does (src/utility.cuh:164-195).  Batches below
// kDropinPersistentMin windows take the plain form: its fixed cost (no
// window sort, no chunk compaction) is far below the persistent form's,
// which wins on large batches.
constexpr int64_t kDropinPersistentMin = 32768;

static int query_dropin(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                        const crt_bbox_f32* d_qbox, crt_idpair* d_dq, cudaStream_t stream)
{
  if (!tree_ok(d_rt) || !box_ok(d_rbox) || !box_ok(d_qbox) || !d_dq)
    return fail(CRT_ERR_INVALID_ARG, "query: null or negative-size argument");
  init_device();
  crt_query_opts o;
  crt_query_opts_default(&o);
  const int64_t nq = d_qbox->sz;
  if (nq < kDropinPersistentMin) o.mode = CRT_QUERY_PLAIN;
  int64_t want = (int64_t)(g_pairs_per_window.load() * (double)nq * 1.25) + 1024;
  crt_query_result* res = nullptr;
  if (cudaMallocAsync((void**)&res, sizeof(crt_query_result), stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(CRT_ERR_OOM, "query: result block allocation failed");
  }
  int rc = CRT_OK;
  int32_t* work = nullptr;
  int64_t cap = 0;
  crt_query_result h{};
  for (int attempt = 0; attempt < 3; attempt++) {
    cap = query_capacity(want, o);
    if (cudaMallocAsync((void**)&work, 2 * sizeof(int32_t) * (size_t)cap, stream) != cudaSuccess) {
      cudaGetLastError();
      work = nullptr;
      rc = fail(CRT_ERR_OOM, "query: output allocation failed");
      break;
    }
    rc = query_into(*d_rt, *d_rbox, *d_qbox, work, work + cap, cap, res, nullptr, o, stream);
    if (rc != CRT_OK) break;
    cudaError_t e = cudaMemcpyAsync(&h, res, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      rc = cuda_fail(e, "query");
      break;
    }
    if (h.error) {
      rc = fail(h.error, "query: device-side error");
      break;
    }
    if (!h.overflow) break;
    cudaFreeAsync(work, stream);
    work = nullptr;
    want = h.required;  // exact: the retry cannot overflow
  }
  if (rc == CRT_OK && h.overflow) rc = fail(CRT_ERR_CUDA, "query: output overflow after retry");
  if (rc == CRT_OK && h.count > INT32_MAX)
    rc = fail(CRT_ERR_OVERFLOW_INT32, "query: more than INT32_MAX pairs; use crt_query_into_f32");
  int32_t *fid = nullptr, *tid = nullptr;
  if (rc == CRT_OK) {
    const size_t bytes = sizeof(int32_t) * (size_t)std::max<int64_t>(h.count, 1);
    // two allocations, as idpair_d_alloc makes them, from the device's
    // stream-ordered pool: cudaFree (the reference's idpair_d_free) accepts
    // them, and they cost no device-wide synchronisation here
    if (cudaMallocAsync((void**)&fid, bytes, stream) != cudaSuccess ||
        cudaMallocAsync((void**)&tid, bytes, stream) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(CRT_ERR_OOM, "query: output allocation failed");
    } else if (h.count > 0) {
      cudaMemcpyAsync(fid, work, sizeof(int32_t) * (size_t)h.count, cudaMemcpyDeviceToDevice, stream);
      cudaMemcpyAsync(tid, work + cap, sizeof(int32_t) * (size_t)h.count, cudaMemcpyDeviceToDevice,
                      stream);
    }
  }
  if (work) cudaFreeAsync(work, stream);
  cudaFreeAsync(res, stream);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (rc == CRT_OK && e != cudaSuccess) rc = cuda_fail(e, "query: copy");
  if (rc != CRT_OK) {
    if (fid) cudaFreeAsync(fid, stream);
    if (tid) cudaFreeAsync(tid, stream);
    cudaStreamSynchronize(stream);
    return rc;
  }
  if (nq > 0) g_pairs_per_window.store(std::max(1.0, (double)h.count / (double)nq));
  d_dq->sz = (int)h.count;
  d_dq->fid = fid;
  d_dq->tid = tid;
  return CRT_OK;
}

}  // namespace crt

using namespace crt;

extern "C" {

const char* crt_status_string(int s)
{
  switch (s) {
    case CRT_OK: return "ok";
    case CRT_ERR_INVALID_ARG: return "invalid argument";
    case CRT_ERR_OOM: return "out of memory";
    case CRT_ERR_OVERFLOW_INT32: return "result does not fit int32";
    case CRT_ERR_OUTPUT_OVERFLOW: return "output buffer too small";
    case CRT_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case CRT_ERR_CUDA: return "CUDA error";
    case CRT_ERR_NOT_SUPPORTED: return "not supported";
    case CRT_ERR_BUSY: return "busy";
    default: return "unknown status";
  }
}

const char* crt_last_error(void) { return t_last_error.c_str(); }
const char* crt_version(void) { return "crtree-b200 0.1 (sm_100a)"; }
uint64_t crt_kernel_launches(void) { return g_launches.load(); }

int64_t crt_tree_size(int64_t n, int fanout)
{
  std::vector<int64_t> lv;
  if (tree_levels(n, fanout, lv) < 0) return -1;
  int64_t r = 0;
  for (auto x : lv) r += x;
  return r;
}

int crt_tree_levels(int64_t n, int fanout, int64_t* levels, int max_levels)
{
  std::vector<int64_t> lv;
  int L = tree_levels(n, fanout, lv);
  if (L < 0) return fail(CRT_ERR_INVALID_ARG, "levels: need n >= 1 and fanout >= 2"), -1;
  if (levels)
    for (int i = 0; i < L && i < max_levels; i++) levels[i] = lv[i];
  return L;
}

int crt_build_f32(crt_bbox_f32* d_box, crt_rtree_f32* d_rt, crt_stream_t stream, int32_t* out_r_sz)
{
  if (!box_ok(d_box) || !d_rt) return fail(CRT_ERR_INVALID_ARG, "build: null argument");
  const int64_t n = d_box->sz;
  const int fanout = d_rt->fanout;
  const int64_t rsz = crt_tree_size(n, fanout);
  if (rsz < 0) return fail(CRT_ERR_INVALID_ARG, "build: need sz >= 1 and fanout >= 2");
  if (n + rsz > INT32_MAX) return fail(CRT_ERR_INVALID_ARG, "build: sz + R_sz exceeds INT32_MAX");
  init_device();
  // node arrays: six allocations, as rt_d_alloc makes them
  // (src/utility.cuh:114-135), from the device's stream-ordered pool:
  // cudaFree (the reference's rt_d_free) accepts them; build_tree synchronises
  // the stream before this returns
  crt_rtree_f32 t = *d_rt;
  t.sz = (int)rsz;
  t.xmin = t.ymin = t.xmax = t.ymax = nullptr;
  t.pos = t.len = nullptr;
  if (rsz > 0) {
    void** arr[6] = {(void**)&t.xmin, (void**)&t.ymin, (void**)&t.xmax, (void**)&t.ymax,
                     (void**)&t.pos, (void**)&t.len};
    for (int a = 0; a < 6; a++) {
      if (cudaMallocAsync(arr[a], sizeof(float) * (size_t)rsz, (cudaStream_t)stream) != cudaSuccess) {
        cudaGetLastError();
        for (int b = 0; b < a; b++) cudaFreeAsync(*arr[b], (cudaStream_t)stream);
        cudaStreamSynchronize((cudaStream_t)stream);
        return fail(CRT_ERR_OOM, "build: node allocation failed");
      }
    }
  }
  int rc = build_tree(d_box->xmin, d_box->ymin, d_box->xmax, d_box->ymax, d_box->id, n, fanout,
                      d_box->xmin, d_box->ymin, d_box->xmax, d_box->ymax, d_box->id, t.xmin,
                      t.ymin, t.xmax, t.ymax, t.pos, t.len, (cudaStream_t)stream);
  if (rc != CRT_OK) {
    if (rsz > 0) {
      cudaFree(t.xmin); cudaFree(t.ymin); cudaFree(t.xmax); cudaFree(t.ymax);
      cudaFree(t.pos); cudaFree(t.len);
    }
    return rc;
  }
  *d_rt = t;
  if (out_r_sz) *out_r_sz = (int32_t)rsz;
  return CRT_OK;
}

int crt_build_into_f32(const crt_bbox_f32* d_in, crt_bbox_f32* d_sorted, crt_rtree_f32* d_rt,
                       crt_stream_t stream)
{
  if (!box_ok(d_in) || !box_ok(d_sorted) || !d_rt || d_sorted->sz != d_in->sz)
    return fail(CRT_ERR_INVALID_ARG, "build_into: bad box arguments");
  const int64_t rsz = crt_tree_size(d_in->sz, d_rt->fanout);
  if (rsz < 0) return fail(CRT_ERR_INVALID_ARG, "build_into: need sz >= 1 and fanout >= 2");
  if (rsz > 0 && !(d_rt->xmin && d_rt->ymin && d_rt->xmax && d_rt->ymax && d_rt->pos && d_rt->len))
    return fail(CRT_ERR_INVALID_ARG, "build_into: node arrays are required");
  init_device();
  int rc = build_tree(d_in->xmin, d_in->ymin, d_in->xmax, d_in->ymax, d_in->id, d_in->sz,
                      d_rt->fanout, d_sorted->xmin, d_sorted->ymin, d_sorted->xmax,
                      d_sorted->ymax, d_sorted->id, d_rt->xmin, d_rt->ymin, d_rt->xmax,
                      d_rt->ymax, d_rt->pos, d_rt->len, (cudaStream_t)stream);
  if (rc == CRT_OK) d_rt->sz = (int)rsz;
  return rc;
}

int crt_query_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                  const crt_bbox_f32* d_qbox, crt_idpair* d_dq, crt_stream_t stream)
{
  return query_dropin(d_rt, d_rbox, d_qbox, d_dq, (cudaStream_t)stream);
}

int crt_query_thrust_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                         const crt_bbox_f32* d_qbox, crt_idpair* d_dq, crt_stream_t stream)
{
  return query_dropin(d_rt, d_rbox, d_qbox, d_dq, (cudaStream_t)stream);
}

int crt_rtree_free(crt_rtree_f32* d_rt)
{
  if (!d_rt) return fail(CRT_ERR_INVALID_ARG, "rtree_free: null");
  float** f[4] = {&d_rt->xmin, &d_rt->ymin, &d_rt->xmax, &d_rt->ymax};
  for (auto p : f) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (d_rt->pos) cudaFree(d_rt->pos);
  if (d_rt->len) cudaFree(d_rt->len);
  d_rt->pos = d_rt->len = nullptr;
  return CRT_OK;
}

int crt_idpair_free(crt_idpair* d_dq)
{
  if (!d_dq) return fail(CRT_ERR_INVALID_ARG, "idpair_free: null");
  if (d_dq->fid) cudaFree(d_dq->fid);
  if (d_dq->tid) cudaFree(d_dq->tid);
  d_dq->fid = d_dq->tid = nullptr;
  return CRT_OK;
}

void crt_query_opts_default(crt_query_opts* o)
{
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->mode = CRT_QUERY_PERSISTENT;
  o->sort_windows = 1;
  o->stage_levels = 2;
  o->warps_per_window = 1;
}

int64_t crt_query_capacity(int64_t pairs, const crt_query_opts* opts)
{
  crt_query_opts o;
  crt_query_opts_default(&o);
  if (opts) o = *opts;
  return query_capacity(pairs, o);
}

int crt_query_into_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                       const crt_bbox_f32* d_qbox, int32_t* d_fid, int32_t* d_tid,
                       int64_t capacity, crt_query_result* d_result, int64_t* d_offsets,
                       const crt_query_opts* opts, crt_stream_t stream)
{
  if (!tree_ok(d_rt) || !box_ok(d_rbox) || !box_ok(d_qbox) || capacity < 0)
    return fail(CRT_ERR_INVALID_ARG, "query_into: bad arguments");
  init_device();
  crt_query_opts o;
  crt_query_opts_default(&o);
  if (opts) o = *opts;
  if (capacity > 0 && !d_fid) return fail(CRT_ERR_INVALID_ARG, "query_into: no id output");
  if (capacity > 0 && !d_tid && (o.mode != CRT_QUERY_PLAIN || !d_offsets))
    return fail(CRT_ERR_INVALID_ARG, "query_into: a window column is needed unless PLAIN writes offsets");
  return query_into(*d_rt, *d_rbox, *d_qbox, d_fid, d_tid, capacity, d_result, d_offsets, o,
                    (cudaStream_t)stream);
}

int crt_query_sync_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                       const crt_bbox_f32* d_qbox, int32_t* d_fid, int32_t* d_tid,
                       int64_t capacity, int64_t* count, int64_t* required,
                       const crt_query_opts* opts, crt_stream_t stream)
{
  crt_query_result* res = nullptr;
  CRT_CUDA(cudaMalloc((void**)&res, sizeof(crt_query_result)));
  int rc = crt_query_into_f32(d_rt, d_rbox, d_qbox, d_fid, d_tid, capacity, res, nullptr, opts,
                              stream);
  crt_query_result h{};
  if (rc == CRT_OK) {
    cudaError_t e = cudaMemcpyAsync(&h, res, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) rc = cuda_fail(e, "query_sync");
  }
  cudaFree(res);
  if (rc != CRT_OK) return rc;
  if (count) *count = h.count;
  if (required) *required = h.required;
  if (h.error) return fail(h.error, "query_sync: device-side error");
  if (h.overflow) return fail(CRT_ERR_OUTPUT_OVERFLOW, "query_sync: output too small");
  return CRT_OK;
}

int crt_pairs_canonicalize(int32_t* d_fid, int32_t* d_tid, int64_t n, crt_stream_t stream)
{
  init_device();
  return pairs_canonicalize(d_fid, d_tid, n, (cudaStream_t)stream);
}

int crt_pairs_digest(const int32_t* d_fid, const int32_t* d_tid, int64_t n, int64_t window_base,
                     int64_t nq, int64_t* d_counts, uint64_t* d_hashes, int64_t* d_bad,
                     crt_stream_t stream)
{
  return pairs_digest(d_fid, d_tid, n, window_base, nq, d_counts, d_hashes, d_bad,
                      (cudaStream_t)stream);
}

int crt_query_plain_noalloc_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                                const crt_bbox_f32* d_qbox, int32_t* d_fid, int32_t* d_tid,
                                int64_t capacity, crt_query_result* d_result, crt_stream_t stream)
{
  if (!tree_ok(d_rt) || !box_ok(d_rbox) || !box_ok(d_qbox))
    return fail(CRT_ERR_INVALID_ARG, "query_plain_noalloc: bad arguments");
  return query_plain_noalloc(*d_rt, *d_rbox, *d_qbox, d_fid, d_tid, capacity, d_result,
                             (cudaStream_t)stream);
}

int crt_query_stats_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                        const crt_bbox_f32* d_qbox, int64_t* d_hits, int64_t* d_tested,
                        int64_t* totals, crt_stream_t stream)
{
  if (!tree_ok(d_rt) || !box_ok(d_rbox) || !box_ok(d_qbox))
    return fail(CRT_ERR_INVALID_ARG, "query_stats: bad arguments");
  init_device();
  return query_stats(*d_rt, *d_rbox, *d_qbox, d_hits, d_tested, totals, (cudaStream_t)stream);
}

int crt_plan_create(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                    const crt_bbox_f32* d_qbox, int64_t max_nq, int32_t* d_fid, int32_t* d_tid,
                    int64_t capacity, crt_query_result* d_result, const crt_query_opts* opts,
                    crt_stream_t stream, crt_plan* out)
{
  if (!tree_ok(d_rt) || !box_ok(d_rbox) || !d_qbox || !out)
    return fail(CRT_ERR_INVALID_ARG, "plan_create: bad arguments");
  init_device();
  crt_query_opts o;
  crt_query_opts_default(&o);
  if (opts) o = *opts;
  void* p = nullptr;
  int rc = plan_create(*d_rt, *d_rbox, *d_qbox, max_nq, d_fid, d_tid, capacity, d_result, o,
                       (cudaStream_t)stream, &p);
  if (rc == CRT_OK) *out = (crt_plan)p;
  return rc;
}

int crt_plan_set_nq(crt_plan plan, int64_t nq, crt_stream_t stream)
{
  if (!plan) return fail(CRT_ERR_INVALID_ARG, "plan_set_nq: null plan");
  return plan_set_nq(plan, nq, (cudaStream_t)stream);
}

int crt_plan_launch(crt_plan plan, crt_stream_t stream)
{
  if (!plan) return fail(CRT_ERR_INVALID_ARG, "plan_launch: null plan");
  return plan_launch(plan, (cudaStream_t)stream);
}

int crt_plan_destroy(crt_plan plan) { return plan_destroy(plan); }

}  // extern "C"
