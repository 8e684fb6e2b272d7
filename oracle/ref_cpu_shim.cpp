// C entry points around the reference's own CPU brute force
// (nested_loop_query, src/utility.h:22-45), compiled from the reference
// sources where they lie into oracle/_ref/libref_cpu.so by oracle/Makefile.
// TEST INFRASTRUCTURE ONLY: used to pin the oracle and as the timed CPU
// baseline of the benchmark; never linked into the product library.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <iterator>
#include <thread>
#include <vector>

#include <thrust/copy.h>
#include <thrust/equal.h>
#include <thrust/execution_policy.h>
#include <thrust/host_vector.h>
#include <thrust/iterator/constant_iterator.h>
#include <thrust/reduce.h>

#include "rtree.h"
#include "utility.h"

namespace {
BBOX<float> make_box(const float* xmin, const float* ymin, const float* xmax, const float* ymax,
                     const int* id, int n)
{
  BBOX<float> b;
  b.sz   = n;
  b.xmin = const_cast<float*>(xmin);
  b.ymin = const_cast<float*>(ymin);
  b.xmax = const_cast<float*>(xmax);
  b.ymax = const_cast<float*>(ymax);
  b.id   = const_cast<int*>(id);
  return b;
}
}  // namespace

// Runs the reference nested_loop_query once and copies up to `cap` pairs
// (did, qid) out in the reference's order.  Returns the pair count.
extern "C" int64_t ref_nested_loop_query(const float* qxmin, const float* qymin,
                                         const float* qxmax, const float* qymax, const int* qid,
                                         int nq, const float* dxmin, const float* dymin,
                                         const float* dxmax, const float* dymax, const int* did,
                                         int nd, int* out_did, int* out_qid, int64_t cap)
{
  BBOX<float> q = make_box(qxmin, qymin, qxmax, qymax, qid, nq);
  BBOX<float> d = make_box(dxmin, dymin, dxmax, dymax, did, nd);
  thrust::host_vector<int> v_did, v_qid;
  int n = nested_loop_query<float>(q, d, v_did, v_qid);
  for (int64_t i = 0; i < n && i < cap; i++) {
    out_did[i] = v_did[i];
    out_qid[i] = v_qid[i];
  }
  return n;
}

// Runs nested_loop_query over `nthreads` contiguous query slices, one host
// thread each; returns the total pair count.  This is the multi-core form of
// the reference's CPU path timed by the benchmark's reference arm.
extern "C" int64_t ref_nested_loop_query_mt(const float* qxmin, const float* qymin,
                                            const float* qxmax, const float* qymax,
                                            const int* qid, int nq, const float* dxmin,
                                            const float* dymin, const float* dxmax,
                                            const float* dymax, const int* did, int nd,
                                            int nthreads)
{
  if (nthreads < 1) nthreads = 1;
  std::vector<int64_t> counts(nthreads, 0);
  std::vector<std::thread> th;
  int per = (nq + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; t++) {
    int q0 = t * per, q1 = std::min(nq, (t + 1) * per);
    if (q0 >= q1) break;
    th.emplace_back([=, &counts] {
      BBOX<float> q = make_box(qxmin + q0, qymin + q0, qxmax + q0, qymax + q0, qid + q0, q1 - q0);
      BBOX<float> d = make_box(dxmin, dymin, dxmax, dymax, did, nd);
      thrust::host_vector<int> v_did, v_qid;
      counts[t] = nested_loop_query<float>(q, d, v_did, v_qid);
    });
  }
  for (auto& t : th) t.join();
  int64_t total = 0;
  for (auto c : counts) total += c;
  return total;
}

namespace {
// splitmix64 finaliser: the per-pair digest of the oracle (orc_pair_hash).
inline uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
}  // namespace

// ref_nested_loop_query_mt, keeping each slice's output: after the
// reference's nested_loop_query calls (timed alone, wall clock of the
// parallel section, into *query_seconds), each thread reduces its pairs to
// per-query counts and order-independent digests, counts[i] / hashes[i] for
// query i, digest = sum of mix64((uint64)(uint32)qid << 32 | (uint32)did)
// over the pairs the reference emitted for it (qid[i] is its window index).
// Returns the total pair count.
extern "C" int64_t ref_nested_loop_query_mt_digest(const float* qxmin, const float* qymin,
                                                   const float* qxmax, const float* qymax,
                                                   const int* qid, int nq, const float* dxmin,
                                                   const float* dymin, const float* dxmax,
                                                   const float* dymax, const int* did, int nd,
                                                   int nthreads, int64_t* counts,
                                                   uint64_t* hashes, double* query_seconds)
{
  if (nthreads < 1) nthreads = 1;
  std::vector<int64_t> total(nthreads, 0);
  std::vector<std::chrono::steady_clock::time_point> ends(nthreads);
  std::vector<std::thread> th;
  int per = (nq + nthreads - 1) / nthreads;
  const auto start = std::chrono::steady_clock::now();
  for (int t = 0; t < nthreads; t++) {
    int q0 = t * per, q1 = std::min(nq, (t + 1) * per);
    if (q0 >= q1) {
      ends[t] = start;
      continue;
    }
    th.emplace_back([=, &total, &ends] {
      BBOX<float> q = make_box(qxmin + q0, qymin + q0, qxmax + q0, qymax + q0, qid + q0, q1 - q0);
      BBOX<float> d = make_box(dxmin, dymin, dxmax, dymax, did, nd);
      thrust::host_vector<int> v_did, v_qid;
      total[t] = nested_loop_query<float>(q, d, v_did, v_qid);
      ends[t] = std::chrono::steady_clock::now();
      for (int i = q0; i < q1; i++) {
        counts[i] = 0;
        hashes[i] = 0;
      }
      // the reference emits queries in order, each query's pairs together
      int i = q0;
      for (size_t k = 0; k < v_did.size(); k++) {
        while (i < q1 && v_qid[k] != qid[i]) i++;
        if (i >= q1) break;
        counts[i]++;
        hashes[i] += mix64(((uint64_t)(uint32_t)v_qid[k] << 32) | (uint32_t)v_did[k]);
      }
    });
  }
  for (auto& t : th) t.join();
  auto end = start;
  for (auto e : ends) end = std::max(end, e);
  if (query_seconds) *query_seconds = std::chrono::duration<double>(end - start).count();
  int64_t sum = 0;
  for (auto c : total) sum += c;
  return sum;
}

// The reference's readMBR (src/utility.cpp:5-40), compiled from its source,
// copied out into caller arrays.  Returns 0, or -1 when it throws (it exits on
// a missing file, so callers pass existing files only).
extern "C" int ref_read_mbr(const char* path, int size, float r, float* xmin, float* ymin,
                            float* xmax, float* ymax, int* id)
{
  float *a = nullptr, *b = nullptr, *c = nullptr, *d = nullptr;
  int* e = nullptr;
  try {
    readMBR(const_cast<char*>(path), size, r, a, b, c, d, e);
  } catch (const std::exception&) {
    return -1;
  }
  for (int i = 0; i < size; i++) {
    xmin[i] = a[i];
    ymin[i] = b[i];
    xmax[i] = c[i];
    ymax[i] = d[i];
    id[i] = e[i];
  }
  delete[] a; delete[] b; delete[] c; delete[] d; delete[] e;
  return 0;
}
