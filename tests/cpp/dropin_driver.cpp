// Drop-in check: a caller written like the reference's driver
// (src/rtree_test_frontier.cu:37-137) -- read boxes and windows, copy them to
// the device, build_rtree, bfs_frontier / bfs_thrust, copy the pairs back,
// canonicalise with two stable sorts (by box id, then by window) -- compiled
// against crtree/rtree_compat.h instead of the reference's Thrust headers.
//
// Built twice (tests/cpp/Makefile):
//   dropin_standalone  with crtree/rtree.h and local copy helpers
//   dropin_refutil     with the reference's own rtree.h and utility.cuh
//                      (box_h2d, idpair_d2h, rt_d_free, idpair_d_free), i.e.
//                      the reference's caller-side code unchanged
//
//   dropin_* <boxes.crtb> <windows.crtb> <fanout> <out_prefix>
// writes <out_prefix>_frontier.bin and <out_prefix>_thrust.bin: int64 count,
// int32 fid[count], int32 tid[count] in canonical order, plus the node
// arrays in <out_prefix>_tree.bin (int64 R_sz, then xmin..ymax, pos, len).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <string>
#include <vector>

#ifdef CRT_WITH_REFERENCE_UTILITY
#include <iostream>
#include "rtree.h"
#include "utility.cuh"
#else
#include <crtree/rtree.h>
#endif
#include <crtree/rtree_compat.h>

#include "../../oracle/crtb_io.h"

#ifndef CRT_WITH_REFERENCE_UTILITY
// the copy/free helpers the reference keeps in src/utility.cuh, restated
static void box_h2d(BBOX<float>& d, const BBOX<float>& h)
{
  d.sz = h.sz;
  float** dp[4] = {&d.xmin, &d.ymin, &d.xmax, &d.ymax};
  float* hp[4] = {h.xmin, h.ymin, h.xmax, h.ymax};
  for (int a = 0; a < 4; a++) {
    cudaMalloc((void**)dp[a], sizeof(float) * (size_t)h.sz);
    cudaMemcpy(*dp[a], hp[a], sizeof(float) * (size_t)h.sz, cudaMemcpyHostToDevice);
  }
  cudaMalloc((void**)&d.id, sizeof(int) * (size_t)h.sz);
  cudaMemcpy(d.id, h.id, sizeof(int) * (size_t)h.sz, cudaMemcpyHostToDevice);
}
static void idpair_d2h(IDPAIR& h, const IDPAIR& d)
{
  h.sz = d.sz;
  h.fid = new int[d.sz > 0 ? d.sz : 1];
  h.tid = new int[d.sz > 0 ? d.sz : 1];
  cudaMemcpy(h.fid, d.fid, sizeof(int) * (size_t)d.sz, cudaMemcpyDeviceToHost);
  cudaMemcpy(h.tid, d.tid, sizeof(int) * (size_t)d.sz, cudaMemcpyDeviceToHost);
}
static void idpair_d_free(IDPAIR& p)
{
  cudaFree(p.fid);
  cudaFree(p.tid);
  p.fid = p.tid = nullptr;
}
static void rt_d_free(RTREE<float>& t)
{
  cudaFree(t.xmin); cudaFree(t.ymin); cudaFree(t.xmax); cudaFree(t.ymax);
  cudaFree(t.pos); cudaFree(t.len);
}
#endif

static BBOX<float> view(CrtbBoxes& b)
{
  BBOX<float> h;
  h.sz = (int)b.n; h.xmin = b.xmin.data(); h.ymin = b.ymin.data(); h.xmax = b.xmax.data();
  h.ymax = b.ymax.data(); h.id = b.id.data();
  return h;
}

static void write_pairs(const std::string& path, IDPAIR& h)
{
  // first by box id, then (stably) by window: the reference driver's order
  std::vector<int> o(h.sz);
  std::iota(o.begin(), o.end(), 0);
  std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return h.fid[a] < h.fid[b]; });
  std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return h.tid[a] < h.tid[b]; });
  std::vector<int> f(h.sz), t(h.sz);
  for (int i = 0; i < h.sz; i++) { f[i] = h.fid[o[i]]; t[i] = h.tid[o[i]]; }
  int64_t n = h.sz;
  crtb_write_arrays(path, {&n, f.data(), t.data()}, {8, (size_t)n * 4, (size_t)n * 4});
}

int main(int argc, char** argv)
{
  if (argc != 5) {
    fprintf(stderr, "usage: %s boxes.crtb windows.crtb fanout out_prefix\n", argv[0]);
    return 2;
  }
  CrtbBoxes hb, hq;
  if (!crtb_read(argv[1], hb) || !crtb_read(argv[2], hq)) return 2;
  std::string out = argv[4];
  BBOX<float> h_box = view(hb), h_q = view(hq), d_box, d_q;
  RTREE<float> d_rt;
  d_rt.fanout = atoi(argv[3]);
  box_h2d(d_box, h_box);
  box_h2d(d_q, h_q);
  try {
    int rsz = build_rtree(d_box, d_rt);
    std::vector<float> x0(rsz), y0(rsz), x1(rsz), y1(rsz);
    std::vector<int> pos(rsz), len(rsz);
    cudaMemcpy(x0.data(), d_rt.xmin, 4 * (size_t)rsz, cudaMemcpyDeviceToHost);
    cudaMemcpy(y0.data(), d_rt.ymin, 4 * (size_t)rsz, cudaMemcpyDeviceToHost);
    cudaMemcpy(x1.data(), d_rt.xmax, 4 * (size_t)rsz, cudaMemcpyDeviceToHost);
    cudaMemcpy(y1.data(), d_rt.ymax, 4 * (size_t)rsz, cudaMemcpyDeviceToHost);
    cudaMemcpy(pos.data(), d_rt.pos, 4 * (size_t)rsz, cudaMemcpyDeviceToHost);
    cudaMemcpy(len.data(), d_rt.len, 4 * (size_t)rsz, cudaMemcpyDeviceToHost);
    int64_t r64 = rsz;
    crtb_write_arrays(out + "_tree.bin",
                      {&r64, x0.data(), y0.data(), x1.data(), y1.data(), pos.data(), len.data()},
                      {8, 4 * (size_t)rsz, 4 * (size_t)rsz, 4 * (size_t)rsz, 4 * (size_t)rsz,
                       4 * (size_t)rsz, 4 * (size_t)rsz});
    IDPAIR d_dq, h_dq;
    bfs_frontier(d_rt, d_box, d_q, d_dq);
    idpair_d2h(h_dq, d_dq);
    write_pairs(out + "_frontier.bin", h_dq);
    idpair_d_free(d_dq);
    IDPAIR d_dq2, h_dq2;
    bfs_thrust(d_rt, d_box, d_q, d_dq2);
    idpair_d2h(h_dq2, d_dq2);
    write_pairs(out + "_thrust.bin", h_dq2);
    idpair_d_free(d_dq2);
    if (rsz) rt_d_free(d_rt);
    printf("ok R_sz=%d pairs=%d\n", rsz, h_dq.sz);
  } catch (const crtree::error& e) {
    fprintf(stderr, "crtree error: %s\n", e.what());
    return 1;
  }
  return 0;
}
