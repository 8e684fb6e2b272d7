// Warp-cooperative traversal of one window, shared by the batch query
// (query.cu) and the serving loop (server.cu).
//
// Semantics kept from the reference: the root is never tested; a node whose
// children are nodes passes on the children whose MBR intersects the window
// (src/rtree_bfs_frontier.cuh:110-124); a leaf-parent (pos >= R_sz) tests its
// boxes at slots [pos - R_sz, pos - R_sz + len) (count_hit/write_hit,
// src/rtree_bfs_frontier.cuh:191-289); a hit emits (fid = sorted box's id,
// tid = window index).
//
// The warp keeps its frontier in shared memory as a stack of node indices.
// Each step pops up to K = 32 / fanout nodes (one child per lane, children
// read in SoA layout, coalesced), tests the children, compacts the
// intersecting inner children back onto the stack with a ballot/popc prefix,
// and emits leaf hits warp-collectively.  Popping the top K entries and
// pushing shallower parents' children first keeps the stack ordered by depth,
// so it never holds more than K*fanout entries per level: (levels - 1) * K *
// fanout + 1 in total, which the host sizes exactly.
#pragma once

#include "common.cuh"

namespace crt {

struct TreeView {
  const float* __restrict__ nxmin;
  const float* __restrict__ nymin;
  const float* __restrict__ nxmax;
  const float* __restrict__ nymax;
  const int* __restrict__ npos;
  const int* __restrict__ nlen;
  int rsz;
  int fanout;
  const float* __restrict__ bxmin;
  const float* __restrict__ bymin;
  const float* __restrict__ bxmax;
  const float* __restrict__ bymax;
  const int* __restrict__ bid;
  int nbox;
};

struct WindowView {
  const float* __restrict__ xmin;
  const float* __restrict__ ymin;
  const float* __restrict__ xmax;
  const float* __restrict__ ymax;
  int64_t n;
};

// Top tree levels staged in shared memory (node index < n), or none.
struct NodeCache {
  const float* xmin;
  const float* ymin;
  const float* xmax;
  const float* ymax;
  const int* pos;
  const int* len;
  int n;
};

__device__ __forceinline__ void load_node_box(const TreeView& T, const NodeCache& C, int i,
                                              float& a, float& b, float& c, float& d)
{
  if (i < C.n) {
    a = C.xmin[i]; b = C.ymin[i]; c = C.xmax[i]; d = C.ymax[i];
  } else {
    a = __ldg(T.nxmin + i); b = __ldg(T.nymin + i); c = __ldg(T.nxmax + i); d = __ldg(T.nymax + i);
  }
}
__device__ __forceinline__ void load_node_link(const TreeView& T, const NodeCache& C, int i,
                                               int& p, int& l)
{
  if (i < C.n) {
    p = C.pos[i]; l = C.len[i];
  } else {
    p = __ldg(T.npos + i); l = __ldg(T.nlen + i);
  }
}

// ---------------------------------------------------------------------------
// Warp traversal of one window
// ---------------------------------------------------------------------------
// One frontier entry: the children range [pos, pos + len) of a node that
// intersected the window.  Carrying the range on the stack (it is loaded with
// the node's MBR when the node is tested) saves a dependent load per level.
typedef int2 FrontierEntry;

template <class Emit>
__device__ __forceinline__ void traverse(const TreeView& T, const NodeCache& C, int K,
                                         int lane_g, int lane_c, float x1, float y1, float x2,
                                         float y2, FrontierEntry* stack, int stack_cap,
                                         Emit& emit, int* err)
{
  const int lane = (int)lane_id();
  const uint32_t lt = lanemask_lt();
  const int f = T.fanout;
  if (T.rsz == 0) {
    // one-box (or empty) tree: no nodes, test the boxes directly
    for (int base = 0; base < T.nbox; base += 32) {
      int s = base + lane;
      bool hit = s < T.nbox &&
                 intersects(x1, y1, x2, y2, T.bxmin[s], T.bymin[s], T.bxmax[s], T.bymax[s]);
      if constexpr (Emit::kCountsTests) emit.leaf_tests(min(32, T.nbox - base));
      emit(hit, hit ? T.bid[s] : 0);
    }
    return;
  }
  // the root is never tested: its children range starts the frontier
  {
    int rp, rl;
    load_node_link(T, C, 0, rp, rl);
    if (lane == 0) stack[0] = make_int2(rp, rl);
  }
  int sp = 1;
  __syncwarp();
  while (sp > 0) {
    const int k = min(sp, K);
    sp -= k;
    // popped entries stack[sp .. sp+k): lower index = shallower; lane g holds entry g
    FrontierEntry e = make_int2(0, 0);
    if (lane < k) e = stack[sp + lane];
    __syncwarp();
    const int span = f <= 32 ? 32 : f;  // children covered per node group
    for (int base = 0; base < span; base += 32) {
      int g, c;
      if (f <= 32) { g = lane_g; c = lane_c; }
      else { g = 0; c = base + lane; }
      const int gs = min(g, k - 1);
      const int pos = __shfl_sync(0xffffffffu, e.x, gs);
      const int len = __shfl_sync(0xffffffffu, e.y, gs);
      const bool valid = g < k && c < len;
      const int child = pos + c;
      bool hit = false, push = false;
      int hid = 0, cpos = 0, clen = 0;
      if (valid) {
        if (pos >= T.rsz) {
          const int s = child - T.rsz;
          if (s < T.nbox) {
            hit = intersects(x1, y1, x2, y2, __ldg(T.bxmin + s), __ldg(T.bymin + s),
                             __ldg(T.bxmax + s), __ldg(T.bymax + s));
            if (hit) hid = __ldg(T.bid + s);
          }
        } else if (child < T.rsz) {
          float a, b, cc, d;
          load_node_box(T, C, child, a, b, cc, d);
          load_node_link(T, C, child, cpos, clen);
          push = intersects(x1, y1, x2, y2, a, b, cc, d);
        }
      }
      if constexpr (Emit::kCountsTests)
        emit.leaf_tests(__popc(__ballot_sync(0xffffffffu, valid && pos >= T.rsz && child - T.rsz < T.nbox)));
      const uint32_t pm = __ballot_sync(0xffffffffu, push);
      if (pm) {
        const int np = __popc(pm);
        if (sp + np > stack_cap) {
          // cannot happen with the host-sized stack; never write past it
          raise_error(err, CRT_ERR_NOT_SUPPORTED);
          return;
        }
        if (push) stack[sp + __popc(pm & lt)] = make_int2(cpos, clen);
        sp += np;
      }
      emit(hit, hid);
    }
    __syncwarp();
  }
}

// Lane -> (node group, child) for fanout <= 32.
__device__ __forceinline__ void lane_map(int f, int K, int& g, int& c)
{
  const int lane = (int)lane_id();
  if (f <= 32) {
    g = lane / f;
    c = lane - g * f;
    if (g >= K) { g = 32; c = 0; }
  } else {
    g = 0;
    c = lane;
  }
}

}  // namespace crt
