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

// Deepest tree the containment shortcut handles (a tree of 2^31 boxes at
// fanout 2 has 31 levels).
constexpr int kMaxLevels = 40;

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
  // Packed-layout tables for the containment shortcut (nlev == 0: off).  In
  // the reference's bulk-load layout the subtree of the g-th node of height h
  // (h = 0: leaf-parents) holds the sorted slots
  // [g * span[h], min(nbox, (g + 1) * span[h])), span[h] = fanout^(h + 1).
  int nlev;
  const int* __restrict__ lvl_first;        // first node index of height h
  const long long* __restrict__ lvl_span;   // boxes under a full node of height h
  // Non-zero word: some box is not ordinary, and the shortcut is off (null:
  // every box was found ordinary when the tables were made).
  const int* __restrict__ lvl_odd;
};

// Host image of the containment tables: kMaxLevels ints (first node of each
// height) then kMaxLevels int64 (boxes under a full node of that height).  On
// the device a flag word follows them: set when some box is not ordinary.
struct LevelTables {
  int nlev = 0;
  int first[kMaxLevels];
  long long span[kMaxLevels];
};
constexpr size_t kLevelOddOffset = sizeof(int) * kMaxLevels + sizeof(long long) * kMaxLevels;
constexpr size_t kLevelTableBytes = kLevelOddOffset + 16;
// Tables of a tree in the reference's packed layout; nlev == 0 otherwise.
LevelTables level_tables(const crt_rtree_f32& rt, int64_t nbox);
// Zeroes *odd, then sets it when some of the n boxes is not ordinary
// (xmin <= xmax and ymin <= ymax, which a NaN coordinate also fails).
void launch_odd_boxes(const float* xmin, const float* ymin, const float* xmax, const float* ymax,
                      int64_t n, int* odd, cudaStream_t stream);

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
// With the containment shortcut on, the high 8 bits of `len` hold the height
// of the nodes in the range.
typedef int2 FrontierEntry;
constexpr int kLenBits = 24;
constexpr int kLenMask = (1 << kLenBits) - 1;

// Emits every box of the sorted slot range [first, first + count) as a hit,
// 32 at a time (warp-collective); emitters with a faster bulk path override it.
template <class Emit>
__device__ __forceinline__ void emit_range_default(Emit& emit, const int* __restrict__ bid,
                                                   long long first, long long count)
{
  const int lane = (int)lane_id();
  for (long long base = 0; base < count; base += 32) {
    const long long i = base + lane;
    const bool hit = i < count;
    emit(hit, hit ? __ldg(bid + first + i) : 0);
  }
}

// Emits every lane's slot range one after the other through emit.range
// (warp-collective).
template <class Emit>
__device__ __forceinline__ void emit_ranges_each(Emit& emit, const int* __restrict__ bid, bool mine,
                                                 long long first, long long count)
{
  uint32_t im = __ballot_sync(0xffffffffu, mine);
  while (im) {
    const int src = __ffs(im) - 1;
    im &= im - 1;
    emit.range(bid, __shfl_sync(0xffffffffu, first, src), __shfl_sync(0xffffffffu, count, src));
  }
}

// Contained subtrees below this many boxes (a leaf-parent holds `fanout`)
// are emitted together, all of one step's at once; larger ones one at a
// time, each into an output reservation of its own.
constexpr int kSmallRange = 256;

// Emits the ids of every lane's slot range [first, first + count) (count <
// kSmallRange; a lane with mine == false adds none), 32 ids per warp pass
// whatever the ranges' sizes: each lane finds the range holding its id by a
// binary search over the lanes' inclusive count prefix (warp-collective).
template <class Emit>
__device__ __forceinline__ void emit_small_ranges(Emit& emit, const int* __restrict__ bid, bool mine,
                                                  long long first, int count)
{
  const int lane = (int)lane_id();
  const int c = mine ? count : 0;
  int x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const int total = __shfl_sync(0xffffffffu, x, 31);
  // element t of the concatenation, inside lane j's range, is id bid[base_j + t]
  const long long base = first - (x - c);
  for (int t0 = 0; t0 < total; t0 += 32) {
    const int t = t0 + lane;
    int j = 0;  // lanes whose inclusive prefix is <= t: the owner of t
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      const int v = __shfl_sync(0xffffffffu, x, j + s - 1);
      if (v <= t) j += s;
    }
    const long long b = __shfl_sync(0xffffffffu, base, j);
    const bool ok = t < total;
    emit(ok, ok ? __ldg(bid + b + t) : 0);
  }
}

// Pair stores use the evict-first hint (st.global.cs): the output streams
// through L2 once, and keeping it out of the way leaves L2 to the tree's
// boxes and ids (measured: 1-3% on the uniform batch, 7-10% on road
// geometry).
__device__ __forceinline__ void put_pair(int32_t* __restrict__ fid, int32_t* __restrict__ tid,
                                         long long slot, long long cap, int id, int q)
{
  if (slot < cap) {
    __stcs(fid + slot, id);
    if (tid) __stcs(tid + slot, q);  // no window column: CSR output
  }
}

// Four pairs at output slot sl (16-byte aligned in fid and tid), or one by
// one where they reach cap.
__device__ __forceinline__ void put_pairs4(int32_t* __restrict__ fid, int32_t* __restrict__ tid,
                                           long long sl, long long cap, int4 v, int q)
{
  if (sl + 3 < cap) {
    __stcs(reinterpret_cast<int4*>(fid + sl), v);
    if (tid) __stcs(reinterpret_cast<int4*>(tid + sl), make_int4(q, q, q, q));
  } else {
    put_pair(fid, tid, sl + 0, cap, v.x, q);
    put_pair(fid, tid, sl + 1, cap, v.y, q);
    put_pair(fid, tid, sl + 2, cap, v.z, q);
    put_pair(fid, tid, sl + 3, cap, v.w, q);
  }
}

// Writes the pairs (bid[first + i], q) to output slots slot0 + i for
// i < count, skipping slots at or past `cap` (warp-collective).  A contained
// subtree can hold millions of boxes, so the ids are read as 16-byte vectors
// (128 ids per warp step, kRangeUnroll steps in flight) instead of one 4-byte
// load per lane; one step keeps the kernels within their register budgets.
// Where the output is not 16-byte aligned with the source the stores are
// single; this form needs fewer registers than copy_range_realign (below),
// and the plain and serving kernels run faster with it.
constexpr int kRangeUnroll = 1;

__device__ __forceinline__ void copy_range(const int* __restrict__ bid, long long first,
                                           long long count, int32_t* __restrict__ fid,
                                           int32_t* __restrict__ tid, long long slot0,
                                           long long cap, int q)
{
  const int lane = (int)lane_id();
  const int* src = bid + first;
  // head: ids before the first 16-byte boundary of the source
  long long head = (long long)((4 - (((uintptr_t)src >> 2) & 3)) & 3);
  if (head > count) head = count;
  if (lane < head) put_pair(fid, tid, slot0 + lane, cap, __ldg(src + lane), q);
  const int4* v = reinterpret_cast<const int4*>(src + head);
  const long long nv = (count - head) >> 2;
  const long long s = slot0 + head;
  for (long long g0 = 0; g0 < nv; g0 += 32 * kRangeUnroll) {
    int4 r[kRangeUnroll];
#pragma unroll
    for (int u = 0; u < kRangeUnroll; u++) {
      const long long g = g0 + u * 32 + lane;
      if (g < nv) r[u] = __ldg(v + g);
    }
#pragma unroll
    for (int u = 0; u < kRangeUnroll; u++) {
      const long long g = g0 + u * 32 + lane;
      if (g < nv) {
        const long long sl = s + 4 * g;
        const uintptr_t al = (uintptr_t)(fid + sl) | (tid ? (uintptr_t)(tid + sl) : (uintptr_t)0);
        if (sl + 3 < cap && (al & 15) == 0) {
          __stcs(reinterpret_cast<int4*>(fid + sl), r[u]);
          if (tid) __stcs(reinterpret_cast<int4*>(tid + sl), make_int4(q, q, q, q));
        } else {
          put_pair(fid, tid, sl + 0, cap, r[u].x, q);
          put_pair(fid, tid, sl + 1, cap, r[u].y, q);
          put_pair(fid, tid, sl + 2, cap, r[u].z, q);
          put_pair(fid, tid, sl + 3, cap, r[u].w, q);
        }
      }
    }
  }
  // tail: the last (count - head) % 4 ids
  const long long done = head + 4 * nv;
  if (lane < count - done) put_pair(fid, tid, slot0 + done + lane, cap, __ldg(src + done + lane), q);
}

// copy_range with 16-byte stores wherever the reservation starts (the
// persistent kernel's large-subtree reservations start anywhere in a
// 16-byte line): the output is aligned first (up to 3 ids one by one); when
// the source then sits at another offset within its 16 bytes, each lane's
// four ids come from its own aligned source vector and its neighbour's (one
// shuffle per component), so loads and stores both stay 16-byte accesses.
// Only aligned vectors inside [bid, bid + first + count) are read.
__device__ __forceinline__ void copy_range_realign(const int* __restrict__ bid, long long first,
                                                   long long count, int32_t* __restrict__ fid,
                                                   int32_t* __restrict__ tid, long long slot0,
                                                   long long cap, int q)
{
  const int lane = (int)lane_id();
  if (count <= 0) return;
  const uintptr_t fa = (uintptr_t)(fid + slot0);
  // vectors need bid 16-byte aligned and fid, tid at one offset within 16 bytes
  const bool vec = ((uintptr_t)bid & 15) == 0 &&
                   (!tid || (((uintptr_t)(tid + slot0) ^ fa) & 15) == 0);
  if (!vec) {
    for (long long i = lane; i < count; i += 32)
      put_pair(fid, tid, slot0 + i, cap, __ldg(bid + first + i), q);
    return;
  }
  // head: ids before the output's first 16-byte boundary
  long long head = (long long)((4 - ((fa >> 2) & 3)) & 3);
  if (head > count) head = count;
  if (lane < head) put_pair(fid, tid, slot0 + lane, cap, __ldg(bid + first + lane), q);
  const long long f1 = first + head;  // first source id of the body
  const long long s1 = slot0 + head;  // its output slot, 16-byte aligned
  const long long end = first + count;
  const int r = (int)(f1 & 3);  // source offset within its 16 bytes
  const long long B = f1 - r;   // the aligned source vector holding f1
  const int4* __restrict__ v = reinterpret_cast<const int4*>(bid + B);
  long long ng;  // output vectors of the body
  if (r == 0) {
    ng = (end - f1) >> 2;
    for (long long g = lane; g < ng; g += 32) put_pairs4(fid, tid, s1 + 4 * g, cap, __ldg(v + g), q);
  } else {
    // output vector g takes source vectors g and g + 1, both inside [B, end)
    // for g < ng
    ng = end - B >= 8 ? ((end - B - 8) >> 2) + 1 : 0;
    for (long long g0 = 0; g0 < ng; g0 += 32) {
      const long long g = g0 + lane;
      int4 x = make_int4(0, 0, 0, 0);
      if (g <= ng) x = __ldg(v + g);
      int4 n;
      n.x = __shfl_down_sync(0xffffffffu, x.x, 1);
      n.y = __shfl_down_sync(0xffffffffu, x.y, 1);
      n.z = __shfl_down_sync(0xffffffffu, x.z, 1);
      n.w = __shfl_down_sync(0xffffffffu, x.w, 1);
      if (lane == 31 && g + 1 <= ng) n = __ldg(v + g + 1);
      if (g < ng) {
        int4 o;
        if (r == 1) o = make_int4(x.y, x.z, x.w, n.x);
        else if (r == 2) o = make_int4(x.z, x.w, n.x, n.y);
        else o = make_int4(x.w, n.x, n.y, n.z);
        put_pairs4(fid, tid, s1 + 4 * g, cap, o, q);
      }
    }
  }
  // tail: the ids past the body (fewer than 8)
  for (long long i = f1 + 4 * ng + lane; i < end; i += 32)
    put_pair(fid, tid, s1 + (i - f1), cap, __ldg(bid + i), q);
}

// Outcome of testing one child slot of a step.
struct ChildTest {
  bool valid, hit, push, inside;
  int hid, cpos, clen;
  long long rfirst, rcount;
  bool leaf;  // a box slot (counted as a leaf test)
};

// Tests child c of popped entry g (of k popped; lane e of the warp holds
// entry e): a leaf box against the window, or an inner node (intersects:
// push its children range; contained: emit its boxes' slot range).
__device__ __forceinline__ void test_child(const TreeView& T, const NodeCache& C, FrontierEntry e,
                                           int k, int g, int c, bool contain, float x1, float y1,
                                           float x2, float y2, ChildTest& t)
{
  const int gs = min(g, k - 1);
  const int pos = __shfl_sync(0xffffffffu, e.x, gs);
  const int ey = __shfl_sync(0xffffffffu, e.y, gs);
  const int len = contain ? (ey & kLenMask) : ey;
  const int hc = contain ? (ey >> kLenBits) : 0;  // height of the nodes [pos, pos+len)
  t.valid = g < k && c < len;
  const int child = pos + c;
  t.hit = t.push = t.inside = t.leaf = false;
  t.hid = t.cpos = t.clen = 0;
  t.rfirst = t.rcount = 0;
  if (!t.valid) return;
  if (pos >= T.rsz) {
    const int s = child - T.rsz;
    if (s < T.nbox) {
      t.leaf = true;
      // the id is loaded with the box (one round trip; most tested boxes of
      // a leaf-parent that straddles the window hit)
      const float m1 = __ldg(T.bxmin + s), n1 = __ldg(T.bymin + s);
      const float m2 = __ldg(T.bxmax + s), n2 = __ldg(T.bymax + s);
      const int id = __ldg(T.bid + s);
      t.hit = intersects(x1, y1, x2, y2, m1, n1, m2, n2);
      t.hid = id;
    }
  } else if (child < T.rsz) {
    float a, b, cc, d;
    load_node_box(T, C, child, a, b, cc, d);
    load_node_link(T, C, child, t.cpos, t.clen);
    t.push = intersects(x1, y1, x2, y2, a, b, cc, d);
    if (contain && t.push && x1 <= a && cc <= x2 && y1 <= b && d <= y2) {
      t.inside = true;
      t.push = false;
      const long long span = __ldg(T.lvl_span + hc);
      t.rfirst = (long long)(child - __ldg(T.lvl_first + hc)) * span;
      t.rcount = min((long long)T.nbox - t.rfirst, span);
    } else if (contain) {
      t.clen |= max(hc - 1, 0) << kLenBits;
    }
  }
}

// part / nparts: this warp takes the part-th of nparts equal shares of the
// root's children (several warps sharing one window); the shares' subtrees
// are disjoint, so their hits together are the window's.
template <class Emit, bool kContain = true>
__device__ __forceinline__ void traverse(const TreeView& T, const NodeCache& C, int K,
                                         int lane_g, int lane_c, float x1, float y1, float x2,
                                         float y2, FrontierEntry* stack, int stack_cap,
                                         Emit& emit, int* err, int part = 0, int nparts = 1)
{
  const int lane = (int)lane_id();
  const uint32_t lt = lanemask_lt();
  const int f = T.fanout;
  if (T.rsz == 0) {
    if (part != 0) return;
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
  // A window that contains a node's MBR hits every ordinary box under it:
  // x1 <= MBR.xmin <= xmin <= xmax <= MBR.xmax <= x2, and the same in y, so
  // none of the predicate's four exclusions holds.  The subtree's slot range
  // is then emitted without descending.  A box that is not ordinary (xmin >
  // xmax, ymin > ymax, or a NaN coordinate, which the MBR's min/max skip) can
  // fail the predicate under a contained MBR, so any such box in the set
  // turns the shortcut off.  A NaN in the window or the MBR fails the
  // containment test and takes the normal path.
  const bool contain = kContain && T.nlev > 0 && (T.lvl_odd == nullptr || *T.lvl_odd == 0);
  // the root is never tested: its children range starts the frontier
  {
    int rp, rl;
    load_node_link(T, C, 0, rp, rl);
    if (nparts > 1) {
      const int a = (int)((long long)rl * part / nparts);
      const int b = (int)((long long)rl * (part + 1) / nparts);
      rp += a;
      rl = b - a;
    }
    if (contain) rl |= max(T.nlev - 2, 0) << kLenBits;
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
      ChildTest t;
      if (f <= 32) test_child(T, C, e, k, lane_g, lane_c, contain, x1, y1, x2, y2, t);
      else test_child(T, C, e, k, 0, base + lane, contain, x1, y1, x2, y2, t);
      if constexpr (Emit::kCountsTests) emit.leaf_tests(__popc(__ballot_sync(0xffffffffu, t.leaf)));
      const uint32_t pm = __ballot_sync(0xffffffffu, t.push);
      if (pm) {
        const int np = __popc(pm);
        if (sp + np > stack_cap) {
          // cannot happen with the host-sized stack; never write past it
          raise_error(err, CRT_ERR_NOT_SUPPORTED);
          return;
        }
        if (t.push) stack[sp + __popc(pm & lt)] = make_int2(t.cpos, t.clen);
        sp += np;
      }
      emit(t.hit, t.hid);
      if (contain) {
        const bool small = t.inside && t.rcount < kSmallRange;
        if (__any_sync(0xffffffffu, small)) emit.small_ranges(T.bid, small, t.rfirst, (int)t.rcount);
        const bool big = t.inside && !small;
        if (__any_sync(0xffffffffu, big)) emit.big_ranges(T.bid, big, t.rfirst, t.rcount);
      }
    }
    __syncwarp();
  }
}

// Lane -> (node group, child) of its first child slot, for fanout <= 32;
// lanes past the last whole group get group 32 (never valid).
__device__ __forceinline__ void lane_map(int f, int& g, int& c)
{
  const int lane = (int)lane_id();
  if (f <= 32) {
    g = lane / f;
    c = lane - g * f;
    if (g >= 32 / f) { g = 32; c = 0; }
  } else {
    g = 0;
    c = lane;
  }
}

}  // namespace crt
