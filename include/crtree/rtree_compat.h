/*
 * Drop-in C++ surface over the crtree C ABI: the reference's build and query
 * templates, with the same names, argument order, ownership and results.
 *
 *   build_rtree(d_box, d_rt)             trxcllnt/curtree src/rtree_bulkload_thrust.cuh:62
 *   bfs_frontier(d_rt, d_rbox, d_qbox, d_dq)   src/rtree_bfs_frontier.cuh:292
 *   bfs_thrust(d_rt, d_rbox, d_qbox, d_dq)     src/rtree_bfs_thrust.cuh:59
 *
 * They work with the reference's own BBOX/RTREE/IDPAIR (src/rtree.h) or with
 * crtree/rtree.h: the templates deduce whichever struct templates are in
 * scope and check their layout against the C structs at compile time.  The
 * arrays build and query allocate are plain cudaMalloc allocations, so the
 * reference's rt_d_free / idpair_d_free (src/utility.cuh) release them.
 *
 * Errors: where the reference calls exit() or loops forever (n == 0,
 * fanout == 1, an overflowing frontier), these throw crtree::error carrying
 * the crt_status code.  Only float boxes exist, as in the reference's callers.
 */
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>

#include "../crtree.h"

namespace crtree {

struct error : std::runtime_error {
  int status;
  error(int s, const char* where)
    : std::runtime_error(std::string(where) + ": " + crt_status_string(s) + ": " + crt_last_error()),
      status(s)
  {
  }
};

namespace detail {
template <class Box>
inline crt_bbox_f32* as_c_box(Box& b)
{
  static_assert(sizeof(Box) == sizeof(crt_bbox_f32), "BBOX<float> layout");
  static_assert(offsetof(Box, sz) == offsetof(crt_bbox_f32, sz) &&
                  offsetof(Box, xmin) == offsetof(crt_bbox_f32, xmin) &&
                  offsetof(Box, ymin) == offsetof(crt_bbox_f32, ymin) &&
                  offsetof(Box, xmax) == offsetof(crt_bbox_f32, xmax) &&
                  offsetof(Box, ymax) == offsetof(crt_bbox_f32, ymax) &&
                  offsetof(Box, id) == offsetof(crt_bbox_f32, id),
                "BBOX<float> member offsets");
  return reinterpret_cast<crt_bbox_f32*>(&b);
}
template <class Tree>
inline crt_rtree_f32* as_c_tree(Tree& t)
{
  static_assert(sizeof(Tree) == sizeof(crt_rtree_f32), "RTREE<float> layout");
  static_assert(offsetof(Tree, sz) == offsetof(crt_rtree_f32, sz) &&
                  offsetof(Tree, fanout) == offsetof(crt_rtree_f32, fanout) &&
                  offsetof(Tree, xmin) == offsetof(crt_rtree_f32, xmin) &&
                  offsetof(Tree, pos) == offsetof(crt_rtree_f32, pos) &&
                  offsetof(Tree, len) == offsetof(crt_rtree_f32, len),
                "RTREE<float> member offsets");
  return reinterpret_cast<crt_rtree_f32*>(&t);
}
template <class Pair>
inline crt_idpair* as_c_pair(Pair& p)
{
  static_assert(sizeof(Pair) == sizeof(crt_idpair), "IDPAIR layout");
  static_assert(offsetof(Pair, sz) == offsetof(crt_idpair, sz) &&
                  offsetof(Pair, fid) == offsetof(crt_idpair, fid) &&
                  offsetof(Pair, tid) == offsetof(crt_idpair, tid),
                "IDPAIR member offsets");
  return reinterpret_cast<crt_idpair*>(&p);
}
}  // namespace detail
}  // namespace crtree

/* build_rtree: sorts d_box in place into Z-order, allocates the node arrays of
 * d_rt (d_rt.fanout set by the caller) and returns R_sz. */
template <template <class> class Box, template <class> class Tree>
inline int build_rtree(Box<float>& d_box, Tree<float>& d_rt)
{
  int32_t rsz = 0;
  int s = crt_build_f32(crtree::detail::as_c_box(d_box), crtree::detail::as_c_tree(d_rt), nullptr,
                        &rsz);
  if (s != CRT_OK) throw crtree::error(s, "build_rtree");
  return rsz;
}

/* bfs_frontier: allocates d_dq and fills it with every (box id, window index)
 * pair whose boxes intersect. */
template <template <class> class Box, template <class> class Tree, class Pair>
inline void bfs_frontier(const Tree<float>& d_rt, const Box<float>& d_rbox,
                         const Box<float>& d_qbox, Pair& d_dq)
{
  int s = crt_query_f32(crtree::detail::as_c_tree(const_cast<Tree<float>&>(d_rt)),
                        crtree::detail::as_c_box(const_cast<Box<float>&>(d_rbox)),
                        crtree::detail::as_c_box(const_cast<Box<float>&>(d_qbox)),
                        crtree::detail::as_c_pair(d_dq), nullptr);
  if (s != CRT_OK) throw crtree::error(s, "bfs_frontier");
}

/* bfs_thrust: the same pair set as bfs_frontier. */
template <template <class> class Box, template <class> class Tree, class Pair>
inline void bfs_thrust(const Tree<float>& d_rt, const Box<float>& d_rbox, const Box<float>& d_qbox,
                       Pair& d_dq)
{
  int s = crt_query_thrust_f32(crtree::detail::as_c_tree(const_cast<Tree<float>&>(d_rt)),
                               crtree::detail::as_c_box(const_cast<Box<float>&>(d_rbox)),
                               crtree::detail::as_c_box(const_cast<Box<float>&>(d_qbox)),
                               crtree::detail::as_c_pair(d_dq), nullptr);
  if (s != CRT_OK) throw crtree::error(s, "bfs_thrust");
}
