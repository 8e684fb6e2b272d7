/*
 * BBOX / RTREE / IDPAIR for callers that do not have the reference's own
 * src/rtree.h.  The member names, order and types are those of
 * trxcllnt/curtree src/rtree.h:3-29 so that code written against the
 * reference compiles unchanged and the structs are passed through the C ABI
 * of crtree.h as-is (layouts are checked in crtree/rtree_compat.h).
 * Include either this header or the reference's rtree.h, not both.
 */
#pragma once

template <class T>
struct BBOX {
  int sz;
  T* xmin;
  T* ymin;
  T* xmax;
  T* ymax;
  int* id;
};

template <class T>
struct RTREE {
  int sz;
  int fanout;
  T* xmin;
  T* ymin;
  T* xmax;
  T* ymax;
  int* pos;
  int* len;
};

struct IDPAIR {
  int sz;
  int* fid;
  int* tid;
};
