/*
 * CPU restatement of the reference R-tree hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the oracle that the CUDA library is checked against.  Only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark load
 * it; nothing in the product library links, calls or falls back to it.
 *
 * Each function restates one piece of trxcllnt/curtree (paths are relative to
 * that project's root):
 *   - Morton key          src/rtree_bulkload_thrust.cuh:52-60, src/z_order.cuh:63-69
 *   - stable signed sort  src/rtree_bulkload_thrust.cuh:72, 83-86 (thrust::sort_by_key
 *                         on an int key: CUB's stable LSD radix sort, signed order)
 *   - level sizes         src/rtree_bulkload_thrust.cuh:103-117
 *   - node build          src/rtree_bulkload_thrust.cuh:32-50, 127-172
 *   - tree query          src/rtree_bfs_frontier.cuh:40-44, 60-182, 191-289 and
 *                         src/rtree_bfs_thrust.cuh:44-47, 95-250
 *   - brute force         src/utility.h:16-45 (intersect_cpu, nested_loop_query)
 *
 * Pinning: the brute force is checked against the reference's own
 * nested_loop_query compiled from its sources (oracle/Makefile, target ref),
 * and the build against node arrays written by the reference's own
 * build_rtree run on a B200 (tests/golden/).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* Morton key                                                                */
/* ------------------------------------------------------------------------ */

/* Float -> uint16 conversion as the reference's device build performs its
 * `(ushort)` cast (src/rtree_bulkload_thrust.cuh:55-56): truncate toward zero
 * to an unsigned 32-bit integer, saturating (negative and NaN -> 0,
 * >= 2^32 -> 2^32 - 1), then keep the low 16 bits.  Pinned by the golden
 * fixtures whose box centres lie outside [0, 65536). */
uint16_t orc_f2u16(float v)
{
  if (v != v) return 0;
  if (v <= 0.0f) return 0;
  if (v >= 4294967296.0f) return 0xFFFF;
  return (uint16_t)((uint32_t)v & 0xFFFFu);
}

/* Spread the 16 bits of v over the even bit positions of a 32-bit word: the
 * value the reference's 256-entry dilation table pair produces
 * (src/z_order.cuh:63-65). */
uint32_t orc_dilate16(uint16_t v)
{
  uint32_t x = v;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

/* z_order(x, y) = dilate(y) << 1 | dilate(x)  (src/z_order.cuh:67-69). */
uint32_t orc_zorder(uint16_t x, uint16_t y) { return (orc_dilate16(y) << 1) | orc_dilate16(x); }

/* mbr2key (src/rtree_bulkload_thrust.cuh:52-60): key of the box centre,
 * stored as a signed int (src/rtree_bulkload_thrust.cuh:72). */
int32_t orc_key(float xmin, float ymin, float xmax, float ymax)
{
  float cx = (xmin + xmax) / 2;
  float cy = (ymin + ymax) / 2;
  return (int32_t)orc_zorder(orc_f2u16(cx), orc_f2u16(cy));
}

void orc_keys(const float* xmin, const float* ymin, const float* xmax, const float* ymax,
              int64_t n, int32_t* keys)
{
  for (int64_t i = 0; i < n; i++) keys[i] = orc_key(xmin[i], ymin[i], xmax[i], ymax[i]);
}

/* Stable sort of positions by signed 32-bit key: perm[k] = input position of
 * the k-th smallest key, ties in input order.  LSD counting sort with 8-bit
 * digits on key ^ 0x80000000 (signed order as unsigned). */
int orc_sort_perm(const int32_t* keys, int64_t n, int32_t* perm)
{
  uint32_t* k0 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
  uint32_t* k1 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
  int32_t* p1 = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
  if (!k0 || !k1 || !p1) { free(k0); free(k1); free(p1); return -1; }
  for (int64_t i = 0; i < n; i++) { k0[i] = (uint32_t)keys[i] ^ 0x80000000u; perm[i] = (int32_t)i; }
  uint32_t* ks = k0; uint32_t* kd = k1; int32_t* ps = perm; int32_t* pd = p1;
  for (int shift = 0; shift < 32; shift += 8) {
    int64_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (int64_t i = 0; i < n; i++) cnt[((ks[i] >> shift) & 0xFF) + 1]++;
    for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
    for (int64_t i = 0; i < n; i++) {
      int64_t d = cnt[(ks[i] >> shift) & 0xFF]++;
      kd[d] = ks[i];
      pd[d] = ps[i];
    }
    uint32_t* tk = ks; ks = kd; kd = tk;
    int32_t* tp = ps; ps = pd; pd = tp;
  }
  /* four passes: the result is back in `perm` */
  free(k0); free(k1); free(p1);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Level sizes                                                               */
/* ------------------------------------------------------------------------ */

/* Node count per level, leaf-parent level first, root last
 * (src/rtree_bulkload_thrust.cuh:103-115), with an exact integer ceiling.
 * Returns the number of levels; 0 for n == 1 (the reference allocates an
 * empty tree there); -1 for n < 1 or fanout < 2 (the reference never
 * terminates on those). */
int orc_levels(int64_t n, int fanout, int64_t* levels, int max_levels)
{
  if (n < 1 || fanout < 2) return -1;
  int lev = 0;
  int64_t len = n;
  while (len != 1) {
    len = (len + fanout - 1) / fanout;
    if (lev >= max_levels) return -2;
    levels[lev++] = len;
  }
  return lev;
}

/* The reference's own float formula `ceil((float)length / d)`
 * (src/rtree_bulkload_thrust.cuh:109); used only to show where it departs from
 * the exact ceiling. */
int orc_levels_ref_float(int64_t n, int fanout, int64_t* levels, int max_levels)
{
  if (n < 1 || fanout < 2) return -1;
  int lev = 0;
  int len = (int)n;
  while (len != 1) {
    int num_nodes = (int)ceil((double)((float)len / (float)fanout));
    if (lev >= max_levels) return -2;
    levels[lev++] = num_nodes;
    len = num_nodes;
  }
  return lev;
}

/* ------------------------------------------------------------------------ */
/* Node build                                                                */
/* ------------------------------------------------------------------------ */

/* min()/max() of the reference's reduce_op (src/rtree_bulkload_thrust.cuh:
 * 42-45): NaN loses to a number; -0 orders below +0. */
static float fmin_dev(float a, float b)
{
  if (a != a) return b;
  if (b != b) return a;
  if (a == b) return signbit(a) ? a : b;
  return a < b ? a : b;
}
static float fmax_dev(float a, float b)
{
  if (a != a) return b;
  if (b != b) return a;
  if (a == b) return signbit(a) ? b : a;
  return a > b ? a : b;
}

/* build_rtree (src/rtree_bulkload_thrust.cuh:62-213): sort the boxes by key
 * (stable, signed), then reduce groups of `fanout` consecutive children level
 * by level.  Node storage: root at 0, levels downward, the leaf-parent level
 * last; a leaf-parent's pos is R_sz + first box slot, an upper node's pos is
 * the index of its first child node.  Writes the permuted boxes to out_* and
 * returns R_sz (negative on bad arguments). */
int64_t orc_build(const float* xmin, const float* ymin, const float* xmax, const float* ymax,
                  const int32_t* id, int64_t n, int fanout,
                  float* oxmin, float* oymin, float* oxmax, float* oymax, int32_t* oid,
                  float* nxmin, float* nymin, float* nxmax, float* nymax,
                  int32_t* npos, int32_t* nlen)
{
  int64_t levels[64];
  int nlev = orc_levels(n, fanout, levels, 64);
  if (nlev < 0) return -1;
  int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!keys || !perm) { free(keys); free(perm); return -2; }
  orc_keys(xmin, ymin, xmax, ymax, n, keys);
  if (orc_sort_perm(keys, n, perm) != 0) { free(keys); free(perm); return -2; }
  for (int64_t s = 0; s < n; s++) {
    int64_t p = perm[s];
    oxmin[s] = xmin[p]; oymin[s] = ymin[p]; oxmax[s] = xmax[p]; oymax[s] = ymax[p]; oid[s] = id[p];
  }
  free(keys); free(perm);

  int64_t rsz = 0;
  for (int l = 0; l < nlev; l++) rsz += levels[l];
  int64_t start = rsz;
  int64_t child_start = 0, child_count = n;
  for (int l = 0; l < nlev; l++) {
    start -= levels[l];
    for (int64_t g = 0; g < levels[l]; g++) {
      int64_t c0 = g * fanout;
      int64_t c1 = c0 + fanout < child_count ? c0 + fanout : child_count;
      float a, b, c, d;
      if (l == 0) {
        a = oxmin[c0]; b = oymin[c0]; c = oxmax[c0]; d = oymax[c0];
        for (int64_t k = c0 + 1; k < c1; k++) {
          a = fmin_dev(a, oxmin[k]); b = fmin_dev(b, oymin[k]);
          c = fmax_dev(c, oxmax[k]); d = fmax_dev(d, oymax[k]);
        }
        npos[start + g] = (int32_t)(rsz + c0);
      } else {
        int64_t base = child_start;
        a = nxmin[base + c0]; b = nymin[base + c0]; c = nxmax[base + c0]; d = nymax[base + c0];
        for (int64_t k = c0 + 1; k < c1; k++) {
          a = fmin_dev(a, nxmin[base + k]); b = fmin_dev(b, nymin[base + k]);
          c = fmax_dev(c, nxmax[base + k]); d = fmax_dev(d, nymax[base + k]);
        }
        npos[start + g] = (int32_t)(base + c0);
      }
      nxmin[start + g] = a; nymin[start + g] = b; nxmax[start + g] = c; nymax[start + g] = d;
      nlen[start + g] = (int32_t)(c1 - c0);
    }
    child_start = start;
    child_count = levels[l];
  }
  return rsz;
}

/* ------------------------------------------------------------------------ */
/* Queries                                                                   */
/* ------------------------------------------------------------------------ */

/* intersect / intersect_cpu (src/rtree_bfs_frontier.cuh:40-44,
 * src/utility.h:16-20): closed intervals; a NaN compares false, so it never
 * excludes. */
static inline int isect(float x1, float y1, float x2, float y2, float m1, float n1, float m2, float n2)
{
  return !(x1 > m2 || x2 < m1 || y1 > n2 || y2 < n1);
}

static inline uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Order-independent digest of one hit pair (query index, box id). */
uint64_t orc_pair_hash(int32_t q, int32_t id)
{
  return mix64(((uint64_t)(uint32_t)q << 32) | (uint32_t)id);
}

typedef struct {
  /* tree */
  const float *nxmin, *nymin, *nxmax, *nymax;
  const int32_t *npos, *nlen;
  int64_t rsz;
  int fanout;
  /* permuted boxes */
  const float *bxmin, *bymin, *bxmax, *bymax;
  const int32_t* bid;
  int64_t nbox;
  /* queries */
  const float *qxmin, *qymin, *qxmax, *qymax;
  const int32_t* qid;      /* NULL: positional ids */
  int64_t q0, q1;
  /* outputs (per query) */
  int64_t* counts;         /* may be NULL */
  uint64_t* hashes;        /* may be NULL */
  int64_t* tested;         /* leaf boxes tested per query (T_leaf), may be NULL */
  int64_t* nodes_visited;  /* internal node tests per query, may be NULL */
  /* pair output: only for single-threaded calls */
  int32_t *out_fid, *out_tid;
  int64_t out_cap, out_n;
  int status;
} tq_args;

/* The reference's tree query (src/rtree_bfs_frontier.cuh:60-182 for the
 * descent, :191-289 for the leaf test; src/rtree_bfs_thrust.cuh:95-250 gives
 * the same set): the root is never tested; a node whose children are nodes
 * (pos < R_sz) passes on the children whose MBR intersects the window; a
 * leaf-parent (pos >= R_sz) tests its boxes [pos - R_sz, pos - R_sz + len).
 * With R_sz == 0 (a single box) the box is tested directly. */
static void tree_query_one(tq_args* a, int64_t q, int64_t* stack, int64_t stack_cap)
{
  float x1 = a->qxmin[q], y1 = a->qymin[q], x2 = a->qxmax[q], y2 = a->qymax[q];
  int32_t qout = a->qid ? a->qid[q] : (int32_t)q;
  int64_t cnt = 0, tested = 0, visited = 0;
  uint64_t h = 0;
  if (a->rsz == 0) {
    for (int64_t s = 0; s < a->nbox; s++) {
      tested++;
      if (isect(x1, y1, x2, y2, a->bxmin[s], a->bymin[s], a->bxmax[s], a->bymax[s])) {
        int32_t fid = a->bid[s];
        cnt++;
        h += orc_pair_hash(qout, fid);
        if (a->out_fid) {
          if (a->out_n < a->out_cap) { a->out_fid[a->out_n] = fid; a->out_tid[a->out_n] = qout; }
          a->out_n++;
        }
      }
    }
  } else {
    int64_t sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      int64_t node = stack[--sp];
      int64_t pos = a->npos[node], len = a->nlen[node];
      if (pos >= a->rsz) {
        int64_t s0 = pos - a->rsz;
        for (int64_t s = s0; s < s0 + len && s < a->nbox; s++) {
          tested++;
          if (isect(x1, y1, x2, y2, a->bxmin[s], a->bymin[s], a->bxmax[s], a->bymax[s])) {
            int32_t fid = a->bid[s];
            cnt++;
            h += orc_pair_hash(qout, fid);
            if (a->out_fid) {
              if (a->out_n < a->out_cap) { a->out_fid[a->out_n] = fid; a->out_tid[a->out_n] = qout; }
              a->out_n++;
            }
          }
        }
      } else {
        /* push in reverse so that children pop in slot order */
        for (int64_t c = pos + len - 1; c >= pos; c--) {
          visited++;
          if (isect(x1, y1, x2, y2, a->nxmin[c], a->nymin[c], a->nxmax[c], a->nymax[c])) {
            if (sp >= stack_cap) { a->status = -3; return; }
            stack[sp++] = c;
          }
        }
      }
    }
  }
  if (a->counts) a->counts[q] = cnt;
  if (a->hashes) a->hashes[q] = h;
  if (a->tested) a->tested[q] = tested;
  if (a->nodes_visited) a->nodes_visited[q] = visited;
}

static void* tree_query_worker(void* p)
{
  tq_args* a = (tq_args*)p;
  int64_t cap = 64 * (int64_t)(a->fanout > 0 ? a->fanout : 2) + 64;
  int64_t* stack = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap);
  if (!stack) { a->status = -2; return NULL; }
  for (int64_t q = a->q0; q < a->q1 && a->status == 0; q++) tree_query_one(a, q, stack, cap);
  free(stack);
  return NULL;
}

/* Per-query hit counts, pair digests and work counters for a window batch
 * against a built tree, over `nthreads` host threads.  qid (may be NULL:
 * positional) gives each query's window index for the digests. */
int orc_tree_query_stats_ids(const float* nxmin, const float* nymin, const float* nxmax,
                             const float* nymax, const int32_t* npos, const int32_t* nlen,
                             int64_t rsz, int fanout,
                             const float* bxmin, const float* bymin, const float* bxmax,
                             const float* bymax, const int32_t* bid, int64_t nbox,
                             const float* qxmin, const float* qymin, const float* qxmax,
                             const float* qymax, const int32_t* qid, int64_t nq,
                             int64_t* counts, uint64_t* hashes, int64_t* tested,
                             int64_t* nodes_visited, int nthreads)
{
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  tq_args args[256];
  int started[256];
  int64_t per = (nq + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; t++) {
    tq_args* a = &args[t];
    memset(a, 0, sizeof(*a));
    a->nxmin = nxmin; a->nymin = nymin; a->nxmax = nxmax; a->nymax = nymax;
    a->npos = npos; a->nlen = nlen; a->rsz = rsz; a->fanout = fanout;
    a->bxmin = bxmin; a->bymin = bymin; a->bxmax = bxmax; a->bymax = bymax; a->bid = bid;
    a->nbox = nbox;
    a->qxmin = qxmin; a->qymin = qymin; a->qxmax = qxmax; a->qymax = qymax; a->qid = qid;
    a->q0 = t * per; a->q1 = (t + 1) * per < nq ? (t + 1) * per : nq;
    a->counts = counts; a->hashes = hashes; a->tested = tested; a->nodes_visited = nodes_visited;
    started[t] = 0;
    if (a->q0 >= a->q1) continue;
    if (pthread_create(&th[t], NULL, tree_query_worker, a) == 0) started[t] = 1;
    else tree_query_worker(a);
  }
  int st = 0;
  for (int t = 0; t < nthreads; t++) {
    if (started[t]) pthread_join(th[t], NULL);
    if (args[t].status != 0) st = args[t].status;
  }
  return st;
}

/* orc_tree_query_stats_ids with positional window indices. */
int orc_tree_query_stats(const float* nxmin, const float* nymin, const float* nxmax,
                         const float* nymax, const int32_t* npos, const int32_t* nlen,
                         int64_t rsz, int fanout,
                         const float* bxmin, const float* bymin, const float* bxmax,
                         const float* bymax, const int32_t* bid, int64_t nbox,
                         const float* qxmin, const float* qymin, const float* qxmax,
                         const float* qymax, int64_t nq,
                         int64_t* counts, uint64_t* hashes, int64_t* tested,
                         int64_t* nodes_visited, int nthreads)
{
  return orc_tree_query_stats_ids(nxmin, nymin, nxmax, nymax, npos, nlen, rsz, fanout, bxmin,
                                  bymin, bxmax, bymax, bid, nbox, qxmin, qymin, qxmax, qymax,
                                  NULL, nq, counts, hashes, tested, nodes_visited, nthreads);
}

/* Tree query writing every hit pair (fid = box id, tid = query index) in
 * query order, then the order the descent meets the boxes.  Single thread;
 * returns the total hit count (pairs past `cap` are counted, not written) or
 * a negative status. */
int64_t orc_tree_query_pairs(const float* nxmin, const float* nymin, const float* nxmax,
                             const float* nymax, const int32_t* npos, const int32_t* nlen,
                             int64_t rsz, int fanout,
                             const float* bxmin, const float* bymin, const float* bxmax,
                             const float* bymax, const int32_t* bid, int64_t nbox,
                             const float* qxmin, const float* qymin, const float* qxmax,
                             const float* qymax, int64_t nq,
                             int32_t* out_fid, int32_t* out_tid, int64_t cap)
{
  tq_args a;
  memset(&a, 0, sizeof(a));
  a.nxmin = nxmin; a.nymin = nymin; a.nxmax = nxmax; a.nymax = nymax;
  a.npos = npos; a.nlen = nlen; a.rsz = rsz; a.fanout = fanout;
  a.bxmin = bxmin; a.bymin = bymin; a.bxmax = bxmax; a.bymax = bymax; a.bid = bid; a.nbox = nbox;
  a.qxmin = qxmin; a.qymin = qymin; a.qxmax = qxmax; a.qymax = qymax;
  a.q0 = 0; a.q1 = nq;
  a.out_fid = out_fid; a.out_tid = out_tid; a.out_cap = cap;
  tree_query_worker(&a);
  if (a.status != 0) return a.status;
  return a.out_n;
}

/* ------------------------------------------------------------------------ */
/* Brute force (nested_loop_query, src/utility.h:22-45)                      */
/* ------------------------------------------------------------------------ */

typedef struct {
  const float *qxmin, *qymin, *qxmax, *qymax;
  const int32_t* qid;
  const float *dxmin, *dymin, *dxmax, *dymax;
  const int32_t* did;
  int64_t nd, q0, q1;
  int64_t* counts;
  uint64_t* hashes;
} nl_args;

static void* nested_worker(void* p)
{
  nl_args* a = (nl_args*)p;
  for (int64_t i = a->q0; i < a->q1; i++) {
    float x1 = a->qxmin[i], y1 = a->qymin[i], x2 = a->qxmax[i], y2 = a->qymax[i];
    int32_t qo = a->qid ? a->qid[i] : (int32_t)i;
    int64_t c = 0;
    uint64_t h = 0;
    for (int64_t j = 0; j < a->nd; j++) {
      if (isect(x1, y1, x2, y2, a->dxmin[j], a->dymin[j], a->dxmax[j], a->dymax[j])) {
        c++;
        h += orc_pair_hash(qo, a->did ? a->did[j] : (int32_t)j);
      }
    }
    if (a->counts) a->counts[i] = c;
    if (a->hashes) a->hashes[i] = h;
  }
  return NULL;
}

/* Per-query counts and digests of the brute force over `nthreads` threads. */
int orc_nested_loop_stats(const float* qxmin, const float* qymin, const float* qxmax,
                          const float* qymax, const int32_t* qid, int64_t nq,
                          const float* dxmin, const float* dymin, const float* dxmax,
                          const float* dymax, const int32_t* did, int64_t nd,
                          int64_t* counts, uint64_t* hashes, int nthreads)
{
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  nl_args args[256];
  int started[256];
  int64_t per = (nq + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; t++) {
    nl_args* a = &args[t];
    a->qxmin = qxmin; a->qymin = qymin; a->qxmax = qxmax; a->qymax = qymax; a->qid = qid;
    a->dxmin = dxmin; a->dymin = dymin; a->dxmax = dxmax; a->dymax = dymax; a->did = did;
    a->nd = nd;
    a->q0 = t * per; a->q1 = (t + 1) * per < nq ? (t + 1) * per : nq;
    a->counts = counts; a->hashes = hashes;
    started[t] = 0;
    if (a->q0 >= a->q1) continue;
    if (pthread_create(&th[t], NULL, nested_worker, a) == 0) started[t] = 1;
    else nested_worker(a);
  }
  for (int t = 0; t < nthreads; t++)
    if (started[t]) pthread_join(th[t], NULL);
  return 0;
}

/* Brute-force pairs in the reference's order: queries ascending, then data in
 * input order (src/utility.h:25-43).  Returns the hit count (pairs past `cap`
 * are counted, not written). */
int64_t orc_nested_loop_pairs(const float* qxmin, const float* qymin, const float* qxmax,
                              const float* qymax, const int32_t* qid, int64_t nq,
                              const float* dxmin, const float* dymin, const float* dxmax,
                              const float* dymax, const int32_t* did, int64_t nd,
                              int32_t* out_did, int32_t* out_qid, int64_t cap)
{
  int64_t n = 0;
  for (int64_t i = 0; i < nq; i++) {
    for (int64_t j = 0; j < nd; j++) {
      if (isect(qxmin[i], qymin[i], qxmax[i], qymax[i], dxmin[j], dymin[j], dxmax[j], dymax[j])) {
        if (n < cap) {
          out_did[n] = did ? did[j] : (int32_t)j;
          out_qid[n] = qid ? qid[i] : (int32_t)i;
        }
        n++;
      }
    }
  }
  return n;
}

/* ---------------------------------------------------------------------------
 * The reference's CPU check builds a Boost.Geometry rtree<value,
 * quadratic<16>> by inserting the boxes one at a time and then queries it
 * box by box (src/verify.hpp:35-95).  Boost is not available here, so this
 * restates the algorithm that parameter set names: Guttman's R-tree with the
 * quadratic split (A. Guttman, "R-trees: a dynamic index structure for
 * spatial searching", SIGMOD 1984), at most 16 and at least 4 entries per
 * node (Boost's default minimum for quadratic<16> is 0.3 x 16).  Insertion
 * descends to the child needing the least area enlargement (ties: the
 * smaller area), splits an overflowing node by the quadratic method (seeds:
 * the pair wasting the most area; then the entry with the greatest
 * preference for one group, to the group it enlarges least, keeping every
 * group at the minimum), and adjusts the covering rectangles up the path.
 * CPU baseline only: its tree shape differs from the reference's packed
 * tree, its pair set is the brute force's.
 * ------------------------------------------------------------------------- */
#define QR_MAX 16
#define QR_MIN 4

typedef struct { float x0, y0, x1, y1; } qr_rect;

typedef struct qr_node {
  int leaf, n;
  qr_rect r[QR_MAX + 1];
  intptr_t ent[QR_MAX + 1]; /* child node, or box id in a leaf */
} qr_node;

typedef struct {
  qr_node* root;
  int height;
  qr_node** blocks;
  int64_t nblocks, cap_blocks, used; /* nodes handed out of the last block */
} qr_tree;

#define QR_BLOCK 65536

static qr_node* qr_alloc(qr_tree* t, int leaf)
{
  if (t->nblocks == 0 || t->used == QR_BLOCK) {
    if (t->nblocks == t->cap_blocks) {
      int64_t c = t->cap_blocks ? 2 * t->cap_blocks : 64;
      qr_node** b = (qr_node**)realloc(t->blocks, sizeof(qr_node*) * (size_t)c);
      if (!b) return NULL;
      t->blocks = b;
      t->cap_blocks = c;
    }
    qr_node* blk = (qr_node*)malloc(sizeof(qr_node) * QR_BLOCK);
    if (!blk) return NULL;
    t->blocks[t->nblocks++] = blk;
    t->used = 0;
  }
  qr_node* nd = &t->blocks[t->nblocks - 1][t->used++];
  nd->leaf = leaf;
  nd->n = 0;
  return nd;
}

static inline float qr_area(qr_rect a) { return (a.x1 - a.x0) * (a.y1 - a.y0); }
static inline qr_rect qr_union(qr_rect a, qr_rect b)
{
  qr_rect u = {a.x0 < b.x0 ? a.x0 : b.x0, a.y0 < b.y0 ? a.y0 : b.y0, a.x1 > b.x1 ? a.x1 : b.x1,
               a.y1 > b.y1 ? a.y1 : b.y1};
  return u;
}
static qr_rect qr_cover(const qr_node* nd)
{
  qr_rect u = nd->r[0];
  for (int i = 1; i < nd->n; i++) u = qr_union(u, nd->r[i]);
  return u;
}

/* Splits the QR_MAX + 1 entries of nd between nd and a new node (quadratic). */
static qr_node* qr_split(qr_tree* t, qr_node* nd)
{
  const int m = nd->n;
  qr_rect r[QR_MAX + 1];
  intptr_t e[QR_MAX + 1];
  memcpy(r, nd->r, sizeof(qr_rect) * (size_t)m);
  memcpy(e, nd->ent, sizeof(intptr_t) * (size_t)m);
  int s1 = 0, s2 = 1;
  float worst = -INFINITY;
  for (int i = 0; i < m; i++)
    for (int j = i + 1; j < m; j++) {
      const float d = qr_area(qr_union(r[i], r[j])) - qr_area(r[i]) - qr_area(r[j]);
      if (d > worst) { worst = d; s1 = i; s2 = j; }
    }
  qr_node* b = qr_alloc(t, nd->leaf);
  if (!b) return NULL;
  char done[QR_MAX + 1];
  memset(done, 0, sizeof(done));
  nd->n = 0;
  nd->r[0] = r[s1]; nd->ent[0] = e[s1]; nd->n = 1;
  b->r[0] = r[s2]; b->ent[0] = e[s2]; b->n = 1;
  done[s1] = done[s2] = 1;
  qr_rect ca = r[s1], cb = r[s2];
  int left = m - 2;
  while (left > 0) {
    qr_node* all = NULL;
    if (nd->n + left == QR_MIN) all = nd;
    else if (b->n + left == QR_MIN) all = b;
    if (all) {
      for (int k = 0; k < m; k++)
        if (!done[k]) { all->r[all->n] = r[k]; all->ent[all->n] = e[k]; all->n++; done[k] = 1; }
      break;
    }
    int pick = -1;
    float best = -1.f, pd1 = 0.f, pd2 = 0.f;
    for (int k = 0; k < m; k++) {
      if (done[k]) continue;
      const float d1 = qr_area(qr_union(ca, r[k])) - qr_area(ca);
      const float d2 = qr_area(qr_union(cb, r[k])) - qr_area(cb);
      const float diff = fabsf(d1 - d2);
      if (pick < 0 || diff > best) { best = diff; pick = k; pd1 = d1; pd2 = d2; }
    }
    int to_a;
    if (pd1 != pd2) to_a = pd1 < pd2;
    else if (qr_area(ca) != qr_area(cb)) to_a = qr_area(ca) < qr_area(cb);
    else to_a = nd->n <= b->n;
    qr_node* g = to_a ? nd : b;
    g->r[g->n] = r[pick]; g->ent[g->n] = e[pick]; g->n++;
    if (to_a) ca = qr_union(ca, r[pick]); else cb = qr_union(cb, r[pick]);
    done[pick] = 1;
    left--;
  }
  return b;
}

static int qr_insert(qr_tree* t, qr_rect rc, int id)
{
  qr_node* path[64];
  int slot[64];
  int d = 0;
  qr_node* nd = t->root;
  while (!nd->leaf) {
    int best = 0;
    float be = INFINITY, ba = INFINITY;
    for (int i = 0; i < nd->n; i++) {
      const float a = qr_area(nd->r[i]);
      const float en = qr_area(qr_union(nd->r[i], rc)) - a;
      if (en < be || (en == be && a < ba)) { be = en; ba = a; best = i; }
    }
    path[d] = nd; slot[d] = best; d++;
    nd = (qr_node*)nd->ent[best];
  }
  nd->r[nd->n] = rc; nd->ent[nd->n] = id; nd->n++;
  qr_node* split = NULL;
  if (nd->n > QR_MAX && !(split = qr_split(t, nd))) return -2;
  qr_node* child = nd;
  while (d > 0) {
    d--;
    qr_node* p = path[d];
    p->r[slot[d]] = qr_cover(child);
    if (split) {
      p->r[p->n] = qr_cover(split); p->ent[p->n] = (intptr_t)split; p->n++;
      split = NULL;
      if (p->n > QR_MAX && !(split = qr_split(t, p))) return -2;
    }
    child = p;
  }
  if (split) {  /* the root split: a new root over both halves */
    qr_node* r = qr_alloc(t, 0);
    if (!r) return -2;
    r->r[0] = qr_cover(t->root); r->ent[0] = (intptr_t)t->root;
    r->r[1] = qr_cover(split); r->ent[1] = (intptr_t)split;
    r->n = 2;
    t->root = r;
    t->height++;
  }
  return 0;
}

static double qr_now(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* Inserts the n boxes in input order; *seconds receives the build time. */
void* orc_qrtree_build(const float* xmin, const float* ymin, const float* xmax, const float* ymax,
                       const int32_t* id, int64_t n, double* seconds)
{
  const double t0 = qr_now();
  qr_tree* t = (qr_tree*)calloc(1, sizeof(qr_tree));
  if (!t) return NULL;
  t->root = qr_alloc(t, 1);
  t->height = 1;
  for (int64_t i = 0; i < n && t->root; i++) {
    qr_rect rc = {xmin[i], ymin[i], xmax[i], ymax[i]};
    if (qr_insert(t, rc, id[i]) != 0) { t->root = NULL; break; }
  }
  if (seconds) *seconds = qr_now() - t0;
  return t;
}

void orc_qrtree_free(void* h)
{
  qr_tree* t = (qr_tree*)h;
  if (!t) return;
  for (int64_t b = 0; b < t->nblocks; b++) free(t->blocks[b]);
  free(t->blocks);
  free(t);
}

typedef struct {
  const qr_tree* t;
  const float *qx0, *qy0, *qx1, *qy1;
  const int32_t* qid;
  int64_t q0, q1;
  int64_t* counts;
  uint64_t* hashes;
  int status;
} qr_args;

static void* qr_query_worker(void* p)
{
  qr_args* a = (qr_args*)p;
  const int cap = 64 * QR_MAX;
  const qr_node** st = (const qr_node**)malloc(sizeof(qr_node*) * (size_t)cap);
  if (!st) { a->status = -2; return NULL; }
  for (int64_t q = a->q0; q < a->q1; q++) {
    const float x1 = a->qx0[q], y1 = a->qy0[q], x2 = a->qx1[q], y2 = a->qy1[q];
    const int32_t qo = a->qid ? a->qid[q] : (int32_t)q;
    int64_t cnt = 0;
    uint64_t h = 0;
    int sp = 0;
    st[sp++] = a->t->root;
    while (sp > 0) {
      const qr_node* nd = st[--sp];
      for (int i = 0; i < nd->n; i++) {
        const qr_rect r = nd->r[i];
        if (!isect(x1, y1, x2, y2, r.x0, r.y0, r.x1, r.y1)) continue;
        if (nd->leaf) {
          cnt++;
          h += orc_pair_hash(qo, (int32_t)nd->ent[i]);
        } else if (sp < cap) {
          st[sp++] = (const qr_node*)nd->ent[i];
        } else {
          a->status = -3;
        }
      }
    }
    if (a->counts) a->counts[q] = cnt;
    if (a->hashes) a->hashes[q] = h;
  }
  free(st);
  return NULL;
}

/* Per-window counts and pair digests over `nthreads` host threads (the tree
 * is read-only); *seconds receives the wall time of the queries. */
int orc_qrtree_query_stats(void* h, const float* qxmin, const float* qymin, const float* qxmax,
                           const float* qymax, const int32_t* qid, int64_t nq, int64_t* counts,
                           uint64_t* hashes, int nthreads, double* seconds)
{
  qr_tree* t = (qr_tree*)h;
  if (!t || !t->root) return -1;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  qr_args args[256];
  int started[256];
  const double t0 = qr_now();
  const int64_t per = (nq + nthreads - 1) / nthreads;
  for (int i = 0; i < nthreads; i++) {
    qr_args* a = &args[i];
    memset(a, 0, sizeof(*a));
    a->t = t;
    a->qx0 = qxmin; a->qy0 = qymin; a->qx1 = qxmax; a->qy1 = qymax; a->qid = qid;
    a->q0 = i * per; a->q1 = (i + 1) * per < nq ? (i + 1) * per : nq;
    a->counts = counts; a->hashes = hashes;
    started[i] = 0;
    if (a->q0 >= a->q1) continue;
    if (pthread_create(&th[i], NULL, qr_query_worker, a) == 0) started[i] = 1;
    else qr_query_worker(a);
  }
  int st = 0;
  for (int i = 0; i < nthreads; i++) {
    if (started[i]) pthread_join(th[i], NULL);
    if (args[i].status != 0) st = args[i].status;
  }
  if (seconds) *seconds = qr_now() - t0;
  return st;
}
