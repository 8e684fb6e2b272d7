/*
 * crtree -- B200-native 2-D bounding-box R-tree: Z-order bulk load and
 * batched window query behind a C ABI.
 *
 * The drop-in entry points replace the reference's (trxcllnt/curtree)
 * header templates one for one; every declaration below names the reference
 * interface it replaces (paths relative to that project's root).  The
 * extended entry points add what the reference lacks: 64-bit result counts,
 * caller-owned output with overflow-and-retry, explicit streams, persistent
 * batches captured in CUDA graphs, and a serving loop.
 *
 * Conventions
 *   - Every function returns a crt_status code; none exits, aborts or traps.
 *     crt_last_error() gives a message for the calling thread's last failure.
 *   - Pointers inside crt_bbox_f32 / crt_rtree_f32 / crt_idpair are device
 *     pointers (cudaMalloc or equivalent), unless a function says otherwise.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).
 *   - Arithmetic is the reference's: fp32 centre (xmin + xmax) / 2 truncated
 *     to uint16 per axis, a 32-bit Morton key sorted as a signed int (stable),
 *     fp32 min/max node boxes, and the closed-interval intersection test
 *     !(q.xmin > b.xmax || q.xmax < b.xmin || q.ymin > b.ymax || q.ymax < b.ymin).
 */
#ifndef CRTREE_H_
#define CRTREE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* crt_stream_t; /* same type as cudaStream_t */

typedef enum {
  CRT_OK                  = 0,
  CRT_ERR_INVALID_ARG     = 1, /* n < 1, fanout < 2, null pointer, n + R_sz > INT32_MAX ... */
  CRT_ERR_OOM             = 2, /* a device or host allocation failed */
  CRT_ERR_OVERFLOW_INT32  = 3, /* result count does not fit the reference's int sz */
  CRT_ERR_OUTPUT_OVERFLOW = 4, /* caller-owned output too small; *required holds the size */
  CRT_ERR_DEVICE_TIMEOUT  = 5, /* a bounded device-side wait ran out */
  CRT_ERR_CUDA            = 6, /* a CUDA runtime call failed */
  CRT_ERR_NOT_SUPPORTED   = 7,
  CRT_ERR_BUSY            = 8  /* serving: admission rejected (queue or memory full) */
} crt_status;

/* Layout-identical to BBOX<float> (src/rtree.h:3-11). */
typedef struct {
  int sz;
  float* xmin;
  float* ymin;
  float* xmax;
  float* ymax;
  int* id;
} crt_bbox_f32;

/* Layout-identical to RTREE<float> (src/rtree.h:13-23).  Nodes [0, sz): root
 * first, then each level downward; the children of node i are
 * [pos[i], pos[i] + len[i]); pos[i] >= sz means the children are boxes at
 * sorted slots pos[i] - sz ... */
typedef struct {
  int sz;
  int fanout;
  float* xmin;
  float* ymin;
  float* xmax;
  float* ymax;
  int* pos;
  int* len;
} crt_rtree_f32;

/* Layout-identical to IDPAIR (src/rtree.h:25-29): fid = box id, tid = query
 * index. */
typedef struct {
  int sz;
  int* fid;
  int* tid;
} crt_idpair;

const char* crt_status_string(int status);
const char* crt_last_error(void);
/* Library version string and the number of kernels launched by this process
 * so far (a cheap counter the benchmark reports). */
const char* crt_version(void);
uint64_t crt_kernel_launches(void);

/* ---------------------------------------------------------------------- */
/* Drop-in entry points                                                     */
/* ---------------------------------------------------------------------- */

/* Replaces `template <class T> int build_rtree(BBOX<T>& d_box, RTREE<T>& d_rt)`
 * (src/rtree_bulkload_thrust.cuh:62-213).
 * Reads d_rt->fanout, sorts d_box IN PLACE into Z-order (its five arrays are
 * permuted; id[] then holds the original ids), allocates the six node arrays
 * of d_rt from the device's stream-ordered pool (cudaMallocAsync on stream;
 * free with crt_rtree_free or the reference's rt_d_free, both cudaFree), fills them bit-exactly as the reference does, sets d_rt->sz and
 * *out_r_sz to R_sz.  Returns after the tree is complete on the device.
 * d_box->sz == 1 gives R_sz == 0, as in the reference; d_box->sz < 1 or
 * fanout < 2 (where the reference never returns) give CRT_ERR_INVALID_ARG. */
int crt_build_f32(crt_bbox_f32* d_box, crt_rtree_f32* d_rt, crt_stream_t stream,
                  int32_t* out_r_sz);

/* Replaces `bfs_frontier(const RTREE<T>&, const BBOX<T>& d_rbox,
 * const BBOX<T>& d_qbox, IDPAIR& d_dq)` (src/rtree_bfs_frontier.cuh:292-529).
 * d_rbox is the box set build sorted (same arrays as d_box after
 * crt_build_f32).  Allocates d_dq->fid / d_dq->tid from the stream-ordered
 * pool (free with crt_idpair_free or the reference's idpair_d_free) and fills them with every
 * (box id, query index) pair whose boxes intersect, in unspecified order.
 * Never overflows (the reference aborts when a 32-query block expands past
 * 1024 nodes); results past INT32_MAX pairs give CRT_ERR_OVERFLOW_INT32.
 * With R_sz == 0 (a one-box tree) the box is tested directly. */
int crt_query_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                  const crt_bbox_f32* d_qbox, crt_idpair* d_dq, crt_stream_t stream);

/* Replaces `bfs_thrust(...)` (src/rtree_bfs_thrust.cuh:59-256), which returns
 * the same pair set as bfs_frontier; same contract as crt_query_f32. */
int crt_query_thrust_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                         const crt_bbox_f32* d_qbox, crt_idpair* d_dq, crt_stream_t stream);

/* Replace rt_d_free / idpair_d_free (src/utility.cuh:137-162, 187-195):
 * cudaFree the arrays and null the pointers. */
int crt_rtree_free(crt_rtree_f32* d_rt);
int crt_idpair_free(crt_idpair* d_dq);

/* ---------------------------------------------------------------------- */
/* Extended entry points (no reference counterpart)                         */
/* ---------------------------------------------------------------------- */

/* Out-of-place build: reads d_in (unchanged), writes the Z-ordered boxes into
 * the caller-allocated arrays of d_sorted (same sz), and writes the nodes into
 * the caller-allocated arrays of d_rt (capacity crt_tree_size(sz, fanout)).
 * Asynchronous on `stream`; scratch comes from the stream-ordered allocator. */
int crt_build_into_f32(const crt_bbox_f32* d_in, crt_bbox_f32* d_sorted, crt_rtree_f32* d_rt,
                       crt_stream_t stream);

/* R_sz for n boxes at this fanout (exact integer ceiling per level), or -1. */
int64_t crt_tree_size(int64_t n, int fanout);
/* Number of levels (root .. leaf-parents) and the node count of each level,
 * leaf-parent level first, as in the reference's levels vector. */
int crt_tree_levels(int64_t n, int fanout, int64_t* levels, int max_levels);

/* Query modes. */
enum {
  CRT_QUERY_PERSISTENT = 0, /* one persistent work-stealing launch, Morton-ordered windows */
  CRT_QUERY_PLAIN      = 1  /* one warp per window in input order: count pass, scan, write pass */
};

typedef struct {
  int mode;             /* CRT_QUERY_PERSISTENT or CRT_QUERY_PLAIN */
  int sort_windows;     /* persistent: visit windows in Morton order of their centres (default 1) */
  int stage_levels;     /* persistent: whole tree levels below the root staged in shared memory
                           with bulk async copies (default 2, 0 = none; levels that do not fit
                           beside the warps' frontier stacks are left out) */
  int warps_per_cta;    /* persistent: 8, 16 or 32 warps per CTA (0 = default) */
  int chunk;            /* persistent: output slots a warp reserves at a time (0 = default) */
  int no_contain;       /* 1: test every box even under nodes the window contains */
  int warps_per_window; /* persistent: warps sharing one window, each taking an equal share of
                           the root's children (1, 2 or 4; 0 = 1) */
  int reserved[1];
} crt_query_opts;

void crt_query_opts_default(crt_query_opts* o);

/* Device-resident result block of an extended query (caller-allocated,
 * 64 bytes, device memory).  count = pairs written (valid when overflow == 0),
 * required = exact pair count, overflow = 1 when required > capacity,
 * error = a crt_status raised on the device. */
typedef struct {
  int64_t count;
  int64_t required;
  int32_t overflow;
  int32_t error;
  int64_t reserved[5];
} crt_query_result;

/* Windows against a tree into caller-owned output.  Asynchronous: enqueues
 * the work on `stream` and writes *d_result on the device.  When the output is
 * too small, d_result->overflow is set and d_result->required holds the exact
 * pair count: grow the output to crt_query_capacity(required, ...) and call
 * again (overflow-and-retry).  PLAIN mode also writes per-window hit counts
 * (int64, nq + 1 entries, exclusive prefix) into d_offsets when non-NULL, and
 * its pairs come grouped by window in window order.  PLAIN mode with
 * d_offsets may pass d_tid = NULL: the result is then CSR (box ids of window
 * w at d_fid[d_offsets[w] .. d_offsets[w + 1])), half the bytes of pairs. */
int crt_query_into_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                       const crt_bbox_f32* d_qbox, int32_t* d_fid, int32_t* d_tid,
                       int64_t capacity, crt_query_result* d_result, int64_t* d_offsets,
                       const crt_query_opts* opts, crt_stream_t stream);

/* Sorts n pairs in place into (window, box id) order, both ascending as
 * signed ints: the order the reference's drivers produce with two host
 * stable sorts (src/rtree_test_frontier.cu:102-105), here on the GPU.
 * Synchronous; at most INT32_MAX pairs per call. */
int crt_pairs_canonicalize(int32_t* d_fid, int32_t* d_tid, int64_t n, crt_stream_t stream);

/* Per-window pair counts and order-independent digests of a pair list, for
 * checking a result of billions of pairs without sorting it.  The reference's
 * drivers verify a query by sorting the pairs and comparing vectors
 * (src/rtree_test_frontier.cu:102-123); this is that check in a form whose
 * value does not depend on pair order.  For each pair i with window
 * w = d_tid[i] + window_base in [0, nq): d_counts[w] += 1 and
 * d_hashes[w] += mix(((uint64_t)w << 32) | (uint32_t)d_fid[i]) mod 2^64, where
 * mix is the splitmix64 finaliser.  Pairs whose window falls outside [0, nq)
 * are skipped and counted in *d_bad (device int64; may be NULL).  The arrays
 * accumulate (zero them first), so a result streamed in batches is digested
 * batch by batch with each batch's window_base.  Asynchronous on `stream`. */
int crt_pairs_digest(const int32_t* d_fid, const int32_t* d_tid, int64_t n, int64_t window_base,
                     int64_t nq, int64_t* d_counts, uint64_t* d_hashes, int64_t* d_bad,
                     crt_stream_t stream);

/* Output slots to allocate for `pairs` hit pairs so that a PERSISTENT query
 * cannot overflow (adds the per-warp reservation slack). */
int64_t crt_query_capacity(int64_t pairs, const crt_query_opts* opts);

/* Synchronous convenience over crt_query_into_f32: runs, reads the result
 * block, and returns CRT_ERR_OUTPUT_OVERFLOW with *required set when the
 * output was too small. */
int crt_query_sync_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                       const crt_bbox_f32* d_qbox, int32_t* d_fid, int32_t* d_tid,
                       int64_t capacity, int64_t* count, int64_t* required,
                       const crt_query_opts* opts, crt_stream_t stream);

/* The plain query (CRT_QUERY_PLAIN of crt_query_into_f32: the same pairs in
 * the same order, grouped by window) for callers that cannot allocate device
 * memory while they run -- a process whose device memory belongs to another
 * allocator or budget, or a loop that cannot take cudaMalloc's implicit
 * synchronisation.  No counterpart in the reference.  It allocates nothing:
 * its scratch is a fixed 1 MiB device array inside the library (held by every
 * GPU that loads the library until exit), so a call takes at most 65536
 * windows (more gives CRT_ERR_INVALID_ARG).  The caller passes the tree, the
 * windows, the output arrays and the device result block as usual.  The first
 * call on a device looks up the array's device address (with that device
 * current).  Calls share the array: calls whose work overlaps on the GPU
 * race, so serialise them (one stream, one thread at a time). */
int crt_query_plain_noalloc_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                                const crt_bbox_f32* d_qbox, int32_t* d_fid, int32_t* d_tid,
                                int64_t capacity, crt_query_result* d_result, crt_stream_t stream);

/* Per-window workload statistics: hit count and number of leaf boxes the
 * reference's algorithm tests (int64 device arrays of nq entries, either may
 * be NULL); totals (host, 4 entries, may be NULL): [0] all hits, [1] leaf
 * boxes tested box by box (the reference's algorithm), [2] leaf boxes tested
 * with the containment shortcut (this library's queries), [3] hits emitted
 * as contained slot ranges.  Synchronous.  Sizes outputs before a query and
 * gives the benchmark its algorithmic bytes. */
int crt_query_stats_f32(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                        const crt_bbox_f32* d_qbox, int64_t* d_hits, int64_t* d_tested,
                        int64_t* totals, crt_stream_t stream);

/* Persistent batch plan: binds a tree, a window buffer of up to max_nq
 * windows and an output buffer, and records the whole query (counter reset,
 * window ordering, persistent traversal, output compaction) as one CUDA
 * graph.  crt_plan_launch replays it for the windows currently in the bound
 * buffer (nq may change between launches; the graph reads it from device
 * memory).  The plan owns its scratch. */
typedef struct crt_plan_s* crt_plan;
int crt_plan_create(const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                    const crt_bbox_f32* d_qbox, int64_t max_nq, int32_t* d_fid, int32_t* d_tid,
                    int64_t capacity, crt_query_result* d_result, const crt_query_opts* opts,
                    crt_stream_t stream, crt_plan* out);
int crt_plan_set_nq(crt_plan plan, int64_t nq, crt_stream_t stream);
int crt_plan_launch(crt_plan plan, crt_stream_t stream);
int crt_plan_destroy(crt_plan plan);

/* ---------------------------------------------------------------------- */
/* Ingest and persistence                                                   */
/* ---------------------------------------------------------------------- */

/* Replaces readMBR (src/utility.cpp:5-40): reads n records
 * "x1,y1,x2,y2,id,pid,nume" from a text file into HOST arrays as the boxes
 * [min(x1,x2) - r, max(x1,x2) + r] x [min(y1,y2) - r, max(y1,y2) + r] with
 * their ids (fp32 arithmetic and %f/%d parsing as the reference's fscanf).
 * A missing file, a malformed record or fewer than n records give
 * CRT_ERR_INVALID_ARG (the reference exits or throws); *n_read = records
 * parsed before the problem. */
int crt_read_mbr_csv(const char* path, int64_t n, float r, float* xmin, float* ymin, float* xmax,
                     float* ymax, int32_t* id, int64_t* n_read);
/* Replaces readMBR followed by box_h2d (src/utility.cpp:5-40,
 * src/utility.cuh:42-66): the same format, values, statuses and *n_read as
 * crt_read_mbr_csv, with the records found and parsed on the GPU.  The boxes
 * land in newly cudaMalloc'd arrays *d_box (free with crt_bbox_free); n = -1
 * reads every record of the file.  On an error nothing is allocated.
 * Records the device parser cannot convert with certainty (hex or inf/nan
 * spellings, values within a few double ulps of a float rounding boundary,
 * malformed records, ...) are parsed by the host parser, so the result is
 * always the host loader's.  Returns after the boxes are on the device. */
int crt_read_mbr_csv_device(const char* path, int64_t n, float r, crt_bbox_f32* d_box,
                            int64_t* n_read, crt_stream_t stream);
/* Binary form of the same records (no reference counterpart: the reference
 * reads text only): a file of 28-byte little-endian records, float32 x1, y1,
 * x2, y2 then int32 id, pid, nume, read into newly cudaMalloc'd arrays *d_box
 * with readMBR's box [min(x1,x2) - r, max(x1,x2) + r] x [min(y1,y2) - r,
 * max(y1,y2) + r] (free with crt_bbox_free).  n = -1 reads every record; a
 * file size that is not a multiple of 28, or fewer than n records, is
 * CRT_ERR_INVALID_ARG (*n_read = records present). */
int crt_read_mbr_bin_device(const char* path, int64_t n, float r, crt_bbox_f32* d_box,
                            int64_t* n_read, crt_stream_t stream);
/* The same for text already in host memory (len bytes), into the caller's
 * device arrays of n entries. */
int crt_parse_mbr_csv_device(const char* text, int64_t len, int64_t n, float r, float* d_xmin,
                             float* d_ymin, float* d_xmax, float* d_ymax, int32_t* d_id,
                             int64_t* n_read, crt_stream_t stream);

/* Writes a built tree and its sorted box set to a file (no reference
 * counterpart; format in curtree_b200/csrc/io.cu). */
int crt_tree_save(const char* path, const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox);
/* Reads such a file into newly cudaMalloc'd device arrays (free with
 * crt_rtree_free and crt_bbox_free); the result can be queried at once. */
int crt_tree_load(const char* path, crt_rtree_f32* d_rt, crt_bbox_f32* d_rbox);
/* Replaces box_d_free (src/utility.cuh:68-89): cudaFree the five arrays. */
int crt_bbox_free(crt_bbox_f32* d_box);

/* ---------------------------------------------------------------------- */
/* Serving loop (no reference counterpart: the reference answers one batch   */
/* per call)                                                                 */
/* ---------------------------------------------------------------------- */

/* Continuous batching of window-query requests against device-resident
 * trees.  One persistent kernel serves every admitted request; requests that
 * arrive while others run are admitted as soon as a request slot and arena
 * memory are free, and their windows are processed alongside the others'.
 * A request is admitted by its HBM footprint: 16 bytes per window plus an
 * output estimate of 8 bytes per expected pair (host windows: their area,
 * clipped to the tree's root MBR, times the tree's box density and a learned
 * correction; device windows: the tree's running pairs-per-window average;
 * either times output_slack).  A request whose output outgrows
 * the estimate is re-run with its exact size (overflow-and-retry) before it
 * completes.  Results stay in the arena until crt_server_release.
 * While requests are in flight the device loop holds all but one SM's worth
 * of the GPU's CTA slots.  A kernel of another stream runs beside it on the
 * slots left free when its stream has a hardware queue of its own
 * (CUDA_DEVICE_MAX_CONNECTIONS); otherwise it waits until the loop stops,
 * idle_ms after the last request completes. */
typedef struct crt_server_s* crt_server;

typedef struct {
  int64_t arena_bytes;     /* device memory for windows and outputs in flight (default 8 GiB) */
  int max_requests;        /* request slots admitted at once (default 4096) */
  int max_trees;           /* default 16 */
  double pairs_per_window; /* initial output estimate per window (default 64) */
  double output_slack;     /* multiplier on the estimate (default 1.5; below 1 forces re-runs) */
  int idle_ms;             /* stop the device loop after this long without work (default 20) */
  int64_t device_wait_us;  /* bound on any device-side wait (default 2 s) */
  int reserved[4];
} crt_server_opts;

typedef struct {
  int64_t request_id;
  int tree_id;
  int status;           /* CRT_OK, or the error that ended the request */
  int64_t nq;
  int64_t count;        /* hit pairs */
  int32_t* d_fid;       /* device, count entries: box ids */
  int32_t* d_tid;       /* device, count entries: window index within the request */
  double submit_time_s; /* steady clock, seconds */
  double complete_time_s;
  int retries;          /* overflow re-runs */
  int reserved;
} crt_server_completion;

void crt_server_opts_default(crt_server_opts* o);
int crt_server_create(const crt_server_opts* opts, crt_server* out);
/* Registers a built tree (crt_build_f32 output: d_rbox is the sorted box set).
 * The arrays must outlive the server.  Trees are added before the first
 * submission. */
int crt_server_add_tree(crt_server s, const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox,
                        int* tree_id);
/* Admits nq windows (host or device pointers; copied before return) for one
 * tree, or returns CRT_ERR_BUSY when no slot or arena space is free now. */
int crt_server_submit(crt_server s, int tree_id, const float* xmin, const float* ymin,
                      const float* xmax, const float* ymax, int64_t nq, int64_t* request_id);
/* Takes up to max_out completions, waiting up to wait_ms for the first. */
int crt_server_poll(crt_server s, crt_server_completion* out, int max_out, int* n_out,
                    int wait_ms);
/* Frees a completed request's windows and output. */
int crt_server_release(crt_server s, int64_t request_id);
/* Counters; returns the device loop's last error status (CRT_OK if none). */
int crt_server_stats(crt_server s, int64_t* submitted, int64_t* completed, int64_t* retried,
                     int64_t* arena_used);
int crt_server_destroy(crt_server s);

/* ---------------------------------------------------------------------- */
/* Kernel timing (no reference counterpart; the reference prints host        */
/* gettimeofday timers, src/rtree_bulkload_thrust.cuh:74-89)                */
/* ---------------------------------------------------------------------- */

/* When enabled, the library brackets each major kernel launch (encode,
 * onesweep passes, level reductions, query traversal kernels, graph replays)
 * with CUDA events on its own stream.  crt_profile_collect waits for them and
 * sums the durations of the launches named `name` (all when NULL/empty):
 * "encode", "sort_pass", "level", "traverse_persistent", "traverse_plain",
 * "plan". */
void crt_profile_enable(int on);
int crt_profile_collect(const char* name, double* total_ms, int64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* CRTREE_H_ */
