// GPU ingest of the reference's MBR text format (readMBR,
// src/utility.cpp:5-40): the text is copied to the device through pinned
// staging buffers by several host threads, record starts are found by a
// three-kernel line scan, and one thread parses each record.  The boxes,
// ids, statuses and *n_read are those of the host loader crt_read_mbr_csv
// (io.cu): numbers are converted by an exact fast path, and every record the
// fast path cannot decide with certainty is handed to the host parser.
//
// Record starts (the host loader's rule): the first byte of a line that is
// not ' ', '\t' or '\r', unless that byte is the line's '\n'.  Put another
// way, a byte that is neither blank nor '\n' starts a record when the last
// non-blank byte before it is a '\n', or when there is none.  The text is cut
// into 16 KiB tiles of 32 bytes per thread:
//   1. line_tile_kernel: per tile, the number of starts whose previous
//      non-blank byte lies in the tile, whether the tile's first non-blank
//      byte is a record byte (it starts a record if the tiles before end a
//      line), and the class of its last non-blank byte (none, '\n', other);
//   2. line_scan_kernel (one CTA): carries that class across the tiles and
//      sums the counts, giving each tile its first record index;
//   3. line_emit_kernel: writes the byte offset of each start at its record
//      index, for the first n records.
//
// Numbers (after Clinger, "How to read floating point numbers accurately",
// PLDI 1990): the decimal significand is kept to 19 digits w (digits past
// them are dropped, a relative change below 1e-18) and the decimal exponent
// e10 must lie in [-44, 44]; d = w * 10^e10 is formed in double with at most
// three roundings (w to double, then one or two exact powers of ten up to
// 1e22), so |d - x| < 7 units in the last place of d.  Rounding d to float
// then gives the correctly rounded float of x, as strtof does, unless d lies
// within 16 double ulps of a point halfway between two floats, or outside the
// normal float range: those records go to the host parser (about one random
// value in 2^24 is that close).  So do spellings the fast path does not take:
// hex and inf/nan forms, integers of more than 18 digits, exponents of more
// than five digits, fields of 63 bytes or more, long blank runs and blanks
// other than ' ', '\t', '\r', and records continued on the next line.  A
// malformed record always goes to the host parser, which reports it.
#include <cuda_runtime.h>
#include <errno.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"
#include "profile.h"

namespace crt {

namespace {

constexpr int kLineThreads = 512;
constexpr int kLineBytes = 32;  // per thread
constexpr int kLineTile = kLineThreads * kLineBytes;
constexpr int kScanThreads = 1024;
constexpr int kParseThreads = 256;
constexpr int kTextPad = 64;        // '\n' bytes after the last tile
constexpr int kFieldMax = 62;       // longest field the fast path takes
constexpr int64_t kFallbackList = 1 << 20;  // undecided records listed at first
constexpr int kStageThreads = 16;
constexpr size_t kStageChunk = size_t(4) << 20;

// classes of a non-blank byte; kNone also means "no such byte"
constexpr int kNone = 0, kNl = 1, kOther = 2;

__device__ __forceinline__ int byte_class(unsigned c)
{
  return (c == ' ' || c == '\t' || c == '\r') ? kNone : (c == '\n' ? kNl : kOther);
}

struct LastOp {
  __device__ int operator()(int a, int b) const { return b ? b : a; }
};
struct SumOp {
  __device__ int64_t operator()(int64_t a, int64_t b) const { return a + b; }
};

// Exclusive scan over the block (kThreads a multiple of 32, at most 1024);
// total = the inclusive result of the last thread.
template <int kThreads, typename T, typename Op>
__device__ T block_exclusive_scan(T v, T identity, Op op, T& total)
{
  constexpr int kWarps = kThreads / 32;
  __shared__ T s_warp[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x = op(y, x);
  }
  T ex = __shfl_up_sync(0xFFFFFFFFu, x, 1);
  if (lane == 0) ex = identity;
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T s = lane < kWarps ? s_warp[lane] : identity;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s = op(y, s);
    }
    s_warp[lane] = s;
  }
  __syncthreads();
  const T res = op(warp ? s_warp[warp - 1] : identity, ex);
  total = s_warp[kWarps - 1];
  __syncthreads();
  return res;
}

// A thread's 32 bytes: starts preceded (past blanks) by a '\n' among them,
// and the classes of the first and last non-blank bytes.
struct Walk {
  int cnt, first, last;
};

__device__ __forceinline__ void load32(const uint8_t* text, uint32_t w[8])
{
  const uint4* src = reinterpret_cast<const uint4*>(text + (size_t)blockIdx.x * kLineTile) +
                     2 * threadIdx.x;
  const uint4 a = src[0], b = src[1];
  w[0] = a.x, w[1] = a.y, w[2] = a.z, w[3] = a.w;
  w[4] = b.x, w[5] = b.y, w[6] = b.z, w[7] = b.w;
}

__device__ __forceinline__ Walk walk32(const uint32_t w[8])
{
  Walk r{0, kNone, kNone};
#pragma unroll
  for (int i = 0; i < kLineBytes; i++) {
    const int k = byte_class((w[i >> 2] >> (8 * (i & 3))) & 0xFFu);
    if (k == kNone) continue;
    if (k == kOther && r.last == kNl) r.cnt++;
    if (r.first == kNone) r.first = k;
    r.last = k;
  }
  return r;
}

// tile_word: bits 0-15 starts, bit 16 first non-blank byte is a record byte,
// bits 24-25 class of the last non-blank byte; bits 28-29 are set by the scan
// to the class carried into the tile.
__global__ void __launch_bounds__(kLineThreads)
    line_tile_kernel(const uint8_t* __restrict__ text, uint32_t* __restrict__ tile_word)
{
  uint32_t w[8];
  load32(text, w);
  const Walk r = walk32(w);
  int tile_last;
  const int in = block_exclusive_scan<kLineThreads>(r.last, kNone, LastOp(), tile_last);
  const int64_t mine = r.cnt + (r.first == kOther && in == kNl);
  int64_t cnt;
  block_exclusive_scan<kLineThreads>(mine, (int64_t)0, SumOp(), cnt);
  const int lead = __syncthreads_or(r.first == kOther && in == kNone);
  if (threadIdx.x == 0)
    tile_word[blockIdx.x] = (uint32_t)cnt | ((uint32_t)(lead != 0) << 16) | ((uint32_t)tile_last << 24);
}

__global__ void __launch_bounds__(kScanThreads)
    line_scan_kernel(uint32_t* __restrict__ tile_word, int64_t* __restrict__ tile_base,
                     int64_t ntiles, unsigned long long* __restrict__ total)
{
  const int64_t per = (ntiles + kScanThreads - 1) / kScanThreads;
  const int64_t b = min(ntiles, per * (int64_t)threadIdx.x), e = min(ntiles, b + per);
  int last = kNone;
  for (int64_t t = b; t < e; t++) {
    const int l = (tile_word[t] >> 24) & 3;
    if (l) last = l;
  }
  int unused;
  const int in = block_exclusive_scan<kScanThreads>(last, kNone, LastOp(), unused);
  int64_t sum = 0;
  int st = in;
  for (int64_t t = b; t < e; t++) {
    const uint32_t w = tile_word[t];
    sum += (w & 0xFFFFu) + (((w >> 16) & 1u) && st != kOther);
    const int l = (w >> 24) & 3;
    if (l) st = l;
  }
  int64_t all;
  int64_t base = block_exclusive_scan<kScanThreads>(sum, (int64_t)0, SumOp(), all);
  st = in;
  for (int64_t t = b; t < e; t++) {
    const uint32_t w = tile_word[t];
    tile_base[t] = base;
    tile_word[t] = (w & ~(3u << 28)) | ((uint32_t)st << 28);
    base += (w & 0xFFFFu) + (((w >> 16) & 1u) && st != kOther);
    const int l = (w >> 24) & 3;
    if (l) st = l;
  }
  if (threadIdx.x == 0) *total = (unsigned long long)all;
}

__global__ void __launch_bounds__(kLineThreads)
    line_emit_kernel(const uint8_t* __restrict__ text, const uint32_t* __restrict__ tile_word,
                     const int64_t* __restrict__ tile_base, int64_t m, int64_t* __restrict__ starts)
{
  const int64_t tb = tile_base[blockIdx.x];
  if (tb >= m) return;  // uniform over the block
  uint32_t w[8];
  load32(text, w);
  const Walk r = walk32(w);
  int unused;
  int in = block_exclusive_scan<kLineThreads>(r.last, kNone, LastOp(), unused);
  if (in == kNone) in = (tile_word[blockIdx.x] >> 28) & 3;
  const int64_t mine = r.cnt + (r.first == kOther && in != kOther);
  int64_t tot;
  int64_t pos = tb + block_exclusive_scan<kLineThreads>(mine, (int64_t)0, SumOp(), tot);
  if (mine == 0 || pos >= m) return;
  const int64_t off = (int64_t)blockIdx.x * kLineTile + (int64_t)threadIdx.x * kLineBytes;
  int prev = in;
#pragma unroll
  for (int i = 0; i < kLineBytes; i++) {
    const int k = byte_class((w[i >> 2] >> (8 * (i & 3))) & 0xFFu);
    if (k == kNone) continue;
    if (k == kOther && prev != kOther) {
      if (pos < m) starts[pos] = off + i;
      pos++;
    }
    prev = k;
  }
}

__constant__ double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                                  1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                                  1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

__device__ __forceinline__ unsigned at(const uint8_t* t, int64_t p) { return __ldg(t + p); }
__device__ __forceinline__ bool is_digit(unsigned c) { return c - '0' < 10u; }

// w * 10^e10 rounded to float; false when the fast path cannot be sure.
__device__ __forceinline__ bool decimal_to_float(uint64_t w, int e10, bool neg, float* out)
{
  if (w == 0) {
    *out = neg ? -0.0f : 0.0f;
    return true;
  }
  if (e10 < -44 || e10 > 44) return false;
  double d = __ull2double_rn(w);
  if (e10 > 22) {
    d = __dmul_rn(d, 1e22);
    e10 -= 22;
  } else if (e10 < -22) {
    d = __ddiv_rn(d, 1e22);
    e10 += 22;
  }
  if (e10 > 0) d = __dmul_rn(d, kPow10[e10]);
  else if (e10 < 0) d = __ddiv_rn(d, kPow10[-e10]);
  const uint64_t bits = (uint64_t)__double_as_longlong(d);
  const int be = (int)(bits >> 52) & 0x7FF;
  if (be < 1023 - 125 || be > 1023 + 126) return false;  // keep to normal floats
  const int low = (int)(bits & ((1u << 29) - 1));         // bits below float precision
  if (abs(low - (1 << 28)) <= 16) return false;           // near a halfway point
  const float f = __double2float_rn(d);
  *out = neg ? -f : f;
  return true;
}

// A float field at p (its leading blanks skipped): returns the index of the
// ',' that ends it, or -1 for the host parser.
__device__ __forceinline__ int64_t float_field(const uint8_t* t, int64_t p, float* v)
{
  const int64_t p0 = p, lim = p + kFieldMax;
  unsigned c = at(t, p);
  const bool neg = c == '-';
  if (c == '-' || c == '+') c = at(t, ++p);
  uint64_t w = 0;
  int nd = 0, e10 = 0;
  bool any = false;
  while (p < lim && is_digit(c)) {
    any = true;
    const unsigned d = c - '0';
    if (w || d) {
      if (nd < 19) {
        w = w * 10 + d;
        nd++;
      } else {
        e10++;
      }
    }
    c = at(t, ++p);
  }
  if (c == '.' && p < lim) {
    c = at(t, ++p);
    while (p < lim && is_digit(c)) {
      any = true;
      const unsigned d = c - '0';
      if (!w && !d) {
        e10--;
      } else if (nd < 19) {
        w = w * 10 + d;
        nd++;
        e10--;
      }
      c = at(t, ++p);
    }
  }
  if (!any) return -1;
  if ((c == 'e' || c == 'E') && p < lim) {
    c = at(t, ++p);
    const bool eneg = c == '-';
    if ((c == '-' || c == '+') && p < lim) c = at(t, ++p);
    int ev = 0, ed = 0;
    while (p < lim && is_digit(c)) {
      if (ed < 6) ev = ev * 10 + (int)(c - '0');
      ed++;
      c = at(t, ++p);
    }
    if (ed == 0 || ed > 5) return -1;
    e10 += eneg ? -ev : ev;
  }
  if (p - p0 > kFieldMax || c != ',') return -1;
  return decimal_to_float(w, e10, neg, v) ? p : -1;
}

// An integer field at p: the low 32 bits of its value (what (int) of strtol
// keeps); the others end at ','; the last one may be followed by ' ', '\t'
// or '\r' and must end its line (the fast path takes one record per line:
// then the next record starts on the next line, as fscanf finds it).
__device__ __forceinline__ int64_t int_field(const uint8_t* t, int64_t p, bool last, int32_t* v)
{
  const int64_t p0 = p, lim = p + kFieldMax;
  unsigned c = at(t, p);
  const bool neg = c == '-';
  if (c == '-' || c == '+') c = at(t, ++p);
  uint64_t x = 0;
  int nd = 0;
  while (p < lim && is_digit(c)) {
    x = x * 10 + (c - '0');
    nd++;
    c = at(t, ++p);
  }
  if (nd == 0 || nd > 18) return -1;
  if (last)
    while (p < lim && (c == ' ' || c == '\t' || c == '\r')) c = at(t, ++p);
  if (p - p0 > kFieldMax) return -1;
  if (last ? c != '\n' : c != ',') return -1;
  *v = (int32_t)(uint32_t)(neg ? 0 - x : x);
  return p;
}

// The record starting at p (a non-blank byte): false for the host parser.
__device__ __forceinline__ bool record_fast(const uint8_t* t, int64_t p, float v[4], int32_t& id)
{
#pragma unroll
  for (int f = 0; f < 7; f++) {
    if (f) {
      // past the ',' ending the previous field, then the blanks fscanf skips
      unsigned c = at(t, ++p);
      int s = 0;
      while (s < kFieldMax && (c == ' ' || c == '\t' || c == '\r')) {
        c = at(t, ++p);
        s++;
      }
      if (c == ' ' || c == '\t' || c == '\r' || c == '\n') return false;
    }
    int32_t x = 0;
    const int64_t e = f < 4 ? float_field(t, p, &v[f]) : int_field(t, p, f == 6, &x);
    if (e < 0) return false;
    if (f == 4) id = x;
    p = e;
  }
  return true;
}

// a - r and a + r with the host's NaN rule: x86 arithmetic returns the NaN
// operand itself, quieted (the first one when both are NaN), where the GPU
// returns its canonical NaN; readMBR runs on the host, so its boxes keep the
// input NaN's sign and payload.
__device__ __forceinline__ float quiet_nan(float x) { return __int_as_float(__float_as_int(x) | 0x400000); }

__device__ __forceinline__ float sub_host(float a, float r)
{
  return isnan(a) ? quiet_nan(a) : isnan(r) ? quiet_nan(r) : __fsub_rn(a, r);
}

__device__ __forceinline__ float add_host(float a, float r)
{
  return isnan(a) ? quiet_nan(a) : isnan(r) ? quiet_nan(r) : __fadd_rn(a, r);
}

__global__ void __launch_bounds__(kParseThreads, 4)
    mbr_parse_kernel(const uint8_t* __restrict__ text, const int64_t* __restrict__ starts, int64_t m,
                     float r, float* __restrict__ xmin, float* __restrict__ ymin,
                     float* __restrict__ xmax, float* __restrict__ ymax, int32_t* __restrict__ id,
                     unsigned long long* __restrict__ n_fallback, int64_t* __restrict__ fallback,
                     int64_t fallback_cap)
{
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = starts[k];
    float v[4];
    int32_t rid = 0;
    if (record_fast(text, s, v, rid)) {
      // readMBR: std::min / std::max of the endpoints, then -/+ r in fp32
      xmin[k] = sub_host(v[2] < v[0] ? v[2] : v[0], r);
      ymin[k] = sub_host(v[3] < v[1] ? v[3] : v[1], r);
      xmax[k] = add_host(v[0] < v[2] ? v[2] : v[0], r);
      ymax[k] = add_host(v[1] < v[3] ? v[3] : v[1], r);
      id[k] = rid;
    } else {
      // for the host parser: the record, its start, and the next record's
      // start (-1 for the last), against which the host checks where the
      // record really ends
      const unsigned long long j = atomicAdd(n_fallback, 1ull);
      if ((int64_t)j < fallback_cap) {
        fallback[3 * j] = k;
        fallback[3 * j + 1] = s;
        fallback[3 * j + 2] = k + 1 < m ? starts[k + 1] : -1;
      }
    }
  }
}

struct FixRecord {
  int64_t k;
  float xmin, ymin, xmax, ymax;
  int32_t id, pad;
};

__global__ void mbr_fix_kernel(const FixRecord* __restrict__ rec, int64_t c, float* __restrict__ xmin,
                               float* __restrict__ ymin, float* __restrict__ xmax,
                               float* __restrict__ ymax, int32_t* __restrict__ id)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c;
       i += (int64_t)gridDim.x * blockDim.x) {
    const FixRecord f = rec[i];
    xmin[f.k] = f.xmin;
    ymin[f.k] = f.ymin;
    xmax[f.k] = f.xmax;
    ymax[f.k] = f.ymax;
    id[f.k] = f.id;
  }
}

// Binary MBR records: 28 bytes each, little-endian float32 x1, y1, x2, y2 and
// int32 id, pid, nume (the text record's fields in binary); the box is the one
// readMBR makes of the text record.
constexpr int64_t kBinRecord = 28;

__global__ void __launch_bounds__(kParseThreads)
    mbr_bin_kernel(const uint32_t* __restrict__ words, int64_t n, float r, float* __restrict__ xmin,
                   float* __restrict__ ymin, float* __restrict__ xmax, float* __restrict__ ymax,
                   int32_t* __restrict__ id)
{
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t* w = words + 7 * k;
    const float x1 = __uint_as_float(__ldg(w)), y1 = __uint_as_float(__ldg(w + 1));
    const float x2 = __uint_as_float(__ldg(w + 2)), y2 = __uint_as_float(__ldg(w + 3));
    xmin[k] = sub_host(x2 < x1 ? x2 : x1, r);
    ymin[k] = sub_host(y2 < y1 ? y2 : y1, r);
    xmax[k] = add_host(x1 < x2 ? x2 : x1, r);
    ymax[k] = add_host(y1 < y2 ? y2 : y1, r);
    id[k] = (int32_t)__ldg(w + 4);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// Pinned staging slots, two per copy thread, allocated on first use and kept
// for the life of the process.
struct StagePool {
  std::mutex mu;
  char* slot[kStageThreads][2] = {};
};

StagePool& stage_pool()
{
  static StagePool* p = new StagePool;
  return *p;
}

// The source text: a host buffer, or a file read with pread; the host view
// (for records the device leaves to the host parser) maps the file on demand.
struct Source {
  const char* mem = nullptr;
  int fd = -1;
  int64_t len = 0;
  void* map = nullptr;
  std::string owned;

  const char* view()
  {
    if (mem) return mem;
    if (map) return (const char*)map;
    if (!owned.empty()) return owned.data();
    if (len == 0) return "";
    void* p = mmap(nullptr, (size_t)len, PROT_READ, MAP_PRIVATE, fd, 0);
    if (p != MAP_FAILED) {
      map = p;
      return (const char*)p;
    }
    owned.resize((size_t)len);
    if (!read_at(&owned[0], 0, (size_t)len)) {
      owned.clear();
      return nullptr;
    }
    return owned.data();
  }

  bool read_at(char* dst, int64_t off, size_t m) const
  {
    size_t got = 0;
    while (got < m) {
      const ssize_t k = pread(fd, dst + got, m - got, (off_t)(off + (int64_t)got));
      if (k < 0 && errno == EINTR) continue;
      if (k <= 0) return false;
      got += (size_t)k;
    }
    return true;
  }

  ~Source()
  {
    if (map) munmap(map, (size_t)len);
  }
};

// Copies the text into d_text: copy threads (up to 16, one per host thread of
// the machine) take 4 MiB chunks in turn, each filling its two pinned slots
// alternately (pread or memcpy) while the other slot's copy to the device
// runs on the thread's own stream.  Measured on a 16-thread host with a
// 266 MB file in the page cache: 16 threads x 4 MiB 11.6 ms per call, 8 x 4
// MiB 13.0, 16 x 8 MiB 12.0, 12 x 2 MiB 11.9; a memcpy from an mmap of the
// file instead of pread 14.8.
int stage_text(char* d_text, Source& src, int dev)
{
  const int64_t nchunks = cdiv(src.len, (int64_t)kStageChunk);
  if (nchunks == 0) return CRT_OK;
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min<int64_t>(std::min(kStageThreads, hw), nchunks);
  StagePool& P = stage_pool();
  std::lock_guard<std::mutex> lock(P.mu);
  for (int t = 0; t < nt; t++)  // the slots of the threads this call uses
    for (int s = 0; s < 2; s++)
      if (!P.slot[t][s] &&
          cudaHostAlloc((void**)&P.slot[t][s], kStageChunk, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        P.slot[t][s] = nullptr;
        return fail(CRT_ERR_OOM, "read_mbr_csv_device: pinned staging allocation failed");
      }
  std::vector<int> bad_read(nt, 0);
  std::vector<cudaError_t> err(nt, cudaSuccess);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++) {
    th.emplace_back([&, t] {
      cudaError_t& e = err[t];
      e = cudaSetDevice(dev);
      cudaStream_t st;
      cudaEvent_t ev[2];
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
      if (e != cudaSuccess) return;
      cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
      cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
      int it = 0;
      for (int64_t c = t; c < nchunks && e == cudaSuccess && !bad_read[t]; c += nt, it++) {
        const int s = it & 1;
        if (it >= 2) e = cudaEventSynchronize(ev[s]);  // the slot's previous copy is done
        if (e != cudaSuccess) break;
        const int64_t off = c * (int64_t)kStageChunk;
        const size_t m = (size_t)std::min<int64_t>((int64_t)kStageChunk, src.len - off);
        if (src.mem) std::memcpy(P.slot[t][s], src.mem + off, m);
        else if (!src.read_at(P.slot[t][s], off, m)) bad_read[t] = 1;
        if (!bad_read[t]) e = cudaMemcpyAsync(d_text + off, P.slot[t][s], m, cudaMemcpyHostToDevice, st);
        if (!bad_read[t] && e == cudaSuccess) e = cudaEventRecord(ev[s], st);
      }
      const cudaError_t es = cudaStreamSynchronize(st);
      if (e == cudaSuccess) e = es;
      cudaEventDestroy(ev[0]);
      cudaEventDestroy(ev[1]);
      cudaStreamDestroy(st);
    });
  }
  for (auto& x : th) x.join();
  for (int t = 0; t < nt; t++) {
    if (err[t] != cudaSuccess) return cuda_fail(err[t], "read_mbr_csv_device: staging copy");
    if (bad_read[t]) return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv_device: reading the file failed");
  }
  return CRT_OK;
}

// Stream-ordered device allocations released when the call returns.
struct Scratch {
  cudaStream_t stream;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : stream(s) {}
  template <typename T>
  T* get(size_t bytes)
  {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    ptrs.push_back(p);
    return (T*)p;
  }
  ~Scratch()
  {
    for (void* p : ptrs) cudaFreeAsync(p, stream);
  }
};

struct Outputs {
  float *xmin = nullptr, *ymin = nullptr, *xmax = nullptr, *ymax = nullptr;
  int32_t* id = nullptr;
};

// The loader proper.  n < 0: every record (only when `alloc`).  alloc: the
// outputs are cudaMalloc'd here for the records found (*box_out, freed on
// failure); otherwise they are the caller's, of n entries.
int ingest(Source& src, int64_t n, float r, bool alloc, Outputs out, crt_bbox_f32* box_out,
           int64_t* n_read, cudaStream_t stream)
{
  if (n_read) *n_read = 0;
  int dev = 0;
  CRT_CUDA(cudaGetDevice(&dev));
  const int64_t ntiles = cdiv(src.len, kLineTile);
  const size_t text_bytes = (size_t)ntiles * kLineTile + kTextPad;
  Scratch S(stream);
  // 256-byte aligned for the tiles' 16-byte loads
  char* d_text_raw = S.get<char>(text_bytes + 256);
  char* d_text = d_text_raw ? (char*)(((uintptr_t)d_text_raw + 255) & ~(uintptr_t)255) : nullptr;
  unsigned long long* ctr = S.get<unsigned long long>(256);  // [0] records, [1] fallbacks
  uint32_t* tile_word = S.get<uint32_t>((size_t)ntiles * 4);
  int64_t* tile_base = S.get<int64_t>((size_t)ntiles * 8);
  if (!d_text || !ctr || !tile_word || !tile_base)
    return fail(CRT_ERR_OOM, "read_mbr_csv_device: device allocation failed");
  CRT_CUDA(cudaMemsetAsync(d_text + src.len, '\n', text_bytes - (size_t)src.len, stream));
  CRT_CUDA(cudaMemsetAsync(ctr, 0, 256, stream));
  CRT_CUDA(cudaStreamSynchronize(stream));  // the copy threads write d_text on their own streams
  const auto t0 = std::chrono::steady_clock::now();
  int rc = stage_text(d_text, src, dev);
  if (rc != CRT_OK) return rc;
  if (profiling())
    prof_add("ingest_stage",
             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());

  unsigned long long h_ctr[2] = {0, 0};
  if (ntiles > 0) {
    {
      ProfScope ps("ingest_lines", stream);
      line_tile_kernel<<<(unsigned)ntiles, kLineThreads, 0, stream>>>((const uint8_t*)d_text, tile_word);
      line_scan_kernel<<<1, kScanThreads, 0, stream>>>(tile_word, tile_base, ntiles, ctr);
    }
    CRT_LAUNCHED(2);
    CRT_CUDA(cudaGetLastError());
    CRT_CUDA(cudaMemcpyAsync(h_ctr, ctr, 8, cudaMemcpyDeviceToHost, stream));
    CRT_CUDA(cudaStreamSynchronize(stream));
  }
  const int64_t total = (int64_t)h_ctr[0];
  int64_t m = n < 0 ? total : std::min(total, n);
  if (alloc) {
    if (m > INT32_MAX) return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv_device: more than 2^31-1 records");
    void** dst[5] = {(void**)&out.xmin, (void**)&out.ymin, (void**)&out.xmax, (void**)&out.ymax,
                     (void**)&out.id};
    for (int a = 0; a < 5 && m > 0; a++)
      if (cudaMalloc(dst[a], (size_t)m * 4) != cudaSuccess) {
        cudaGetLastError();
        for (int b = 0; b < a; b++) cudaFree(*dst[b]);
        return fail(CRT_ERR_OOM, "read_mbr_csv_device: output allocation failed");
      }
  }
  auto release = [&] {
    if (alloc) {
      void* p[5] = {out.xmin, out.ymin, out.xmax, out.ymax, out.id};
      for (void* q : p)
        if (q) cudaFree(q);
    }
  };

  int64_t first_bad = -1;
  if (m > 0) {
    int64_t cap = std::min<int64_t>(m, kFallbackList);
    int64_t* starts = S.get<int64_t>((size_t)m * 8);
    int64_t* fb = S.get<int64_t>((size_t)cap * 24);
    if (!starts || !fb) {
      release();
      return fail(CRT_ERR_OOM, "read_mbr_csv_device: device allocation failed");
    }
    {
      ProfScope ps("ingest_emit", stream);
      line_emit_kernel<<<(unsigned)ntiles, kLineThreads, 0, stream>>>(
          (const uint8_t*)d_text, tile_word, tile_base, m, starts);
    }
    const int64_t grid = std::min<int64_t>(cdiv(m, kParseThreads), (int64_t)sm_count() * 16);
    {
      ProfScope ps("ingest_parse", stream);
      mbr_parse_kernel<<<(unsigned)grid, kParseThreads, 0, stream>>>(
          (const uint8_t*)d_text, starts, m, r, out.xmin, out.ymin, out.xmax, out.ymax, out.id,
          ctr + 1, fb, cap);
    }
    CRT_LAUNCHED(2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_ctr[1], ctr + 1, 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      release();
      return cuda_fail(e, "read_mbr_csv_device: parse");
    }
    const int64_t c = (int64_t)h_ctr[1];
    if (c > cap) {
      // more undecided records than the list holds: list them all (the
      // parse runs again into a list of their exact count)
      cap = c;
      fb = S.get<int64_t>((size_t)cap * 24);
      if (!fb) {
        release();
        return fail(CRT_ERR_OOM, "read_mbr_csv_device: device allocation failed");
      }
      e = cudaMemsetAsync(ctr + 1, 0, 8, stream);
      if (e == cudaSuccess) {
        mbr_parse_kernel<<<(unsigned)grid, kParseThreads, 0, stream>>>(
            (const uint8_t*)d_text, starts, m, r, out.xmin, out.ymin, out.xmax, out.ymax, out.id,
            ctr + 1, fb, cap);
        CRT_LAUNCHED(1);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "read_mbr_csv_device: parse");
      }
    }
    if (c > 0) {
      const char* base = src.view();
      if (!base) {
        release();
        return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv_device: reading the file failed");
      }
      const char* end = base + src.len;
      std::vector<FixRecord> fix;
      bool whole = false;
      if (!whole) {
        std::vector<int64_t> h_fb((size_t)c * 3);
        e = cudaMemcpy(h_fb.data(), fb, (size_t)c * 24, cudaMemcpyDeviceToHost);
        // host threads parse the listed records, each into its own part
        const int nt = (int)std::max<int64_t>(
            1, std::min<int64_t>(std::min(32u, std::max(1u, std::thread::hardware_concurrency())),
                                 c / 4096 + 1));
        std::vector<std::vector<FixRecord>> parts((size_t)nt);
        std::vector<int64_t> bad((size_t)nt, -1);
        std::vector<char> moved((size_t)nt, 0);
        auto work = [&](int t) {
          const int64_t j0 = c * t / nt, j1 = c * (t + 1) / nt;
          for (int64_t j = j0; j < j1; j++) {
            const int64_t k = h_fb[3 * j], s0 = h_fb[3 * j + 1], next = h_fb[3 * j + 2];
            float v[4];
            int rid = 0;
            const char* stop = parse_mbr_record(base + s0, end, v, rid);
            if (!stop) {
              if (bad[t] < 0 || k < bad[t]) bad[t] = k;
              continue;
            }
            // a record that does not end where the line scan put the next one
            // (records across lines, several on a line): fscanf's records are
            // not the lines here, so the host loader reads the whole file
            if (next >= 0 ? stop != base + next : (m < n || n < 0) && stop != end) {
              moved[t] = 1;
              return;
            }
            FixRecord f{k, 0, 0, 0, 0, rid, 0};
            mbr_box(v, r, &f.xmin, &f.ymin, &f.xmax, &f.ymax);
            parts[t].push_back(f);
          }
        };
        if (e == cudaSuccess) {
          std::vector<std::thread> th;
          for (int t = 1; t < nt; t++) th.emplace_back(work, t);
          work(0);
          for (auto& x : th) x.join();
        }
        for (int t = 0; t < nt; t++) {
          whole = whole || moved[t];
          if (bad[t] >= 0 && (first_bad < 0 || bad[t] < first_bad)) first_bad = bad[t];
          fix.insert(fix.end(), parts[t].begin(), parts[t].end());
        }
      }
      if (whole && e == cudaSuccess) {
        MbrRecords rec;
        scan_mbr_text(base, (size_t)src.len, n, r, rec);
        first_bad = rec.malformed || (n >= 0 && rec.count < n) ? rec.count : -1;
        if (first_bad < 0 && rec.count != m && !alloc) {
          m = rec.count;  // the caller's arrays hold n >= rec.count records
        } else if (first_bad < 0 && rec.count != m) {
          // fscanf finds another number of records than the line scan
          release();
          m = rec.count;
          if (m > INT32_MAX)
            return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv_device: more than 2^31-1 records");
          void** dst[5] = {(void**)&out.xmin, (void**)&out.ymin, (void**)&out.xmax,
                           (void**)&out.ymax, (void**)&out.id};
          for (int a2 = 0; a2 < 5; a2++) *dst[a2] = nullptr;
          for (int a2 = 0; a2 < 5 && m > 0; a2++)
            if (cudaMalloc(dst[a2], (size_t)m * 4) != cudaSuccess) {
              cudaGetLastError();
              for (int b2 = 0; b2 < a2; b2++) cudaFree(*dst[b2]);
              return fail(CRT_ERR_OOM, "read_mbr_csv_device: output allocation failed");
            }
        }
        const size_t bytes = (size_t)std::min<int64_t>(rec.count, m) * 4;
        float* dv[4] = {out.xmin, out.ymin, out.xmax, out.ymax};
        for (int a2 = 0; a2 < 4 && bytes && e == cudaSuccess; a2++)
          e = cudaMemcpy(dv[a2], rec.v[a2].data(), bytes, cudaMemcpyHostToDevice);
        if (bytes && e == cudaSuccess) e = cudaMemcpy(out.id, rec.id.data(), bytes, cudaMemcpyHostToDevice);
        if (first_bad >= 0 && !rec.malformed) {
          // fewer records than asked for: reported below with the count
          first_bad = -1;
          m = rec.count;
        }
      } else if (!fix.empty() && e == cudaSuccess) {
        FixRecord* d_fix = S.get<FixRecord>(fix.size() * sizeof(FixRecord));
        if (!d_fix) {
          release();
          return fail(CRT_ERR_OOM, "read_mbr_csv_device: device allocation failed");
        }
        e = cudaMemcpyAsync(d_fix, fix.data(), fix.size() * sizeof(FixRecord),
                            cudaMemcpyHostToDevice, stream);
        const int64_t g = std::min<int64_t>(cdiv((int64_t)fix.size(), 256), (int64_t)sm_count() * 4);
        if (e == cudaSuccess) {
          mbr_fix_kernel<<<(unsigned)g, 256, 0, stream>>>(d_fix, (int64_t)fix.size(), out.xmin,
                                                         out.ymin, out.xmax, out.ymax, out.id);
          CRT_LAUNCHED(1);
          e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      }
      if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "read_mbr_csv_device: host-parsed records");
      }
    }
  }
  if (first_bad >= 0) {
    release();
    if (n_read) *n_read = first_bad;
    return fail(CRT_ERR_INVALID_ARG,
                "read_mbr_csv: record " + std::to_string(first_bad) + " is not x1,y1,x2,y2,id,pid,nume");
  }
  if (n_read) *n_read = m;
  if (n >= 0 && m < n) {
    release();
    return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv: file holds " + std::to_string(m) + " records, " +
                                         std::to_string(n) + " requested");
  }
  if (alloc && box_out) {
    box_out->xmin = out.xmin;
    box_out->ymin = out.ymin;
    box_out->xmax = out.xmax;
    box_out->ymax = out.ymax;
    box_out->id = out.id;
    box_out->sz = (int)m;
  }
  return CRT_OK;
}

// The binary loader: the first m records of the file staged to the device
// like the text, then one thread per record.
int ingest_bin(Source& src, int64_t n, float r, crt_bbox_f32* box_out, int64_t* n_read,
               cudaStream_t stream)
{
  if (n_read) *n_read = 0;
  if (src.len % kBinRecord)
    return fail(CRT_ERR_INVALID_ARG, "read_mbr_bin_device: the file is not a whole number of "
                                     "28-byte records");
  const int64_t total = src.len / kBinRecord;
  if (n > total) {
    if (n_read) *n_read = total;
    return fail(CRT_ERR_INVALID_ARG, "read_mbr_bin_device: file holds " + std::to_string(total) +
                                         " records, " + std::to_string(n) + " requested");
  }
  const int64_t m = n < 0 ? total : n;
  if (m > INT32_MAX) return fail(CRT_ERR_INVALID_ARG, "read_mbr_bin_device: more than 2^31-1 records");
  crt_bbox_f32 box{};
  box.sz = (int)m;
  if (m > 0) {
    int dev = 0;
    CRT_CUDA(cudaGetDevice(&dev));
    Scratch S(stream);
    char* raw = S.get<char>((size_t)(m * kBinRecord) + 256);
    if (!raw) return fail(CRT_ERR_OOM, "read_mbr_bin_device: device allocation failed");
    char* d_rec = (char*)(((uintptr_t)raw + 255) & ~(uintptr_t)255);
    CRT_CUDA(cudaStreamSynchronize(stream));  // the copy threads write d_rec on their own streams
    src.len = m * kBinRecord;                 // only the records asked for
    int rc = stage_text(d_rec, src, dev);
    if (rc != CRT_OK) return rc;
    void** dst[5] = {(void**)&box.xmin, (void**)&box.ymin, (void**)&box.xmax, (void**)&box.ymax,
                     (void**)&box.id};
    for (int a = 0; a < 5; a++)
      if (cudaMalloc(dst[a], (size_t)m * 4) != cudaSuccess) {
        cudaGetLastError();
        for (int b = 0; b < a; b++) cudaFree(*dst[b]);
        return fail(CRT_ERR_OOM, "read_mbr_bin_device: output allocation failed");
      }
    const int64_t grid = std::min<int64_t>(cdiv(m, kParseThreads), (int64_t)sm_count() * 16);
    mbr_bin_kernel<<<(unsigned)grid, kParseThreads, 0, stream>>>(
        (const uint32_t*)d_rec, m, r, box.xmin, box.ymin, box.xmax, box.ymax, box.id);
    CRT_LAUNCHED(1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      crt_bbox_free(&box);
      return cuda_fail(e, "read_mbr_bin_device");
    }
  }
  if (n_read) *n_read = m;
  *box_out = box;
  return CRT_OK;
}

}  // namespace

}  // namespace crt

using namespace crt;

extern "C" {

int crt_read_mbr_csv_device(const char* path, int64_t n, float r, crt_bbox_f32* d_box,
                            int64_t* n_read, crt_stream_t stream)
{
  if (!path || !d_box || n < -1) return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv_device: bad arguments");
  if (n_read) *n_read = 0;
  const int fd = open(path, O_RDONLY | O_CLOEXEC);
  if (fd < 0) return fail(CRT_ERR_INVALID_ARG, std::string("read_mbr_csv_device: cannot open ") + path);
  struct stat sb;
  if (fstat(fd, &sb) != 0 || !S_ISREG(sb.st_mode)) {
    close(fd);
    return fail(CRT_ERR_INVALID_ARG, std::string("read_mbr_csv_device: not a regular file: ") + path);
  }
  int rc;
  {
    Source src;
    src.fd = fd;
    src.len = (int64_t)sb.st_size;
    crt_bbox_f32 box{};
    rc = ingest(src, n, r, true, Outputs{}, &box, n_read, (cudaStream_t)stream);
    if (rc == CRT_OK) *d_box = box;
  }
  close(fd);
  return rc;
}

int crt_read_mbr_bin_device(const char* path, int64_t n, float r, crt_bbox_f32* d_box,
                            int64_t* n_read, crt_stream_t stream)
{
  if (!path || !d_box || n < -1) return fail(CRT_ERR_INVALID_ARG, "read_mbr_bin_device: bad arguments");
  if (n_read) *n_read = 0;
  const int fd = open(path, O_RDONLY | O_CLOEXEC);
  if (fd < 0) return fail(CRT_ERR_INVALID_ARG, std::string("read_mbr_bin_device: cannot open ") + path);
  struct stat sb;
  if (fstat(fd, &sb) != 0 || !S_ISREG(sb.st_mode)) {
    close(fd);
    return fail(CRT_ERR_INVALID_ARG, std::string("read_mbr_bin_device: not a regular file: ") + path);
  }
  int rc;
  {
    Source src;
    src.fd = fd;
    src.len = (int64_t)sb.st_size;
    crt_bbox_f32 box{};
    rc = ingest_bin(src, n, r, &box, n_read, (cudaStream_t)stream);
    if (rc == CRT_OK) *d_box = box;
  }
  close(fd);
  return rc;
}

int crt_parse_mbr_csv_device(const char* text, int64_t len, int64_t n, float r, float* d_xmin,
                             float* d_ymin, float* d_xmax, float* d_ymax, int32_t* d_id,
                             int64_t* n_read, crt_stream_t stream)
{
  if ((!text && len > 0) || len < 0 || n < 0 ||
      (n > 0 && !(d_xmin && d_ymin && d_xmax && d_ymax && d_id)))
    return fail(CRT_ERR_INVALID_ARG, "parse_mbr_csv_device: bad arguments");
  Source src;
  src.mem = len > 0 ? text : nullptr;
  src.len = len;
  Outputs out{d_xmin, d_ymin, d_xmax, d_ymax, d_id};
  return ingest(src, n, r, false, out, nullptr, n_read, (cudaStream_t)stream);
}

}  // extern "C"
