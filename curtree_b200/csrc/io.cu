// Host-side I/O around the tree: the reference's MBR text loader and a tree
// file format.
//
// crt_read_mbr_csv restates readMBR (src/utility.cpp:5-40): each record is a
// line "x1,y1,x2,y2,id,pid,nume"; the box is [min(x1,x2) - r, max(x1,x2) + r]
// x [min(y1,y2) - r, max(y1,y2) + r] in fp32, id is the fifth field, pid and
// nume are read and dropped.  Numbers parse as fscanf's %f / %d do (strtof /
// strtol, correctly rounded); blanks may precede a number and end a line, but
// not precede a ',' (the format's literal commas do not skip blanks); one
// record per line, blank lines skipped.  Where the
// reference exits (missing file) or throws (a malformed record), this
// returns a status.  Records are parsed by several host threads.
//
// crt_tree_save / crt_tree_load write and read a built tree with its sorted
// box set, a format the reference does not have:
//   8 bytes   magic "CRTREE\0\1"
//   int64     n (boxes), int64 R_sz, int32 fanout, int32 0
//   R_sz x float32 xmin, ymin, xmax, ymax; R_sz x int32 pos, len
//   n x float32 xmin, ymin, xmax, ymax; n x int32 id
// all little-endian.  Loading allocates the device arrays with cudaMalloc
// (free with crt_rtree_free / crt_bbox_free).
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace crt {

namespace {

const char kMagic[8] = {'C', 'R', 'T', 'R', 'E', 'E', 0, 1};

bool read_file(const char* path, std::string& out)
{
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  out.resize(sz > 0 ? (size_t)sz : 0);
  const bool ok = sz <= 0 || std::fread(&out[0], 1, (size_t)sz, f) == (size_t)sz;
  std::fclose(f);
  return ok;
}

inline const char* skip_ws(const char* p, const char* end)
{
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) p++;
  return p;
}

}  // namespace

// One record "x1,y1,x2,y2,id,pid,nume" starting at p; false if malformed.
bool parse_mbr_record(const char* p, const char* end, float v[4], int& id)
{
  char buf[64];
  for (int f = 0; f < 7; f++) {
    p = skip_ws(p, end);
    size_t m = 0;
    while (p + m < end && p[m] != ',' && p[m] != '\n' && p[m] != '\r' && m < sizeof(buf) - 1) m++;
    if (m == 0) return false;
    std::memcpy(buf, p, m);
    buf[m] = 0;
    char* stop = nullptr;
    errno = 0;
    if (f < 4) {
      v[f] = std::strtof(buf, &stop);
    } else {
      const long x = std::strtol(buf, &stop, 10);
      if (f == 4) id = (int)x;
    }
    // fscanf skips blanks before a number, and the format's closing newline
    // matches blanks after the last one; a blank before a ',' fails the match
    if (f == 6)
      while (stop && (*stop == ' ' || *stop == '\t')) stop++;
    if (!stop || *stop != 0) return false;
    p += m;
    if (f < 6) {
      if (p >= end || *p != ',') return false;
      p++;
    }
  }
  return true;
}

namespace {

// Class of a stretch's last byte that is not ' ', '\t' or '\r'.
constexpr int kNoByte = 0, kNewline = 1, kOtherByte = 2;

inline bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

int last_class(const char* p, const char* e)
{
  while (e > p) {
    const char c = *--e;
    if (!is_blank(c)) return c == '\n' ? kNewline : kOtherByte;
  }
  return kNoByte;
}

// Record starts in [b, e), at most `cap`, given the class of the last
// non-blank byte before b.
void chunk_starts(const char* base, size_t b, size_t e, int in, int64_t cap,
                  std::vector<size_t>& out)
{
  int prev = in;
  for (size_t i = b; i < e && (int64_t)out.size() < cap; i++) {
    const char c = base[i];
    if (is_blank(c)) continue;
    if (c != '\n' && prev != kOtherByte) out.push_back(i);
    prev = c == '\n' ? kNewline : kOtherByte;
  }
}

}  // namespace

// The first n record starts: the first byte of each line that is not ' ',
// '\t' or '\r', unless it is the line's '\n' -- the same as "a byte that is
// neither blank nor '\n' whose previous non-blank byte is a '\n' or absent".
// The second form splits: host threads take 8 MiB chunks, the class each
// chunk ends with is carried across the chunks, then each thread lists its
// chunk's starts.
std::vector<size_t> record_starts(const char* base, size_t L, int64_t n)
{
  constexpr size_t kChunk = size_t(8) << 20;
  const int hw = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const int nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)hw, (L + kChunk - 1) / kChunk));
  const size_t per = (L + nt - 1) / std::max(nt, 1);
  std::vector<int> last(nt, kNoByte);
  std::vector<std::vector<size_t>> part(nt);
  auto run = [&](auto&& body) {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(body, t);
    body(0);
    for (auto& x : th) x.join();
  };
  run([&](int t) {
    const size_t b = std::min(L, t * per), e = std::min(L, b + per);
    last[t] = last_class(base + b, base + e);
  });
  run([&](int t) {
    int in = kNoByte;
    for (int u = 0; u < t; u++)
      if (last[u] != kNoByte) in = last[u];
    const size_t b = std::min(L, t * per), e = std::min(L, b + per);
    chunk_starts(base, b, e, in, n, part[t]);
  });
  std::vector<size_t> starts;
  starts.reserve((size_t)std::max<int64_t>(0, n));
  for (int t = 0; t < nt && (int64_t)starts.size() < n; t++) {
    const size_t take = (size_t)std::min<int64_t>((int64_t)part[t].size(), n - (int64_t)starts.size());
    starts.insert(starts.end(), part[t].begin(), part[t].begin() + take);
  }
  return starts;
}

void mbr_box(const float v[4], float r, float* xmin, float* ymin, float* xmax, float* ymax)
{
  // readMBR: min/max of the endpoints, then -/+ r (fp32)
  *xmin = std::min(v[0], v[2]) - r;
  *ymin = std::min(v[1], v[3]) - r;
  *xmax = std::max(v[0], v[2]) + r;
  *ymax = std::max(v[1], v[3]) + r;
}

int read_mbr_text(const char* base, size_t L, int64_t n, float r, float* xmin, float* ymin,
                  float* xmax, float* ymax, int32_t* id, int64_t* n_read)
{
  const std::vector<size_t> starts = record_starts(base, L, n);
  const int64_t m = (int64_t)starts.size();
  const char* end = base + L;
  int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<int64_t> bad(nt, -1);
  std::vector<std::thread> th;
  const int64_t per = (m + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    th.emplace_back([&, t] {
      for (int64_t k = t * per; k < std::min(m, (t + 1) * per); k++) {
        float v[4];
        int rid = 0;
        if (!parse_mbr_record(base + starts[k], end, v, rid)) {
          bad[t] = k;
          return;
        }
        mbr_box(v, r, &xmin[k], &ymin[k], &xmax[k], &ymax[k]);
        id[k] = rid;
      }
    });
  }
  for (auto& x : th) x.join();
  int64_t first_bad = -1;
  for (auto b : bad)
    if (b >= 0 && (first_bad < 0 || b < first_bad)) first_bad = b;
  if (first_bad >= 0) {
    if (n_read) *n_read = first_bad;
    return fail(CRT_ERR_INVALID_ARG,
                "read_mbr_csv: record " + std::to_string(first_bad) + " is not x1,y1,x2,y2,id,pid,nume");
  }
  if (n_read) *n_read = m;
  if (m < n)
    return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv: file holds " + std::to_string(m) +
                                         " records, " + std::to_string(n) + " requested");
  return CRT_OK;
}

}  // namespace crt

using namespace crt;

extern "C" {

int crt_read_mbr_csv(const char* path, int64_t n, float r, float* xmin, float* ymin, float* xmax,
                     float* ymax, int32_t* id, int64_t* n_read)
{
  if (!path || n < 0 || (n > 0 && !(xmin && ymin && xmax && ymax && id)))
    return fail(CRT_ERR_INVALID_ARG, "read_mbr_csv: bad arguments");
  if (n_read) *n_read = 0;
  std::string text;
  if (!read_file(path, text)) return fail(CRT_ERR_INVALID_ARG, std::string("read_mbr_csv: cannot open ") + path);
  return read_mbr_text(text.data(), text.size(), n, r, xmin, ymin, xmax, ymax, id, n_read);
}

int crt_bbox_free(crt_bbox_f32* b)
{
  if (!b) return fail(CRT_ERR_INVALID_ARG, "bbox_free: null");
  void* p[5] = {b->xmin, b->ymin, b->xmax, b->ymax, b->id};
  for (void* q : p)
    if (q) cudaFree(q);
  b->xmin = b->ymin = b->xmax = b->ymax = nullptr;
  b->id = nullptr;
  return CRT_OK;
}

static int copy_out(FILE* f, const void* dev, size_t bytes, std::vector<char>& buf)
{
  size_t done = 0;
  while (done < bytes) {
    const size_t m = std::min(buf.size(), bytes - done);
    cudaError_t e = cudaMemcpy(buf.data(), (const char*)dev + done, m, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "tree_save");
    if (std::fwrite(buf.data(), 1, m, f) != m) return fail(CRT_ERR_INVALID_ARG, "tree_save: write failed");
    done += m;
  }
  return CRT_OK;
}

int crt_tree_save(const char* path, const crt_rtree_f32* d_rt, const crt_bbox_f32* d_rbox)
{
  if (!path || !d_rt || !d_rbox || d_rt->sz < 0 || d_rbox->sz < 0)
    return fail(CRT_ERR_INVALID_ARG, "tree_save: bad arguments");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(CRT_ERR_INVALID_ARG, std::string("tree_save: cannot create ") + path);
  const int64_t n = d_rbox->sz, rsz = d_rt->sz;
  const int32_t hdr2[2] = {d_rt->fanout, 0};
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&n, 8, 1, f) == 1 &&
            std::fwrite(&rsz, 8, 1, f) == 1 && std::fwrite(hdr2, 4, 2, f) == 2;
  int rc = ok ? CRT_OK : fail(CRT_ERR_INVALID_ARG, "tree_save: write failed");
  std::vector<char> buf(64 << 20);
  const void* arrs[11] = {d_rt->xmin, d_rt->ymin, d_rt->xmax, d_rt->ymax, d_rt->pos, d_rt->len,
                          d_rbox->xmin, d_rbox->ymin, d_rbox->xmax, d_rbox->ymax, d_rbox->id};
  for (int a = 0; a < 11 && rc == CRT_OK; a++) {
    const size_t bytes = (size_t)(a < 6 ? rsz : n) * 4;
    if (bytes && !arrs[a]) rc = fail(CRT_ERR_INVALID_ARG, "tree_save: null array");
    else if (bytes) rc = copy_out(f, arrs[a], bytes, buf);
  }
  if (std::fclose(f) != 0 && rc == CRT_OK) rc = fail(CRT_ERR_INVALID_ARG, "tree_save: close failed");
  return rc;
}

int crt_tree_load(const char* path, crt_rtree_f32* d_rt, crt_bbox_f32* d_rbox)
{
  if (!path || !d_rt || !d_rbox) return fail(CRT_ERR_INVALID_ARG, "tree_load: bad arguments");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(CRT_ERR_INVALID_ARG, std::string("tree_load: cannot open ") + path);
  char magic[8];
  int64_t n = 0, rsz = 0;
  int32_t hdr2[2] = {0, 0};
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
            std::fread(&n, 8, 1, f) == 1 && std::fread(&rsz, 8, 1, f) == 1 &&
            std::fread(hdr2, 4, 2, f) == 2;
  if (!ok || n < 0 || rsz < 0 || n > INT32_MAX || rsz > INT32_MAX || n + rsz > INT32_MAX ||
      (rsz > 0 && hdr2[0] < 2) || crt_tree_size(std::max<int64_t>(n, 1), std::max(hdr2[0], 2)) != rsz) {
    std::fclose(f);
    return fail(CRT_ERR_INVALID_ARG, "tree_load: not a tree file, or a damaged one");
  }
  crt_rtree_f32 t{};
  crt_bbox_f32 b{};
  t.sz = (int)rsz;
  t.fanout = hdr2[0];
  b.sz = (int)n;
  void** dst[11] = {(void**)&t.xmin, (void**)&t.ymin, (void**)&t.xmax, (void**)&t.ymax,
                    (void**)&t.pos,  (void**)&t.len,  (void**)&b.xmin, (void**)&b.ymin,
                    (void**)&b.xmax, (void**)&b.ymax, (void**)&b.id};
  std::vector<char> buf(64 << 20);
  int rc = CRT_OK;
  for (int a = 0; a < 11 && rc == CRT_OK; a++) {
    const size_t bytes = (size_t)(a < 6 ? rsz : n) * 4;
    if (!bytes) continue;
    if (cudaMalloc(dst[a], bytes) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(CRT_ERR_OOM, "tree_load: allocation failed");
      break;
    }
    size_t done = 0;
    while (done < bytes && rc == CRT_OK) {
      const size_t m = std::min(buf.size(), bytes - done);
      if (std::fread(buf.data(), 1, m, f) != m) {
        rc = fail(CRT_ERR_INVALID_ARG, "tree_load: file is truncated");
        break;
      }
      cudaError_t e = cudaMemcpy((char*)*dst[a] + done, buf.data(), m, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) rc = cuda_fail(e, "tree_load");
      done += m;
    }
  }
  std::fclose(f);
  if (rc != CRT_OK) {
    for (int a = 0; a < 11; a++)
      if (*dst[a]) cudaFree(*dst[a]);
    return rc;
  }
  *d_rt = t;
  *d_rbox = b;
  return CRT_OK;
}

}  // extern "C"
