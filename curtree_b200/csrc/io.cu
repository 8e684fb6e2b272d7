// Host-side I/O around the tree: the reference's MBR text loader and a tree
// file format.
//
// crt_read_mbr_csv restates readMBR (src/utility.cpp:5-40), which reads each
// record with fscanf(fp, "%f,%f,%f,%f,%d,%d,%d\n", ...): the box is
// [min(x1,x2) - r, max(x1,x2) + r] x [min(y1,y2) - r, max(y1,y2) + r] in fp32,
// id is the fifth field, pid and nume are read and dropped.  Numbers parse as
// fscanf's %f / %d do (strtof / strtol, correctly rounded); whitespace
// (newlines included) may precede a number but not a ',' (the format's
// literal commas do not skip it), and the closing "\n" skips any whitespace,
// so records need not sit one per line.  Where the reference exits (missing
// file) or throws (a malformed record), this returns a status.  Records are
// parsed by several host threads.
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

// fscanf's whitespace (isspace in the C locale)
inline bool is_space(char c)
{
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

inline const char* skip_ws(const char* p, const char* end)
{
  while (p < end && is_space(*p)) p++;
  return p;
}

}  // namespace

// One record of readMBR's fscanf(fp, "%f,%f,%f,%f,%d,%d,%d\n", ...) at p:
// each number may be preceded by whitespace (newlines too); the literal ','
// must follow a number at once; after the last number the format's closing
// "\n" skips any whitespace, and whatever follows begins the next record.
// Returns the position after the record and that whitespace, or nullptr
// where fscanf would read fewer than seven fields.
const char* parse_mbr_record(const char* p, const char* end, float v[4], int& id)
{
  char buf[64];
  std::string big;
  for (int f = 0; f < 7; f++) {
    p = skip_ws(p, end);
    size_t m = 0;
    while (p + m < end && p[m] != ',' && !is_space(p[m])) m++;
    if (m == 0) return nullptr;
    const char* tok = buf;
    if (m < sizeof(buf)) {
      std::memcpy(buf, p, m);
      buf[m] = 0;
    } else {
      big.assign(p, m);
      tok = big.c_str();
    }
    char* stop = nullptr;
    if (f < 4) {
      v[f] = std::strtof(tok, &stop);
    } else {
      const long x = std::strtol(tok, &stop, 10);
      if (f == 4) id = (int)x;
    }
    if (!stop || stop == tok) return nullptr;  // no number here
    const size_t used = (size_t)(stop - tok);
    if (f < 6) {
      if (used != m || p + m >= end || p[m] != ',') return nullptr;
      p += m + 1;
    } else {
      p += used;
    }
  }
  return skip_ws(p, end);
}

namespace {

// Class of a stretch's last byte that is not whitespace.
constexpr int kNoByte = 0, kComma = 1, kOtherByte = 2;

int last_class(const char* p, const char* e)
{
  while (e > p) {
    const char c = *--e;
    if (!is_space(c)) return c == ',' ? kComma : kOtherByte;
  }
  return kNoByte;
}

// Candidate record starts in [b, e), at most `cap`: a byte that is neither
// whitespace nor ',' whose previous byte is whitespace (or absent) and whose
// last non-whitespace predecessor is not a ',' (or absent).  `in` is the
// class of the last non-whitespace byte before b.
void chunk_starts(const char* base, size_t b, size_t e, int in, int64_t cap,
                  std::vector<size_t>& out)
{
  int prev = in;
  bool ws = b == 0 || is_space(base[b - 1]);
  for (size_t i = b; i < e && (int64_t)out.size() < cap; i++) {
    const char c = base[i];
    if (is_space(c)) {
      ws = true;
      continue;
    }
    if (c != ',' && ws && prev != kComma) out.push_back(i);
    prev = c == ',' ? kComma : kOtherByte;
    ws = false;
  }
}

}  // namespace

// The first n candidate record starts (n < 0: all).  In a text that fscanf
// reads record after record, these are where its records begin: every
// record's first number follows whitespace (or begins the text), and no
// other number is both preceded by whitespace and not preceded by a ','.
// Host threads take 8 MiB chunks; the class each chunk ends with is carried
// across the chunks, then each thread lists its chunk's starts.
std::vector<size_t> record_starts(const char* base, size_t L, int64_t n)
{
  if (n < 0) n = INT64_MAX;
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

// Records in readMBR's order: the candidate starts are parsed by host
// threads, and the records are kept up to the first one that does not begin
// exactly where the one before ended (after its trailing whitespace) or does
// not parse; from there the text is read one record after another, as
// fscanf reads it.  So the result is fscanf's for any text, and parallel for
// the usual one: records separated by whitespace, no record ending in a
// byte that runs into the next number.
void scan_mbr_text(const char* base, size_t L, int64_t limit, float r, MbrRecords& out)
{
  const char* end = base + L;
  const std::vector<size_t> starts = record_starts(base, L, limit);
  const int64_t m = (int64_t)starts.size();
  for (auto& v : out.v) v.resize((size_t)m);
  out.id.resize((size_t)m);
  std::vector<int64_t> ends((size_t)m, -1);
  const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  const int64_t per = (m + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    th.emplace_back([&, t] {
      for (int64_t k = t * per; k < std::min(m, (t + 1) * per); k++) {
        float v[4];
        int rid = 0;
        const char* e = parse_mbr_record(base + starts[k], end, v, rid);
        if (!e) continue;
        ends[k] = e - base;
        mbr_box(v, r, &out.v[0][k], &out.v[1][k], &out.v[2][k], &out.v[3][k]);
        out.id[k] = rid;
      }
    });
  }
  for (auto& x : th) x.join();
  // keep the records fscanf would read the same way
  int64_t expect = skip_ws(base, end) - base;
  int64_t good = 0;
  while (good < m && (int64_t)starts[good] == expect && ends[good] >= 0) expect = ends[good++];
  for (auto& v : out.v) v.resize((size_t)good);
  out.id.resize((size_t)good);
  out.count = good;
  out.malformed = false;
  // then one record after another from where the last kept one ended
  const char* p = base + expect;
  while (limit < 0 || out.count < limit) {
    p = skip_ws(p, end);
    if (p >= end) break;  // end of text: fewer records than asked for
    float v[4];
    int rid = 0;
    const char* e = parse_mbr_record(p, end, v, rid);
    if (!e) {
      out.malformed = true;
      break;
    }
    float b[4];
    mbr_box(v, r, &b[0], &b[1], &b[2], &b[3]);
    for (int a = 0; a < 4; a++) out.v[a].push_back(b[a]);
    out.id.push_back(rid);
    out.count++;
    p = e;
  }
}

int read_mbr_text(const char* base, size_t L, int64_t n, float r, float* xmin, float* ymin,
                  float* xmax, float* ymax, int32_t* id, int64_t* n_read)
{
  MbrRecords rec;
  scan_mbr_text(base, L, n, r, rec);
  const int64_t m = rec.count;
  float* dst[4] = {xmin, ymin, xmax, ymax};
  for (int a = 0; a < 4; a++)
    if (m) std::memcpy(dst[a], rec.v[a].data(), sizeof(float) * (size_t)m);
  if (m) std::memcpy(id, rec.id.data(), sizeof(int32_t) * (size_t)m);
  if (n_read) *n_read = m;
  if (rec.malformed)
    return fail(CRT_ERR_INVALID_ARG,
                "read_mbr_csv: record " + std::to_string(m) + " is not x1,y1,x2,y2,id,pid,nume");
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
