// Box-file reader/writer shared by the reference runners (oracle/ref_gpu_*.cu).
// Format ("CRTB"): 4-byte magic, int64 count n, then n float32 xmin, ymin,
// xmax, ymax and n int32 ids, little-endian.  Test infrastructure only.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

struct CrtbBoxes {
  std::vector<float> xmin, ymin, xmax, ymax;
  std::vector<int> id;
  int64_t n = 0;
};

inline bool crtb_read(const std::string& path, CrtbBoxes& b)
{
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[4];
  bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "CRTB", 4) == 0 &&
            std::fread(&b.n, sizeof(int64_t), 1, f) == 1 && b.n >= 0;
  if (ok) {
    b.xmin.resize(b.n); b.ymin.resize(b.n); b.xmax.resize(b.n); b.ymax.resize(b.n); b.id.resize(b.n);
    size_t n = (size_t)b.n;
    ok = std::fread(b.xmin.data(), 4, n, f) == n && std::fread(b.ymin.data(), 4, n, f) == n &&
         std::fread(b.xmax.data(), 4, n, f) == n && std::fread(b.ymax.data(), 4, n, f) == n &&
         std::fread(b.id.data(), 4, n, f) == n;
  }
  std::fclose(f);
  return ok;
}

inline bool crtb_write_arrays(const std::string& path, const std::vector<const void*>& arrays,
                              const std::vector<size_t>& bytes)
{
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = true;
  for (size_t i = 0; i < arrays.size(); i++)
    if (bytes[i] && std::fwrite(arrays[i], 1, bytes[i], f) != bytes[i]) ok = false;
  std::fclose(f);
  return ok;
}
