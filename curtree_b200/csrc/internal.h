// Internal host interfaces shared between the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace crt {

// Radix-sort scratch shared by the box build and the window ordering.
struct SortBufs {
  uint32_t* keys[2];
  uint32_t* vals[2];
};

// Radix digits of the 32-bit sort keys: kDigits digits of kDigitBits bits
// from the least significant end, the last one narrower when kDigitBits does
// not divide 32.  Histograms and bucket starts keep kBins entries per digit.
// 8-bit digits (four passes, uniform digits skipped) measured faster on a
// B200 than 10 + 10 + 10 + 2 (three passes for 30-bit Morton keys): 2.74
// against 3.43 ms for 100M keys, the 1024-bin passes paying more for ranking,
// bin scans and look-back than the fourth pass costs.
#ifndef CRT_SORT_DIGIT_BITS
#define CRT_SORT_DIGIT_BITS 8
#endif
constexpr int kDigitBits = CRT_SORT_DIGIT_BITS;
constexpr int kBins = 1 << kDigitBits;
constexpr int kDigits = (32 + kDigitBits - 1) / kDigitBits;
static_assert(kDigits == 4, "four digit passes at most");
constexpr int kSortTile = 8192;

__host__ __device__ constexpr int digit_bits(int d)
{
  return 32 - d * kDigitBits < kDigitBits ? 32 - d * kDigitBits : kDigitBits;
}
__device__ __forceinline__ uint32_t key_digit(uint32_t k, int d)
{
  return (k >> (d * kDigitBits)) & ((1u << digit_bits(d)) - 1u);
}

// Control block of one sort (int32 words, zero-initialised by the caller).
struct SortCtrl {
  int tile_ctr[4];  // per pass: next tile index
  int error;        // first device error
  int active;       // bit d: digit d is non-uniform
  int n_active;     // number of active passes: the order is in vals[n_active & 1]
  int pad[9];
  int bucket_start[kDigits * kBins];
};

// Bytes of zero-initialised state a sort of n keys needs: SortCtrl, the
// digit histograms (kDigits x kBins words, filled by the caller's key kernel
// with key_digit) and the look-back status words (in that order).
size_t sort_zero_bytes(int64_t n);
// Enqueues plan + four onesweep passes; keys must be in bufs.keys[0] and the
// histograms filled.  The sorted positions end in bufs.vals[n_active & 1]
// (identity when no pass is active).
// flags: kSortGivenValues -- the values are in bufs.vals[0] (otherwise the
// first pass makes them: positions 0..n-1); kSortKeepKeys -- the sorted keys
// are kept too, in bufs.keys[n_active & 1] (otherwise the last pass drops them).
constexpr int kSortGivenValues = 1;
constexpr int kSortKeepKeys = 2;
void sort_passes(SortBufs bufs, int64_t n, void* zero_block, cudaStream_t stream, int flags = 0);
uint32_t* sort_hist(void* zero_block);
SortCtrl* sort_ctrl(void* zero_block);

int tree_levels(int64_t n, int fanout, std::vector<int64_t>& lv);

int build_tree(const float* in_xmin, const float* in_ymin, const float* in_xmax,
               const float* in_ymax, const int* in_id, int64_t n, int fanout, float* out_xmin,
               float* out_ymin, float* out_xmax, float* out_ymax, int* out_id, float* nxmin,
               float* nymin, float* nxmax, float* nymax, int* npos, int* nlen,
               cudaStream_t stream);

int pairs_canonicalize(int32_t* fid, int32_t* tid, int64_t n, cudaStream_t stream);
int pairs_digest(const int32_t* fid, const int32_t* tid, int64_t n, int64_t window_base,
                 int64_t nq, int64_t* d_counts, uint64_t* d_hashes, int64_t* d_bad,
                 cudaStream_t stream);

// Query entry used by the C ABI.
int query_into(const crt_rtree_f32& rt, const crt_bbox_f32& rbox, const crt_bbox_f32& qbox,
               int32_t* fid, int32_t* tid, int64_t capacity, crt_query_result* d_result,
               int64_t* d_offsets, const crt_query_opts& opts, cudaStream_t stream);
int64_t query_capacity(int64_t pairs, const crt_query_opts& opts);

// Host parser of the reference's MBR text format (io.cu), with the rules of
// readMBR's fscanf(fp, "%f,%f,%f,%f,%d,%d,%d\n", ...): one record at p (the
// position after it and the whitespace that follows, or nullptr where fscanf
// reads fewer than seven fields), the box readMBR makes of its four numbers,
// and whole texts: scan_mbr_text reads up to `limit` records (limit < 0:
// all) in fscanf's order, stopping at the end of the text or at a malformed
// record; read_mbr_text does so into caller arrays (statuses and *n_read as
// crt_read_mbr_csv).
const char* parse_mbr_record(const char* p, const char* end, float v[4], int& id);
void mbr_box(const float v[4], float r, float* xmin, float* ymin, float* xmax, float* ymax);
struct MbrRecords {
  std::vector<float> v[4];  // xmin, ymin, xmax, ymax
  std::vector<int32_t> id;
  int64_t count = 0;
  bool malformed = false;  // stopped at a record fscanf cannot read
};
void scan_mbr_text(const char* base, size_t len, int64_t limit, float r, MbrRecords& out);
int read_mbr_text(const char* base, size_t len, int64_t n, float r, float* xmin, float* ymin,
                  float* xmax, float* ymax, int32_t* id, int64_t* n_read);

}  // namespace crt
