// Stable in-cell order of the grid build for crowded cells.
//
// The grid build sorts particles by cell key with a counting sort whose
// scatter leaves each cell's ids in atomic arrival order; the reference's
// stable radix sort (wp.HashGrid.build) leaves them ascending.  Cells of up
// to kSmallCell particles take their rank by counting smaller ids (at most
// kSmallCell loads per particle).  The ids of a more crowded cell are sorted
// by one thread block: a bitonic sort in shared memory up to kSmemSortMax
// ids, else an LSD radix sort of the ids (8-bit digits, stable scatter
// through per-warp digit counts) over a global ping-pong pair.  Work stays
// O(N) per build whatever the occupancy: a cell of 200,000 particles (or a
// blown-up state, whose non-finite particles share one bucket) costs a few
// radix passes instead of k^2 comparisons.
#pragma once

#include <stdint.h>

namespace fs {

constexpr int kSmallCell = 64;        // cells up to this size rank in place
constexpr int kSortThreads = 1024;    // threads of a crowded-cell sorting block
constexpr int kSmemSortMax = 4096;    // largest cell sorted in shared memory
constexpr int kRadixWarps = kSortThreads / 32;
// dynamic shared memory of a sorting block: the bitonic buffer, or the radix
// pass's per-warp digit counts + digit bases
constexpr int kSortSmemInts =
    (kSmemSortMax > kRadixWarps * 256 + 256) ? kSmemSortMax : kRadixWarps * 256 + 256;
constexpr size_t kSortSmemBytes = sizeof(int32_t) * kSortSmemInts;

// Largest number of crowded cells a build of n particles can have.
__host__ __device__ inline int64_t max_big_cells(int64_t n) { return n / (kSmallCell + 1) + 1; }

// Bits that hold every id below n.
__device__ __forceinline__ int id_bits(int64_t n) {
  const uint32_t m = n > 1 ? (uint32_t)(n - 1) : 1u;
  return 32 - __clz(m);
}

// Ascending sort of v[0, len) (len <= kSmemSortMax) in shared memory s; the
// whole block calls it.
__device__ inline void block_bitonic_sort(int32_t* v, int len, int32_t* s) {
  int p = 1;
  while (p < len) p <<= 1;
  for (int k = threadIdx.x; k < p; k += blockDim.x) s[k] = k < len ? v[k] : 0x7fffffff;
  __syncthreads();
  for (int k = 2; k <= p; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < p; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const int32_t a = s[i], b = s[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int k = threadIdx.x; k < len; k += blockDim.x) v[k] = s[k];
  __syncthreads();
}

// One stable LSD pass: dst = src ordered by digit (src >> shift) & 255,
// equal digits in src order.  The whole block (kSortThreads threads) calls
// it; smem holds kSortSmemInts ints.
__device__ inline void block_radix_pass(const int32_t* src, int32_t* dst, int len, int shift, int32_t* smem) {
  int32_t* wcnt = smem;                      // [kRadixWarps][256]
  int32_t* base = smem + kRadixWarps * 256;  // [256] running start of each digit
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int d = tid; d < 256; d += blockDim.x) base[d] = 0;
  __syncthreads();
  for (int k = tid; k < len; k += blockDim.x) atomicAdd(&base[(src[k] >> shift) & 255], 1);
  __syncthreads();
  if (w == 0) {  // exclusive prefix of the 256 digit counts, 8 per lane
    int32_t v[8], s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      v[q] = base[lane * 8 + q];
      s += v[q];
    }
    int32_t inc = s;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    int32_t run = inc - s;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      base[lane * 8 + q] = run;
      run += v[q];
    }
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int c0 = 0; c0 < len; c0 += blockDim.x) {
    for (int q = tid; q < kRadixWarps * 256; q += blockDim.x) wcnt[q] = 0;
    __syncthreads();
    const int k = c0 + tid;
    const bool valid = k < len;
    const int32_t v = valid ? src[k] : 0;
    const int d = valid ? (v >> shift) & 255 : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & lt);
    if (valid && rank == 0) wcnt[w * 256 + d] = __popc(peers);
    __syncthreads();
    for (int dd = tid; dd < 256; dd += blockDim.x) {  // warps in order: earlier warps hold earlier ids
      int32_t run = base[dd];
      for (int ww = 0; ww < kRadixWarps; ++ww) {
        const int32_t t = wcnt[ww * 256 + dd];
        wcnt[ww * 256 + dd] = run;
        run += t;
      }
      base[dd] = run;
    }
    __syncthreads();
    if (valid) dst[wcnt[w * 256 + d] + rank] = v;
    __syncthreads();
  }
}

// Sorts the ids a[0, len) ascending (the whole block calls it).  b[0, len)
// is scratch of the same size; the result is in a or in b: returns the one.
__device__ inline int32_t* block_sort_ids(int32_t* a, int32_t* b, int len, int bits, int32_t* smem) {
  if (len <= kSmemSortMax) {
    block_bitonic_sort(a, len, smem);
    return a;
  }
  int32_t* src = a;
  int32_t* dst = b;
  for (int shift = 0; shift < bits; shift += 8) {
    block_radix_pass(src, dst, len, shift, smem);
    int32_t* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

}  // namespace fs
