// Result assembly on opened match bitmaps: candidate lists, per-query final
// results and the in-batch deduplication.
//
// Bitmaps are u32 words [query][stride/32] (bit j of word w = entry 32w + j).
// Each thread owns one word and touches memory only for set bits; the list
// appends use one atomic per warp (ballot + popc) instead of one per match.
// Semantics follow iris-mpc-gpu/src/dot/kernel.cu: partialDbResults 212-239,
// mergeDbResults 241-282, mergeDbResultsWithOrPolicyBitmap 284-349,
// mergeBatchResults 352-387 (MAX_MATCHES_LEN = 256).
#include <cuda_runtime.h>
#include <stdint.h>
#include "results.h"

namespace irs {

namespace {

__global__ void compact_kernel(const uint32_t* __restrict__ bitmap, uint32_t n_queries, uint32_t db_len,
                               uint32_t stride_words, uint32_t* __restrict__ out, uint32_t* __restrict__ counter,
                               uint32_t cap) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t words = (db_len + 31) / 32;
  const bool in_range = i < (uint64_t)n_queries * words;
  uint32_t bits = 0, q = 0, w = 0;
  if (in_range) {
    q = (uint32_t)(i / words);
    w = (uint32_t)(i % words);
    bits = bitmap[(size_t)q * stride_words + w];
    const uint32_t valid = db_len - w * 32;
    if (valid < 32) bits &= (1u << valid) - 1u;
  }
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = (uint32_t)__popc(bits);
  // warp-level exclusive scan of n
  uint32_t incl = n;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= (uint32_t)d) incl += t;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(0xFFFFFFFFu, base, 31);
  uint32_t pos = base + incl - n;
  while (bits) {
    const int b = __ffs(bits) - 1;
    bits &= bits - 1;
    if (pos < cap) out[pos] = w * 32 + (uint32_t)b;
    pos++;
  }
}

// Ordered compaction of selected bitmap rows (one block per listed row): the
// row's set bits below db_len become ascending entry ids (the lowest `cap`
// kept, the total counted), and the words are zeroed when `clear` so the row
// can be reused.  256 threads sweep the row 256 words at a time; a block-wide
// exclusive scan of the per-word popcounts gives each set bit its position.
__global__ void take_rows_kernel(uint32_t* __restrict__ bitmap, uint32_t stride_words,
                                 const uint32_t* __restrict__ rows, uint32_t db_len, int clear,
                                 uint32_t* __restrict__ counts, uint32_t* __restrict__ ids, uint32_t cap) {
  __shared__ uint32_t warp_sums[8];
  __shared__ uint32_t running;
  const uint32_t row = rows[blockIdx.x];
  uint32_t* src = bitmap + (size_t)row * stride_words;
  uint32_t* out = ids + (size_t)blockIdx.x * cap;
  const uint32_t words = (db_len + 31) / 32;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) running = 0;
  __syncthreads();
  for (uint32_t base = 0; base < words; base += blockDim.x) {
    const uint32_t w = base + threadIdx.x;
    uint32_t bits = 0;
    if (w < words) {
      bits = src[w];
      const uint32_t valid = db_len - w * 32;
      if (valid < 32) bits &= (1u << valid) - 1u;
      if (clear) src[w] = 0;
    }
    const uint32_t n = (uint32_t)__popc(bits);
    uint32_t incl = n;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= (uint32_t)d) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    uint32_t before = running;
    for (uint32_t k = 0; k < warp; k++) before += warp_sums[k];
    uint32_t pos = before + incl - n;
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      if (pos < cap) out[pos] = w * 32 + (uint32_t)b;
      pos++;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t tot = 0;
      for (uint32_t k = 0; k < blockDim.x / 32; k++) tot += warp_sums[k];
      running += tot;
    }
    __syncthreads();
  }
  if (clear) {  // words past db_len (appends not yet scanned by this row's request) are cleared too
    for (uint32_t w = words + threadIdx.x; w < stride_words; w += blockDim.x) src[w] = 0;
  }
  if (threadIdx.x == 0) counts[blockIdx.x] = running;
}

// mergeDbResults / mergeDbResultsWithOrPolicyBitmap with one or two eyes.
__global__ void merge_db_kernel(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                                const uint32_t* __restrict__ or_policy, uint32_t n_queries, uint32_t db_len,
                                uint32_t stride_words, uint32_t* __restrict__ final_results,
                                uint32_t* __restrict__ match_counter, uint32_t* __restrict__ all_matches) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t words = (db_len + 31) / 32;
  if (i >= (uint64_t)n_queries * words) return;
  const uint32_t q = (uint32_t)(i / words), w = (uint32_t)(i % words);
  const size_t idx = (size_t)q * stride_words + w;
  const uint32_t l = left[idx];
  uint32_t bits = l;
  if (right) {
    const uint32_t r = right[idx];
    const uint32_t pol = or_policy ? or_policy[idx] : 0u;
    bits = (l & r & ~pol) | ((l | r) & pol);
  }
  const uint32_t valid = db_len - w * 32;
  if (valid < 32) bits &= (1u << valid) - 1u;
  while (bits) {
    const int b = __ffs(bits) - 1;
    bits &= bits - 1;
    const uint32_t db = w * 32 + (uint32_t)b;
    atomicMin(&final_results[q], db);
    const uint32_t c = atomicAdd(&match_counter[q], 1u);
    if (c < kMaxMatchesLen) all_matches[(size_t)kMaxMatchesLen * q + c] = db;
  }
}

// mergeBatchResults: self bitmap [query][j] of query q against the centre
// (DB-format) share of batch query j; only strictly earlier queries count.
__global__ void merge_batch_kernel(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                                   uint32_t n_queries, uint32_t stride_words, uint32_t* __restrict__ final_results,
                                   uint32_t* __restrict__ match_counter, uint32_t* __restrict__ all_matches) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t words = (n_queries + 31) / 32;
  if (i >= (uint64_t)n_queries * words) return;
  const uint32_t q = (uint32_t)(i / words), w = (uint32_t)(i % words);
  const size_t idx = (size_t)q * stride_words + w;
  uint32_t bits = left[idx];
  if (right) bits &= right[idx];
  // keep j < q only (above the diagonal in the reference's orientation)
  const uint32_t lo = w * 32;
  if (lo >= q) bits = 0;
  else if (q - lo < 32) bits &= (1u << (q - lo)) - 1u;
  while (bits) {
    const int b = __ffs(bits) - 1;
    bits &= bits - 1;
    const uint32_t j = lo + (uint32_t)b;
    atomicMin(&final_results[q], 0xFFFFFFFFu - 1u);
    const uint32_t c = atomicAdd(&match_counter[q], 1u);
    if (c < kMaxMatchesLen) all_matches[(size_t)kMaxMatchesLen * q + c] = 0xFFFFFFFFu - j;
  }
}

}  // namespace

cudaError_t launch_compact(const uint32_t* bitmap, uint32_t n_queries, uint32_t db_len, uint32_t stride_words,
                           uint32_t* out, uint32_t* counter, uint32_t cap, cudaStream_t stream) {
  const uint64_t n = (uint64_t)n_queries * ((db_len + 31) / 32);
  if (!n) return cudaSuccess;
  compact_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(bitmap, n_queries, db_len, stride_words, out,
                                                                  counter, cap);
  return cudaGetLastError();
}

cudaError_t launch_merge_db(const uint32_t* left, const uint32_t* right, const uint32_t* or_policy, uint32_t n_queries,
                            uint32_t db_len, uint32_t stride_words, uint32_t* final_results, uint32_t* match_counter,
                            uint32_t* all_matches, cudaStream_t stream) {
  const uint64_t n = (uint64_t)n_queries * ((db_len + 31) / 32);
  if (!n) return cudaSuccess;
  merge_db_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(left, right, or_policy, n_queries, db_len,
                                                                   stride_words, final_results, match_counter,
                                                                   all_matches);
  return cudaGetLastError();
}

cudaError_t launch_merge_batch(const uint32_t* left, const uint32_t* right, uint32_t n_queries, uint32_t stride_words,
                               uint32_t* final_results, uint32_t* match_counter, uint32_t* all_matches,
                               cudaStream_t stream) {
  const uint64_t n = (uint64_t)n_queries * ((n_queries + 31) / 32);
  if (!n) return cudaSuccess;
  merge_batch_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(left, right, n_queries, stride_words,
                                                                      final_results, match_counter, all_matches);
  return cudaGetLastError();
}

cudaError_t launch_take_rows(uint32_t* bitmap, uint32_t stride_words, const uint32_t* rows, uint32_t n_rows,
                             uint32_t db_len, int clear, uint32_t* counts, uint32_t* ids, uint32_t cap,
                             cudaStream_t stream) {
  if (!n_rows) return cudaSuccess;
  take_rows_kernel<<<n_rows, 256, 0, stream>>>(bitmap, stride_words, rows, db_len, clear, counts, ids, cap);
  return cudaGetLastError();
}

}  // namespace irs
