// Launch interface of the fused threshold kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"

namespace irs {

struct ThresholdParams {
  const uint16_t* code[3];  // party p's own additive component of the code dots
  const uint16_t* mask[3];  // ... of the (x2) mask dots
  ChaChaKey key[3];         // stream p = party p's own seed
  uint64_t nonce;
  uint64_t batch;
  const uint64_t* batch_dev;  // when set, the batch id is read from device memory
  uint32_t threshold_a;
  // flat mode
  uint64_t n_words;
  uint64_t word_base;
  uint32_t* revealed;   // [n_words], optional
  uint32_t* res_comp;   // [3][n_words], optional: component p of the result
  // bitmap mode
  uint32_t n_entries;   // entries in this call
  uint32_t m0;          // global index of the first entry (multiple of 32)
  uint32_t n_pad;       // dot-share row stride in elements (multiple of 32)
  uint32_t n_slots;     // 32-row query slots evaluated
  const uint32_t* slot_valid;  // [n_slots] valid-row mask, NULL = rows 0..30
  const uint32_t* slot_query;  // [n_slots] query index owning the slot, NULL = identity
  // Optional segment table (several queries per 32-row slot): segments
  // seg_start[s] .. seg_start[s+1]-1 of slot s report rows seg_mask[k] to
  // query seg_query[k].  Overrides slot_valid / slot_query when set.
  const uint32_t* seg_start;
  const uint32_t* seg_query;
  const uint32_t* seg_mask;
  uint32_t* bitmap;     // [queries][bitmap_stride/32], optional
  uint32_t bitmap_stride;      // bits per bitmap row (multiple of 32)
  uint32_t* match_count;
  uint32_t* match_list; // pairs (query, entry), optional
  uint32_t match_cap;
  // Optional distance capture (anonymised statistics): every opened match of
  // a valid row appends (entry, row, the three parties' code and mask dot
  // components) at position atomicAdd(dist_count, 1) when below dist_cap.
  uint32_t* dist_count;
  uint32_t* dist_entry;  // [dist_cap] global DB entry
  uint32_t* dist_row;    // [dist_cap] query row (32 * slot + row of the slot)
  uint16_t* dist_code;   // [3][dist_cap]
  uint16_t* dist_mask;   // [3][dist_cap]
  uint32_t dist_cap;
  // (query, entry) pairs recorded for every valid row whether or not they
  // match (the reference's anon_stats_idx: reauth targets), n_forced <= 256
  const uint32_t* forced_query;
  const uint32_t* forced_entry;
  uint32_t n_forced;
};

cudaError_t launch_threshold_flat(const ThresholdParams& P, int stage, cudaStream_t stream);
cudaError_t launch_threshold_bitmap(const ThresholdParams& P, cudaStream_t stream);
cudaError_t launch_lift_flat(const ThresholdParams& P, uint16_t* corr, cudaStream_t stream);

}  // namespace irs
