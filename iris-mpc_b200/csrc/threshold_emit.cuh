// Result emission of the bitmap-mode threshold (internal to the library):
// the rotation OR of a 32-row word's opened bits per query, one ballot per
// warp into the match bitmap (openResults, iris-mpc-gpu/src/dot/kernel.cu:
// 54-116), the (query, entry) match list, and the anonymised-statistics
// distance capture (kernel.cu:73-106).  Shared by the standalone threshold
// kernel (threshold.cu) and the fused GEMM + threshold scan (fused_scan.cu),
// so both write identical results.
#pragma once
#include <stdint.h>
#include "threshold.h"

namespace irs {

// One warp, lane = entry m_global (valid lanes only count), one 32-row slot.
// `opened` = the lane's opened comparison bits of the slot's 32 rows.
// share(p, is_mask, r) returns party p's code (is_mask = 0) or mask dot share
// of row r of this (entry, slot) word; it is only called for the distance
// capture, which is rare.
template <typename Share>
__device__ __forceinline__ void emit_word(const ThresholdParams& P, uint32_t opened, bool valid, uint32_t lane,
                                          uint32_t slot, uint64_t m_global, size_t bitmap_word, Share share) {
  // Rotation OR of one query's rows, one ballot for the warp's 32 entries.
  auto emit = [&](uint32_t query, uint32_t row_mask, bool shared_word) {
    const bool match = valid && (opened & row_mask) != 0;
    const uint32_t bits = __ballot_sync(0xFFFFFFFFu, match);
    if (P.bitmap && lane == 0) {
      uint32_t* w = P.bitmap + (size_t)query * (P.bitmap_stride / 32) + bitmap_word;
      if (shared_word) {
        if (bits) atomicOr(w, bits);
      } else {
        *w = bits;
      }
    }
    if (P.match_list && bits) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(P.match_count, (uint32_t)__popc(bits));
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (match) {
        const uint32_t pos = base + (uint32_t)__popc(bits & ((1u << lane) - 1u));
        if (pos < P.match_cap) {
          P.match_list[2 * pos] = query;
          P.match_list[2 * pos + 1] = (uint32_t)m_global;
        }
      }
    }
  };
  uint32_t rows = 0;  // valid rows of the slot (for the distance capture)
  if (P.seg_start) {
    const uint32_t s0 = P.seg_start[slot], s1 = P.seg_start[slot + 1];
    for (uint32_t k = s0; k < s1; k++) {
      emit(P.seg_query[k], P.seg_mask[k], true);
      rows |= P.seg_mask[k];
    }
  } else {
    rows = P.slot_valid ? P.slot_valid[slot] : 0x7FFFFFFFu;
    emit(P.slot_query ? P.slot_query[slot] : slot, rows, false);
  }
  // Distance capture of the per-rotation matches: rare, so one atomic per record.
  if (P.dist_count && valid) {
    uint32_t hits = opened & rows;
    // forced pairs: every valid row of a listed (query, entry) is recorded
    for (uint32_t j = 0; j < P.n_forced; j++) {
      if (P.forced_entry[j] != (uint32_t)m_global) continue;
      if (P.seg_start) {
        for (uint32_t k = P.seg_start[slot]; k < P.seg_start[slot + 1]; k++)
          if (P.seg_query[k] == P.forced_query[j]) hits |= P.seg_mask[k];
      } else if ((P.slot_query ? P.slot_query[slot] : slot) == P.forced_query[j]) {
        hits |= rows;
      }
    }
    while (hits) {
      const int r = __ffs(hits) - 1;
      hits &= hits - 1;
      const uint32_t pos = atomicAdd(P.dist_count, 1u);
      if (pos < P.dist_cap) {
        P.dist_entry[pos] = (uint32_t)m_global;
        P.dist_row[pos] = slot * 32 + (uint32_t)r;
#pragma unroll
        for (int p = 0; p < 3; p++) {
          P.dist_code[(size_t)p * P.dist_cap + pos] = share(p, 0, r);
          P.dist_mask[(size_t)p * P.dist_cap + pos] = share(p, 1, r);
        }
      }
    }
  }
}

}  // namespace irs
