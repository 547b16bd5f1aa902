// Launch interface of the fused GEMM + threshold scan (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "gemm_limb.h"
#include "threshold.h"

namespace irs {

constexpr int kFusedEngines = 6;       // code p0..p2 (K = 12800), mask p0..p2 (K = 6400)
constexpr int kFusedBlockN = 128;      // query rows per tile
// Dot shares of one CTA's current tile, all six engines: [6][128 entries][128 rows] u16.
constexpr size_t kFusedRingBytesPerCta = (size_t)kFusedEngines * 128 * kFusedBlockN * 2;

struct FusedParams {
  GemmProblem prob[kFusedEngines];  // same m0, m_len, n_pad; query maps with 128-row boxes
  ThresholdParams T;                // bitmap mode: keys, batch, slots or segments, outputs
  uint16_t* ring;                   // [grid][6][128][128] u16 scratch
  int tiles_m, tiles_n;             // 128-entry x 128-row tiles of the chunk
  int total_work;                   // tiles_m * tiles_n
  int* err;
  uint64_t wait_timeout_ns;         // 0 = kGemmWaitTimeoutNs
};

// Grid size of a launch (one CTA per SM, at most one per work item); the ring
// must hold kFusedRingBytesPerCta for each of its CTAs.
int fused_scan_grid(const FusedParams& F, int n_sms);
cudaError_t launch_fused_scan(FusedParams& F, int n_sms, cudaStream_t stream);

}  // namespace irs
