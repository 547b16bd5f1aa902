// Launch interface of the tcgen05 limb GEMM (internal to the library).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"

namespace irs {

// One dot-product problem: a party's DB limb planes against its query limb
// planes, for the entries [m0, m0 + m_len).
struct alignas(64) GemmProblem {
  CUtensorMap tm_a_lo;  // DB low bytes   [rows][K]
  CUtensorMap tm_a_hi;  // DB high bytes  [rows][K]
  CUtensorMap tm_b_lo;  // query low bytes  [n_pad][K]
  CUtensorMap tm_b_hi;  // query high bytes [n_pad][K]
  uint16_t* out;        // [m_len][n_pad]
  uint32_t m0;
  uint32_t m_len;
  uint32_t n_pad;
  uint32_t k_iters;     // K / 128
  uint32_t mult;        // 1 for codes, 2 for trimmed masks
  uint32_t mask_on;     // add ks_own - ks_prev
  ChaChaKey key_own;
  ChaChaKey key_prev;
  uint64_t nonce;
  uint64_t batch;
  const uint64_t* batch_dev;  // when set, the batch id is read from device memory
  uint32_t tiles_m;     // filled by launch_limb_gemm
  uint32_t tiles_n;
};

constexpr int kMaxGemmProblems = 6;
constexpr uint64_t kGemmWaitTimeoutNs = 2000000000ull;  // default limit of a bounded wait: 2 s

struct GemmParams {
  GemmProblem prob[kMaxGemmProblems];
  int n_prob;
  int total_tiles;
  int* err;
  // L2 eviction priority of the TMA loads: bit 0 = query planes evict_last
  // (re-read by every DB tile), bit 1 = DB planes evict_first (streamed).
  uint32_t l2_hint;
  // Limit of the MMA's wait for a TMA stage; the other waits get twice this.
  // 0 = kGemmWaitTimeoutNs.
  uint64_t wait_timeout_ns;
  // Test hook: CTA 0 issues no TMA loads, so its MMA's first stage wait runs
  // out (kErrTimeoutFull) and the kernel returns with the error word set.
  uint32_t test_stall;
  // Serpentine K order: a CTA walks K backwards on its odd tile iterations,
  // so the query K blocks the previous wave of CTAs loaded last are the first
  // this wave needs.  Integer accumulation: the result does not depend on it.
  uint32_t serpentine;
};

// Builds a 2-D u8 tensor map (inner dim K, outer dim rows) with 128x`box_rows`
// boxes and 128-byte swizzle.  Returns 0 on success.
int make_tmap_u8(CUtensorMap* map, const void* base, uint64_t rows, uint64_t k, uint32_t box_rows);

// Tile width along the query rows that divides n_pad (256, 128 or 64; 0 if none).
int gemm_block_n_for(uint32_t n_pad);

// True when launch_limb_gemm runs the two-SM (cta_group::2) kernel: asked for
// (`pair`) and the 256-row tile; its query tensor maps must then use boxes of
// block_n / 2 rows.
bool gemm_pair_applies(bool pair, int block_n);

cudaError_t launch_limb_gemm(GemmParams& P, int block_n, bool pair, int n_sms, cudaStream_t stream);

}  // namespace irs
