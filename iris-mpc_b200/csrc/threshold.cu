// Fused 3-party threshold comparison, open and rotation OR.
//
// One thread evaluates the whole Phase-2 protocol for one 32-element word of
// all three co-resident parties (circuit.cuh): the lift of the mask dot
// shares from Z_2^16 to Z_2^32, the bit injection of the two lift carries,
// mask*A - code*2^16 - 1, the 32-bit MSB adder, and the opening of the result.
// The per-gate "send to next party" of the reference (NCCL send/recv around
// every AND round, iris-mpc-gpu/src/threshold_ring/protocol.rs:894-1032) is the
// component store inside the thread, so the ~52 dependent rounds and ~7
// launches per round collapse into straight-line code, and HBM sees each input
// share exactly once.
//
// Modes:
//   flat   -- elements e = 0..n-1, word w = e/32 (Circuits API: results are
//             the per-party shares of the msb bit plus the opened bits);
//   bitmap -- dot shares laid out [entry][n_pad], each query iris owning a
//             32-row slot; a warp covers 32 consecutive entries of one slot,
//             the opened word OR-ed over the slot's valid rows is the match bit
//             (the rotation OR of openResults, dot/kernel.cu:54-116), written
//             with one ballot per warp, and matches are appended to a list.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include "circuit.cuh"
#include "threshold.h"
#include "threshold_emit.cuh"
#include "launch_attr.cuh"

namespace irs {

namespace {

constexpr int kThreshThreads = 128;
// Shared memory per thread of the keystream (WordRandShared): 18 prepared
// words-of-four and 48 keystream words.
constexpr int kRandSmemPerThread = 18 * 16 + 48 * 4;

template <class WR>
__device__ __forceinline__ void init_rand(WR& wr, const ThresholdParams& P, uint64_t word_id) {
#pragma unroll
  for (int s = 0; s < 3; s++) wr.key[s] = P.key[s];
  wr.nonce = P.nonce;
  wr.base = counter_of(P.batch_dev ? *P.batch_dev : P.batch, word_id * (uint64_t)kCircuitBlocksPerWord);
}

// This thread's keystream columns in the block's shared memory ([element][thread]).
template <int THREADS>
__device__ __forceinline__ void bind_rand(WordRandShared& wr) {
  extern __shared__ uint4 rand_smem[];
  wr.pre = rand_smem + threadIdx.x;
  wr.ks = reinterpret_cast<uint32_t*>(rand_smem + 18 * THREADS) + threadIdx.x;
  wr.nt = THREADS;
}

template <int STAGE>
__global__ void __launch_bounds__(kThreshThreads) threshold_flat_kernel(const ThresholdParams P) {
  const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.n_words) return;
  WordRandShared wr;
  bind_rand<kThreshThreads>(wr);
  init_rand(wr, P, P.word_base + w);
  const uint16_t* code[3] = {P.code[0] + 32 * w, P.code[1] + 32 * w, P.code[2] + 32 * w};
  const uint16_t* mask[3] = {P.mask[0] + 32 * w, P.mask[1] + 32 * w, P.mask[2] + 32 * w};
  Comp msb;
  const uint32_t r = threshold_word<STAGE>(code, mask, P.threshold_a, wr, msb);
  if (P.revealed) P.revealed[w] = r;
  if (P.res_comp) {
    P.res_comp[w] = msb.c0;
    P.res_comp[P.n_words + w] = msb.c1;
    P.res_comp[2 * P.n_words + w] = msb.c2;
  }
}

// The bitmap kernel indexes by global warp only, so its block size is free:
// THREADS x MIN_BLOCKS sets the resident warps per SM the registers are sized for.
template <int THREADS, int MIN_BLOCKS>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) threshold_bitmap_kernel(const ThresholdParams P) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t gwarp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t n_groups = (P.n_entries + 31) / 32;
  const uint64_t total = (uint64_t)n_groups * P.n_slots;
  if (gwarp >= total) return;  // warp-uniform
  const uint32_t slot = (uint32_t)(gwarp % P.n_slots);
  const uint32_t group = (uint32_t)(gwarp / P.n_slots);
  const uint32_t m_local = group * 32 + lane;
  const bool valid = m_local < P.n_entries;
  const uint32_t m_read = valid ? m_local : (P.n_entries - 1);
  const uint64_t m_global = (uint64_t)P.m0 + m_local;

  WordRandShared wr;
  bind_rand<THREADS>(wr);
  init_rand(wr, P, ((uint64_t)P.m0 + m_read) * (uint64_t)(P.n_pad / 32) + slot);
  const size_t off = (size_t)m_read * P.n_pad + (size_t)slot * 32;
  uint32_t opened;
  {
    // The share pointers die here; the rare distance capture below rebuilds
    // them from `off`, which keeps 12 registers free through the circuit.
    const uint16_t* code[3] = {P.code[0] + off, P.code[1] + off, P.code[2] + off};
    const uint16_t* mask[3] = {P.mask[0] + off, P.mask[1] + off, P.mask[2] + off};
    Comp msb;
    opened = threshold_word<kStageFull>(code, mask, P.threshold_a, wr, msb);
  }
  const size_t bitmap_word = (size_t)((P.m0 + group * 32) / 32);
  // The capture rebuilds the share pointers from `off` (rare).
  emit_word(P, opened, valid, lane, slot, m_global, bitmap_word,
            [&](int p, int is_mask, int r) { return (is_mask ? P.mask[p] : P.code[p])[off + r]; });
}

__global__ void __launch_bounds__(kThreshThreads) lift_flat_kernel(const ThresholdParams P, uint16_t* corr) {
  const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.n_words) return;
  WordRand wr;
  init_rand(wr, P, P.word_base + w);
  const uint16_t* mask[3] = {P.mask[0] + 32 * w, P.mask[1] + 32 * w, P.mask[2] + 32 * w};
  uint16_t c1[3][32], c2[3][32];
  lift_word(mask, wr, c1, c2);
  const uint64_t n = P.n_words * 32;
#pragma unroll
  for (int p = 0; p < 3; p++) {
    uint16_t* o1 = corr + (size_t)(2 * p) * n + 32 * w;
    uint16_t* o2 = corr + (size_t)(2 * p + 1) * n + 32 * w;
#pragma unroll
    for (int j = 0; j < 32; j++) { o1[j] = c1[p][j]; o2[j] = c2[p][j]; }
  }
}

}  // namespace

constexpr int kRandSmem = kThreshThreads * kRandSmemPerThread;  // 61,440 bytes per block

template <class K>
static cudaError_t allow_rand_smem(K kernel, std::atomic<uint64_t>& done) {
  return smem_limit_once(kernel, kRandSmem, done);
}

cudaError_t launch_threshold_flat(const ThresholdParams& P, int stage, cudaStream_t stream) {
  if (P.n_words == 0) return cudaSuccess;
  static std::atomic<uint64_t> done_full{0}, done_msb{0};
  cudaError_t attr = allow_rand_smem(threshold_flat_kernel<kStageFull>, done_full);
  if (attr == cudaSuccess) attr = allow_rand_smem(threshold_flat_kernel<kStageMsbOnly>, done_msb);
  if (attr != cudaSuccess) return attr;
  const unsigned grid = (unsigned)((P.n_words + kThreshThreads - 1) / kThreshThreads);
  if (stage == kStageFull) threshold_flat_kernel<kStageFull><<<grid, kThreshThreads, kRandSmem, stream>>>(P);
  else threshold_flat_kernel<kStageMsbOnly><<<grid, kThreshThreads, kRandSmem, stream>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_threshold_bitmap(const ThresholdParams& P, cudaStream_t stream) {
  if (P.n_entries == 0 || P.n_slots == 0) return cudaSuccess;
  const uint64_t warps = (uint64_t)((P.n_entries + 31) / 32) * P.n_slots;
  // Resident warps per SM the kernel's registers are sized for: 12 (3 per
  // SM sub-partition, 168-register cap) measured 2-6% faster than 8 on
  // 512K-entry batches.  Other
  // counts give the same register cap as one of these two, since each
  // sub-partition holds a quarter of the register file.
  // IRS_THRESHOLD_WARPS_PER_SM=8 selects the other variant for tuning runs.
  static const bool eight = [] {
    const char* e = getenv("IRS_THRESHOLD_WARPS_PER_SM");
    return e && atoi(e) == 8;
  }();
  static std::atomic<uint64_t> done_8{0}, done_12{0};
  cudaError_t attr = eight ? allow_rand_smem(threshold_bitmap_kernel<kThreshThreads, 2>, done_8)
                           : allow_rand_smem(threshold_bitmap_kernel<kThreshThreads, 3>, done_12);
  if (attr != cudaSuccess) return attr;
  const unsigned grid = (unsigned)((warps * 32 + kThreshThreads - 1) / kThreshThreads);
  if (eight) threshold_bitmap_kernel<kThreshThreads, 2><<<grid, kThreshThreads, kRandSmem, stream>>>(P);
  else threshold_bitmap_kernel<kThreshThreads, 3><<<grid, kThreshThreads, kRandSmem, stream>>>(P);
  return cudaGetLastError();
}

cudaError_t launch_lift_flat(const ThresholdParams& P, uint16_t* corr, cudaStream_t stream) {
  if (P.n_words == 0) return cudaSuccess;
  const unsigned grid = (unsigned)((P.n_words + kThreshThreads - 1) / kThreshThreads);
  lift_flat_kernel<<<grid, kThreshThreads, 0, stream>>>(P, corr);
  return cudaGetLastError();
}

}  // namespace irs
