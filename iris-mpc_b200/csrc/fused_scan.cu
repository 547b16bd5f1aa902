// Fused scan of one DB chunk: the six limb GEMMs (3 parties x code/mask) and
// the 3-party threshold comparison, open and rotation OR in ONE persistent
// kernel.
//
// Replaces, per DB chunk, the reference's Phase 1 (dot + dot_reduce_and_multiply
// + reshare, iris-mpc-gpu/src/dot/share_db.rs:800-1036), Phase 2
// (compare_threshold_masked_many, threshold_ring/protocol.rs:2519-2546) and the
// open + openResults (server/actor.rs:2376-2519, 2928-2997; dot/kernel.cu:54-116)
// -- the library's other path runs them as one GEMM launch and one threshold
// launch with the dot shares round-tripping through HBM.
//
// One CTA per SM, persistent over work items = (128 DB entries) x (128 query
// rows), each processed for the six engines in turn:
//   warp 0      TMA loads (128-byte swizzle) of the engine's DB and query limb
//               tiles into a 3-stage ring of 64 KB stages;
//   warp 1      tcgen05.mma (u8 x u8 -> s32, three per 32-byte K step) into one
//               of two TMEM accumulator buffers (2 x 256 columns), alternating
//               per engine, so it runs up to two engine tiles ahead of the
//               epilogue;
//   warps 2..9  drain the accumulator (tcgen05.ld), release it, form the
//               masked u16 dot share ((acc0 + (acc1 << 8)) x multiplier +
//               ks_own - ks_prev, ChaCha12) and store it into the CTA's slot of
//               an L2 ring in global memory ([6][128][128] u16, 196 KB per CTA);
//               after the sixth engine the same warps evaluate the threshold
//               circuit on the slot (two (entry, 32-row word) pairs per thread:
//               4 words x 128 entries per tile), open the bits and emit the
//               rotation OR with one ballot per warp, while the MMA warp
//               already computes the next tile's first two engines.
// The dot shares and the circuit keystream sit at the same positions as in
// the two-launch path, so both give bit-identical per-party shares and
// results.  All waits are bounded (the GEMM's limits); the epilogue warps agree
// on a failure at their barrier (bar.red.or), so no warp waits for one that
// gave up.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "circuit.cuh"
#include "common.cuh"
#include "fused_scan.h"
#include "gemm_limb.h"
#include "tc_sm100.cuh"
#include "launch_attr.cuh"
#include "threshold.h"
#include "threshold_emit.cuh"

namespace irs {

namespace {

constexpr int kFBN = kFusedBlockN;
constexpr int kFThreads = 320;
constexpr int kFStageBytes = 2 * kBM * kBK + 2 * kFBN * kBK;  // 64 KB
constexpr int kFStages = 3;
constexpr int kFTmemCols = 512;                                // two buffers x (acc0 | acc1)
constexpr int kFSmem = kFStages * kFStageBytes + 1024 /*align*/ + 256 /*barriers*/;
constexpr int kRingTile = kBM * kFBN;                          // u16 per engine per tile
constexpr int kEpiThreads = 256;

// Named barrier 1 of the eight epilogue warps; returns whether any of them
// passed `fail` (bar.red.or).
__device__ __forceinline__ bool epi_sync_any(bool fail) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)fail), "n"(kEpiThreads)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory"); }

__device__ __forceinline__ void st_ring(void* p, uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.b32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "r"(a), "r"(b), "r"(c),
               "r"(d), "l"(pol)
               : "memory");
}

__global__ void __launch_bounds__(kFThreads, 1) fused_scan_kernel(const __grid_constant__ FusedParams F) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* a_lo = smem;
  uint8_t* a_hi = a_lo + kFStages * kBM * kBK;
  uint8_t* b_lo = a_hi + kFStages * kBM * kBK;
  uint8_t* b_hi = b_lo + kFStages * kFBN * kBK;
  uint64_t* bars = reinterpret_cast<uint64_t*>(b_hi + kFStages * kFBN * kBK);
  uint64_t* full_bar = bars;
  uint64_t* empty_bar = bars + kFStages;
  uint64_t* acc_full = bars + 2 * kFStages;   // [2]
  uint64_t* acc_empty = acc_full + 2;         // [2]
  uint64_t* done_bar = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int* err = F.err;
  const uint64_t lim = F.wait_timeout_ns, lim2 = 2 * F.wait_timeout_ns;
  const int total = F.total_work;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kFStages; s++) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 8);  // one arrive per epilogue warp
    }
    mbar_init(done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)kFTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued_phase[kFStages];
      bool issued[kFStages];
      for (int s = 0; s < kFStages; s++) issued[s] = false;
      bool ok = true;
      for (int w = blockIdx.x; ok && w < total; w += gridDim.x) {
        const int m_tile = w / F.tiles_n, yb = (w % F.tiles_n) * kFBN;
        for (int e = 0; ok && e < kFusedEngines; e++) {
          const GemmProblem& pr = F.prob[e];
          const int ya0 = (int)pr.m0 + m_tile * kBM;
          for (uint32_t ki = 0; ki < pr.k_iters; ki++) {
            if (!mbar_wait(&empty_bar[stage], phase ^ 1u, err, kErrTimeoutEmpty, lim2)) { ok = false; break; }
            mbar_expect_tx(&full_bar[stage], (uint32_t)kFStageBytes);
            const int x = (int)ki * kBK;
            tma_load_2d(a_lo + stage * kBM * kBK, &pr.tm_a_lo, &full_bar[stage], x, ya0);
            tma_load_2d(a_hi + stage * kBM * kBK, &pr.tm_a_hi, &full_bar[stage], x, ya0);
            tma_load_2d(b_lo + stage * kFBN * kBK, &pr.tm_b_lo, &full_bar[stage], x, yb);
            tma_load_2d(b_hi + stage * kFBN * kBK, &pr.tm_b_hi, &full_bar[stage], x, yb);
            issued[stage] = true;
            issued_phase[stage] = (int)phase;
            if (++stage == kFStages) { stage = 0; phase ^= 1u; }
          }
        }
      }
      // Exit: no copy into this CTA's shared memory may still be in flight.
      for (int s = 0; s < kFStages; s++)
        if (issued[s]) mbar_wait_drain(&full_bar[s], (uint32_t)issued_phase[s], err, lim2);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t use_phase[2] = {0u, 0u};
      int buf = 0;
      bool ok = true;
      constexpr uint32_t idesc = idesc_u8(kFBN);
      for (int w = blockIdx.x; ok && w < total; w += gridDim.x) {
        for (int e = 0; ok && e < kFusedEngines; e++) {
          const GemmProblem& pr = F.prob[e];
          if (!mbar_wait(&acc_empty[buf], use_phase[buf] ^ 1u, err, kErrTimeoutAccEmpty, lim2)) { ok = false; break; }
          use_phase[buf] ^= 1u;
          tc_fence_after();
          const uint32_t d = tmem + (uint32_t)(buf * 2 * kFBN);
          for (uint32_t ki = 0; ki < pr.k_iters; ki++) {
            if (!mbar_wait(&full_bar[stage], phase, err, kErrTimeoutFull, lim)) { ok = false; break; }
            tc_fence_after();
            const uint64_t dal = smem_desc(a_lo + stage * kBM * kBK);
            const uint64_t dah = smem_desc(a_hi + stage * kBM * kBK);
            const uint64_t dbl = smem_desc(b_lo + stage * kFBN * kBK);
            const uint64_t dbh = smem_desc(b_hi + stage * kFBN * kBK);
#pragma unroll
            for (int kk = 0; kk < kBK / 32; kk++) {
              const uint32_t acc = (ki > 0 || kk > 0) ? 1u : 0u;
              const uint64_t o = (uint64_t)(2 * kk);  // 32 bytes along K, in 16-byte units
              mma_u8(d, dal + o, dbl + o, idesc, acc);
              mma_u8(d + kFBN, dal + o, dbh + o, idesc, acc);
              mma_u8(d + kFBN, dah + o, dbl + o, idesc, 1u);
            }
            mma_commit(&empty_bar[stage]);
            if (++stage == kFStages) { stage = 0; phase ^= 1u; }
          }
          if (ok) mma_commit(&acc_full[buf]);
          buf ^= 1;
        }
      }
      // Exit: wait until every MMA issued by this thread has completed.
      mma_commit(done_bar);
      mbar_wait_drain(done_bar, 0, err, lim2);
    }
  } else {
    // ---------------- Epilogue + threshold (warps 2..9) ----------------
    const int quad = warp & 3;         // TMEM lanes 32*quad .. 32*quad+31
    const int half = (warp - 2) >> 2;  // column half (64 rows) of the tile
    const int row = quad * 32 + lane;  // entry within the tile
    const int ep_warp = warp - 2;      // 0..7
    constexpr int kCols = kFBN / 2;    // query rows per thread
    uint16_t* ring = F.ring + (size_t)blockIdx.x * kFusedEngines * kRingTile;
    const uint64_t pol = policy_evict_last();
    const ThresholdParams& T = F.T;
    uint32_t use_phase[2] = {0u, 0u};
    int buf = 0;
    bool failed = false;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
      const int m_tile = w / F.tiles_n, n_tile = w % F.tiles_n;
      for (int e = 0; e < kFusedEngines; e++) {
        if (failed) break;
        const GemmProblem& pr = F.prob[e];
        if (!mbar_wait(&acc_full[buf], use_phase[buf], err, kErrTimeoutAccFull, lim2)) {
          failed = true;
          break;
        }
        use_phase[buf] ^= 1u;
        tc_fence_after();
        uint32_t packed[kCols / 2];
        const uint32_t tbase = tmem + (uint32_t)(buf * 2 * kFBN) + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * kCols);
#pragma unroll
        for (int c = 0; c < kCols / 32; c++) {
          uint32_t r0[32], r1[32];
          tmem_ld32(tbase + (uint32_t)(c * 32), r0);
          tmem_ld32(tbase + (uint32_t)(kFBN + c * 32), r1);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const uint32_t lo = (r0[2 * j] + (r1[2 * j] << 8)) & 0xFFFFu;
            const uint32_t hi = (r0[2 * j + 1] + (r1[2 * j + 1] << 8)) << 16;
            packed[c * 16 + j] = lo | hi;
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[buf]);
        buf ^= 1;

        const uint32_t m_local = (uint32_t)(m_tile * kBM + row);
        if (m_local < pr.m_len) {
          const uint64_t m_global = (uint64_t)pr.m0 + m_local;
          uint16_t* dst = ring + (size_t)e * kRingTile + (size_t)row * kFBN;
#pragma unroll
          for (int c = 0; c < kCols / 32; c++) {
            const uint32_t nl = (uint32_t)(half * kCols + c * 32);
            const uint32_t n = (uint32_t)(n_tile * kFBN) + nl;
            uint32_t v[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
              const uint32_t x = packed[c * 16 + j];
              v[j] = (pr.mult == 1) ? x : (((x & 0xFFFFu) * pr.mult) & 0xFFFFu) | (((x >> 16) * pr.mult) << 16);
            }
            if (pr.mask_on) {
              const uint64_t blk = (m_global * pr.n_pad + n) >> 5;
              const uint64_t batch = pr.batch_dev ? *pr.batch_dev : pr.batch;
              uint32_t ks[32];
              chacha12_pair(&pr.key_own, &pr.key_prev, counter_of(batch, blk), pr.nonce, ks);
#pragma unroll
              for (int j = 0; j < 16; j++) v[j] = sub2(add2(v[j], ks[j]), ks[16 + j]);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) st_ring(dst + nl + 8 * q, v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3], pol);
          }
        }
      }
      // The six engines' shares of this tile are in the ring (or some warp
      // gave up, in which case all leave together).
      if (epi_sync_any(failed)) break;
      // Threshold, open and rotation OR of the tile: warp item k = (32-row
      // word k / 4, 32-entry group k % 4), two per warp.
#pragma unroll 1
      for (int r = 0; r < 2; r++) {
        const int k = ep_warp + 8 * r;
        const int word = k >> 2, group = k & 3;
        const uint32_t slot = (uint32_t)(n_tile * (kFBN / 32) + word);
        if (slot >= T.n_slots) continue;  // warp-uniform: padded rows beyond the evaluated slots
        const int entry = group * 32 + lane;
        const uint32_t m_local = (uint32_t)(m_tile * kBM + entry);
        const bool valid = m_local < T.n_entries;
        const int e_read = valid ? entry : 0;  // entry 0 of a tile is always valid
        WordRand wr;
#pragma unroll
        for (int s = 0; s < 3; s++) wr.key[s] = T.key[s];
        wr.nonce = T.nonce;
        // the word's keystream position, as in threshold_bitmap_kernel
        const uint64_t word_id = ((uint64_t)T.m0 + (uint64_t)(m_tile * kBM + e_read)) * (uint64_t)(T.n_pad / 32) + slot;
        wr.base = counter_of(T.batch_dev ? *T.batch_dev : T.batch, word_id * (uint64_t)kCircuitBlocksPerWord);
        const size_t off = (size_t)e_read * kFBN + (size_t)word * 32;
        uint32_t opened;
        {
          const uint16_t* code[3] = {ring + off, ring + kRingTile + off, ring + 2 * kRingTile + off};
          const uint16_t* mask[3] = {ring + 3 * kRingTile + off, ring + 4 * kRingTile + off,
                                     ring + 5 * kRingTile + off};
          Comp msb;
          opened = threshold_word<kStageFull, true>(code, mask, T.threshold_a, wr, msb);
        }
        const uint64_t m_global = (uint64_t)T.m0 + m_local;
        const size_t bitmap_word = (size_t)((T.m0 + (uint32_t)(m_tile * kBM + group * 32)) / 32);
        emit_word(T, opened, valid, (uint32_t)lane, slot, m_global, bitmap_word, [&](int p, int is_mask, int rr) {
          return ring[(size_t)(is_mask ? 3 + p : p) * kRingTile + off + rr];
        });
      }
      epi_sync();  // the next tile's epilogue overwrites the ring slot
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kFTmemCols));
  }
}

}  // namespace

int fused_scan_grid(const FusedParams& F, int n_sms) { return F.total_work < n_sms ? F.total_work : n_sms; }

cudaError_t launch_fused_scan(FusedParams& F, int n_sms, cudaStream_t stream) {
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = smem_limit_once(fused_scan_kernel, kFSmem, attr_done);
  if (e != cudaSuccess) return e;
  if (F.wait_timeout_ns == 0) F.wait_timeout_ns = kGemmWaitTimeoutNs;
  const int grid = fused_scan_grid(F, n_sms);
  if (grid <= 0) return cudaSuccess;
  fused_scan_kernel<<<grid, kFThreads, kFSmem, stream>>>(F);
  return cudaGetLastError();
}

}  // namespace irs
