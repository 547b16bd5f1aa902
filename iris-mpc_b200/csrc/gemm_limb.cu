// Exact mod-2^16 dot products of u16 share matrices on tcgen05 INT8 tensor cores.
//
// Replaces the reference's three cublasGemmEx int8 limb GEMMs plus the
// matmul_correct_and_reduce kernel (iris-mpc-gpu/src/dot/share_db.rs:62-112,
// 800-905; iris-mpc-gpu/src/dot/kernel.cu:16-28).  Each u16 is split into two
// unsigned bytes (lo, hi); since
//     d*q mod 2^16 = dlo*qlo + 2^8 * (dlo*qhi + dhi*qlo)   (mod 2^16)
// one pass over K issues three u8 x u8 -> s32 MMAs per K step into two TMEM
// accumulators: acc0 += Dlo.Qlo and acc1 += Dlo.Qhi + Dhi.Qlo.  The epilogue
// forms (acc0 + (acc1 << 8)) mod 2^16, multiplies by the engine multiplier
// (2 for trimmed masks), adds the zero-share mask ks_own - ks_prev computed in
// registers with ChaCha12, and stores u16 dot shares.  Unsigned limbs need no
// sum correction (the reference's signed limbs do).
//
// Layouts: DB limb planes [entries][K] u8, query limb planes [rows][K] u8
// (both K-major, K a multiple of 128), output [entries][n_pad] u16 with the
// query row fastest.  Keystream u16 of element (entry m, row n) sits at index
// m * n_pad + n of the engine's stream (32 u16 per ChaCha block).
//
// Kernel structure (one CTA per SM, persistent over tiles of 128 entries x BN
// rows): warp 0 issues TMA loads (128B swizzle) into a STAGES-deep ring,
// warp 1 allocates TMEM and issues the MMAs from one thread, warps 2..9 drain
// the accumulators (tcgen05.ld), release TMEM to the next tile and then run
// the ChaCha mask and the stores while the next tile's MMAs proceed.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include "common.cuh"
#include "gemm_limb.h"
#include "tc_sm100.cuh"
#include "launch_attr.cuh"

namespace irs {

namespace {

constexpr int kThreads = 320;

template <int BN>
struct Cfg {
  static constexpr int kStageBytes = 2 * kBM * kBK + 2 * BN * kBK;
  static constexpr int kStages = (196608 / kStageBytes) > 6 ? 6 : (196608 / kStageBytes);
  static constexpr int kTmemCols = 2 * BN;  // acc0 | acc1
  static constexpr int kColsPerThread = BN / 2;  // two epilogue warps per TMEM lane quadrant
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;
};

struct Tile {
  int prob, m_tile, n_tile;
};

__device__ __forceinline__ bool tile_of(const GemmParams& P, int t, Tile& out) {
  for (int i = 0; i < P.n_prob; i++) {
    const int nt = (int)(P.prob[i].tiles_m * P.prob[i].tiles_n);
    if (t < nt) {
      out.prob = i;
      out.m_tile = t / (int)P.prob[i].tiles_n;
      out.n_tile = t % (int)P.prob[i].tiles_n;
      return true;
    }
    t -= nt;
  }
  return false;
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1) limb_gemm_kernel(const __grid_constant__ GemmParams P) {
  using C = Cfg<BN>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* a_lo = smem;
  uint8_t* a_hi = a_lo + C::kStages * kBM * kBK;
  uint8_t* b_lo = a_hi + C::kStages * kBM * kBK;
  uint8_t* b_hi = b_lo + C::kStages * BN * kBK;
  uint64_t* bars = reinterpret_cast<uint64_t*>(b_hi + C::kStages * BN * kBK);
  uint64_t* full_bar = bars;
  uint64_t* empty_bar = bars + C::kStages;
  uint64_t* acc_full = bars + 2 * C::kStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* done_bar = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 3);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int* err = P.err;
  // The MMA's wait for a TMA stage has the launch's limit; every other wait
  // (which in a failing launch only follows that one) twice as long, so the
  // first expiry names the stage that never arrived.
  const uint64_t lim = P.wait_timeout_ns, lim2 = 2 * P.wait_timeout_ns;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; s++) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 8);  // one arrive per epilogue warp
    mbar_init(done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)C::kTmemCols));
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
      int issued_phase[8];
      bool issued[8];
      for (int s = 0; s < C::kStages; s++) issued[s] = false;
      bool ok = true;
      const bool hinted = P.l2_hint != 0;
      const uint64_t pol_a = (P.l2_hint & 2u) ? policy_evict_first() : policy_evict_normal();
      const uint64_t pol_b = (P.l2_hint & 1u) ? policy_evict_last() : policy_evict_normal();
      // Test hook (GemmParams::test_stall): CTA 0 issues no loads at all, so
      // its MMA's first stage wait runs out.  Nothing is in flight to drain.
      if (P.test_stall && blockIdx.x == 0) ok = false;
      int it = 0;
      for (int t = blockIdx.x; ok && t < P.total_tiles; t += gridDim.x, it++) {
        Tile tl;
        if (!tile_of(P, t, tl)) break;
        const GemmProblem& pr = P.prob[tl.prob];
        const int ya = (int)pr.m0 + tl.m_tile * kBM;
        const int yb = tl.n_tile * BN;
        const bool rev = P.serpentine && (it & 1);
        for (uint32_t ki = 0; ki < pr.k_iters; ki++) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1u, err, kErrTimeoutEmpty, lim2)) { ok = false; break; }
          mbar_expect_tx(&full_bar[stage], (uint32_t)C::kStageBytes);
          const int x = (int)(rev ? pr.k_iters - 1 - ki : ki) * kBK;
          if (hinted) {
            tma_load_2d_hint(a_lo + stage * kBM * kBK, &pr.tm_a_lo, &full_bar[stage], x, ya, pol_a);
            tma_load_2d_hint(a_hi + stage * kBM * kBK, &pr.tm_a_hi, &full_bar[stage], x, ya, pol_a);
            tma_load_2d_hint(b_lo + stage * BN * kBK, &pr.tm_b_lo, &full_bar[stage], x, yb, pol_b);
            tma_load_2d_hint(b_hi + stage * BN * kBK, &pr.tm_b_hi, &full_bar[stage], x, yb, pol_b);
          } else {
            tma_load_2d(a_lo + stage * kBM * kBK, &pr.tm_a_lo, &full_bar[stage], x, ya);
            tma_load_2d(a_hi + stage * kBM * kBK, &pr.tm_a_hi, &full_bar[stage], x, ya);
            tma_load_2d(b_lo + stage * BN * kBK, &pr.tm_b_lo, &full_bar[stage], x, yb);
            tma_load_2d(b_hi + stage * BN * kBK, &pr.tm_b_hi, &full_bar[stage], x, yb);
          }
          issued[stage] = true;
          issued_phase[stage] = (int)phase;
          if (++stage == C::kStages) { stage = 0; phase ^= 1u; }
        }
      }
      // Exit: make sure no copy into this CTA's shared memory is still in flight.
      for (int s = 0; s < C::kStages; s++)
        if (issued[s]) mbar_wait_drain(&full_bar[s], (uint32_t)issued_phase[s], err, lim2);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      constexpr uint32_t idesc = idesc_u8(BN);
      for (int t = blockIdx.x; ok && t < P.total_tiles; t += gridDim.x) {
        Tile tl;
        if (!tile_of(P, t, tl)) break;
        const GemmProblem& pr = P.prob[tl.prob];
        if (!mbar_wait(acc_empty, acc_phase ^ 1u, err, kErrTimeoutAccEmpty, lim2)) { ok = false; break; }
        acc_phase ^= 1u;
        tc_fence_after();
        for (uint32_t ki = 0; ki < pr.k_iters; ki++) {
          if (!mbar_wait(&full_bar[stage], phase, err, kErrTimeoutFull, lim)) { ok = false; break; }
          tc_fence_after();
          const uint64_t dal = smem_desc(a_lo + stage * kBM * kBK);
          const uint64_t dah = smem_desc(a_hi + stage * kBM * kBK);
          const uint64_t dbl = smem_desc(b_lo + stage * BN * kBK);
          const uint64_t dbh = smem_desc(b_hi + stage * BN * kBK);
#pragma unroll
          for (int kk = 0; kk < kBK / 32; kk++) {
            const uint32_t acc = (ki > 0 || kk > 0) ? 1u : 0u;
            const uint64_t o = (uint64_t)(2 * kk);  // 32 bytes along K, in 16-byte units
            mma_u8(tmem, dal + o, dbl + o, idesc, acc);
            mma_u8(tmem + BN, dal + o, dbh + o, idesc, acc);
            mma_u8(tmem + BN, dah + o, dbl + o, idesc, 1u);
          }
          mma_commit(&empty_bar[stage]);
          if (++stage == C::kStages) { stage = 0; phase ^= 1u; }
        }
        if (ok) mma_commit(acc_full);
      }
      // Exit: wait until every MMA issued by this thread has completed.
      mma_commit(done_bar);
      mbar_wait_drain(done_bar, 0, err, lim2);
    }
  } else {
    // ---------------- Epilogue (warps 2..9) ----------------
    const int quad = warp & 3;                 // TMEM lanes 32*quad .. 32*quad+31
    const int half = (warp - 2) >> 2;          // column half of the tile
    const int row = quad * 32 + lane;          // entry within the tile
    constexpr int kCols = C::kColsPerThread;
    uint32_t acc_phase = 0;
    for (int t = blockIdx.x; t < P.total_tiles; t += gridDim.x) {
      Tile tl;
      if (!tile_of(P, t, tl)) break;
      const GemmProblem& pr = P.prob[tl.prob];
      if (!mbar_wait(acc_full, acc_phase, err, kErrTimeoutAccFull, lim2)) break;
      acc_phase ^= 1u;
      tc_fence_after();
      uint32_t packed[kCols / 2];
      const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * kCols);
#pragma unroll
      for (int c = 0; c < kCols / 32; c++) {
        uint32_t r0[32], r1[32];
        tmem_ld32(tbase + (uint32_t)(c * 32), r0);
        tmem_ld32(tbase + (uint32_t)(BN + c * 32), r1);
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
      if (lane == 0) mbar_arrive(acc_empty);

      const uint32_t m_local = (uint32_t)(tl.m_tile * kBM + row);
      if (m_local < pr.m_len) {
        const uint64_t m_global = (uint64_t)pr.m0 + m_local;
        uint16_t* out_row = pr.out + (size_t)m_local * pr.n_pad;
#pragma unroll
        for (int c = 0; c < kCols / 32; c++) {
          const uint32_t n = (uint32_t)(tl.n_tile * BN + half * kCols + c * 32);
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
          uint4* dst = reinterpret_cast<uint4*>(out_row + n);
#pragma unroll
          for (int q = 0; q < 4; q++) dst[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)C::kTmemCols));
  }
}

// ---------------------------------------------------------------------------
// Two-SM variant: a cluster of two CTAs computes a 256-entry x 256-row tile
// with tcgen05.mma.cta_group::2 (M = 256).  Each CTA loads its own 128 entries
// (A) and half of the 256 query rows (B); the leader CTA (rank 0) issues the
// MMAs, which read the A and B halves from both CTAs' shared memory, and each
// CTA's TMEM receives the accumulator rows of its own entries.  Per SM this
// halves the B bytes written into and read from shared memory, which is what
// bounds the one-SM kernel (about 156 of 128 B/clk at full MMA rate).
// TMA completions of both CTAs land on the leader's stage barriers; stage and
// accumulator barriers are released to both CTAs with multicast commits; the
// follower's epilogue releases the accumulator on the leader's barrier.
// ---------------------------------------------------------------------------
constexpr int kBM2 = 256;

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t map_to_rank(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar_cluster_addr, int x,
                                                 int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster_addr)
      : "memory");
}

__device__ __forceinline__ void mma_u8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// Arrives on the barrier at the same offset in both CTAs of the pair once the
// leader's preceding MMAs have completed.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar) {
  const uint16_t mask = 0x3;
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"(mask)
      : "memory");
}

__host__ __device__ constexpr uint32_t idesc_u8_m256(int bn) {
  return (2u << 4) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(kBM2 >> 4) << 24);
}

struct Cfg2 {
  static constexpr int BN = 256;
  static constexpr int kHalfN = BN / 2;
  static constexpr int kStageBytes = 2 * 128 * kBK + 2 * kHalfN * kBK;  // per CTA
  static constexpr int kStages = 3;
  static constexpr int kTmemCols = 2 * BN;
  static constexpr int kColsPerThread = BN / 2;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 + 256;
};

__device__ __forceinline__ bool tile_of2(const GemmParams& P, int t, Tile& out) {
  for (int i = 0; i < P.n_prob; i++) {
    const int nt = (int)(P.prob[i].tiles_m * P.prob[i].tiles_n);
    if (t < nt) {
      out.prob = i;
      out.m_tile = t / (int)P.prob[i].tiles_n;
      out.n_tile = t % (int)P.prob[i].tiles_n;
      return true;
    }
    t -= nt;
  }
  return false;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    limb_gemm_pair_kernel(const __grid_constant__ GemmParams P) {
  using C = Cfg2;
  constexpr int BN = C::BN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* a_lo = smem;
  uint8_t* a_hi = a_lo + C::kStages * 128 * kBK;
  uint8_t* b_lo = a_hi + C::kStages * 128 * kBK;
  uint8_t* b_hi = b_lo + C::kStages * C::kHalfN * kBK;
  uint64_t* bars = reinterpret_cast<uint64_t*>(b_hi + C::kStages * C::kHalfN * kBK);
  uint64_t* full_bar = bars;
  uint64_t* empty_bar = bars + C::kStages;
  uint64_t* acc_full = bars + 2 * C::kStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* done_bar = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 3);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const int cluster = blockIdx.x >> 1;
  const int n_clusters = gridDim.x >> 1;
  int* err = P.err;
  const uint64_t lim = P.wait_timeout_ns, lim2 = 2 * P.wait_timeout_ns;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; s++) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 16);  // 8 epilogue warps in each CTA
    mbar_init(done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)C::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // peer barriers initialised before any remote arrive
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued_phase[C::kStages];
      bool issued[C::kStages];
      for (int s = 0; s < C::kStages; s++) issued[s] = false;
      bool ok = true;
      int it = 0;  // both CTAs of a pair walk the same tiles, so they agree on the order
      for (int t = cluster; ok && t < P.total_tiles; t += n_clusters, it++) {
        Tile tl;
        if (!tile_of2(P, t, tl)) break;
        const GemmProblem& pr = P.prob[tl.prob];
        const int ya = (int)pr.m0 + tl.m_tile * kBM2 + (int)rank * 128;
        const int yb = tl.n_tile * BN + (int)rank * C::kHalfN;
        const bool rev = P.serpentine && (it & 1);
        for (uint32_t ki = 0; ki < pr.k_iters; ki++) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1u, err, kErrTimeoutEmpty, lim2)) { ok = false; break; }
          if (leader) mbar_expect_tx(&full_bar[stage], (uint32_t)(2 * C::kStageBytes));
          const uint32_t fb = map_to_rank(&full_bar[stage], 0);
          const int x = (int)(rev ? pr.k_iters - 1 - ki : ki) * kBK;
          tma_load_2d_pair(a_lo + stage * 128 * kBK, &pr.tm_a_lo, fb, x, ya);
          tma_load_2d_pair(a_hi + stage * 128 * kBK, &pr.tm_a_hi, fb, x, ya);
          tma_load_2d_pair(b_lo + stage * C::kHalfN * kBK, &pr.tm_b_lo, fb, x, yb);
          tma_load_2d_pair(b_hi + stage * C::kHalfN * kBK, &pr.tm_b_hi, fb, x, yb);
          issued[stage] = true;
          issued_phase[stage] = (int)phase;
          if (++stage == C::kStages) { stage = 0; phase ^= 1u; }
        }
      }
      // Exit: the leader's stage barriers complete only when both CTAs' copies
      // of that stage have landed.
      if (leader)
        for (int s = 0; s < C::kStages; s++)
          if (issued[s]) mbar_wait_drain(&full_bar[s], (uint32_t)issued_phase[s], err, lim2);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (leader CTA only) ----------------
    if (lane == 0 && leader) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      constexpr uint32_t idesc = idesc_u8_m256(BN);
      for (int t = cluster; ok && t < P.total_tiles; t += n_clusters) {
        Tile tl;
        if (!tile_of2(P, t, tl)) break;
        const GemmProblem& pr = P.prob[tl.prob];
        if (!mbar_wait(acc_empty, acc_phase ^ 1u, err, kErrTimeoutAccEmpty, lim2)) { ok = false; break; }
        acc_phase ^= 1u;
        tc_fence_after();
        for (uint32_t ki = 0; ki < pr.k_iters; ki++) {
          if (!mbar_wait(&full_bar[stage], phase, err, kErrTimeoutFull, lim)) { ok = false; break; }
          tc_fence_after();
          const uint64_t dal = smem_desc(a_lo + stage * 128 * kBK);
          const uint64_t dah = smem_desc(a_hi + stage * 128 * kBK);
          const uint64_t dbl = smem_desc(b_lo + stage * C::kHalfN * kBK);
          const uint64_t dbh = smem_desc(b_hi + stage * C::kHalfN * kBK);
#pragma unroll
          for (int kk = 0; kk < kBK / 32; kk++) {
            const uint32_t acc = (ki > 0 || kk > 0) ? 1u : 0u;
            const uint64_t o = (uint64_t)(2 * kk);
            mma_u8_pair(tmem, dal + o, dbl + o, idesc, acc);
            mma_u8_pair(tmem + BN, dal + o, dbh + o, idesc, acc);
            mma_u8_pair(tmem + BN, dah + o, dbl + o, idesc, 1u);
          }
          mma_commit_pair(&empty_bar[stage]);
          if (++stage == C::kStages) { stage = 0; phase ^= 1u; }
        }
        if (ok) mma_commit_pair(acc_full);
      }
      asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(done_bar))
                   : "memory");
      mbar_wait_drain(done_bar, 0, err, lim2);
    }
  } else {
    // ---------------- Epilogue (warps 2..9, both CTAs) ----------------
    const int quad = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = quad * 32 + lane;
    constexpr int kCols = C::kColsPerThread;
    const uint32_t acc_empty_leader = map_to_rank(acc_empty, 0);
    uint32_t acc_phase = 0;
    for (int t = cluster; t < P.total_tiles; t += n_clusters) {
      Tile tl;
      if (!tile_of2(P, t, tl)) break;
      const GemmProblem& pr = P.prob[tl.prob];
      if (!mbar_wait(acc_full, acc_phase, err, kErrTimeoutAccFull, lim2)) break;
      acc_phase ^= 1u;
      tc_fence_after();
      uint32_t packed[kCols / 2];
      const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * kCols);
#pragma unroll
      for (int c = 0; c < kCols / 32; c++) {
        uint32_t r0[32], r1[32];
        tmem_ld32(tbase + (uint32_t)(c * 32), r0);
        tmem_ld32(tbase + (uint32_t)(BN + c * 32), r1);
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
      if (lane == 0) mbar_arrive_cluster(acc_empty_leader);

      const uint32_t m_local = (uint32_t)(tl.m_tile * kBM2 + (int)rank * 128 + row);
      if (m_local < pr.m_len) {
        const uint64_t m_global = (uint64_t)pr.m0 + m_local;
        uint16_t* out_row = pr.out + (size_t)m_local * pr.n_pad;
#pragma unroll
        for (int c = 0; c < kCols / 32; c++) {
          const uint32_t n = (uint32_t)(tl.n_tile * BN + half * kCols + c * 32);
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
          uint4* dst = reinterpret_cast<uint4*>(out_row + n);
#pragma unroll
          for (int q = 0; q < 4; q++) dst[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // no CTA leaves while its peer may still touch its memory
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)C::kTmemCols));
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

}  // namespace

int make_tmap_u8(CUtensorMap* map, const void* base, uint64_t rows, uint64_t k, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return -1;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (k % kBK) || box_rows > 256) return -2;
  cuuint64_t dims[2] = {k, rows};
  cuuint64_t strides[1] = {k};
  cuuint32_t box[2] = {(cuuint32_t)kBK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -3;
}

template <int BN>
static cudaError_t launch_bn(const GemmParams& P, int n_sms, cudaStream_t stream) {
  using C = Cfg<BN>;
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = smem_limit_once(limb_gemm_kernel<BN>, C::kSmemBytes, attr_done);
  if (e != cudaSuccess) return e;
  const int grid = P.total_tiles < n_sms ? P.total_tiles : n_sms;
  if (grid <= 0) return cudaSuccess;
  limb_gemm_kernel<BN><<<grid, kThreads, C::kSmemBytes, stream>>>(P);
  return cudaGetLastError();
}

static cudaError_t launch_pair(const GemmParams& P, int n_sms, cudaStream_t stream) {
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = smem_limit_once(limb_gemm_pair_kernel, Cfg2::kSmemBytes, attr_done);
  if (e != cudaSuccess) return e;
  const int clusters = P.total_tiles < n_sms / 2 ? P.total_tiles : n_sms / 2;
  if (clusters <= 0) return cudaSuccess;
  limb_gemm_pair_kernel<<<2 * clusters, kThreads, Cfg2::kSmemBytes, stream>>>(P);
  return cudaGetLastError();
}

// The pair kernel reaches a higher MAC rate per clock but, at the B200's
// 1000 W limit, pulls the SM clock down about as far as it gains, so the
// one-SM kernel is the default and the batch autotuner decides per batch
// shape (irs_sharedb_set_pair).
bool gemm_pair_applies(bool pair, int block_n) { return pair && block_n == 256; }

// Measured on 65,536-entry chunks of the six engines: up to 768 query rows
// the 128-row tile (3 pipeline stages) beats the 256-row tile (2 stages) by
// 5-20%, since the pass is still close to streaming the DB; from 1024 rows,
// and on whole-DB passes, the 256-row tile wins (1024 rows: 66.8 against
// 76.9 ms on 524,288 entries).
int gemm_block_n_for(uint32_t n_pad) {
  if (n_pad <= 768 && n_pad % 128 == 0) return 128;
  if (n_pad % 256 == 0) return 256;
  if (n_pad % 128 == 0) return 128;
  if (n_pad % 64 == 0) return 64;
  return 0;
}

// L2 policy of the one-SM kernel's loads (GemmParams::l2_hint), opt-in through
// IRS_GEMM_L2HINT.  Measured at 524,288 entries x 2048 query rows: the query
// planes are re-read from DRAM once per sweep of the 148 CTAs over the DB
// (about 1.8x the algorithmic bytes in all), but DRAM runs at ~16% of its
// bandwidth under this tensor-bound kernel, and keeping the queries with
// evict_last saved 2% of the traffic while slowing the GEMM by 3% and the
// following threshold kernel by 18% (the pinned lines outlive the GEMM).
// Marking the streaming DB evict_first (value 2) instead tripled the reads
// on 65,536-entry chunks (31-48 GB against 13.7 GB per launch: each DB tile
// is read by the wave's 8 query-tile CTAs, and the hint drops it between
// them), and under the power cap the clock fell from 1567 to ~1365 MHz, 14%
// slower per batch.
static uint32_t gemm_l2_hint() {
  static const uint32_t hint = [] {
    const char* e = getenv("IRS_GEMM_L2HINT");
    return e ? (uint32_t)atoi(e) & 3u : 0u;
  }();
  return hint;
}

cudaError_t launch_limb_gemm(GemmParams& P, int block_n, bool pair_wanted, int n_sms, cudaStream_t stream) {
  // the stall hook is the one-SM kernel's
  const bool pair = gemm_pair_applies(pair_wanted, block_n) && !P.test_stall;
  if (P.wait_timeout_ns == 0) P.wait_timeout_ns = kGemmWaitTimeoutNs;
  P.l2_hint = gemm_l2_hint();
  // Serpentine K order (GemmParams::serpentine), on unless IRS_GEMM_SERPENTINE=0.
  // Measured with the query planes re-read once per wave: DRAM reads per
  // 65,536-entry one-SM launch 11.46 GB against 13.2-13.9 GB in K order, per
  // 32,768-entry two-SM launch 11.1-11.6 against 11.8-12.2 GB on the same
  // GPU; batch times unchanged (within 0.3%), results identical.
  static const uint32_t serp = [] {
    const char* e = getenv("IRS_GEMM_SERPENTINE");
    return e ? (uint32_t)(atoi(e) != 0) : 1u;
  }();
  P.serpentine = serp;
  const uint32_t bm = pair ? (uint32_t)kBM2 : (uint32_t)kBM;
  P.total_tiles = 0;
  for (int i = 0; i < P.n_prob; i++) {
    GemmProblem& pr = P.prob[i];
    pr.tiles_m = (pr.m_len + bm - 1) / bm;
    pr.tiles_n = pr.n_pad / (uint32_t)block_n;
    P.total_tiles += (int)(pr.tiles_m * pr.tiles_n);
  }
  if (pair) return launch_pair(P, n_sms, stream);
  switch (block_n) {
    case 256: return launch_bn<256>(P, n_sms, stream);
    case 128: return launch_bn<128>(P, n_sms, stream);
    case 64: return launch_bn<64>(P, n_sms, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace irs
