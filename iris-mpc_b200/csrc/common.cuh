// Shared device helpers for the iris B200 kernels: ChaCha12 keystream blocks,
// the position-addressable keystream layout, error reporting and bounded
// waits.  Everything here is __host__ __device__ where it can be, so the
// host-side unit harness exercises the same code the kernels run.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

#define IRS_HD __host__ __device__ __forceinline__

namespace irs {

constexpr int kIrisCodeLength = 12800;
constexpr int kMaskCodeLength = 6400;
constexpr int kRotations = 31;
constexpr int kRowLen = 800;        // coefficients per iris row (200 columns x 4)
constexpr int kSlotRows = 32;       // query rows reserved per query iris (31 rotations + 1 pad)

// Keystream domains: nonce = (domain << 32) | device index.
constexpr uint32_t kDomCodeDot = 1;
constexpr uint32_t kDomMaskDot = 2;
constexpr uint32_t kDomCircuit = 3;
constexpr uint32_t kDomOrTree = 4;
// Circuit keystream: 8 blocks (128 words) per 32-element word and stream.
constexpr int kCircuitBlocksPerWord = 8;

// Threshold circuit variants: the full compare_threshold_masked_many, or the
// msb of -code*2^16 - 1 alone (lifted mask and corrections at zero).
enum : int { kStageFull = 0, kStageMsbOnly = 1 };

// Error codes written to the device error word (first error wins).
enum : int {
  kErrNone = 0,
  kErrTimeoutFull = 1,      // MMA waited too long for a TMA stage
  kErrTimeoutEmpty = 2,     // producer waited too long for a free stage
  kErrTimeoutAccFull = 3,   // epilogue waited too long for the accumulator
  kErrTimeoutAccEmpty = 4,  // MMA waited too long for the epilogue
  kErrTimeoutDrain = 5,     // exit-time wait on in-flight copies gave up
  kErrBadShape = 6,
  kErrOverflow = 7,         // a result list exceeded its capacity (counted, not fatal)
};

IRS_HD uint64_t nonce_of(uint32_t domain, uint32_t dev) { return ((uint64_t)domain << 32) | dev; }
IRS_HD uint64_t counter_of(uint64_t batch, uint64_t blk) { return (batch << 40) | blk; }

struct ChaChaKey {
  uint32_t k[8];
};

IRS_HD uint32_t rotl32(uint32_t v, int n) {
#ifdef __CUDA_ARCH__
  return __funnelshift_l(v, v, n);
#else
  return (v << n) | (v >> (32 - n));
#endif
}

// Rotations by 16 and 8 are byte permutes on the device (one PRMT each,
// measured 1.7% faster threshold kernels than funnel shifts); same values.
#ifdef __CUDA_ARCH__
#define IRS_ROT16(x) __byte_perm((x), (x), 0x1032)
#define IRS_ROT8(x) __byte_perm((x), (x), 0x2103)
#else
#define IRS_ROT16(x) rotl32((x), 16)
#define IRS_ROT8(x) rotl32((x), 8)
#endif
#define IRS_QR(a, b, c, d)        \
  a += b; d ^= a; d = IRS_ROT16(d); \
  c += d; b ^= c; b = rotl32(b, 12); \
  a += b; d ^= a; d = IRS_ROT8(d);  \
  c += d; b ^= c; b = rotl32(b, 7);

// One keystream block: state = "expand 32-byte k" | key | counter | nonce,
// ROUNDS/2 double rounds, feed-forward add.  Same construction as the
// reference's chacha12 kernel (iris-mpc-gpu/src/rng/chacha.cu:74-138), with
// the whole state in registers.
template <int ROUNDS = 12>
IRS_HD void chacha_block(const ChaChaKey& key, uint64_t counter, uint64_t nonce, uint32_t out[16]) {
  const uint32_t c0 = 0x61707865u, c1 = 0x3320646eu, c2 = 0x79622d32u, c3 = 0x6b206574u;
  uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
  uint32_t x4 = key.k[0], x5 = key.k[1], x6 = key.k[2], x7 = key.k[3];
  uint32_t x8 = key.k[4], x9 = key.k[5], x10 = key.k[6], x11 = key.k[7];
  uint32_t x12 = (uint32_t)counter, x13 = (uint32_t)(counter >> 32);
  uint32_t x14 = (uint32_t)nonce, x15 = (uint32_t)(nonce >> 32);
#pragma unroll
  for (int i = 0; i < ROUNDS / 2; i++) {
    IRS_QR(x0, x4, x8, x12) IRS_QR(x1, x5, x9, x13) IRS_QR(x2, x6, x10, x14) IRS_QR(x3, x7, x11, x15)
    IRS_QR(x0, x5, x10, x15) IRS_QR(x1, x6, x11, x12) IRS_QR(x2, x7, x8, x13) IRS_QR(x3, x4, x9, x14)
  }
  out[0] = x0 + c0; out[1] = x1 + c1; out[2] = x2 + c2; out[3] = x3 + c3;
  out[4] = x4 + key.k[0]; out[5] = x5 + key.k[1]; out[6] = x6 + key.k[2]; out[7] = x7 + key.k[3];
  out[8] = x8 + key.k[4]; out[9] = x9 + key.k[5]; out[10] = x10 + key.k[6]; out[11] = x11 + key.k[7];
  out[12] = x12 + (uint32_t)counter; out[13] = x13 + (uint32_t)(counter >> 32);
  out[14] = x14 + (uint32_t)nonce; out[15] = x15 + (uint32_t)(nonce >> 32);
}

// The first ChaCha round's column quarter rounds 1..3 read only the key, the
// high counter word and the nonce, so blocks that share those (the eight blocks
// of one circuit word: their counters never carry into the high word) share them.
// pre[24] = key[8] | ctr_hi | nonce_lo | nonce_hi | 0 | the twelve words of
// columns 1..3 after the first round (x1 x5 x9 x13, x2 x6 x10 x14, x3 x7 x11 x15).
IRS_HD void chacha_prepare(const ChaChaKey& key, uint32_t ctr_hi, uint64_t nonce, uint32_t pre[24]) {
  for (int i = 0; i < 8; i++) pre[i] = key.k[i];
  pre[8] = ctr_hi;
  pre[9] = (uint32_t)nonce;
  pre[10] = (uint32_t)(nonce >> 32);
  pre[11] = 0;
  uint32_t x1 = 0x3320646eu, x5 = key.k[1], x9 = key.k[5], x13 = ctr_hi;
  uint32_t x2 = 0x79622d32u, x6 = key.k[2], x10 = key.k[6], x14 = pre[9];
  uint32_t x3 = 0x6b206574u, x7 = key.k[3], x11 = key.k[7], x15 = pre[10];
  IRS_QR(x1, x5, x9, x13) IRS_QR(x2, x6, x10, x14) IRS_QR(x3, x7, x11, x15)
  pre[12] = x1; pre[13] = x5; pre[14] = x9; pre[15] = x13;
  pre[16] = x2; pre[17] = x6; pre[18] = x10; pre[19] = x14;
  pre[20] = x3; pre[21] = x7; pre[22] = x11; pre[23] = x15;
}

// ChaCha12 block with counter (ctr_hi << 32 | ctr_lo) from the six prepared
// words-of-four of chacha_prepare (k0 = key 0..3, k1 = key 4..7, cn = ctr_hi,
// nonce, c1..c3 = the prepared columns): the same keystream as
// chacha_block<12>.  Word j goes to out[j * stride].
IRS_HD void chacha12_core(uint4 k0, uint4 k1, uint4 cn, uint4 c1, uint4 c2, uint4 c3, uint32_t ctr_lo,
                          uint32_t* out, int stride) {
  const uint32_t s0 = 0x61707865u, s1 = 0x3320646eu, s2 = 0x79622d32u, s3 = 0x6b206574u;
  uint32_t x0 = s0, x4 = k0.x, x8 = k1.x, x12 = ctr_lo;
  IRS_QR(x0, x4, x8, x12)
  uint32_t x1 = c1.x, x5 = c1.y, x9 = c1.z, x13 = c1.w;
  uint32_t x2 = c2.x, x6 = c2.y, x10 = c2.z, x14 = c2.w;
  uint32_t x3 = c3.x, x7 = c3.y, x11 = c3.z, x15 = c3.w;
  IRS_QR(x0, x5, x10, x15) IRS_QR(x1, x6, x11, x12) IRS_QR(x2, x7, x8, x13) IRS_QR(x3, x4, x9, x14)
#pragma unroll
  for (int i = 1; i < 6; i++) {
    IRS_QR(x0, x4, x8, x12) IRS_QR(x1, x5, x9, x13) IRS_QR(x2, x6, x10, x14) IRS_QR(x3, x7, x11, x15)
    IRS_QR(x0, x5, x10, x15) IRS_QR(x1, x6, x11, x12) IRS_QR(x2, x7, x8, x13) IRS_QR(x3, x4, x9, x14)
  }
  out[0 * stride] = x0 + s0; out[1 * stride] = x1 + s1; out[2 * stride] = x2 + s2; out[3 * stride] = x3 + s3;
  out[4 * stride] = x4 + k0.x; out[5 * stride] = x5 + k0.y; out[6 * stride] = x6 + k0.z;
  out[7 * stride] = x7 + k0.w; out[8 * stride] = x8 + k1.x; out[9 * stride] = x9 + k1.y;
  out[10 * stride] = x10 + k1.z; out[11 * stride] = x11 + k1.w; out[12 * stride] = x12 + ctr_lo;
  out[13 * stride] = x13 + cn.x; out[14 * stride] = x14 + cn.y; out[15 * stride] = x15 + cn.z;
}

// chacha12_core from a contiguous prepared array pre[24] (16-byte aligned).
IRS_HD void chacha12_block_prepared(const uint32_t* pre, uint32_t ctr_lo, uint32_t out[16]) {
  const uint4* q = reinterpret_cast<const uint4*>(pre);
  chacha12_core(q[0], q[1], q[2], q[3], q[4], q[5], ctr_lo, out, 1);
}
#undef IRS_QR
#undef IRS_ROT16
#undef IRS_ROT8

// Packed 16-bit lane arithmetic (two u16 per u32, no carry across lanes).
IRS_HD uint32_t add2(uint32_t a, uint32_t b) {
  return ((a & 0x7fff7fffu) + (b & 0x7fff7fffu)) ^ ((a ^ b) & 0x80008000u);
}
IRS_HD uint32_t sub2(uint32_t a, uint32_t b) {
  return ((a | 0x80008000u) - (b & 0x7fff7fffu)) ^ ((a ^ ~b) & 0x80008000u);
}

#ifdef __CUDACC__
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void set_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}
__device__ __forceinline__ bool has_error(const int* err) {
  return err && *(const volatile int*)err != 0;
}
#endif

}  // namespace irs
