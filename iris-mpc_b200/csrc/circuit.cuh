// Bit-sliced 3-party threshold circuit for one 32-element word.
//
// The three co-resident parties hold replicated shares: party p holds the
// pair (component p, component p-1) of every secret.  This file keeps the
// three components of each secret bit plane in a Comp and evaluates every
// gate as the three party-local computations the protocol prescribes:
//   - XOR: each party XORs its own pair (component-wise XOR);
//   - AND: party p computes (xa&ya)^(xb&ya)^(xa&yb)^r_p from its view only,
//     with r_p = keystream(seed p) ^ keystream(seed p-1) (zero-sharing), then
//     "sends" the result to p+1 -- which on one GPU is the component store.
// Protocol steps follow iris-mpc-gpu/src/threshold_ring/protocol.rs:
//   lift_mpc 2041-2074, binary_add_3_get_two_carries 2137-2241,
//   bit_inject_party_{0,1,2} 1302-1643 (kernel.cu:526-629),
//   lift_mul_sub 1831-1872 (kernel.cu:181-195,407-426),
//   extract_msb 2243-2258, binary_add_3_get_msb 2262-2359.
//
// Keystream layout per 32-element word and stream s (party s's own seed):
// 8 ChaCha12 blocks = 128 words, block b at counter (batch<<40)|(word*8+b).
//   words 0..31  : lift adder gates  (2k = carry-save AND of plane k, k<15;
//                  2k+1 = ripple step k, k<15; 30 = plane 15; 31 = final AND)
//   words 32..92 : msb adder gates   (32+2k = carry-save AND of plane k, k<31;
//                  33+2k = ripple step k, k<30)
//   words 96..111: bit-inject randomness of carry c1 (u16 j at word 96+j/2)
//   words 112..127: bit-inject randomness of carry c2
// Stream 0 feeds r01, stream 1 r12, stream 2 r02 of the bit injection.
#pragma once
#include "common.cuh"

namespace irs {

struct Comp {
  uint32_t c0, c1, c2;
};

IRS_HD Comp cxor(Comp a, Comp b) { return {a.c0 ^ b.c0, a.c1 ^ b.c1, a.c2 ^ b.c2}; }

// and_pre_inner (threshold_ring/cuda/kernel.cu:37-41): the local part of a
// party's AND share from its view (xa, xb), (ya, yb) and its randomness.
IRS_HD uint32_t and_local(uint32_t xa, uint32_t xb, uint32_t ya, uint32_t yb, uint32_t r) {
  return (xa & ya) ^ (xb & ya) ^ (xa & yb) ^ r;
}

// One AND gate for the three parties.  k0/k1/k2: this gate's keystream word
// from streams 0/1/2.  Party p's randomness is k_p ^ k_{p-1}.
IRS_HD Comp cand(Comp x, Comp y, uint32_t k0, uint32_t k1, uint32_t k2) {
  Comp z;
  z.c0 = and_local(x.c0, x.c2, y.c0, y.c2, k0 ^ k2);  // party 0 views (c0, c2)
  z.c1 = and_local(x.c1, x.c0, y.c1, y.c0, k1 ^ k0);  // party 1 views (c1, c0)
  z.c2 = and_local(x.c2, x.c1, y.c2, y.c1, k2 ^ k1);  // party 2 views (c2, c1)
  return z;
}

// Block `counter` of the three streams into ks[3][16].  Kept out of line: the
// circuit draws 24 blocks per word, and one shared copy of the ChaCha code
// keeps the kernel's instruction working set inside the instruction cache.
#ifdef __CUDACC__
static __host__ __device__ __noinline__
#else
static
#endif
void chacha12_x3(const uint32_t* pre, uint32_t ctr_lo, uint32_t* ks) {
#pragma unroll 1
  for (int s = 0; s < 3; s++) chacha12_block_prepared(pre + 24 * s, ctr_lo, ks + 16 * s);
}

// Keystream of one word: the current block of each of the three streams.
// The eight blocks of a word share their counter's high word (the low word
// of block 0's counter is a multiple of 8), so the first ChaCha round's constant columns
// are prepared once per word and stream (chacha_prepare).
struct WordRand {
  ChaChaKey key[3];
  uint64_t nonce;
  uint64_t base;  // counter of block 0 of this word
  uint32_t ks[3][16];
  int block;
  bool prepared = false;
  alignas(16) uint32_t pre[3][24];
  IRS_HD void load(int b) {
    block = b;
    if (!prepared) {
      for (int s = 0; s < 3; s++) chacha_prepare(key[s], (uint32_t)(base >> 32), nonce, pre[s]);
      prepared = true;
    }
    chacha12_x3(&pre[0][0], (uint32_t)(base + (uint64_t)b), &ks[0][0]);
  }
  // word j of stream s's current block
  IRS_HD uint32_t k(int s, int j) const { return ks[s][j]; }
};

#ifdef __CUDACC__
// The three streams' current blocks from prepared words-of-four in shared
// memory, element i of this thread at pre[i * nt] (18 of them) and keystream
// word (s, j) written to ks[(16 s + j) * nt].  Out of line for the same
// instruction-cache reason as chacha12_x3.
static __device__ __noinline__ void chacha12_x3_strided(const uint4* pre, uint32_t* ks, int nt, uint32_t ctr_lo) {
#pragma unroll 1
  for (int s = 0; s < 3; s++) {
    const uint4* q = pre + 6 * s * nt;
    chacha12_core(q[0], q[nt], q[2 * nt], q[3 * nt], q[4 * nt], q[5 * nt], ctr_lo, ks + 16 * s * nt, nt);
  }
}

// WordRand with its keystream and prepared columns in shared memory instead
// of the thread's local memory: the block's threads interleave them
// ([element][thread], so a warp's accesses hit consecutive words and never
// conflict), `pre` and `ks` point at this thread's column and nt is the
// thread count of the block.  Same keystream as WordRand.
struct WordRandShared {
  ChaChaKey key[3];
  uint64_t nonce;
  uint64_t base;
  bool prepared = false;
  uint4* pre;    // [18][nt] words-of-four: 6 per stream
  uint32_t* ks;  // [48][nt]: 16 per stream
  int nt;
  __device__ void load(int b) {
    if (!prepared) {
      for (int s = 0; s < 3; s++) {
        alignas(16) uint32_t t[24];
        chacha_prepare(key[s], (uint32_t)(base >> 32), nonce, t);
#pragma unroll
        for (int q = 0; q < 6; q++) pre[(6 * s + q) * nt] = make_uint4(t[4 * q], t[4 * q + 1], t[4 * q + 2], t[4 * q + 3]);
      }
      prepared = true;
    }
    chacha12_x3_strided(pre, ks, nt, (uint32_t)(base + (uint64_t)b));
  }
  __device__ uint32_t k(int s, int j) const { return ks[(16 * s + j) * nt]; }
};
#endif

// Gate g (compile-time after unrolling) must lie in the loaded block.
#define IRS_GATE(wr, x, y, g) cand((x), (y), (wr).k(0, (g) & 15), (wr).k(1, (g) & 15), (wr).k(2, (g) & 15))

// Byte select from the pair (a, b): result byte i = byte ((sel >> 4i) & 7)
// of the 8-byte value b:a (one PRMT on the device).
IRS_HD uint32_t select_bytes(uint32_t a, uint32_t b, uint32_t sel) {
#ifdef __CUDA_ARCH__
  return __byte_perm(a, b, sel);
#else
  const uint64_t v = ((uint64_t)b << 32) | a;
  uint32_t r = 0;
  for (int i = 0; i < 4; i++) r |= (uint32_t)((v >> (8 * ((sel >> (4 * i)) & 7))) & 0xFFu) << (8 * i);
  return r;
#endif
}

// The first two butterfly stages of the transpose, which move whole half
// words and bytes: (lo a | lo b << 16, hi a | hi b << 16) and the byte
// interleave of the stage with mask 0x00FF00FF -- one byte select per output.
IRS_HD void swap_halves(uint32_t& a, uint32_t& b) {
  const uint32_t x = select_bytes(a, b, 0x5410), y = select_bytes(a, b, 0x7632);
  a = x;
  b = y;
}
IRS_HD void swap_bytes(uint32_t& a, uint32_t& b) {
  const uint32_t x = select_bytes(a, b, 0x6240), y = select_bytes(a, b, 0x7351);
  a = x;
  b = y;
}

// In-register 32x32 bit transpose: afterwards A[r] bit c = old A[c] bit r.
IRS_HD void transpose32(uint32_t A[32]) {
#pragma unroll
  for (int k = 0; k < 16; k++) swap_halves(A[k], A[k + 16]);
#pragma unroll
  for (int k = 0; k < 32; k++)
    if ((k & 8) == 0) swap_bytes(A[k], A[k + 8]);
#pragma unroll
  for (int s = 4, m = 0x0F0F0F0F; s > 0; s >>= 1, m ^= (m << s)) {
#pragma unroll
    for (int k = 0; k < 32; k++) {
      if ((k & s) == 0) {
        uint32_t t = ((A[k] >> s) ^ A[k + s]) & (uint32_t)m;
        A[k] ^= t << s;
        A[k + s] ^= t;
      }
    }
  }
}

// 32 u16 values packed two per word (w[i] = v[2i] | v[2i+1] << 16) to 16 bit
// planes: P[k] bit j = bit k of v[j].
IRS_HD void slice16(const uint32_t w[16], uint32_t P[16]) {
  uint32_t A[16];
#pragma unroll
  for (int k = 0; k < 16; k++) {
    // row k holds element k in the low half and element k+16 in the high half
    uint32_t lo = (k & 1) ? (w[k >> 1] >> 16) : (w[k >> 1] & 0xFFFFu);
    uint32_t hi = (k & 1) ? (w[8 + (k >> 1)] >> 16) : (w[8 + (k >> 1)] & 0xFFFFu);
    A[k] = lo | (hi << 16);
  }
  // 16x16 transposes of both halves at once (the s = 8..1 stages of transpose32)
#pragma unroll
  for (int k = 0; k < 16; k++)
    if ((k & 8) == 0) swap_bytes(A[k], A[k + 8]);
#pragma unroll
  for (int s = 4, m = 0x0F0F0F0F; s > 0; s >>= 1, m ^= (m << s)) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      if ((k & s) == 0) {
        uint32_t t = ((A[k] >> s) ^ A[k + s]) & (uint32_t)m;
        A[k] ^= t << s;
        A[k + s] ^= t;
      }
    }
  }
  // A[k]: low half bit j = element j bit k, high half bit j = element 16+j bit k
#pragma unroll
  for (int k = 0; k < 16; k++) P[k] = A[k];
}

// Loads 32 consecutive u16 (64 bytes, 16-byte aligned) as 16 packed words:
// through the read-only path, or (COHERENT) as ordinary loads, for data that
// other threads of the same CTA wrote before a barrier (the read-only path is
// not coherent with writes of the running kernel).
template <bool COHERENT = false>
IRS_HD void load32(const uint16_t* p, uint32_t w[16]) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
  for (int i = 0; i < 4; i++) {
#ifdef __CUDA_ARCH__
    uint4 v = COHERENT ? q[i] : __ldg(q + i);
#else
    uint4 v = q[i];
#endif
    w[4 * i + 0] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
  }
}

// binary_add_3_get_two_carries for K = 16 on the three components of a
// 16-bit value (M[p][k] = plane k of component p).  Returns the carries c1
// (bit 16) and c2 (bit 17) of M0 + M1 + M2.
template <class WR>
IRS_HD void lift_carries(const uint32_t M[3][16], WR& wr, Comp& c1, Comp& c2) {
  // carry-save: s = x1^x2^x3 = (M0, M1, M2); c = AND(x1^x3, x2^x3) ^ x3
  Comp carry = {0, 0, 0};
  Comp b_prev = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < 16; k++) {
    const int gp = (k < 15) ? 2 * k : 30;
    if (k == 0) wr.load(0);
    if (k == 8) wr.load(1);  // gates 16..31
    Comp x1x3 = {M[0][k], 0u, M[2][k]};
    Comp x2x3 = {0u, M[1][k], M[2][k]};
    Comp ck = IRS_GATE(wr, x1x3, x2x3, gp);
    ck.c2 ^= M[2][k];
    if (k == 0) {
      // ripple step 0: carry = AND(s[1], c[0])
      Comp s1 = {M[0][1], M[1][1], M[2][1]};
      carry = IRS_GATE(wr, s1, ck, 1);
    } else if (k < 15) {
      // ripple step k: a = s[k+1]^carry, b = c[k]^carry, carry ^= AND(a, b)
      const int gr = 2 * k + 1;
      Comp a = cxor({M[0][k + 1], M[1][k + 1], M[2][k + 1]}, carry);
      Comp b = cxor(ck, carry);
      carry = cxor(carry, IRS_GATE(wr, a, b, gr));
    } else {
      b_prev = ck;  // c[15]
    }
  }
  // final: c2 = AND(c[15], carry); c1 = carry ^ c[15]
  c2 = IRS_GATE(wr, b_prev, carry, 31);
  c1 = cxor(carry, b_prev);
}

// binary_add_3_get_msb on the three components of a 32-bit value
// (P[p][k] = plane k of component p).  Returns the components of bit 31.
template <class WR>
IRS_HD Comp msb_of_sum(const uint32_t P[3][32], WR& wr) {
  Comp carry = {0, 0, 0};
  Comp a30 = {0, 0, 0}, b30 = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < 31; k++) {
    const int gp = 32 + 2 * k;
    if ((k & 7) == 0) wr.load(2 + (k >> 3));  // gates 32+2k and 33+2k share a block
    Comp x1x3 = {P[0][k], 0u, P[2][k]};
    Comp x2x3 = {0u, P[1][k], P[2][k]};
    Comp ck = IRS_GATE(wr, x1x3, x2x3, gp);
    ck.c2 ^= P[2][k];
    Comp sk1 = {P[0][k + 1], P[1][k + 1], P[2][k + 1]};  // s[k+1]
    if (k == 0) {
      carry = IRS_GATE(wr, sk1, ck, 33);
    } else if (k < 30) {
      const int gr = 33 + 2 * k;
      Comp a = cxor(sk1, carry);
      Comp b = cxor(ck, carry);
      carry = cxor(carry, IRS_GATE(wr, a, b, gr));
    } else {
      a30 = sk1;
      b30 = ck;
    }
  }
  return cxor(cxor(carry, a30), b30);
}

// bit_inject of one carry plane for elements j in [j0, j0+n): returns, per
// party p, the arithmetic component A_p (u16) of element j.  `ks` words hold
// the u16 randomness (stream 0: r01, stream 1: r12, stream 2: r02).
//   party 1: x = (v1 ^ v0) - r01        -> party 2
//   party 0: y = v2 * r01 - r02         -> party 1
//   party 2: z = v2 * x - r12           -> party 0
//   A0 = r01 - 2y,  A1 = x - 2 r12,  A2 = v2 - 2 (r02 + z)
IRS_HD void inject_bit(Comp v, int j, const uint32_t ks[3][16], uint32_t& A0, uint32_t& A1, uint32_t& A2) {
  const uint32_t sh = 16 * (j & 1);
  const uint32_t r01 = (ks[0][(j >> 1) & 15] >> sh) & 0xFFFFu;
  const uint32_t r12 = (ks[1][(j >> 1) & 15] >> sh) & 0xFFFFu;
  const uint32_t r02 = (ks[2][(j >> 1) & 15] >> sh) & 0xFFFFu;
  const uint32_t v0 = (v.c0 >> j) & 1u, v1 = (v.c1 >> j) & 1u, v2 = (v.c2 >> j) & 1u;
  const uint32_t x = ((v1 ^ v0) - r01) & 0xFFFFu;  // party 1 (holds v1, v0)
  const uint32_t y = (v2 * r01 - r02) & 0xFFFFu;   // party 0 (holds v0, v2)
  const uint32_t z = (v2 * x - r12) & 0xFFFFu;     // party 2 (holds v2, v1)
  A0 = (r01 - 2u * y) & 0xFFFFu;
  A1 = (x - 2u * r12) & 0xFFFFu;
  A2 = (v2 - 2u * (r02 + z)) & 0xFFFFu;
}

// Even bits of x to the low half, odd bits to the high half (bit 2k -> k,
// bit 2k+1 -> 16 + k): the carry bits of elements 2i and 2i+1 then sit at
// bits i and 16 + i, one 16-bit lane each.
IRS_HD uint32_t unzip_bits(uint32_t x) {
  uint32_t t;
  t = (x ^ (x >> 1)) & 0x22222222u; x ^= t ^ (t << 1);
  t = (x ^ (x >> 2)) & 0x0C0C0C0Cu; x ^= t ^ (t << 2);
  t = (x ^ (x >> 4)) & 0x00F000F0u; x ^= t ^ (t << 4);
  t = (x ^ (x >> 8)) & 0x0000FF00u; x ^= t ^ (t << 8);
  return x;
}

// inject_bit for the element pair (2i, 2i+1) in packed 16-bit lanes: V0..V2
// hold the pair's carry bits (0 or 1 per lane, from unzip_bits), R01 / R12 /
// R02 the pair's keystream words; returns the parties' packed components.
IRS_HD void inject_pair(uint32_t V0, uint32_t V1, uint32_t V2, uint32_t R01, uint32_t R12, uint32_t R02,
                        uint32_t& A0, uint32_t& A1, uint32_t& A2) {
  const uint32_t X = sub2(V1 ^ V0, R01);  // party 1 -> party 2
  const uint32_t M2 = V2 * 0xFFFFu;       // lane-wise v2 ? 0xFFFF : 0
  const uint32_t Y = sub2(R01 & M2, R02); // party 0 -> party 1
  const uint32_t Z = sub2(M2 & X, R12);   // party 2 -> party 0
  A0 = sub2(R01, (Y << 1) & 0xFFFEFFFEu);
  A1 = sub2(X, (R12 << 1) & 0xFFFEFFFEu);
  A2 = sub2(V2, (add2(R02, Z) << 1) & 0xFFFEFFFEu);
}

// lift_mpc for one word: the injected correction components of both carries
// (corr1[p][j], corr2[p][j] = party p's own component, u16) such that
// mask = sum_p mask_p - (sum_p corr1_p << 16) - (sum_p corr2_p << 17) in Z_2^32.
IRS_HD void lift_word(const uint16_t* const mask[3], WordRand& wr, uint16_t corr1[3][32], uint16_t corr2[3][32]) {
  Comp c1, c2;
  {
    uint32_t M[3][16];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      uint32_t w[16];
      load32(mask[p], w);
      slice16(w, M[p]);
    }
    lift_carries(M, wr, c1, c2);
  }
  wr.load(6);
#pragma unroll
  for (int j = 0; j < 32; j++) {
    uint32_t A0, A1, A2;
    inject_bit(c1, j, wr.ks, A0, A1, A2);
    corr1[0][j] = (uint16_t)A0; corr1[1][j] = (uint16_t)A1; corr1[2][j] = (uint16_t)A2;
  }
  wr.load(7);
#pragma unroll
  for (int j = 0; j < 32; j++) {
    uint32_t A0, A1, A2;
    inject_bit(c2, j, wr.ks, A0, A1, A2);
    corr2[0][j] = (uint16_t)A0; corr2[1][j] = (uint16_t)A1; corr2[2][j] = (uint16_t)A2;
  }
}

// compare_threshold_masked_many for one word of 32 elements.  code[p] and
// mask[p] point at party p's own additive components (64 bytes each).
// Returns the opened comparison bits; msb receives the components of the
// result (party p's shares are (msb.c_p, msb.c_{p-1})).
template <int STAGE, bool COHERENT = false, class WR>
IRS_HD uint32_t threshold_word(const uint16_t* const code[3], const uint16_t* const mask[3], uint32_t threshold_a,
                               WR& wr, Comp& msb) {
  uint32_t X[3][32];
  if (STAGE == kStageFull) {
    Comp c1, c2;
    {
      uint32_t M[3][16];
#pragma unroll
      for (int p = 0; p < 3; p++) {
        uint32_t w[16];
        load32<COHERENT>(mask[p], w);
        slice16(w, M[p]);
      }
      lift_carries(M, wr, c1, c2);
    }
    // Party p's lift correction C_p[j] = inject(c1)_p[j] + 2 inject(c2)_p[j]
    // (mod 2^16), two elements per word.  The injections run as rolled loops
    // over a small per-thread array: one copy of their code instead of 64
    // unrolled ones keeps the kernel's straight-line code (executed once per
    // word) small enough for the instruction cache.
    // Elements 2i and 2i+1 share keystream word i of each stream, so the
    // injection runs on packed 16-bit lanes, a pair per step.
    uint32_t corr[3][16];
    {
      const uint32_t w0 = unzip_bits(c1.c0), w1 = unzip_bits(c1.c1), w2 = unzip_bits(c1.c2);
      wr.load(6);
#pragma unroll 1
      for (int i = 0; i < 16; i++)
        inject_pair((w0 >> i) & 0x00010001u, (w1 >> i) & 0x00010001u, (w2 >> i) & 0x00010001u, wr.k(0, i),
                    wr.k(1, i), wr.k(2, i), corr[0][i], corr[1][i], corr[2][i]);
    }
    {
      const uint32_t w0 = unzip_bits(c2.c0), w1 = unzip_bits(c2.c1), w2 = unzip_bits(c2.c2);
      wr.load(7);
#pragma unroll 1
      for (int i = 0; i < 16; i++) {
        uint32_t a[3];
        inject_pair((w0 >> i) & 0x00010001u, (w1 >> i) & 0x00010001u, (w2 >> i) & 0x00010001u, wr.k(0, i),
                    wr.k(1, i), wr.k(2, i), a[0], a[1], a[2]);
#pragma unroll
        for (int p = 0; p < 3; p++) corr[p][i] = add2(corr[p][i], (a[p] << 1) & 0xFFFEFFFEu);
      }
    }
    // X_p = (mask_p - A1_p<<16 - A2_p<<17) * A - code_p<<16 - [p == 0]
    //     = mask_p * A - ((C_p * A + code_p) << 16) - [p == 0]   (mod 2^32)
#pragma unroll
    for (int p = 0; p < 3; p++) {
      uint32_t wm[16], wc[16];
      load32<COHERENT>(mask[p], wm);
      load32<COHERENT>(code[p], wc);
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const uint32_t m = (wm[j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
        const uint32_t c = (wc[j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
        const uint32_t cr = (corr[p][j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
        X[p][j] = m * threshold_a - ((cr * threshold_a + c) << 16) - (p == 0 ? 1u : 0u);
      }
    }
  } else {
    // extract_msb with the lifted mask and corrections at zero:
    // X_p = -code_p<<16 - [p == 0]
#pragma unroll
    for (int p = 0; p < 3; p++) {
      uint32_t wc[16];
      load32<COHERENT>(code[p], wc);
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const uint32_t c = (wc[j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
        X[p][j] = 0u - (c << 16) - (p == 0 ? 1u : 0u);
      }
    }
  }
#pragma unroll
  for (int p = 0; p < 3; p++) transpose32(X[p]);
  msb = msb_of_sum(X, wr);
  return msb.c0 ^ msb.c1 ^ msb.c2;  // open: a ^ b ^ (third component from prev)
}

}  // namespace irs
