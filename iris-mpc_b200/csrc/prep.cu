// Data-preparation kernels: u16 share records to u8 limb planes, query
// rotation expansion into 32-row slots, the i8 (byte - 128) storage limbs, and
// the seeded synthetic share database used by the benchmark workloads.
//
// Limb split: the reference stores limb_i = byte_i - 128 as i8 for cuBLAS
// (iris-mpc-gpu/src/dot/share_db.rs:45-59,620-655); the tcgen05 GEMM takes the
// unsigned bytes directly, so a stored i8 limb converts with x ^ 0x80.
// Rotations: row r of a query slot is all_rotations()[r] of the query share,
// i.e. every 800-coefficient row rotated left by 4*(15 - r) coefficients
// (iris-mpc-common/src/galois_engine.rs:42-52,197-206).
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"
#include "prep.h"

namespace irs {

namespace {

__global__ void split_limbs_kernel(const uint16_t* __restrict__ in, uint8_t* __restrict__ lo,
                                   uint8_t* __restrict__ hi, size_t n4) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n4) return;
  const uint2 v = reinterpret_cast<const uint2*>(in)[i];  // 4 u16
  const uint32_t l = (v.x & 0xFFu) | ((v.x >> 8) & 0xFF00u) | ((v.y & 0xFFu) << 16) | ((v.y & 0xFF0000u) << 8);
  const uint32_t h = ((v.x >> 8) & 0xFFu) | ((v.x >> 16) & 0xFF00u) | ((v.y & 0xFF00u) << 8) | (v.y & 0xFF000000u);
  reinterpret_cast<uint32_t*>(lo)[i] = l;
  reinterpret_cast<uint32_t*>(hi)[i] = h;
}

__global__ void xor80_kernel(uint8_t* __restrict__ p, size_t n16) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n16) return;
  uint4 v = reinterpret_cast<uint4*>(p)[i];
  v.x ^= 0x80808080u; v.y ^= 0x80808080u; v.z ^= 0x80808080u; v.w ^= 0x80808080u;
  reinterpret_cast<uint4*>(p)[i] = v;
}

// One thread per (slot row, 4-coefficient block).  Slot s row r holds
// rotation rot_lo[s] + r of query slot_src[s] for r < n_rot[s]; other rows 0.
// mirror_flags bit s: use the mirrored query (already mirrored on the host).
__global__ void expand_slots_kernel(const uint16_t* __restrict__ base, uint32_t K, const QuerySlot* __restrict__ slots,
                                    uint32_t n_slots, uint32_t n_pad, uint8_t* __restrict__ lo,
                                    uint8_t* __restrict__ hi) {
  const uint32_t blocks_per_row = K / 4;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)n_pad * blocks_per_row;
  if (i >= total) return;
  const uint32_t row = (uint32_t)(i / blocks_per_row);
  const uint32_t b = (uint32_t)(i % blocks_per_row);
  const uint32_t s = row / kSlotRows, r = row % kSlotRows;
  uint32_t l = 0, h = 0;
  if (s < n_slots && r < slots[s].n_rot) {
    const QuerySlot sl = slots[s];
    const int rot = (int)sl.rot_lo + (int)r;  // index into all_rotations, 15 = centre
    const int left_blocks = 15 - rot;         // net left rotation in 4-coef blocks
    const uint32_t row800 = b / 200, col = b % 200;
    const uint32_t src_col = (uint32_t)(((int)col + left_blocks % 200 + 200) % 200);
    const uint16_t* src = base + (size_t)sl.src * K + (size_t)row800 * kRowLen + (size_t)src_col * 4;
    const uint2 v = *reinterpret_cast<const uint2*>(src);
    l = (v.x & 0xFFu) | ((v.x >> 8) & 0xFF00u) | ((v.y & 0xFFu) << 16) | ((v.y & 0xFF0000u) << 8);
    h = ((v.x >> 8) & 0xFFu) | ((v.x >> 16) & 0xFF00u) | ((v.y & 0xFF00u) << 8) | (v.y & 0xFF000000u);
  }
  reinterpret_cast<uint32_t*>(lo)[i] = l;
  reinterpret_cast<uint32_t*>(hi)[i] = h;
}

// One thread per (row, 4-coefficient block).  row_desc[r] = (src << 8) |
// mirror << 7 | rot puts rotation `rot` (0..30, 15 = centre) of base query
// `src` in row r, of its mirrored form when the mirror bit is set;
// 0xFFFFFFFF leaves the row zero.  Lets a batch pack queries with different
// rotation counts densely (no 32-row slot per query).
//
// Mirror (mirrored_code / mirrored_mask of the query share,
// iris-mpc-common/src/galois_engine.rs:218-225,520-543): 4-coefficient
// column c of each 800-coefficient row moves to 99 - c (c < 100) or 299 - c
// (c >= 100), and a code share's imaginary half (rows 8..15) is negated.
// The column map is its own inverse, so rotated row column `col` reads base
// column mirror((col + left) mod 200).
__global__ void expand_rows_kernel(const uint16_t* __restrict__ base, uint32_t K, const uint32_t* __restrict__ row_desc,
                                   uint32_t n_rows, uint32_t n_pad, uint8_t* __restrict__ lo, uint8_t* __restrict__ hi) {
  const uint32_t blocks_per_row = K / 4;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)n_pad * blocks_per_row) return;
  const uint32_t row = (uint32_t)(i / blocks_per_row);
  const uint32_t b = (uint32_t)(i % blocks_per_row);
  uint32_t l = 0, h = 0;
  const uint32_t d = row < n_rows ? row_desc[row] : 0xFFFFFFFFu;
  if (d != 0xFFFFFFFFu) {
    const uint32_t src = d >> 8, rot = d & 0x7Fu;
    const bool mirror = (d & 0x80u) != 0;
    const int left_blocks = 15 - (int)rot;
    const uint32_t row800 = b / 200, col = b % 200;
    uint32_t src_col = (uint32_t)(((int)col + left_blocks % 200 + 200) % 200);
    if (mirror) src_col = src_col < 100 ? 99 - src_col : 299 - src_col;
    uint2 v = *reinterpret_cast<const uint2*>(base + (size_t)src * K + (size_t)row800 * kRowLen + (size_t)src_col * 4);
    if (mirror && row800 >= 8) {  // imaginary half: only code shares reach it
      v.x = sub2(0u, v.x);
      v.y = sub2(0u, v.y);
    }
    l = (v.x & 0xFFu) | ((v.x >> 8) & 0xFF00u) | ((v.y & 0xFFu) << 16) | ((v.y & 0xFF0000u) << 8);
    h = ((v.x >> 8) & 0xFFu) | ((v.x >> 16) & 0xFF00u) | ((v.y & 0xFF00u) << 8) | (v.y & 0xFF000000u);
  }
  reinterpret_cast<uint32_t*>(lo)[i] = l;
  reinterpret_cast<uint32_t*>(hi)[i] = h;
}

// Copies DB rows ids[k] of (src_lo, src_hi) into rows k of (dst_lo, dst_hi),
// 16 bytes per thread (prefetch_subset, iris-mpc-gpu/src/dot/share_db.rs:344-407,
// done device-to-device because the DB is resident).
__global__ void gather_rows_kernel(const uint8_t* __restrict__ src_lo, const uint8_t* __restrict__ src_hi,
                                   const uint32_t* __restrict__ ids, uint32_t n, uint32_t K, uint8_t* __restrict__ dst_lo,
                                   uint8_t* __restrict__ dst_hi) {
  const uint32_t per_row = K / 16;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)n * per_row) return;
  const uint32_t k = (uint32_t)(i / per_row), c = (uint32_t)(i % per_row);
  const size_t s = (size_t)ids[k] * K + (size_t)c * 16, d = (size_t)k * K + (size_t)c * 16;
  *reinterpret_cast<uint4*>(dst_lo + d) = *reinterpret_cast<const uint4*>(src_lo + s);
  *reinterpret_cast<uint4*>(dst_hi + d) = *reinterpret_cast<const uint4*>(src_hi + s);
}

// ---------------- synthetic share database ----------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t rng64(uint64_t seed, uint64_t ctr) {
  return mix64(seed + (ctr + 1) * 0x9E3779B97F4A7C15ull);
}
__device__ __forceinline__ int remap_new_to_old(int i) {
  const int b = i / 6400, w = i % 6400 / 3200, r1 = i % 3200 / 800, c = i % 800 / 4, r2 = i % 4;
  return 800 * (r2 * 4 + r1) + c * 4 + w * 2 + b;
}
__device__ __forceinline__ void gr4_mul(const uint32_t a[4], const uint32_t b[4], uint32_t o[4]) {
  const uint32_t d4 = a[1] * b[3] + a[2] * b[2] + a[3] * b[1];
  const uint32_t d5 = a[2] * b[3] + a[3] * b[2];
  const uint32_t d6 = a[3] * b[3];
  o[0] = a[0] * b[0] + d4;
  o[1] = a[0] * b[1] + a[1] * b[0] + d4 + d5;
  o[2] = a[0] * b[2] + a[1] * b[1] + a[2] * b[0] + d5 + d6;
  o[3] = a[0] * b[3] + a[1] * b[2] + a[2] * b[1] + a[3] * b[0] + d6;
}

// One CTA per entry.  Mirrors the synthetic generator and the degree-1 Shamir
// encoding the CPU oracle defines (iris bits from rng64, mask pairs kept with
// probability 0.9, share randomness r = rng64(share seed, block)).
// Seeded uniform bytes (splitmix64 of the 8-byte word index): random shares
// for benchmark buffers whose values do not matter, only their bit activity.
__global__ void fill_random_kernel(uint64_t* __restrict__ p, size_t n_words, uint64_t seed) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_words; i += (size_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    p[i] = z ^ (z >> 31);
  }
}

__global__ void synth_db_kernel(uint64_t seed, uint32_t first, uint32_t count, SynthOut out) {
  __shared__ uint64_t code[200], mask[200];
  const uint32_t e = first + blockIdx.x;
  if (blockIdx.x >= count) return;
  const uint64_t s = mix64(seed ^ ((uint64_t)e * 0xD1B54A32D192ED03ull));
  for (int w = threadIdx.x; w < 200; w += blockDim.x) {
    code[w] = rng64(s, (uint64_t)w);
    uint64_t m = 0;
    for (int q = 0; q < 32; q++) {
      const int p = w * 32 + q;  // pair index
      const uint64_t r = rng64(s ^ 0x5bd1e995ull, (uint64_t)(p >> 1));
      const uint32_t v = (p & 1) ? (uint32_t)(r >> 32) : (uint32_t)r;
      if (v < 3865470566u) m |= 3ull << (2 * q);
    }
    mask[w] = m;
  }
  __syncthreads();
  const uint64_t share_seed = rng64(seed ^ 0x5EEDull, e);
  const uint32_t S[4][4] = {{1, 0, 0, 0}, {58082, 1, 0, 0}, {60579, 25194, 1, 0}, {17325, 51956, 57011, 1}};
  const uint32_t BP[3][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {1, 1, 0, 0}};
  for (int blk = threadIdx.x; blk < 3200; blk += blockDim.x) {
    const int i = blk * 4;
    uint32_t vc[4], vm[4];
    for (int k = 0; k < 4; k++) {
      const int o = remap_new_to_old(i + k);
      const uint32_t mb = (uint32_t)((mask[o >> 6] >> (o & 63)) & 1);
      const uint32_t cb = (uint32_t)((code[o >> 6] >> (o & 63)) & 1);
      vc[k] = (mb - 2u * (cb & mb)) & 0xFFFFu;
      vm[k] = mb;
    }
    for (int which = 0; which < 2; which++) {
      if (which == 1 && i >= kMaskCodeLength) break;  // trimmed mask
      const uint32_t* v = which == 0 ? vc : vm;
      uint32_t sm[4];
      for (int r = 0; r < 4; r++) sm[r] = S[r][0] * v[0] + S[r][1] * v[1] + S[r][2] * v[2] + S[r][3] * v[3];
      const uint64_t rr = rng64(which == 0 ? share_seed : (share_seed ^ 0xabcdef12345ull), (uint64_t)blk);
      const uint32_t rv[4] = {(uint32_t)(rr & 0xFFFF), (uint32_t)((rr >> 16) & 0xFFFF), (uint32_t)((rr >> 32) & 0xFFFF),
                              (uint32_t)(rr >> 48)};
      for (int p = 0; p < 3; p++) {
        uint32_t t[4];
        gr4_mul(rv, BP[p], t);
        uint32_t lo = 0, hi = 0;
        for (int k = 0; k < 4; k++) {
          const uint32_t x = (sm[k] + t[k]) & 0xFFFFu;
          lo |= (x & 0xFFu) << (8 * k);
          hi |= (x >> 8) << (8 * k);
        }
        const size_t K = which == 0 ? (size_t)kIrisCodeLength : (size_t)kMaskCodeLength;
        uint8_t* plo = which == 0 ? out.code_lo[p] : out.mask_lo[p];
        uint8_t* phi = which == 0 ? out.code_hi[p] : out.mask_hi[p];
        reinterpret_cast<uint32_t*>(plo + (size_t)e * K)[blk] = lo;
        reinterpret_cast<uint32_t*>(phi + (size_t)e * K)[blk] = hi;
      }
    }
  }
}

}  // namespace

cudaError_t launch_split_limbs(const uint16_t* in, uint8_t* lo, uint8_t* hi, size_t n, cudaStream_t stream) {
  if (n % 4) return cudaErrorInvalidValue;
  const size_t n4 = n / 4;
  if (!n4) return cudaSuccess;
  split_limbs_kernel<<<(unsigned)((n4 + 255) / 256), 256, 0, stream>>>(in, lo, hi, n4);
  return cudaGetLastError();
}

cudaError_t launch_xor80(uint8_t* p, size_t n, cudaStream_t stream) {
  if (n % 16) return cudaErrorInvalidValue;
  const size_t n16 = n / 16;
  if (!n16) return cudaSuccess;
  xor80_kernel<<<(unsigned)((n16 + 255) / 256), 256, 0, stream>>>(p, n16);
  return cudaGetLastError();
}

cudaError_t launch_expand_slots(const uint16_t* base, uint32_t K, const QuerySlot* slots, uint32_t n_slots,
                                uint32_t n_pad, uint8_t* lo, uint8_t* hi, cudaStream_t stream) {
  const size_t total = (size_t)n_pad * (K / 4);
  if (!total) return cudaSuccess;
  expand_slots_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(base, K, slots, n_slots, n_pad, lo, hi);
  return cudaGetLastError();
}

cudaError_t launch_expand_rows(const uint16_t* base, uint32_t K, const uint32_t* row_desc, uint32_t n_rows,
                               uint32_t n_pad, uint8_t* lo, uint8_t* hi, cudaStream_t stream) {
  const size_t total = (size_t)n_pad * (K / 4);
  if (!total) return cudaSuccess;
  expand_rows_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(base, K, row_desc, n_rows, n_pad, lo, hi);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const uint8_t* src_lo, const uint8_t* src_hi, const uint32_t* ids, uint32_t n,
                               uint32_t K, uint8_t* dst_lo, uint8_t* dst_hi, cudaStream_t stream) {
  const size_t total = (size_t)n * (K / 16);
  if (!total) return cudaSuccess;
  gather_rows_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(src_lo, src_hi, ids, n, K, dst_lo, dst_hi);
  return cudaGetLastError();
}

cudaError_t launch_fill_random(void* p, size_t bytes, uint64_t seed, cudaStream_t stream) {
  const size_t n = bytes / 8;
  if (n) {
    const size_t blocks = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
    fill_random_kernel<<<(unsigned)blocks, 256, 0, stream>>>(static_cast<uint64_t*>(p), n, seed);
  }
  return cudaGetLastError();
}

cudaError_t launch_synth_db(uint64_t seed, uint32_t first, uint32_t count, const SynthOut& out, cudaStream_t stream) {
  if (!count) return cudaSuccess;
  synth_db_kernel<<<count, 128, 0, stream>>>(seed, first, count, out);
  return cudaGetLastError();
}

}  // namespace irs
