// MPC OR tree over a shared bit vector (or_reduce_result / or_tree_on_gpu,
// iris-mpc-gpu/src/threshold_ring/protocol.rs:2363-2515): the three parties
// reduce all bits of a replicated-shared vector to one shared bit by AND gates
// on their own views (OR(x, y) = x ^ y ^ (x & y)), then open it.
//
// Tree shape (the reference's): at each level the first half of the words is
// combined with the second half, word i with word i + num, and an odd last
// word moves down; after the word tree, the 32 bits of the last word are
// collapsed with shifted copies of itself (16, 8, 4, 2, 1).  One launch per
// level, ping-ponging between two scratch vectors.
//
// Randomness of the AND gate of level L, index i: word 0 of the ChaCha12 block
// at counter (batch << 40) | (L << 34) | i of each party's stream, nonce
// domain 4; party p's mask is k_p ^ k_{p-1} (zero-sharing).  Word levels are
// 1.., the collapse steps 40..44.
#include <cuda_runtime.h>
#include <stdint.h>
#include "or_tree.h"

namespace irs {

namespace {

__device__ __forceinline__ void or_gate(uint32_t x[3], const uint32_t y[3], const OrTreeParams& P, uint64_t gate) {
  const uint64_t batch = P.batch_dev ? *P.batch_dev : P.batch;
  uint32_t k[3];
#pragma unroll 1
  for (int s = 0; s < 3; s++) {
    uint32_t blk[16];
    chacha_block<12>(P.key[s], counter_of(batch, gate), P.nonce, blk);
    k[s] = blk[0];
  }
  uint32_t z[3];
#pragma unroll
  for (int p = 0; p < 3; p++) {
    const int q = (p + 2) % 3;  // party p views (component p, component p-1)
    z[p] = (x[p] & y[p]) ^ (x[q] & y[p]) ^ (x[p] & y[q]) ^ (k[p] ^ k[q]);
  }
#pragma unroll
  for (int p = 0; p < 3; p++) x[p] = x[p] ^ y[p] ^ z[p];
}

__global__ void or_level_kernel(const uint32_t* __restrict__ in, uint64_t in_stride, uint32_t* __restrict__ out,
                                uint64_t out_stride, uint64_t num, int odd, uint32_t level, const OrTreeParams P) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < num) {
    uint32_t x[3], y[3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      x[p] = in[p * in_stride + i];
      y[p] = in[p * in_stride + i + num];
    }
    or_gate(x, y, P, ((uint64_t)level << 34) | i);
#pragma unroll
    for (int p = 0; p < 3; p++) out[p * out_stride + i] = x[p];
  } else if (odd && i == num) {
#pragma unroll
    for (int p = 0; p < 3; p++) out[p * out_stride + num] = in[p * in_stride + 2 * num];
  }
}

__global__ void or_collapse_kernel(const uint32_t* __restrict__ in, uint64_t stride, uint32_t* __restrict__ out4,
                                   const OrTreeParams P) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t x[3] = {in[0], in[stride], in[2 * stride]};
  int j = 0;
  for (int s = 16; s >= 1; s >>= 1, j++) {
    const uint32_t y[3] = {x[0] >> s, x[1] >> s, x[2] >> s};
    or_gate(x, y, P, (uint64_t)(40 + j) << 34);
  }
  out4[0] = x[0] & 1u;
  out4[1] = x[1] & 1u;
  out4[2] = x[2] & 1u;
  out4[3] = (x[0] ^ x[1] ^ x[2]) & 1u;
}

}  // namespace

cudaError_t launch_or_tree(const OrTreeParams& P, const uint32_t* comp, size_t n_words, uint32_t* scratch,
                           uint32_t* out4, cudaStream_t stream) {
  if (n_words == 0) return cudaErrorInvalidValue;
  const uint32_t* cur = comp;
  uint64_t cur_stride = n_words;
  uint32_t* bufs[2] = {scratch, scratch + 3 * n_words};
  int which = 0;
  uint64_t num = n_words;
  uint32_t level = 1;
  while (num > 1) {
    const int odd = (int)(num & 1);
    num >>= 1;
    const uint64_t threads = num + (uint64_t)odd;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    or_level_kernel<<<grid, 256, 0, stream>>>(cur, cur_stride, bufs[which], n_words, num, odd, level, P);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cur = bufs[which];
    cur_stride = n_words;
    which ^= 1;
    num += (uint64_t)odd;
    level++;
  }
  or_collapse_kernel<<<1, 32, 0, stream>>>(cur, cur_stride, out4, P);
  return cudaGetLastError();
}

}  // namespace irs
