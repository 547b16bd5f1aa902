// Launch interface of the MPC OR tree (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"

namespace irs {

struct OrTreeParams {
  ChaChaKey key[3];           // stream p = party p's own seed
  uint64_t nonce;             // nonce_of(kDomOrTree, device)
  uint64_t batch;
  const uint64_t* batch_dev;  // when set, the batch id is read from device memory
};

// OR of every bit of n_words 32-bit words of a shared bit vector, given the
// three components comp[p * n_words + w] (party p's a-share of word w).
// scratch: 2 * 3 * n_words words; out4 (device): the three components of the
// OR bit (bit 0) and the opened bit.
cudaError_t launch_or_tree(const OrTreeParams& P, const uint32_t* comp, size_t n_words, uint32_t* scratch,
                           uint32_t* out4, cudaStream_t stream);

}  // namespace irs
