// Launch interface of the data-preparation kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace irs {

// One 32-row query slot: rows 0..n_rot-1 hold rotations rot_lo..rot_lo+n_rot-1
// (indices into all_rotations(), 15 = centre) of base query `src`.
struct QuerySlot {
  uint32_t src;
  uint32_t rot_lo;
  uint32_t n_rot;
  uint32_t query;  // output query index (bitmap row) the slot reports to
};

struct SynthOut {
  uint8_t* code_lo[3];
  uint8_t* code_hi[3];
  uint8_t* mask_lo[3];
  uint8_t* mask_hi[3];
};

cudaError_t launch_split_limbs(const uint16_t* in, uint8_t* lo, uint8_t* hi, size_t n, cudaStream_t stream);
cudaError_t launch_xor80(uint8_t* p, size_t n, cudaStream_t stream);
cudaError_t launch_expand_slots(const uint16_t* base, uint32_t K, const QuerySlot* slots, uint32_t n_slots,
                                uint32_t n_pad, uint8_t* lo, uint8_t* hi, cudaStream_t stream);
cudaError_t launch_expand_rows(const uint16_t* base, uint32_t K, const uint32_t* row_desc, uint32_t n_rows,
                               uint32_t n_pad, uint8_t* lo, uint8_t* hi, cudaStream_t stream);
cudaError_t launch_gather_rows(const uint8_t* src_lo, const uint8_t* src_hi, const uint32_t* ids, uint32_t n,
                               uint32_t K, uint8_t* dst_lo, uint8_t* dst_hi, cudaStream_t stream);
cudaError_t launch_fill_random(void* p, size_t bytes, uint64_t seed, cudaStream_t stream);
cudaError_t launch_synth_db(uint64_t seed, uint32_t first, uint32_t count, const SynthOut& out, cudaStream_t stream);

}  // namespace irs
