// Launch interface of the result-assembly kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace irs {

constexpr uint32_t kMaxMatchesLen = 256;

cudaError_t launch_compact(const uint32_t* bitmap, uint32_t n_queries, uint32_t db_len, uint32_t stride_words,
                           uint32_t* out, uint32_t* counter, uint32_t cap, cudaStream_t stream);
cudaError_t launch_merge_db(const uint32_t* left, const uint32_t* right, const uint32_t* or_policy, uint32_t n_queries,
                            uint32_t db_len, uint32_t stride_words, uint32_t* final_results, uint32_t* match_counter,
                            uint32_t* all_matches, cudaStream_t stream);
cudaError_t launch_merge_batch(const uint32_t* left, const uint32_t* right, uint32_t n_queries, uint32_t stride_words,
                               uint32_t* final_results, uint32_t* match_counter, uint32_t* all_matches,
                               cudaStream_t stream);

cudaError_t launch_take_rows(uint32_t* bitmap, uint32_t stride_words, const uint32_t* rows, uint32_t n_rows,
                             uint32_t db_len, int clear, uint32_t* counts, uint32_t* ids, uint32_t cap,
                             cudaStream_t stream);

}  // namespace irs
