// Per-device launch attributes of the kernels that need more than 48 KB of
// dynamic shared memory.
#pragma once
#include <atomic>
#include <stdint.h>
#include <cuda_runtime.h>

namespace irs {

// Raises `kernel`'s dynamic shared memory limit to `bytes` on the current
// device, once per device: a function attribute belongs to the device's
// context, so a process that drives several GPUs sets it on each.  `done`
// holds one bit per device ordinal (ordinals >= 64 set it on every call).
template <class K>
cudaError_t smem_limit_once(K kernel, int bytes, std::atomic<uint64_t>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

}  // namespace irs
