// compare_threshold_masked_many without any device allocation.
//
// Some callers cannot allocate device memory once they are running: a server
// that reserves all of HBM for the share database at start-up and runs inside
// a fixed budget, or a host runtime whose own stream-ordered allocator owns the
// device and forbids cudaMalloc/cudaMallocAsync from libraries.  The regular
// entry point draws its per-call scratch (the three parties' result components
// before they are split into each party's (a, b) share words) from a memory
// pool; this variant keeps that scratch in a file-scope device array instead.
//
// The array (kNoallocMaxElements / 32 words per party) is part of the library
// image: every GPU that loads the library holds it until the process exits.
// All calls share it and it keeps the last call's contents; the threshold
// kernel overwrites every word it later reads, so nothing needs clearing.
// Calls whose work overlaps on the GPU (different streams, or several host
// threads) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>

#include "../../include/irisb200.h"
#include "internal.h"
#include "threshold.h"

using namespace irs;

namespace {

constexpr size_t kNoallocMaxElements = IRS_NOALLOC_MAX_ELEMENTS;
constexpr size_t kNoallocWords = kNoallocMaxElements / 32;

// Per-word result components of the three parties: [3][kNoallocWords].
static __device__ __align__(256) uint32_t g_noalloc_comp[3 * kNoallocWords];

// Device addresses of g_noalloc_comp, per device.  A call made outside stream
// capture looks the address up afresh (cudaGetSymbolAddress is a table lookup,
// and a fresh lookup stays right after cudaDeviceReset has reloaded the
// module); a call inside a capture uses the address cached by the last call
// outside one, so the first call on a device must come before any capture.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_comp_ptr[kMaxDevices] = {};

// `device` is the current device.  Returns IRS_OK or an error status with the
// thread's last-error message set.
int comp_ptr_for(int device, bool capturing, uint32_t** out) {
  if (device < 0 || device >= kMaxDevices)
    return set_error(IRS_ERR_INVALID, "device ordinal %d is outside the %d devices the no-allocation entry point "
                     "supports", device, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_mu);
  if (capturing) {
    if (!g_comp_ptr[device])
      return set_error(IRS_ERR_STATE, "the first no-allocation call on device %d must come before any stream "
                       "capture (it resolves the scratch array's device address)", device);
    *out = g_comp_ptr[device];
    return IRS_OK;
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_comp);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return set_error(IRS_ERR_CUDA, "cudaGetSymbolAddress of the no-allocation scratch failed on device %d: %s",
                     device, cudaGetErrorString(e));
  }
  g_comp_ptr[device] = static_cast<uint32_t*>(p);
  *out = g_comp_ptr[device];
  return IRS_OK;
}

__global__ void noalloc_scatter_kernel(const uint32_t* comp, size_t n_words32, uint64_t* a0, uint64_t* a1,
                                       uint64_t* a2, uint64_t* b0, uint64_t* b1, uint64_t* b2, uint64_t* opened) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * i >= n_words32) return;
  const uint32_t* c0p = comp;
  const uint32_t* c1p = comp + n_words32;
  const uint32_t* c2p = comp + 2 * n_words32;
  const uint64_t c0 = (uint64_t)c0p[2 * i] | ((uint64_t)c0p[2 * i + 1] << 32);
  const uint64_t c1 = (uint64_t)c1p[2 * i] | ((uint64_t)c1p[2 * i + 1] << 32);
  const uint64_t c2 = (uint64_t)c2p[2 * i] | ((uint64_t)c2p[2 * i + 1] << 32);
  if (a0) a0[i] = c0;
  if (a1) a1[i] = c1;
  if (a2) a2[i] = c2;
  if (b0) b0[i] = c2;
  if (b1) b1[i] = c0;
  if (b2) b2[i] = c1;
  if (opened) opened[i] = c0 ^ c1 ^ c2;
}

}  // namespace

extern "C" int irs_circuits_compare_threshold_masked_many_noalloc(irs_circuits* c, const uint16_t* const code_a[3],
                                                                  const uint16_t* const mask_a[3], size_t n,
                                                                  uint32_t threshold_a, uint64_t* const res_a[3],
                                                                  uint64_t* const res_b[3], uint64_t* opened,
                                                                  void* stream) {
  CircuitView v;
  int rc = circuit_view(c, &v);
  if (rc) return rc;
  if (!code_a || !mask_a) return set_error(IRS_ERR_INVALID, "share pointers missing");
  if (n % 64) return set_error(IRS_ERR_INVALID, "n = %zu must be a multiple of 64", n);
  if (n > kNoallocMaxElements)
    return set_error(IRS_ERR_INVALID, "n = %zu exceeds the no-allocation limit of %zu elements", n,
                     kNoallocMaxElements);
  for (int p = 0; p < 3; p++) {
    if (!code_a[p] || !mask_a[p]) return set_error(IRS_ERR_INVALID, "share pointer of party %d missing", p);
    if (((uintptr_t)code_a[p] & 15) || ((uintptr_t)mask_a[p] & 15))
      return set_error(IRS_ERR_INVALID, "share pointers must be 16-byte aligned");
  }
  if (cudaSetDevice(v.device) != cudaSuccess) return set_error(IRS_ERR_CUDA, "cudaSetDevice(%d) failed", v.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : v.stream0;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();
    return set_error(IRS_ERR_CUDA, "cudaStreamIsCapturing failed");
  }
  uint32_t* comp = nullptr;
  rc = comp_ptr_for(v.device, cap != cudaStreamCaptureStatusNone, &comp);
  if (rc) return rc;
  if (n == 0) return IRS_OK;
  ThresholdParams P = {};
  for (int p = 0; p < 3; p++) {
    P.key[p] = v.keys[p];
    P.code[p] = code_a[p];
    P.mask[p] = mask_a[p];
  }
  P.nonce = v.nonce;
  P.batch = v.batch;
  P.batch_dev = v.batch_dev;
  P.threshold_a = threshold_a;
  P.n_words = n / 32;
  P.word_base = 0;
  // The flat kernel writes component p of word w at res_comp[p * n_words + w].
  P.res_comp = comp;
  cudaError_t e = launch_threshold_flat(P, kStageFull, s);
  if (e == cudaSuccess) {
    const size_t w64 = n / 64;
    noalloc_scatter_kernel<<<(unsigned)((w64 + 255) / 256), 256, 0, s>>>(
        comp, n / 32, res_a ? res_a[0] : nullptr, res_a ? res_a[1] : nullptr, res_a ? res_a[2] : nullptr,
        res_b ? res_b[0] : nullptr, res_b ? res_b[1] : nullptr, res_b ? res_b[2] : nullptr, opened);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return set_error(IRS_ERR_CUDA, "no-allocation threshold launch: %s", cudaGetErrorString(e));
  return IRS_OK;
}
