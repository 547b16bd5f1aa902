// Library-internal accessors shared between the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/irisb200.h"
#include "common.cuh"

namespace irs {

// What a kernel launch needs from an irs_circuits handle.
struct CircuitView {
  ChaChaKey keys[3];
  uint64_t nonce;
  uint64_t batch;
  const uint64_t* batch_dev;
  int device;
  cudaStream_t stream0;  // party 0's stream
};

// Fills `v` from `c`; returns IRS_ERR_INVALID (and sets the error) for NULL.
int circuit_view(irs_circuits* c, CircuitView* v);

// Sets the calling thread's last-error message and returns `code`.
int set_error(int code, const char* fmt, ...);

}  // namespace irs
