// Error plumbing shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/fishfry.h"

namespace ff {

// Records the message of the last failure on this thread and returns status.
int set_error(int status, const char *fmt, ...);

// Returns FF_ERR_CUDA with the call site if e != cudaSuccess.
#define FF_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return ::ff::set_error(FF_ERR_CUDA, "%s failed at %s:%d: %s (%s)", #call, __FILE__,   \
                             __LINE__, cudaGetErrorName(e_), cudaGetErrorString(e_));       \
  } while (0)

// Prime factors 2, 3, 5 only.
bool smooth235(int n);
// Prime factors 2, 3, 5 and 7 only (the radices of the FFT stages).
bool smooth2357(int n);

}  // namespace ff
