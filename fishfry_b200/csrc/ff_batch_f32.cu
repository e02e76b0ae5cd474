// FP32 batch pass kernels (ff_batch_dev.cuh): butterflies and filter products
// in FP32; twiddles, wavenumbers and the filter's 1/k^2 formed in FP64.
#include "ff_batch_dev.cuh"

namespace ff {
FF_INSTANTIATE_BATCH(float)
}  // namespace ff
