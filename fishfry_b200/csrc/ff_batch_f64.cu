// FP64 batch pass kernels (ff_batch_dev.cuh).
#include "ff_batch_dev.cuh"

namespace ff {
FF_INSTANTIATE_BATCH(double)
}  // namespace ff
