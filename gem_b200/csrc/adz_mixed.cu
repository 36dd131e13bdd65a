// MIXED instantiation: FP64 positions and cell offsets, FP32 weights and
// packed FP32 sums.
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kMixed)
}  // namespace adz
