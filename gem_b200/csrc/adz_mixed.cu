// MIXED instantiation: FP64 positions and cell offsets, FP32 weights and
// packed FP32 sums.  Departure winds are stored as three component planes
// (ADZ_MIXED_SOA in adz_kernels.cuh).  Resident blocks per SM were picked by
// timing the 1024x1024x80 step (trajectory 7 blocks of 128 threads, sets 9,
// BICUBH_QV sets 5: 96 registers, no spills; 27.4 ms for 8 tracers at the
// unbounded 128 registers, 21.4 ms at 5 or 6 blocks, 24.8 ms at 8).
#define ADZ_TRAJ_MINB 7
#define ADZ_SET_MINB 9
#define ADZ_QV_MINB 5
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kMixed)
}  // namespace adz
