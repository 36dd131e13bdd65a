// MIXED instantiation: FP64 positions and cell offsets, FP32 weights and
// packed FP32 sums.  Departure winds are stored as three component planes
// (ADZ_MIXED_SOA in adz_kernels.cuh).  Block shapes and resident blocks per
// SM were picked by timing the 1024x1024x80 step:
//   trajectory  tiles of 32 i by 4 levels, 7 blocks of 128 threads: 9.54 ms
//               (6, 8, 9 blocks: 9.84, 9.72, 10.42; 128 i of one level at
//               8 blocks: 10.31 ms; 64 x 2: 10.00; 32 x 8 in blocks of 256
//               threads at 3, 4 blocks: 9.89, 9.60; 32 x 16 at 2: 10.05;
//               16 x 8: 11.85);
//   sets        128 i of one level, points in (i, k, j) order, 9 blocks:
//               11.25 ms (8, 10 blocks: 11.8, 13.0; 32 x 4 tiles at 8, 9, 10
//               blocks: 11.41, 12.51, 12.40; 64 x 2 at 8, 9: 11.53, 12.62);
//   BICUBH_QV   5 blocks (96 registers, no spills; 27.4 ms for 8 tracers at
//               the unbounded 128 registers, 21.4 ms at 5 or 6 blocks, 24.8
//               ms at 8, before the (i, k, j) order).
#define ADZ_TRAJ_TILE_K 4
#define ADZ_SET_TILE_K 1
#define ADZ_TRAJ_MINB 7
#define ADZ_SET_MINB 9
#define ADZ_QV_MINB 5
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kMixed)
}  // namespace adz
