// MIXED instantiation: FP64 positions and cell offsets, FP32 weights and
// packed FP32 sums.  Departure winds are stored as three component planes
// (ADZ_MIXED_SOA in adz_kernels.cuh).  Block shapes and resident blocks per
// SM were picked by timing the 1024x1024x80 step:
//   trajectory  tiles of 32 i by 4 levels, 7 blocks of 128 threads: 9.54 ms
//               (6, 8, 9 blocks: 9.84, 9.72, 10.42; 128 i of one level at
//               8 blocks: 10.31 ms; 64 x 2: 10.00; 32 x 8 in blocks of 256
//               threads at 3, 4 blocks: 9.89, 9.60; 32 x 16 at 2: 10.05;
//               16 x 8: 11.85);
//   sets        tiles of 32 i by 4 levels, 9 blocks: 10.83 ms against 11.35
//               for 128 i of one level in (i, k, j) order in the same runs
//               (8 blocks on tiles: 11.27).  The tile index is 32-bit
//               arithmetic: with 64-bit indices the kernel spilled 144 bytes
//               at the 56 registers of 9 blocks and took 12.51 ms; blocks of
//               2 rows of such tiles (256 threads) at 4, 5 blocks: 11.75, 12.56;
#define ADZ_SET_TILE_K 4
//   BICUBH_QV   5 blocks (96 registers, no spills; 27.4 ms for 8 tracers at
//               the unbounded 128 registers, 21.4 ms at 5 or 6 blocks, 24.8
//               ms at 8, before the (i, k, j) order).
#define ADZ_TRAJ_TILE_K 4
#define ADZ_TRAJ_MINB 7
#define ADZ_SET_MINB 9
#define ADZ_QV_MINB 5
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kMixed)
}  // namespace adz
