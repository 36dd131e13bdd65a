// REF32 and FP64 instantiations.  Built with -fmad=false: the only fused
// multiply-adds are the explicit fma() calls that mirror the reference build.
// REF32's gather kernels are built for 6 (trajectory) and 7 (sets) resident
// blocks of 128 threads, 80 and 72 registers with about 100 bytes of spill
// (32.7 ms per 1024x1024x80 step at ptxas's 96-98 registers, 28.9 ms at
// 6/7, before the tiles); FP64 keeps ptxas's choice.  Both precisions run
// the trajectory and the sets on tiles of 32 i by 4 levels: FP64 35.6 ms
// per step (38.9 ms at 128 i of one level, 36.0 with sets of 64 x 2), REF32
// 27.3 ms (28.1 ms).
#define ADZ_TRAJ_TILE_K 4
#define ADZ_SET_TILE_K 4
#define ADZ_TRAJ_MINB_REF32 6
#define ADZ_SET_MINB_REF32 7
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kRef32)
ADZ_INSTANTIATE(kFp64)
}  // namespace adz
