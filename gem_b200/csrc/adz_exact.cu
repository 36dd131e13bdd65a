// REF32 and FP64 instantiations.  Built with -fmad=false: the only fused
// multiply-adds are the explicit fma() calls that mirror the reference build.
// Both precisions run the trajectory and the sets on tiles of 32 i by 4
// levels: FP64 35.4 ms per 1024x1024x80 step (38.9 ms at 128 i of one level,
// 36.0 with sets of 64 x 2), REF32 26.8 ms (28.1 ms).  Resident blocks of 128
// threads: REF32 5 (trajectory) and 7 (sets), 96 and 72 registers (26.77 ms;
// 6 and 7: 27.00, 5 and 6: 27.40, 6 and 6: 27.63; 32.7 ms at ptxas's 96-98
// registers before the tiles); FP64 keeps ptxas's choice, 96 registers and 5
// blocks, in both (7 and 7: 1 % faster on momentum + 4 tracers but 9 %
// slower with 8 tracers; 7 and ptxas's: 5 % slower; 6 and 6: 1.5 % slower).
#define ADZ_TRAJ_TILE_K 4
#define ADZ_SET_TILE_K 4
#define ADZ_TRAJ_MINB_REF32 5
#define ADZ_SET_MINB_REF32 7
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kRef32)
ADZ_INSTANTIATE(kFp64)
}  // namespace adz
