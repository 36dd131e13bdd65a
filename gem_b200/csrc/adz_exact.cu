// REF32 and FP64 instantiations.  Built with -fmad=false: the only fused
// multiply-adds are the explicit fma() calls that mirror the reference build.
// REF32's gather kernels are built for 6 (trajectory) and 7 (sets) resident
// blocks of 128 threads, 80 and 72 registers with about 100 bytes of spill:
// 28.9 ms per 1024x1024x80 step against 32.7 ms at the 96-98 registers ptxas
// picks (6/6: 29.8 ms, 7/6: 29.7 ms).  FP64 keeps ptxas's choice (6/6 made it
// 1 % slower).
#define ADZ_TRAJ_MINB_REF32 6
#define ADZ_SET_MINB_REF32 7
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kRef32)
ADZ_INSTANTIATE(kFp64)
}  // namespace adz
