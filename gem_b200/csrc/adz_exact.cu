// REF32 and FP64 instantiations.  Built with -fmad=false: the only fused
// multiply-adds are the explicit fma() calls that mirror the reference build.
// REF32's gather kernels are built for 6 resident blocks of 128 threads (80
// registers, about 100 bytes of spill): 29.9 ms per 1024x1024x80 step against
// 32.7 ms at the 96-98 registers ptxas picks.  FP64 keeps ptxas's choice (the
// same budget made it 1 % slower).
#define ADZ_TRAJ_MINB_REF32 6
#define ADZ_SET_MINB_REF32 6
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kRef32)
ADZ_INSTANTIATE(kFp64)
}  // namespace adz
