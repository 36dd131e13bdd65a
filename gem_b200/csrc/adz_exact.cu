// REF32 and FP64 instantiations.  Built with -fmad=false: the only fused
// multiply-adds are the explicit fma() calls that mirror the reference build.
#include "adz_kernels.cuh"

namespace adz {
ADZ_INSTANTIATE(kRef32)
ADZ_INSTANTIATE(kFp64)
}  // namespace adz
