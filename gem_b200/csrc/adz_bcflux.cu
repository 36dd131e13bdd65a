// LAM boundary fluxes for the Bermejo-Conde fixer.  Aranami et al. (2015)
// (B/adz_BC_LAM_Aranami_hlt.F90:18-236, masks of
// B/adz_BC_LAM_setup.F90:18-92): the masked copies of a
// tracer and the zeroing of the interpolated fluxes.  The interpolation
// between them is the set-t kernel over range b (adzc_bc_lam_flux).
//
// mask_o is 1 on the core (levels k0t..nk and, on each LAM edge the tile
// touches, the span inside its pilot zone); mask_i is 1 on the rest of the
// domain; both are 0 outside the domain.  They are functions of the global
// position, so a tile of a decomposition gets what the reference's halo
// exchange of the masks gives.  The copies select (mask ? value : 0), which
// is the reference's mask * value for finite values and 0 where the reference
// never writes.  Without a tracer the copies are the masks themselves, the
// PSADJ branch (B/adz_BC_LAM_Aranami_hlt.F90:84-101).
#include <cuda_runtime.h>

#include "adz_types.h"

namespace adz {
namespace bcflux {

__device__ __forceinline__ bool in_domain(const BcMask& m, int i, int j) {
  return (!m.west || i >= 1) && (!m.east || i <= m.ni) && (!m.south || j >= 1) && (!m.north || j <= m.nj);
}
__device__ __forceinline__ bool in_core(const BcMask& m, int i, int j, int k) {
  const bool cx = (!m.west || i >= 1 + m.pil_w) && (!m.east || i <= m.ni - m.pil_e);
  const bool cy = (!m.south || j >= 1 + m.pil_s) && (!m.north || j <= m.nj - m.pil_n);
  return cx && cy && k >= m.k0t;
}

template <typename T>
__global__ void __launch_bounds__(256) k_bc_mask(BcMask m, const T* __restrict__ src, T* __restrict__ mo,
                                                 T* __restrict__ mi) {
  const long long plane = (long long)m.nit * m.njt, n = plane * m.nk;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = m.lminx + (int)(e % m.nit), j = m.lminy + (int)((e / m.nit) % m.njt), k = 1 + (int)(e / plane);
    const bool dom = in_domain(m, i, j), core = dom && in_core(m, i, j, k);
    const T v = src ? src[e] : (T)1;  // no tracer: the masks themselves (PSADJ)
    mo[e] = core ? v : (T)0;
    mi[e] = (dom && !core) ? v : (T)0;
  }
}

// FLUX_out = 0 on the core; FLUX_in = 0 on the pilot zones (levels k0t..nk)
// and above k0t on range b (B/adz_BC_LAM_Aranami_hlt.F90:160-226)
template <typename T>
__global__ void __launch_bounds__(256) k_bc_zero(BcMask m, T* __restrict__ fo, T* __restrict__ fi) {
  const long long plane = (long long)m.ni * m.nj, n = plane * m.nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % m.ni), j = 1 + (int)((t / m.ni) % m.nj), k = 1 + (int)(t / plane);
    const long long e = (long long)(i - m.lminx) + (long long)(j - m.lminy) * m.nit + (long long)(k - 1) * m.nit * m.njt;
    if (k >= m.k0t) {
      if (j >= 1 + m.pil_s && j <= m.nj - m.pil_n && i >= 1 + m.pil_w && i <= m.ni - m.pil_e) fo[e] = (T)0;
      if ((m.north && j >= m.nj - m.pil_n + 1) || (m.east && i >= m.ni - m.pil_e + 1) || (m.south && j <= m.pil_s) ||
          (m.west && i <= m.pil_w))
        fi[e] = (T)0;
    } else if (i >= m.i0b && i <= m.inb && j >= m.j0b && j <= m.jnb) {
      fi[e] = (T)0;
    }
  }
}

// adz_BC_LAM_zlf_hlt (B/adz_BC_LAM_zlf_hlt.F90:18-319) on the tile's
// interior 1..ni x 1..nj x 1..nk, each cell by the region it lies in:
//   setup 1  F1 = 0 outside the core widened by ext on the LAM edges the tile
//            touches, and below level nint(k0t/2) inside it (the source);
//   setup 2  F2 = F1 outside the core and below level k0t inside it (keep
//            the piloting values of the destination);
//   setup 3  F1 = 0 outside the BCS_BASE (4) extension on the LAM edges;
//   setup 4  F1 = F2 on the region of setup 2 (restore the piloting values).
// The edge tests use the tile's own pilot widths as the reference does.
template <typename T>
__global__ void __launch_bounds__(256) k_bc_zlf(BcMask m, int setup, ZlfPtrs f) {
  const long long plane = (long long)m.ni * m.nj, n = plane * m.nk;
  const int k0 = m.k0t, k0d2 = (k0 + 1) / 2;  // nint(k0/2.) for k0 >= 1
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % m.ni), j = 1 + (int)((t / m.ni) % m.nj), k = 1 + (int)(t / plane);
    const long long e = (long long)(i - m.lminx) + (long long)(j - m.lminy) * m.nit + (long long)(k - 1) * m.nit * m.njt;
    bool hit;
    if (setup == 1) {
      const int i0e = 1 + m.pil_w - m.ext * m.west, ine = m.ni - m.pil_e + m.ext * m.east;
      const int j0e = 1 + m.pil_s - m.ext * m.south, jne = m.nj - m.pil_n + m.ext * m.north;
      hit = (m.west && i <= i0e - 1) || (m.east && i >= ine + 1) || (m.south && j <= j0e - 1) ||
            (m.north && j >= jne + 1) || (i >= i0e && i <= ine && j >= j0e && j <= jne && k <= k0d2 - 1);
    } else if (setup == 3) {
      const int bcs = 4;
      hit = (m.west && i <= bcs * m.west) || (m.east && i >= m.ni - bcs * m.east + 1) ||
            (m.south && j <= bcs * m.south) || (m.north && j >= m.nj - bcs * m.north + 1);
    } else {  // setups 2 and 4: outside the core, or below k0t inside it
      const int i0c = 1 + m.pil_w, inc = m.ni - m.pil_e, j0c = 1 + m.pil_s, jnc = m.nj - m.pil_n;
      hit = (m.west && i <= i0c - 1) || (m.east && i >= inc + 1) || (m.south && j <= j0c - 1) ||
            (m.north && j >= jnc + 1) || (i >= i0c && i <= inc && j >= j0c && j <= jnc && k <= k0 - 1);
    }
    if (!hit) continue;
    for (int q = 0; q < f.n; q++) {
      T* f1 = (T*)f.f1[q];
      if (setup == 1 || setup == 3) f1[e] = (T)0;
      else if (setup == 2) ((T*)f.f2[q])[e] = f1[e];
      else f1[e] = ((const T*)f.f2[q])[e];
    }
  }
}

inline int grid_of(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148LL * 32 ? 148LL * 32 : b));
}

}  // namespace bcflux

template <typename T>
cudaError_t launch_bc_mask(const BcMask& m, const void* src, void* mo, void* mi, cudaStream_t s) {
  const long long n = (long long)m.nit * m.njt * m.nk;
  bcflux::k_bc_mask<T><<<bcflux::grid_of(n), 256, 0, s>>>(m, (const T*)src, (T*)mo, (T*)mi);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_bc_zero(const BcMask& m, void* fo, void* fi, cudaStream_t s) {
  const long long n = (long long)m.ni * m.nj * m.nk;
  bcflux::k_bc_zero<T><<<bcflux::grid_of(n), 256, 0, s>>>(m, (T*)fo, (T*)fi);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_bc_zlf(const BcMask& m, int setup, const ZlfPtrs& f, cudaStream_t s) {
  const long long n = (long long)m.ni * m.nj * m.nk;
  if (n <= 0 || f.n <= 0) return cudaSuccess;
  bcflux::k_bc_zlf<T><<<bcflux::grid_of(n), 256, 0, s>>>(m, setup, f);
  return cudaGetLastError();
}
template cudaError_t launch_bc_zlf<float>(const BcMask&, int, const ZlfPtrs&, cudaStream_t);
template cudaError_t launch_bc_zlf<double>(const BcMask&, int, const ZlfPtrs&, cudaStream_t);
template cudaError_t launch_bc_mask<float>(const BcMask&, const void*, void*, void*, cudaStream_t);
template cudaError_t launch_bc_mask<double>(const BcMask&, const void*, void*, void*, cudaStream_t);
template cudaError_t launch_bc_zero<float>(const BcMask&, void*, void*, cudaStream_t);
template cudaError_t launch_bc_zero<double>(const BcMask&, void*, void*, cudaStream_t);

}  // namespace adz
