// Kernels of the advection step, templated on the precision mode.
//
//   k_prepare      adz_prepareWinds departure winds (B/adz_prepareWinds.F90:16-107)
//   k_inittraj     adz_inittraj (B/adz_inittraj.F90:25-37)
//   k_traject      all Adz_niter fixed-point iterations of one arrival point in
//                  one thread, arrival winds formed in registers
//                  (B/adz_traject.F90:63-108, B/adz_prepareWinds.F90:40-97)
//   k_tricub_set   position of a set derived in registers (B/adz_interp_traj.F90)
//                  then the multi-field interpolation, mono bounds and clip
//                  (B/adz_interp_hlt.F90:98-182, B/adz_post_tr.F90:81-94)
//   k_interp_pos   the reference interpolators on explicit positions
//                  (B/turbo_tricublin.c:752-1312)
// B/ = src/gemdyn/src/base/.
#pragma once
#include "adz_device.cuh"
#include "adz_qv.cuh"

// launch bounds of the gather kernels (minimum resident blocks of 128 threads
// per SM; 0 lets ptxas choose).  A translation unit may set them before
// including this header; the _REF32 values apply to the REF32 instantiations
// (they default to the others).  The bounds expressions name PREC, the
// precision template parameter of every kernel that uses them.
// levels per block of the gather kernels: 1 walks the points in (i, k, j)
// order, 128 consecutive i per block; 2 or 4 gives every block a tile of
// 128/TK consecutive i by TK consecutive levels (one warp row per level)
#ifndef ADZ_TRAJ_TILE_K
#define ADZ_TRAJ_TILE_K 1
#endif
#ifndef ADZ_SET_TILE_K
#define ADZ_SET_TILE_K 1
#endif
#ifndef ADZ_TRAJ_MINB
#define ADZ_TRAJ_MINB 0
#endif
#ifndef ADZ_SET_MINB
#define ADZ_SET_MINB 0
#endif
#ifndef ADZ_TRAJ_MINB_REF32
#define ADZ_TRAJ_MINB_REF32 ADZ_TRAJ_MINB
#endif
#ifndef ADZ_SET_MINB_REF32
#define ADZ_SET_MINB_REF32 ADZ_SET_MINB
#endif
#define ADZ_TRAJ_BOUNDS __launch_bounds__(128, PREC == kRef32 ? ADZ_TRAJ_MINB_REF32 : ADZ_TRAJ_MINB)
// the tiled trajectory kernel may take wider blocks: ADZ_TRAJ_TILE_I
// consecutive i by ADZ_TRAJ_TILE_K levels, with its own resident-block budget
// (in blocks of that size)
#ifndef ADZ_TRAJ_TILE_I
#define ADZ_TRAJ_TILE_I (128 / ADZ_TRAJ_TILE_K)
#endif
#if ADZ_TRAJ_TILE_K > 1
#define ADZ_TRAJ_TILE_THREADS (ADZ_TRAJ_TILE_I * ADZ_TRAJ_TILE_K)
#else
#define ADZ_TRAJ_TILE_THREADS 128
#endif
#ifndef ADZ_TRAJ_TILE_MINB
#define ADZ_TRAJ_TILE_MINB ADZ_TRAJ_MINB
#endif
#ifndef ADZ_TRAJ_TILE_MINB_REF32
#define ADZ_TRAJ_TILE_MINB_REF32 ADZ_TRAJ_MINB_REF32
#endif
// the iteration to a tolerance (k_traject_tol) has its own resident-block
// budget and walks the trajectory's tiles of 32 i by 4 levels (ADZ_TOL_TILES
// 0: points in (i, k, j) order).  MIXED, 1024x1024x80 cold start to 1e-4:
// tiles at 7 blocks 13.26 ms against 14.82 ms in (i, k, j) order (204 bytes
// of spills there against 40); 6 and 5 blocks were slower either way
#ifndef ADZ_TOL_MINB
#define ADZ_TOL_MINB ADZ_TRAJ_MINB
#endif
#ifndef ADZ_TOL_TILES
#define ADZ_TOL_TILES 1
#endif
#define ADZ_TOL_BOUNDS __launch_bounds__(128, PREC == kRef32 ? ADZ_TRAJ_MINB_REF32 : ADZ_TOL_MINB)
#define ADZ_TRAJ_TILE_BOUNDS \
  __launch_bounds__(ADZ_TRAJ_TILE_THREADS, PREC == kRef32 ? ADZ_TRAJ_TILE_MINB_REF32 : ADZ_TRAJ_TILE_MINB)
#define ADZ_SET_BOUNDS __launch_bounds__(128, PREC == kRef32 ? ADZ_SET_MINB_REF32 : ADZ_SET_MINB)
// rows per block of the interleaved sets launch on tiles (blocks of
// 128 * ADZ_SET_TILE_J threads), with its own budget in such blocks
#ifndef ADZ_SET_TILE_J
#define ADZ_SET_TILE_J 1
#endif
#ifndef ADZ_PARTS_MINB
#define ADZ_PARTS_MINB ADZ_SET_MINB
#endif
#ifndef ADZ_PARTS_MINB_REF32
#define ADZ_PARTS_MINB_REF32 ADZ_SET_MINB_REF32
#endif
#define ADZ_PARTS_BOUNDS \
  __launch_bounds__(128 * ADZ_SET_TILE_J, PREC == kRef32 ? ADZ_PARTS_MINB_REF32 : ADZ_PARTS_MINB)
#ifndef ADZ_QV_MINB
#define ADZ_QV_MINB 0
#endif
// BICUBH_QV on tiles of 32 i by 4 levels (0: points in (i, k, j) order).
// MIXED, 8 tracers at 1024x1024x80, 5 blocks: 17.48 ms against 18.70 ms in
// (i, k, j) order (6 blocks on tiles: 17.64)
#ifndef ADZ_QV_TILES
#define ADZ_QV_TILES 1
#endif
#if ADZ_QV_MINB > 0
#define ADZ_QV_BOUNDS __launch_bounds__(128, ADZ_QV_MINB)
#else
#define ADZ_QV_BOUNDS __launch_bounds__(128)
#endif

// MIXED stores the departure winds as three component planes (u, v, w) instead
// of interleaved triplets: each component gather is then a run of consecutive
// floats across the warp's lanes, like a single field.
#ifndef ADZ_MIXED_SOA
#define ADZ_MIXED_SOA 1
#endif

namespace adz {

template <int PREC>
struct WindLayout {
  static constexpr bool soa = (PREC == kMixed) && (ADZ_MIXED_SOA != 0);
};

__device__ __forceinline__ long long ext_index(const DGrid& g, int i, int j, int k) {
  return (long long)(i - g.lminx) + (long long)(j - g.lminy) * g.nit + (long long)(k - 1) * g.nij;
}
__device__ __forceinline__ long long arr_index(const DGrid& g, int i, int j, int k) {
  return (long long)(i - 1) + (long long)(j - 1) * g.ni + (long long)(k - 1) * g.ni * g.nj;
}
__device__ __forceinline__ long long wp_index(const DGrid& g, int i, int j, int k, int c) {
  const long long nx = g.ni + 4, ny = g.nj + 4;
  return (long long)(i + 1) + (long long)(j + 1) * nx + (long long)(k - 1) * nx * ny +
         (long long)(c - 1) * nx * ny * g.nk;
}
__device__ __forceinline__ double dmin_(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax_(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ int imin_(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax_(int a, int b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// departure winds of one extended cell e (adz_prepareWinds.F90:26-97)
template <int PREC>
__device__ __forceinline__ void prepare_cell(const DGrid& g, const typename Types<PREC>::F* __restrict__ uu,
                                             const typename Types<PREC>::F* __restrict__ vv,
                                             const typename Types<PREC>::F* __restrict__ ww,
                                             typename Types<PREC>::F* __restrict__ uvw_d, long long e) {
  using F = typename Types<PREC>::F;
  const long long n = g.nij * g.nk;
  // the extended volume is below 2^31 cells (adzc_setup refuses larger tiles)
  const int k = (int)e / (int)g.nij + 1;
  const long long r = e - (long long)(k - 1) * g.nij;
  const int jj = (int)r / g.nit;
  const double cyj = __ldg(g.cy + jj);
  const double* vw = g.vw;
  const int nk = g.nk;
  const long long cu = WindLayout<PREC>::soa ? e : 3 * e;
  const long long cs = WindLayout<PREC>::soa ? n : 1;  // component stride
  uvw_d[cu] = (F)(g.inv_rayt * (double)uu[e] * cyj);
  uvw_d[cu + cs] = (F)(g.inv_rayt * (double)vv[e]);
  double w;
  if (k == 1) {
    w = g.vw5 * (double)ww[e];
  } else if (k == nk) {
    w = g.vw6 * (double)ww[e - g.nij];
  } else {
    const int km2 = imax_(1, k - 2);
    const double wx = (k >= 3) ? __ldg(vw + 0 * (nk + 1) + k) : 0.0;
    w = wx * (double)ww[r + (long long)(km2 - 1) * g.nij] + __ldg(vw + 1 * (nk + 1) + k) * (double)ww[e - g.nij] +
        __ldg(vw + 2 * (nk + 1) + k) * (double)ww[e] + __ldg(vw + 3 * (nk + 1) + k) * (double)ww[e + g.nij];
  }
  uvw_d[cu + 2 * cs] = (F)w;
}

// MIXED, component planes: four consecutive cells of a row per thread with
// 16-byte loads and stores (rows of a multiple of 4 cells, 16-byte aligned
// arrays; the launcher checks), the arithmetic of prepare_cell
template <int PREC>
__global__ void __launch_bounds__(256) k_prepare4(DGrid g, const float* __restrict__ uu, const float* __restrict__ vv,
                                                  const float* __restrict__ ww, float* __restrict__ uvw_d) {
  const int nit4 = g.nit >> 2, nk = g.nk;
  const int n4 = nit4 * g.njt * nk;
  const int nij = (int)g.nij;
  const long long n = g.nij * g.nk;
  const double* vw = g.vw;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += gridDim.x * blockDim.x) {
    const int row = t / nit4, c = t - row * nit4;
    const int k = row / g.njt + 1, jj = row - (k - 1) * g.njt;
    const int e = (k - 1) * nij + jj * g.nit + 4 * c;
    const double cyj = __ldg(g.cy + jj);
    const float4 u4 = *reinterpret_cast<const float4*>(uu + e);
    const float4 v4 = *reinterpret_cast<const float4*>(vv + e);
    const float u[4] = {u4.x, u4.y, u4.z, u4.w}, v[4] = {v4.x, v4.y, v4.z, v4.w};
    float ou[4], ov[4], ow[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      ou[q] = (float)(g.inv_rayt * (double)u[q] * cyj);
      ov[q] = (float)(g.inv_rayt * (double)v[q]);
    }
    if (k == 1) {
      const float4 w4 = *reinterpret_cast<const float4*>(ww + e);
      const float w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
      for (int q = 0; q < 4; q++) ow[q] = (float)(g.vw5 * (double)w[q]);
    } else if (k == nk) {
      const float4 w4 = *reinterpret_cast<const float4*>(ww + e - nij);
      const float w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
      for (int q = 0; q < 4; q++) ow[q] = (float)(g.vw6 * (double)w[q]);
    } else {
      const int km2 = imax_(1, k - 2);
      const double wx = (k >= 3) ? __ldg(vw + 0 * (nk + 1) + k) : 0.0;
      const double w1 = __ldg(vw + 1 * (nk + 1) + k), w2 = __ldg(vw + 2 * (nk + 1) + k);
      const double w3 = __ldg(vw + 3 * (nk + 1) + k);
      const int r = e - (k - 1) * nij;
      const float4 a4 = *reinterpret_cast<const float4*>(ww + r + (km2 - 1) * nij);
      const float4 b4 = *reinterpret_cast<const float4*>(ww + e - nij);
      const float4 c4 = *reinterpret_cast<const float4*>(ww + e);
      const float4 d4 = *reinterpret_cast<const float4*>(ww + e + nij);
      const float a[4] = {a4.x, a4.y, a4.z, a4.w}, b[4] = {b4.x, b4.y, b4.z, b4.w};
      const float cc[4] = {c4.x, c4.y, c4.z, c4.w}, d[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
      for (int q = 0; q < 4; q++)
        ow[q] = (float)(wx * (double)a[q] + w1 * (double)b[q] + w2 * (double)cc[q] + w3 * (double)d[q]);
    }
    *reinterpret_cast<float4*>(uvw_d + e) = make_float4(ou[0], ou[1], ou[2], ou[3]);
    *reinterpret_cast<float4*>(uvw_d + n + e) = make_float4(ov[0], ov[1], ov[2], ov[3]);
    *reinterpret_cast<float4*>(uvw_d + 2 * n + e) = make_float4(ow[0], ow[1], ow[2], ow[3]);
  }
}

template <int PREC>
__global__ void __launch_bounds__(256) k_prepare(DGrid g, const typename Types<PREC>::F* __restrict__ uu,
                                                 const typename Types<PREC>::F* __restrict__ vv,
                                                 const typename Types<PREC>::F* __restrict__ ww,
                                                 typename Types<PREC>::F* __restrict__ uvw_d) {
  const long long n = g.nij * g.nk;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    prepare_cell<PREC>(g, uu, vv, ww, uvw_d, e);
}

// departure winds of the extended cells in columns [ci0, ci0+nci) and rows
// [cj0, cj0+ncj) of the extended array (0-based), every level: the strips of
// the halo frame once its values have arrived
template <int PREC>
__global__ void __launch_bounds__(256) k_prepare_box(DGrid g, const typename Types<PREC>::F* __restrict__ uu,
                                                     const typename Types<PREC>::F* __restrict__ vv,
                                                     const typename Types<PREC>::F* __restrict__ ww,
                                                     typename Types<PREC>::F* __restrict__ uvw_d, int ci0, int nci,
                                                     int cj0, int ncj) {
  const long long nbox = (long long)nci * ncj, n = nbox * g.nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int ci = ci0 + (int)(t % nci), cj = cj0 + (int)((t / nci) % ncj), k = (int)(t / nbox);
    prepare_cell<PREC>(g, uu, vv, ww, uvw_d, (long long)k * g.nij + (long long)cj * g.nit + ci);
  }
}

// ---------------------------------------------------------------------------
template <int PREC>
__global__ void __launch_bounds__(256) k_inittraj(DGrid g, float* __restrict__ pxyzm, double* __restrict__ wpxyz) {
  const long long n = (long long)g.ni * g.nj * (g.nk - g.k0m + 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.ni) + 1;
    const int j = (int)((t / g.ni) % g.nj) + 1;
    const int k = (int)(t / ((long long)g.ni * g.nj)) + g.k0m;
    const float x = (float)(i + g.i0g - 1), y = (float)(j + g.j0g - 1), z = (float)k;
    if (PREC == kRef32 && pxyzm) {
      const long long a = arr_index(g, i, j, k);
      pxyzm[3 * a] = x;
      pxyzm[3 * a + 1] = y;
      pxyzm[3 * a + 2] = z;
    }
    wpxyz[wp_index(g, i, j, k, 1)] = x;
    wpxyz[wp_index(g, i, j, k, 2)] = y;
    wpxyz[wp_index(g, i, j, k, 3)] = z;
  }
}

// vertical index search of adz_traject.F90:85-90 / zindx (adz_interp_traj.F90:193-203)
__device__ __forceinline__ int vsearch(double zv, const double* z, double ovdz, const int* tab, int pnz, double sig,
                                       int nk) {
  int kk1 = __double2int_rz((zv - __ldg(z)) * ovdz + 1.0);
  kk1 = imin_(imax_(1, kk1), pnz);
  kk1 = __ldg(tab + kk1 - 1);
  if (sig * zv > sig * __ldg(z + imin_(kk1 + 1, nk + 1))) kk1 = kk1 + 1;
  if (sig * zv < sig * __ldg(z + kk1)) kk1 = kk1 - 1;
  return kk1;
}

__device__ __forceinline__ double zindx_t(const DGrid& g, double posz) {
  posz = dmin_(dmax_(posz, g.zmin), g.zmax);
  int kk1 = vsearch(posz, g.zt, g.ovdzt, g.search_t, g.pnz_t, g.sig, g.nk);
  kk1 = imin_(g.nk + 1, imax_(0, kk1));
  const int nb = imax_(imin_(kk1, g.nk - 1), 1);
  return (posz - __ldg(g.zt + nb)) * __ldg(g.odelz_t + nb) + (double)nb;
}

// stencil of a cell (ix local, x as in the ext array) stays inside the array
__device__ __forceinline__ bool stencil_ok(const DGrid& g, int off) {
  // off = corner offset relative to cell (1,1,1): recover corner (i,j) in ext coords
  const long long e = (long long)off + ext_index(g, 1, 1, 1);
  const long long plane = g.nij;
  long long k = e >= 0 ? e / plane : -1;
  const long long r = e - k * plane;
  const int j = (int)(r / g.nit), i = (int)(r - (long long)j * g.nit);
  return e >= 0 && k >= 0 && k <= g.nk - 1 && i >= 0 && i + 3 < g.nit && j >= 0 && j + 3 < g.njt;
}

// ---------------------------------------------------------------------------
// arrival winds (adz_prepareWinds.F90:40-97); Fortran forms the two sums in ``real``
template <int PREC>
__device__ __forceinline__ void arrival_winds(const DGrid& g, const TrajArgs& a, int j, int k, long long e, double& ua,
                                              double& va, double& wa) {
  using F = typename Types<PREC>::F;
  const F* __restrict__ ut0 = (const F*)a.ut0;
  const F* __restrict__ vt0 = (const F*)a.vt0;
  const F* __restrict__ zdt0 = (const F*)a.zdt0;
  const int nk = g.nk;
  const double alpha1 = -1.0 / 16.0, alpha2 = 9.0 / 16.0;
  const double cyj = __ldg(g.cy + (j - g.lminy));
  const F u1 = ut0[e - 2] + ut0[e + 1], u2 = ut0[e] + ut0[e - 1];
  const F v1 = vt0[e - 2 * g.nit] + vt0[e + g.nit], v2 = vt0[e] + vt0[e - g.nit];
  double uad = ((double)u1 * alpha1 + (double)u2 * alpha2) * g.inv_rayt * cyj;
  double vad = ((double)v1 * alpha1 + (double)v2 * alpha2) * g.inv_rayt;
  double wad;
  if (k == 1) {
    wad = g.vw5 * (double)zdt0[e];
  } else if (k == nk) {
    wad = g.vw6 * (double)zdt0[e - g.nij];
  } else {
    const int km2 = imax_(1, k - 2);
    const double wx = (k >= 3) ? __ldg(g.vw + 0 * (nk + 1) + k) : 0.0;
    wad = wx * (double)zdt0[e - (long long)(k - km2) * g.nij] + __ldg(g.vw + 1 * (nk + 1) + k) * (double)zdt0[e - g.nij] +
          __ldg(g.vw + 2 * (nk + 1) + k) * (double)zdt0[e] + __ldg(g.vw + 3 * (nk + 1) + k) * (double)zdt0[e + g.nij];
  }
  if (PREC == kRef32) {  // Adz_uu_arr etc. are ``real``
    ua = (double)(float)uad; va = (double)(float)vad; wa = (double)(float)wad;
  } else {
    ua = uad; va = vad; wa = wad;
  }
}

// one fixed-point update (adz_traject.F90:66-110): departure winds at
// (px,py,pz), new departure point (xm, ym, w3) and the clipped start of the
// next update in (px,py,pz).  Returns 0, kErrHalo or kErrNonFinite.
// COH: the departure winds were written earlier in the same launch (batch)
template <int PREC, bool COH>
__device__ __forceinline__ int traj_update(const DGrid& g, const TrajArgs& a, int i, int j, int k, double ua,
                                           double va, double wa, double& px, double& py, double& pz, double& xm,
                                           double& ym, double& w3, double& wd) {
  using F = typename Types<PREC>::F;
  const F* __restrict__ uvw = (const F*)a.uvw_d;
  const long long e111 = ext_index(g, 1, 1, 1);
  const F* f3 = uvw + 3 * e111;
  const int nk = g.nk;
  double ud, vd;
  int off;
  if (PREC == kMixed) {
    WF w;
    coef_mixed(w, px, py, pz, g.tab_m);
    off = w.off;
    if (!stencil_ok(g, off)) return kErrHalo;
    if (WindLayout<PREC>::soa) {
      const long long ncell = g.nij * g.nk;
      const float* fu = (const float*)uvw + e111 + off;
      ud = interp1_mixed<COH>(fu, w, g.tab_m.ni, g.tab_m.nij);
      vd = interp1_mixed<COH>(fu + ncell, w, g.tab_m.ni, g.tab_m.nij);
      wd = interp1_mixed<COH>(fu + 2 * ncell, w, g.tab_m.ni, g.tab_m.nij);
    } else {
      float o[3];
      interp3_mixed<COH>((const float*)f3 + 3LL * off, w, g.tab_m.ni, g.tab_m.nij, o);
      ud = o[0]; vd = o[1]; wd = o[2];
    }
  } else {
    double c[20];
    int zl;
    if (PREC == kRef32) zl = coef_f32pos(c, off, (float)px, (float)py, (float)pz, g.tab_m);
    else zl = coef_f64pos(c, off, px, py, pz, g.tab_m);
    if (!stencil_ok(g, off)) return kErrHalo;
    double o[3];
    interp3_exact<F, COH>(f3 + 3LL * off, c, g.tab_m.ni, g.tab_m.nij, zl, o);
    if (PREC == kRef32) {  // Tricublin_zyx3_n returns ``real``
      ud = (double)(float)o[0]; vd = (double)(float)o[1]; wd = (double)(float)o[2];
    } else {
      ud = o[0]; vd = o[1]; wd = o[2];
    }
  }
  xm = (double)(i + g.i0g - 1) - (a.dt.dtD * ud + a.dt.dtA * ua) * g.inv_hx;
  ym = (double)(j + g.j0g - 1) - (a.dt.dtD * vd + a.dt.dtA * va) * g.inv_hy;
  const double pos = __ldg(g.zm + k) - a.dt.dtzD * wd - a.dt.dtzA * wa;
  const double zmv = dmin_(dmax_(pos, g.zmin), g.zmax);
  int kk1 = vsearch(zmv, g.zm, g.ovdzm, g.search_m, g.pnz_m, g.sig, nk);
  kk1 = imin_(nk + 1, imax_(0, kk1));
  const int nb = imax_(imin_(kk1, nk - 1), 1);
  w3 = (zmv - __ldg(g.zm + nb)) * __ldg(g.odelz_m + nb) + (double)nb;
  const double cx = dmin_(dmax_(xm, g.imnx), g.imxx);
  const double cyv = dmin_(dmax_(ym, g.imny), g.imxy);
  if (PREC == kRef32) {
    px = (float)cx; py = (float)cyv; pz = (float)w3;
  } else {
    px = cx; py = cyv; pz = w3;
  }
  if (!isfinite(xm) || !isfinite(ym) || !isfinite(w3)) return kErrNonFinite;
  return 0;
}

// starting position of a warm trajectory: the stored departure point, x and y
// clipped to the interpolation range
template <int PREC>
__device__ __forceinline__ void warm_start(const DGrid& g, const TrajArgs& a, int i, int j, int k, double& px,
                                           double& py, double& pz) {
  if (PREC == kRef32) {
    const long long ar = arr_index(g, i, j, k);
    px = a.pxyzm[3 * ar]; py = a.pxyzm[3 * ar + 1]; pz = a.pxyzm[3 * ar + 2];
  } else {
    px = dmin_(dmax_(a.wpxyz[wp_index(g, i, j, k, 1)], g.imnx), g.imxx);
    py = dmin_(dmax_(a.wpxyz[wp_index(g, i, j, k, 2)], g.imny), g.imxy);
    pz = a.wpxyz[wp_index(g, i, j, k, 3)];
  }
}

// bracketing coarse nodes and weight of coordinate i on an axis of n points
// with nodes at min(1 + s m, n), m = 0..nc-1
__device__ __forceinline__ void coarse_bracket(int i, int s, int n, int nc, int& m0, int& m1, float& w) {
  if (nc < 2) {
    m0 = m1 = 0;
    w = 0.0f;
    return;
  }
  m0 = (i - 1) / s;
  m0 = m0 > nc - 2 ? nc - 2 : m0;
  m1 = m0 + 1;
  const int x0 = 1 + s * m0, x1r = 1 + s * m1, x1 = x1r > n ? n : x1r;
  w = (float)(i - x0) / (float)(x1 - x0);
}

// start point from the coarse guess of the tolerance iteration: the
// displacement interpolated bilinearly, X - dx, Y - dy clipped as a warm
// start is, k - dz clipped to the levels
__device__ __forceinline__ void guess_start(const DGrid& g, const TrajArgs& a, const GuessStart& gs, int i, int j,
                                            int k, double& px, double& py, double& pz) {
  int mx0, mx1, my0, my1;
  float wx, wy;
  coarse_bracket(i, gs.stride, g.ni, gs.nxc, mx0, mx1, wx);
  coarse_bracket(j, gs.stride, g.nj, gs.nyc, my0, my1, wy);
  const long long base = (long long)(k - a.k00) * gs.nxc * gs.nyc;
  const float* c00 = gs.d + 3 * (base + (long long)my0 * gs.nxc + mx0);
  const float* c10 = gs.d + 3 * (base + (long long)my0 * gs.nxc + mx1);
  const float* c01 = gs.d + 3 * (base + (long long)my1 * gs.nxc + mx0);
  const float* c11 = gs.d + 3 * (base + (long long)my1 * gs.nxc + mx1);
  float d[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    // (1 - w) a + w b: exact at both nodes
    const float lo = fmaf(wx, __ldg(c10 + q), (1.0f - wx) * __ldg(c00 + q));
    const float hi = fmaf(wx, __ldg(c11 + q), (1.0f - wx) * __ldg(c01 + q));
    d[q] = fmaf(wy, hi, (1.0f - wy) * lo);
  }
  px = dmin_(dmax_((double)(i + g.i0g - 1) - (double)d[0], g.imnx), g.imxx);
  py = dmin_(dmax_((double)(j + g.j0g - 1) - (double)d[1], g.imny), g.imxy);
  const double z = (double)k - (double)d[2];
  pz = z < 1.0 ? 1.0 : (z > (double)g.nk ? (double)g.nk : z);
}

// store the departure point of (i,j,k) (adz_traject.F90:112-118)
template <int PREC>
__device__ __forceinline__ void traj_store(const DGrid& g, const TrajArgs& a, int i, int j, int k, double xm, double ym,
                                           double w3, double px, double py, double pz, double wd) {
  using F = typename Types<PREC>::F;
  a.wpxyz[wp_index(g, i, j, k, 1)] = xm;
  a.wpxyz[wp_index(g, i, j, k, 2)] = ym;
  a.wpxyz[wp_index(g, i, j, k, 3)] = w3;
  const long long ar = arr_index(g, i, j, k);
  if (PREC == kRef32) {
    a.pxyzm[3 * ar] = (float)px;
    a.pxyzm[3 * ar + 1] = (float)py;
    a.pxyzm[3 * ar + 2] = (float)pz;
  }
  ((F*)a.wdep)[ar] = (F)wd;
}

// ---------------------------------------------------------------------------
// COH: the departure winds were written earlier in the same launch (batch)
template <int PREC, bool COH = false>
__device__ __forceinline__ void traject_point(const DGrid& g, const TrajArgs& a, int i, int j, int k) {
  const long long e = ext_index(g, i, j, k);
  double ua, va, wa;
  arrival_winds<PREC>(g, a, j, k, e, ua, va, wa);
  double px, py, pz;
  if (a.cold) {
    px = (double)(i + g.i0g - 1); py = (double)(j + g.j0g - 1); pz = (double)k;
  } else {
    warm_start<PREC>(g, a, i, j, k, px, py, pz);
  }
  double xm = 0.0, ym = 0.0, w3 = 0.0, wlast = 0.0;
  int st = 0;
  for (int it = 0; it < a.niter; it++) {
    double wd;
    st = traj_update<PREC, COH>(g, a, i, j, k, ua, va, wa, px, py, pz, xm, ym, w3, wd);
    if (st) break;
    wlast = wd;
  }
  if (st) {
    raise_status(g.status, st);
    return;
  }
  if (a.niter > 0) traj_store<PREC>(g, a, i, j, k, xm, ym, w3, px, py, pz, wlast);
}

// Iterate to a convergence tolerance instead of a fixed count: stop once no
// coordinate of the clipped departure point moves by more than ``tol`` grid
// indices, after at most ``maxit`` updates.  The start is the arrival point
// (a.cold) or the stored point (a learned guess).  A guessed start that has
// not converged after ``maxit`` updates falls back to the plain iteration
// from the arrival point.  Per point: updates used (iters, saturating at 255;
// +128 when the fallback ran), and block sums into stats[0] updates,
// stats[1] fallbacks, stats[2] points not converged.
template <int PREC>
__device__ __forceinline__ void traject_point_tol(const DGrid& g, const TrajArgs& a, const GuessStart& gs, int i,
                                                  int j, int k, double tol, int maxit, unsigned char* iters,
                                                  unsigned long long* cnt) {
  const long long e = ext_index(g, i, j, k);
  double ua, va, wa;
  arrival_winds<PREC>(g, a, j, k, e, ua, va, wa);
  const double X = (double)(i + g.i0g - 1), Y = (double)(j + g.j0g - 1), Z = (double)k;
  double px, py, pz;
  if (a.cold) {
    px = X; py = Y; pz = Z;
  } else if (gs.d) {
    guess_start(g, a, gs, i, j, k, px, py, pz);
  } else {
    warm_start<PREC>(g, a, i, j, k, px, py, pz);
  }
  double xm = 0.0, ym = 0.0, w3 = 0.0, wlast = 0.0;
  int st = 0, used = 0, pass = a.cold ? 1 : 0;
  bool conv = false;
  for (;;) {
    for (int it = 0; it < maxit; it++) {
      const double qx = px, qy = py, qz = pz;
      double wd;
      st = traj_update<PREC, false>(g, a, i, j, k, ua, va, wa, px, py, pz, xm, ym, w3, wd);
      if (st) break;
      wlast = wd;
      used++;
      if (fabs(px - qx) <= tol && fabs(py - qy) <= tol && fabs(pz - qz) <= tol) {
        conv = true;
        break;
      }
    }
    if (st || conv || pass == 1) break;
    pass = 1;  // fallback: plain iteration from the arrival point
    cnt[1]++;
    px = X; py = Y; pz = Z;
  }
  cnt[0] += used;
  if (!conv) cnt[2]++;
  if (iters) iters[arr_index(g, i, j, k)] = (unsigned char)(imin_(used, 127) + ((pass == 1 && !a.cold) ? 128 : 0));
  if (st) {
    raise_status(g.status, st);
    return;
  }
  if (used > 0) traj_store<PREC>(g, a, i, j, k, xm, ym, w3, px, py, pz, wlast);
}

template <int PREC>
__global__ void ADZ_TRAJ_TILE_BOUNDS k_traject(DGrid g, TrajArgs a) {
#if ADZ_TRAJ_TILE_K > 1
  constexpr int TK = ADZ_TRAJ_TILE_K, TI = ADZ_TRAJ_TILE_I;
  const int nkp = g.nk - a.k00 + 1;
  const int nic = (g.ni + TI - 1) / TI, nkg = (nkp + TK - 1) / TK;
  const long long b = blockIdx.x;
  const int i = (int)(b % nic) * TI + (threadIdx.x % TI) + 1;
  const int k = (int)((b / nic) % nkg) * TK + (threadIdx.x / TI) + a.k00;
  const int j = (int)(b / ((long long)nic * nkg)) + 1;
  if (i > g.ni || k > g.nk || j > g.nj) return;
  traject_point<PREC>(g, a, i, j, k);
#else
  // points in (i, k, j) order: consecutive blocks walk the levels of one row,
  // so each source row stays in L2 while every level that reads it runs
  const int nkp = g.nk - a.k00 + 1;
  const long long nrow = (long long)g.ni * nkp;
  const long long n = nrow * g.nj;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.ni) + 1;
    const int k = (int)((t / g.ni) % nkp) + a.k00;
    const int j = (int)(t / nrow) + 1;
    traject_point<PREC>(g, a, i, j, k);
  }
#endif
}

// the trajectory of the points of a box of the tile (i0..i0+nx-1,
// j0..j0+ny-1, levels from k00), points in (i, k, j) order: the interior
// and the band of a schedule that overlaps the halo exchange
// TILED: one tile of 32 i by 4 levels per block (boxes that tiles cover with
// few idle lanes, as the interior), else points in (i, k, j) order (bands)
template <int PREC, bool TILED>
__global__ void ADZ_TRAJ_BOUNDS k_traject_box(DGrid g, TrajArgs a, int i0, int nx, int j0, int ny) {
  const int nkp = g.nk - a.k00 + 1;
  if (TILED) {
    const unsigned b = blockIdx.x;
    const unsigned nic = (unsigned)(nx + 31) / 32, nkg = (unsigned)(nkp + 3) / 4;
    const unsigned bj = b / nic;
    const int ii = (int)(b - bj * nic) * 32 + (int)(threadIdx.x % 32);
    const int kk = (int)(bj % nkg) * 4 + (int)(threadIdx.x / 32);
    const int jj = (int)(bj / nkg);
    if (ii < nx && kk < nkp && jj < ny) traject_point<PREC>(g, a, ii + i0, jj + j0, kk + a.k00);
    return;
  }
  const long long nrow = (long long)nx * nkp;
  const long long n = nrow * ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx) + i0;
    const int k = (int)((t / nx) % nkp) + a.k00;
    const int j = (int)(t / nrow) + j0;
    traject_point<PREC>(g, a, i, j, k);
  }
}

template <int PREC>
__global__ void ADZ_TOL_BOUNDS k_traject_tol(DGrid g, TrajArgs a, double tol, int maxit, unsigned char* iters,
                                             unsigned long long* stats, GuessStart gs) {
  unsigned long long cnt[3] = {0, 0, 0};
#if ADZ_TOL_TILES
  // one tile of 32 i by 4 levels per block, as in k_traject; lanes outside
  // the grid still take part in the reduction below
  {
    const int nkp = g.nk - a.k00 + 1;
    const int nic = (g.ni + 31) / 32, nkg = (nkp + 3) / 4;
    const long long b = blockIdx.x;
    const int i = (int)(b % nic) * 32 + (threadIdx.x % 32) + 1;
    const int k = (int)((b / nic) % nkg) * 4 + (threadIdx.x / 32) + a.k00;
    const int j = (int)(b / ((long long)nic * nkg)) + 1;
    if (i <= g.ni && k <= g.nk && j <= g.nj) traject_point_tol<PREC>(g, a, gs, i, j, k, tol, maxit, iters, cnt);
  }
#else
  // points in (i, k, j) order, as in k_traject
  const int nkp = g.nk - a.k00 + 1;
  const long long nrow = (long long)g.ni * nkp;
  const long long n = nrow * g.nj;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.ni) + 1;
    const int k = (int)((t / g.ni) % nkp) + a.k00;
    const int j = (int)(t / nrow) + 1;
    traject_point_tol<PREC>(g, a, gs, i, j, k, tol, maxit, iters, cnt);
  }
#endif
  if (stats) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      unsigned long long v = cnt[q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0 && v) atomicAdd(stats + q, v);
    }
  }
}

// ---------------------------------------------------------------------------
// position of arrival point (i,j,k) of a set, adz_interp_traj.F90:45-187
// CG: read the trajectory arrays through the coherent path (ld.global.ca), for a kernel that
// wrote them itself earlier in the same launch
template <typename T, bool CG>
__device__ __forceinline__ T ld_traj(const T* p) {
  if (CG) return __ldca(p);  // coherent (not the read-only path), L1-cached after the acquire
  return *p;
}

template <int PREC, bool CG = false>
__device__ __forceinline__ void set_position(const DGrid& g, const SetArgs& a, int set, int i, int j, int k, double& px,
                                             double& py, double& pz) {
  using F = typename Types<PREC>::F;
  const double aa = -0.0625, bb = 0.5625, half = 0.5;
  const double* W = a.wpxyz;
#define WPX(ii, jj, kk, cc) ld_traj<double, CG>(W + wp_index(g, ii, jj, kk, cc))
  if (set == 0) {
    if (PREC == kRef32) {
      const long long ar = arr_index(g, i, j, k);
      px = a.pxyzm[3 * ar]; py = a.pxyzm[3 * ar + 1]; pz = a.pxyzm[3 * ar + 2];
    } else {
      px = dmin_(dmax_(WPX(i, j, k, 1), g.imnx), g.imxx);
      py = dmin_(dmax_(WPX(i, j, k, 2), g.imny), g.imxy);
      pz = WPX(i, j, k, 3);
    }
    return;
  }
  if (set == 1 || set == 2) {
    const int di = (set == 1), dj = (set == 2);
    double c[3];
#pragma unroll
    for (int q = 1; q <= 3; q++)
      c[q - 1] = aa * (WPX(i - di, j - dj, k, q) + WPX(i + 2 * di, j + 2 * dj, k, q)) +
                 bb * (WPX(i, j, k, q) + WPX(i + di, j + dj, k, q));
    if (set == 1) c[0] = c[0] - 0.5;
    else c[1] = c[1] - 0.5;
    px = dmin_(dmax_(c[0], g.imnx), g.imxx);
    py = dmin_(dmax_(c[1], g.imny), g.imxy);
    pz = dmin_(dmax_(c[2], 0.0), (double)(g.nk + 1));
    return;
  }
  // set T: Adz_pb
  const F* wd = (const F*)a.wdep;
  const F* zd = (const F*)a.zdt0;
  const int nk = g.nk;
  const long long e = ext_index(g, i, j, k);
#define WD(kk) ld_traj<F, CG>(wd + arr_index(g, i, j, kk))
  double xt, yt, ztv;
  if (k >= imax_(a.k00, 2) && k <= nk - 2) {
    const double* vw = g.vw;
    const double w1 = __ldg(vw + 4 * (nk + 1) + k), w2 = __ldg(vw + 5 * (nk + 1) + k);
    const double w3 = __ldg(vw + 6 * (nk + 1) + k), w4 = __ldg(vw + 7 * (nk + 1) + k);
    xt = w1 * WPX(i, j, k - 1, 1) + w2 * WPX(i, j, k, 1) + w3 * WPX(i, j, k + 1, 1) + w4 * WPX(i, j, k + 2, 1);
    yt = w1 * WPX(i, j, k - 1, 2) + w2 * WPX(i, j, k, 2) + w3 * WPX(i, j, k + 1, 2) + w4 * WPX(i, j, k + 2, 2);
    const double wdt = w1 * (double)WD(k - 1) + w2 * (double)WD(k) + w3 * (double)WD(k + 1) + w4 * (double)WD(k + 2);
    ztv = __ldg(g.zt + k) - a.dt.dtzD * wdt - a.dt.dtzA * (double)zd[e];
  } else if (k == nk - 1) {
    xt = (WPX(i, j, k, 1) + WPX(i, j, k + 1, 1)) * half;
    yt = (WPX(i, j, k, 2) + WPX(i, j, k + 1, 2)) * half;
    const F ws = WD(k) + WD(k + 1);
    const double wdt = (double)ws * half;
    ztv = __ldg(g.zt + k) - a.dt.dtzD * wdt - a.dt.dtzA * (double)zd[e];
  } else if (k == nk) {
    if (g.slt_winds && a.uslt && a.vslt) {
      const long long a2 = (long long)(i - 1) + (long long)(j - 1) * g.ni;
      xt = (double)(i + g.i0g - 1) -
           g.inv_rayt * a.dt.dt * (double)((const F*)a.uslt)[a2] * __ldg(g.cy + (j - g.lminy)) * g.inv_hx;
      yt = (double)(j + g.j0g - 1) - g.inv_rayt * a.dt.dt * (double)((const F*)a.vslt)[a2] * g.inv_hy;
    } else {
      xt = g.wp * WPX(i, j, k, 1) + g.wm * WPX(i, j, k - 1, 1);
      yt = g.wp * WPX(i, j, k, 2) + g.wm * WPX(i, j, k - 1, 2);
    }
    const F ws = WD(k - 1) + WD(k);
    const double wdt = (double)ws * half;
    ztv = __ldg(g.zt + k) - g.ww * (a.dt.dtzD * wdt + a.dt.dtzA * (double)zd[e - g.nij]);
  } else {  // k == 1 (k00 == 1)
    xt = (WPX(i, j, 1, 1) + WPX(i, j, 2, 1)) * half;
    yt = (WPX(i, j, 1, 2) + WPX(i, j, 2, 2)) * half;
    const F ws = WD(1) + WD(2);
    const double wdt = (double)ws * half;
    ztv = __ldg(g.zt + 1) - a.dt.dtzD * wdt - a.dt.dtzA * (double)zd[e];
  }
#undef WD
#undef WPX
  px = dmin_(dmax_(xt, g.imnx), g.imxx);
  py = dmin_(dmax_(yt, g.imny), g.imxy);
  pz = zindx_t(g, ztv);
}

// the ensemble perturbation pattern mcrhsint(i, j) (adz_interp_hlt.F90:99,
// 125-133): dst = value + mcrhsint * |value - lin|, before any clip
template <typename T>
__device__ __forceinline__ T pert_at(const SetArgs& a, int i, int j) {
  return __ldg((const T*)a.pert + (long long)(i - 1) + (long long)(j - 1) * a.pert_ld);
}
__device__ __forceinline__ float fabs_(float x) { return fabsf(x); }
__device__ __forceinline__ double fabs_(double x) { return fabs(x); }

// PERT: the mcrhsint perturbation is set (a.pert); a separate instantiation,
// so the common path carries none of it
template <int PREC, bool CG = false, bool PERT = false>
__device__ __forceinline__ void set_point(const DGrid& g, int set, const SetArgs& a, const FieldPtrs& fp, int i,
                                          int j, int k) {
  using F = typename Types<PREC>::F;
  const DZtab& lv = (set == 3) ? g.tab_t : g.tab_m;
  const long long e111 = ext_index(g, 1, 1, 1);
  double px, py, pz;
  set_position<PREC, CG>(g, a, set, i, j, k, px, py, pz);
  const long long e = ext_index(g, i, j, k);
  if (PREC == kMixed) {
    WF w;
    coef_mixed(w, px, py, pz, lv);
    if (!stencil_ok(g, w.off)) { raise_status(g.status, kErrHalo); return; }
    for (int q = 0; q < fp.nf; q++) {
      const float* f = (const float*)fp.src[q] + e111 + w.off;
      if (((fp.mono_mask >> q) & 1u) || PERT) {
        float d, lin, mn, mx;
        interp_mono_mixed(f, w, lv.ni, lv.nij, d, lin, mn, mx);
        if (PERT) d = d + pert_at<float>(a, i, j) * fabsf(d - lin);
        if ((fp.clip_mask >> q) & 1u) d = fmaxf(mn, fminf(mx, d));
        if ((fp.mono_mask >> q) & 1u) {  // post arrays of mono fields
          if (fp.lin[q]) ((float*)fp.lin[q])[e] = fmaxf(mn, fminf(mx, lin));
          if (fp.mn[q]) ((float*)fp.mn[q])[e] = mn;
          if (fp.mx[q]) ((float*)fp.mx[q])[e] = mx;
        }
        ((float*)fp.dst[q])[e] = d;
      } else {
        ((float*)fp.dst[q])[e] = interp1_mixed(f, w, lv.ni, lv.nij);
      }
    }
  } else {
    double c[20];
    int off, zl;
    if (PREC == kRef32) zl = coef_f32pos(c, off, (float)px, (float)py, (float)pz, lv);
    else zl = coef_f64pos(c, off, px, py, pz, lv);
    if (!stencil_ok(g, off)) { raise_status(g.status, kErrHalo); return; }
    for (int q = 0; q < fp.nf; q++) {
      const F* f = (const F*)fp.src[q] + e111 + off;
      if (((fp.mono_mask >> q) & 1u) || PERT) {
        double d, lin, mn, mx;
        interp_mono_exact<F>(f, c, lv.ni, lv.nij, zl, fp.box222 != 0, d, lin, mn, mx);
        F df = (F)d, lf = (F)lin, mnf = (F)mn, mxf = (F)mx;
        // mcrhsint perturbation in the field type (adz_interp_hlt.F90:125-133)
        if (PERT) df = df + pert_at<F>(a, i, j) * fabs_(df - lf);
        // Adz_post lin/min/max (adz_interp_hlt.F90:156-158), clip of adz_post_tr.F90:86-89
        if ((fp.clip_mask >> q) & 1u) df = (mnf > ((mxf < df) ? mxf : df)) ? mnf : ((mxf < df) ? mxf : df);
        if ((fp.mono_mask >> q) & 1u) {  // post arrays of mono fields
          if (fp.lin[q]) ((F*)fp.lin[q])[e] = (mnf > ((mxf < lf) ? mxf : lf)) ? mnf : ((mxf < lf) ? mxf : lf);
          if (fp.mn[q]) ((F*)fp.mn[q])[e] = mnf;
          if (fp.mx[q]) ((F*)fp.mx[q])[e] = mxf;
        }
        ((F*)fp.dst[q])[e] = df;
      } else {
        ((F*)fp.dst[q])[e] = (F)interp1_exact<F>(f, c, lv.ni, lv.nij, zl);
      }
    }
  }
}

// the positions of a set as adz_interp_traj stores them (Adz_pm, Adz_pmu,
// Adz_pmv, Adz_pt: (3, nx, ny, nz), i fastest): FP32 (the reference's real
// arrays, the FP64 value rounded to nearest) in REF32, FP64 otherwise
template <int PREC>
__global__ void __launch_bounds__(256) k_positions(DGrid g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                                                   SetArgs a, void* __restrict__ pos) {
  const long long nplane = (long long)nx * ny;
  const long long n = nplane * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx) + i0;
    const int j = (int)((t / nx) % ny) + j0;
    const int k = (int)(t / nplane) + k0;
    double px, py, pz;
    set_position<PREC, false>(g, a, set, i, j, k, px, py, pz);
    if (PREC == kRef32) {
      float* o = (float*)pos + 3 * t;
      o[0] = (float)px;
      o[1] = (float)py;
      o[2] = (float)pz;
    } else {
      double* o = (double*)pos + 3 * t;
      o[0] = px;
      o[1] = py;
      o[2] = pz;
    }
  }
}

template <int PREC, bool PERT>
__global__ void ADZ_SET_BOUNDS k_tricub_set(DGrid g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                                            SetArgs a, FieldPtrs fp) {
#if ADZ_SET_TILE_K > 1
  // one tile of 128/TK i by TK levels per block, as in k_tricub_parts
  constexpr int TK = ADZ_SET_TILE_K, TI = 128 / TK;
  const unsigned b = blockIdx.x;
  const unsigned nic = (unsigned)(nx + TI - 1) / TI, nkg = (unsigned)(nz + TK - 1) / TK;
  const unsigned bj = b / nic;
  const int ii = (int)(b - bj * nic) * TI + (int)(threadIdx.x % TI);
  const int kk = (int)(bj % nkg) * TK + (int)(threadIdx.x / TI);
  const int jj = (int)(bj / nkg);
  if (ii >= nx || kk >= nz || jj >= ny) return;
  set_point<PREC, false, PERT>(g, set, a, fp, ii + i0, jj + j0, kk + k0);
#else
  // points in (i, k, j) order, as in k_traject
  const long long nrow = (long long)nx * nz;
  const long long n = nrow * ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx) + i0;
    const int k = (int)((t / nx) % nz) + k0;
    const int j = (int)(t / nrow) + j0;
    set_point<PREC, false, PERT>(g, set, a, fp, i, j, k);
  }
#endif
}

// the tricubic groups of several sets in one launch.  Consecutive blocks
// take consecutive parts (u, v, t ...), so every SM runs a mix of the
// issue-bound one-field sets and the load-bound multi-field set at once;
// each thread interpolates one arrival point of its part as k_tricub_set does
template <int PREC, bool PERT>
__global__ void ADZ_PARTS_BOUNDS k_tricub_parts(DGrid g, SetArgs a, const __grid_constant__ SetParts sp) {
  const int q = (int)(blockIdx.x % (unsigned)sp.n);
  const SetPart& P = sp.p[q];
#if ADZ_SET_TILE_K > 1
  // 32-bit tile arithmetic (the grid stays below 2^31 blocks): 64-bit
  // indices here cost registers the point code needs at 9 resident blocks
  constexpr int TK = ADZ_SET_TILE_K, TI = 128 / TK, TJ = ADZ_SET_TILE_J;
  const unsigned b = blockIdx.x / (unsigned)sp.n;
  const unsigned nic = (unsigned)(P.nx + TI - 1) / TI, nkg = (unsigned)(P.nz + TK - 1) / TK;
  const unsigned bj = b / nic, bk = bj % nkg;
  const int ii = (int)(b - bj * nic) * TI + (int)(threadIdx.x % TI);
  const int kk = (int)bk * TK + (int)((threadIdx.x / TI) % TK);
  const int jj = (int)(bj / nkg) * TJ + (int)(threadIdx.x / 128);
  if (ii >= P.nx || kk >= P.nz || jj >= P.ny) return;
  set_point<PREC, false, PERT>(g, P.set, a, P.fp, ii + P.i0, jj + P.j0, kk + P.k0);
#else
  const long long t = (long long)(blockIdx.x / (unsigned)sp.n) * blockDim.x + threadIdx.x;
  // points in (i, k, j) order, as in k_traject
  const long long nrow = (long long)P.nx * P.nz;
  if (t >= nrow * P.ny) return;
  const int i = (int)(t % P.nx) + P.i0;
  const int k = (int)((t / P.nx) % P.nz) + P.k0;
  const int j = (int)(t / nrow) + P.j0;
  set_point<PREC, false, PERT>(g, P.set, a, P.fp, i, j, k);
#endif
}

// BICUBH_QV fields at position set t (adz_interp_hlt.F90:113-116 with
// F_QV_L): lin/min/max of the inner 2x2x2 box always formed, written where
// asked; clip as adz_post_tr.F90:81-94
template <int PREC, bool PERT>
__device__ __forceinline__ void qv_point(const DGrid& g, const SetArgs& a, const FieldPtrs& fp, int i, int j, int k) {
  using F = typename Types<PREC>::F;
  double px, py, pz;
  set_position<PREC, false>(g, a, 3, i, j, k, px, py, pz);
  if (PREC == kRef32) {  // Adz_pt is ``real``
    px = (double)(float)px;
    py = (double)(float)py;
    pz = (double)(float)pz;
  }
  QvCoef c;
  qv_coef<PREC>(g, px, py, pz, c);
  if (!qv_stencil_ok(g, c)) {
    raise_status(g.status, kErrHalo);
    return;
  }
  const long long e = ext_index(g, i, j, k);
  const long long base = ext_index(g, 1, 1, 1) + c.off;
  if (PREC == kMixed) {
    QvCoefF w;
    qv_to_float(c, w);
    for (int q = 0; q < fp.nf; q++) {
      float d, lin, mn, mx;
      interp_qv_mixed((const float*)fp.src[q] + base, g.nit, g.nij, c, w, d, lin, mn, mx);
      if (PERT) d = d + pert_at<float>(a, i, j) * fabsf(d - lin);
      if ((fp.clip_mask >> q) & 1u) d = fmaxf(mn, fminf(mx, d));
      if (fp.lin[q]) ((float*)fp.lin[q])[e] = fmaxf(mn, fminf(mx, lin));
      if (fp.mn[q]) ((float*)fp.mn[q])[e] = mn;
      if (fp.mx[q]) ((float*)fp.mx[q])[e] = mx;
      ((float*)fp.dst[q])[e] = d;
    }
  } else {
    for (int q = 0; q < fp.nf; q++) {
      F d, lin, mn, mx;
      interp_qv_exact<F>((const F*)fp.src[q] + base, g.nit, g.nij, c, d, lin, mn, mx);
      if (PERT) d = d + pert_at<F>(a, i, j) * fabs_(d - lin);
      if ((fp.clip_mask >> q) & 1u) d = (mn > ((mx < d) ? mx : d)) ? mn : ((mx < d) ? mx : d);
      if (fp.lin[q]) ((F*)fp.lin[q])[e] = (mn > ((mx < lin) ? mx : lin)) ? mn : ((mx < lin) ? mx : lin);
      if (fp.mn[q]) ((F*)fp.mn[q])[e] = mn;
      if (fp.mx[q]) ((F*)fp.mx[q])[e] = mx;
      ((F*)fp.dst[q])[e] = d;
    }
  }
}

template <int PREC, bool PERT>
__global__ void ADZ_QV_BOUNDS k_qv_set(DGrid g, int i0, int nx, int j0, int ny, int k0, int nz, SetArgs a,
                                                FieldPtrs fp) {
#if ADZ_QV_TILES
  // one tile of 32 i by 4 levels per block, 32-bit tile arithmetic
  const unsigned b = blockIdx.x;
  const unsigned nic = (unsigned)(nx + 31) / 32, nkg = (unsigned)(nz + 3) / 4;
  const unsigned bj = b / nic;
  const int ii = (int)(b - bj * nic) * 32 + (int)(threadIdx.x % 32);
  const int kk = (int)(bj % nkg) * 4 + (int)(threadIdx.x / 32);
  const int jj = (int)(bj / nkg);
  if (ii >= nx || kk >= nz || jj >= ny) return;
  qv_point<PREC, PERT>(g, a, fp, ii + i0, jj + j0, kk + k0);
#else
  // points in (i, k, j) order, as in k_traject
  const long long nrow = (long long)nx * nz;
  const long long n = nrow * ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx) + i0;
    const int k = (int)((t / nx) % nz) + k0;
    const int j = (int)(t / nrow) + j0;
    qv_point<PREC, PERT>(g, a, fp, i, j, k);
  }
#endif
}

// ---------------------------------------------------------------------------
// explicit positions; kind 0 = cubic, 1 = mono, 2 = 3-component
template <int PREC, int KIND>
__global__ void __launch_bounds__(128) k_interp_pos(DZtab lv, int n, const void* __restrict__ pos, FieldPtrs fp) {
  using F = typename Types<PREC>::F;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const long long o = (long long)t * fp.ostride;
    if (PREC == kMixed) {
      const double* p = (const double*)pos + 3LL * t;
      WF w;
      coef_mixed(w, p[0], p[1], p[2], lv);
      if (KIND == 2) {
        float r[3];
        interp3_mixed((const float*)fp.src[0] + 3LL * w.off, w, lv.ni, lv.nij, r);
        float* d = (float*)fp.dst[0] + 3LL * t;
        d[0] = r[0]; d[1] = r[1]; d[2] = r[2];
      } else {
        for (int q = 0; q < fp.nf; q++) {
          const float* f = (const float*)fp.src[q] + w.off;
          if (KIND == 1) {
            float d, lin, mn, mx;
            interp_mono_mixed(f, w, lv.ni, lv.nij, d, lin, mn, mx);
            ((float*)fp.dst[q])[o] = d;
            ((float*)fp.lin[q])[o] = lin;
            ((float*)fp.mn[q])[o] = mn;
            ((float*)fp.mx[q])[o] = mx;
          } else {
            ((float*)fp.dst[q])[o] = interp1_mixed(f, w, lv.ni, lv.nij);
          }
        }
      }
    } else {
      double c[20];
      int off, zl;
      if (PREC == kRef32) {
        const float* p = (const float*)pos + 3LL * t;
        zl = coef_f32pos(c, off, p[0], p[1], p[2], lv);
      } else {
        const double* p = (const double*)pos + 3LL * t;
        zl = coef_f64pos(c, off, p[0], p[1], p[2], lv);
      }
      if (KIND == 2) {
        double r[3];
        interp3_exact<F>((const F*)fp.src[0] + 3LL * off, c, lv.ni, lv.nij, zl, r);
        F* d = (F*)fp.dst[0] + 3LL * t;
        d[0] = (F)r[0]; d[1] = (F)r[1]; d[2] = (F)r[2];
      } else {
        for (int q = 0; q < fp.nf; q++) {
          const F* f = (const F*)fp.src[q] + off;
          if (KIND == 1) {
            double d, lin, mn, mx;
            interp_mono_exact<F>(f, c, lv.ni, lv.nij, zl, fp.box222 != 0, d, lin, mn, mx);
            ((F*)fp.dst[q])[o] = (F)d;
            ((F*)fp.lin[q])[o] = (F)lin;
            ((F*)fp.mn[q])[o] = (F)mn;
            ((F*)fp.mx[q])[o] = (F)mx;
          } else {
            ((F*)fp.dst[q])[o] = (F)interp1_exact<F>(f, c, lv.ni, lv.nij, zl);
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// persistent batch kernel: work items (domain, phase, group, first, count) taken
// from an atomic queue; phase p>0 items wait (bounded) on the per-domain count
// of completed phase p-1 items.  Item list and host side: adz_batch.cu.

// block-wide copy of a descriptor into shared memory (8-byte words)
template <typename T>
__device__ __forceinline__ void block_copy(T* dst, const T* src) {
  static_assert(sizeof(T) % 8 == 0, "descriptor size");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int q = threadIdx.x; q < (int)(sizeof(T) / 8); q += blockDim.x) d[q] = s[q];
}

// The points of a batch item, one per thread per unit.  A tiled item counts
// tiles of kBatchTileI i by kBatchTileK levels of a region (nx i by nz levels
// by ny rows from i0, k0, j0) in (i, k, j) tile order, one unit per tile; a
// row item counts points in (i, k, j) order, 128 per unit.  32-bit tile
// arithmetic; the point code is inlined once per phase.
struct BatchRegion {
  int i0, nx, j0, k0, nz;
};
__device__ __forceinline__ long long batch_units(const BItem& item) {
  return item.tiles ? item.count : (item.count + 127) / 128;
}
__device__ __forceinline__ bool batch_point(const BItem& item, const BatchRegion& R, long long u, int& i, int& j,
                                            int& k) {
  if (item.tiles) {
    const unsigned nic = ((unsigned)R.nx + kBatchTileI - 1) / kBatchTileI;
    const unsigned nkg = ((unsigned)R.nz + kBatchTileK - 1) / kBatchTileK;
    const unsigned T = (unsigned)(item.start + u), bj = T / nic;
    const unsigned ii = (T - bj * nic) * kBatchTileI + threadIdx.x % kBatchTileI;
    const unsigned kk = (bj % nkg) * kBatchTileK + threadIdx.x / kBatchTileI;
    i = (int)ii + R.i0;
    k = (int)kk + R.k0;
    j = (int)(bj / nkg) + R.j0;
    return ii < (unsigned)R.nx && kk < (unsigned)R.nz;
  }
  const long long t = item.start + u * 128 + threadIdx.x;
  const long long nrow = (long long)R.nx * R.nz;
  i = (int)(t % R.nx) + R.i0;
  k = (int)((t / R.nx) % R.nz) + R.k0;
  j = (int)(t / nrow) + R.j0;
  return t < item.start + item.count;
}

// The trajectory and interpolation items of the one-launch kernel.  With
// ADZ_BATCH_NOINLINE they are separate functions, so that each phase's point
// code gets its own register allocation rather than the union of the phases'.
// Measured on 16 large domains: 157.3 ms against 145.1 ms inlined (40 small
// domains: 9.35 against 8.53 ms), so they stay inlined.
#ifndef ADZ_BATCH_NOINLINE
#define ADZ_BATCH_NOINLINE 0
#endif
#if ADZ_BATCH_NOINLINE
#define ADZ_BATCH_ITEM_FN __device__ __noinline__
#else
#define ADZ_BATCH_ITEM_FN __device__ __forceinline__
#endif
template <int PREC>
ADZ_BATCH_ITEM_FN void batch_item_traject(const BDomC& C, const BItem& item) {
  // tiles of 32 i by 4 levels in (i, k, j) tile order, as in k_traject
  const BatchRegion R{1, C.g.ni, 1, C.ta.k00, C.g.nk - C.ta.k00 + 1};
  for (long long u = 0; u < batch_units(item); u++) {
    int i, j, k;
    if (batch_point(item, R, u, i, j, k)) traject_point<PREC, true>(C.g, C.ta, i, j, k);
  }
}
template <int PREC>
ADZ_BATCH_ITEM_FN void batch_item_sets(const BDomC& C, const BItem& item, int set, const int* srange,
                                       const FieldPtrs& fp) {
  const BatchRegion R{srange[0], srange[1], srange[2], srange[4], C.g.nk - srange[4] + 1};
  for (long long u = 0; u < batch_units(item); u++) {
    int i, j, k;
    if (batch_point(item, R, u, i, j, k)) set_point<PREC, true>(C.g, set, C.sa, fp, i, j, k);
  }
}

// MINB: minimum resident blocks per SM handed to ptxas (register budget);
// the autotuner picks the variant
template <int PREC, int MINB>
__global__ void __launch_bounds__(128, MINB) k_batch(const __grid_constant__ BatchParams P,
                                                     const BDom* __restrict__ doms, const BItem* __restrict__ items,
                                                     long long nitems, const unsigned* __restrict__ need,
                                                     unsigned long long* __restrict__ next,
                                                     unsigned* __restrict__ done, int* __restrict__ status,
                                                     unsigned long long max_spins) {
  __shared__ long long cur;
  __shared__ int dep_ok;
  __shared__ FieldPtrs sfp;
  __shared__ int sset, srange[5];
  for (;;) {
    if (threadIdx.x == 0) cur = (long long)atomicAdd(next, 1ull);
    __syncthreads();
    const long long it = cur;
    if (it >= nitems) break;
    const BItem item = items[it];
    if (threadIdx.x == 0) {
      dep_ok = 1;
      if (item.phase > 0) {
        const unsigned target = need[item.dom * 2 + item.phase - 1];
        const unsigned* d = done + item.dom * 2 + item.phase - 1;
        unsigned long long spins = 0;
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(d) : "memory");
        while (v < target) {
          if (++spins > max_spins) {
            dep_ok = 0;
            atomicOr(status, kErrTimeout);
            break;
          }
          __nanosleep(64);
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(d) : "memory");
        }
      }
    }
    if (item.phase == 2) {  // field group of the item: global descriptor -> shared
      const BDom& D = doms[item.dom];
      block_copy(&sfp, &D.gfp[item.group]);
      if (threadIdx.x < 5) srange[threadIdx.x] = D.grange[item.group][threadIdx.x];
      if (threadIdx.x == 5) sset = D.gset[item.group];
    }
    __syncthreads();
    if (dep_ok) {
      const BDomC& C = P.d[item.dom];  // constant bank
      const long long end = item.start + item.count;
      if (item.phase == 0) {
        using F = typename Types<PREC>::F;
        for (long long e = item.start + threadIdx.x; e < end; e += blockDim.x)
          prepare_cell<PREC>(C.g, (const F*)C.uu, (const F*)C.vv, (const F*)C.ww, (F*)C.ta.uvw_d, e);
      } else if (item.phase == 1) {
        batch_item_traject<PREC>(C, item);
      } else {
        batch_item_sets<PREC>(C, item, sset, srange, sfp);
      }
    }
    __syncthreads();  // the block's writes of this item precede thread 0's fence
    if (threadIdx.x == 0 && item.phase < 2) {
      __threadfence();
      atomicAdd(done + item.dom * 2 + item.phase, 1u);
    }
  }
}

// One phase of the batch per launch (the phased plan).  The previous phase
// of every domain completed with the previous launch, so there is no
// dependency wait, and data it wrote is read through the read-only path.
template <int PREC, int PH>
__device__ __forceinline__ void batch_phase_body(const BatchParams& P, const BDom* __restrict__ doms,
                                                 const BItem* __restrict__ items, long long nitems,
                                                 unsigned long long* __restrict__ next) {
  __shared__ long long cur;
  __shared__ FieldPtrs sfp;
  __shared__ int sset, srange[5];
  for (;;) {
    if (threadIdx.x == 0) cur = (long long)atomicAdd(next, 1ull);
    __syncthreads();
    const long long it = cur;
    if (it >= nitems) break;
    const BItem item = items[it];
    if (PH == 2) {
      const BDom& D = doms[item.dom];
      block_copy(&sfp, &D.gfp[item.group]);
      if (threadIdx.x < 5) srange[threadIdx.x] = D.grange[item.group][threadIdx.x];
      if (threadIdx.x == 5) sset = D.gset[item.group];
      __syncthreads();
    }
    const BDomC& C = P.d[item.dom];
    const long long end = item.start + item.count;
    if (PH == 0) {
      using F = typename Types<PREC>::F;
      for (long long e = item.start + threadIdx.x; e < end; e += blockDim.x)
        prepare_cell<PREC>(C.g, (const F*)C.uu, (const F*)C.vv, (const F*)C.ww, (F*)C.ta.uvw_d, e);
    } else if (PH == 1) {
      const BatchRegion R{1, C.g.ni, 1, C.ta.k00, C.g.nk - C.ta.k00 + 1};
      for (long long u = 0; u < batch_units(item); u++) {
        int i, j, k;
        if (batch_point(item, R, u, i, j, k)) traject_point<PREC, false>(C.g, C.ta, i, j, k);
      }
    } else {
      const BatchRegion R{srange[0], srange[1], srange[2], srange[4], C.g.nk - srange[4] + 1};
      for (long long u = 0; u < batch_units(item); u++) {
        int i, j, k;
        if (batch_point(item, R, u, i, j, k)) set_point<PREC, false>(C.g, sset, C.sa, sfp, i, j, k);
      }
    }
    __syncthreads();  // every thread is done with cur and sfp
  }
}

template <int PREC>
__global__ void __launch_bounds__(128) k_batch_p0(const __grid_constant__ BatchParams P, const BDom* __restrict__ doms,
                                                  const BItem* __restrict__ items, long long nitems,
                                                  unsigned long long* __restrict__ next) {
  batch_phase_body<PREC, 0>(P, doms, items, nitems, next);
}
template <int PREC>
__global__ void ADZ_TRAJ_BOUNDS k_batch_p1(const __grid_constant__ BatchParams P, const BDom* __restrict__ doms,
                                           const BItem* __restrict__ items, long long nitems,
                                           unsigned long long* __restrict__ next) {
  batch_phase_body<PREC, 1>(P, doms, items, nitems, next);
}
template <int PREC>
__global__ void ADZ_SET_BOUNDS k_batch_p2(const __grid_constant__ BatchParams P, const BDom* __restrict__ doms,
                                          const BItem* __restrict__ items, long long nitems,
                                          unsigned long long* __restrict__ next) {
  batch_phase_body<PREC, 2>(P, doms, items, nitems, next);
}

// ---------------------------------------------------------------------------
// launchers (host)
inline int grid_for(long long n, int block, int max_blocks = 148 * 64) {
  long long b = (n + block - 1) / block;
  if (b > max_blocks) b = max_blocks;
  if (b < 1) b = 1;
  return (int)b;
}

template <int PREC>
cudaError_t launch_prepare(const DGrid& g, const void* uu, const void* vv, const void* ww, void* uvw_d,
                           cudaStream_t s) {
  using F = typename Types<PREC>::F;
  const long long n = g.nij * g.nk;
  if constexpr (WindLayout<PREC>::soa) {
    auto a16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
    if (g.nit % 4 == 0 && a16(uu) && a16(vv) && a16(ww) && a16(uvw_d)) {
      k_prepare4<PREC><<<grid_for(n / 4, 256), 256, 0, s>>>(g, (const float*)uu, (const float*)vv, (const float*)ww,
                                                            (float*)uvw_d);
      return cudaGetLastError();
    }
  }
  k_prepare<PREC><<<grid_for(n, 256), 256, 0, s>>>(g, (const F*)uu, (const F*)vv, (const F*)ww, (F*)uvw_d);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_inittraj(const DGrid& g, float* pxyzm, double* wpxyz, cudaStream_t s) {
  const long long n = (long long)g.ni * g.nj * (g.nk - g.k0m + 1);
  k_inittraj<PREC><<<grid_for(n, 256), 256, 0, s>>>(g, pxyzm, wpxyz);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_traject(const DGrid& g, const TrajArgs& a, cudaStream_t s) {
#if ADZ_TRAJ_TILE_K > 1
  constexpr int TK = ADZ_TRAJ_TILE_K, TI = ADZ_TRAJ_TILE_I;
  const long long nb = (long long)((g.ni + TI - 1) / TI) * ((g.nk - a.k00 + 1 + TK - 1) / TK) * g.nj;
  if (nb > 0x7fffffffLL) return cudaErrorInvalidValue;
  k_traject<PREC><<<(unsigned)nb, TI * TK, 0, s>>>(g, a);
#else
  const long long n = (long long)g.ni * g.nj * (g.nk - a.k00 + 1);
  k_traject<PREC><<<grid_for(n, 128, 1 << 30), 128, 0, s>>>(g, a);
#endif
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_traject_box(const DGrid& g, const TrajArgs& a, int i0, int nx, int j0, int ny, cudaStream_t s) {
  const long long nkp = g.nk - a.k00 + 1, n = (long long)nx * ny * nkp;
  if (n <= 0) return cudaSuccess;
  if (batch_use_tiles(nx, nkp)) {
    const long long nb = (long long)((nx + 31) / 32) * ((nkp + 3) / 4) * ny;
    if (nb > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_traject_box<PREC, true><<<(unsigned)nb, 128, 0, s>>>(g, a, i0, nx, j0, ny);
  } else {
    k_traject_box<PREC, false><<<grid_for(n, 128, 1 << 30), 128, 0, s>>>(g, a, i0, nx, j0, ny);
  }
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_prepare_box(const DGrid& g, const void* uu, const void* vv, const void* ww, void* uvw_d, int ci0,
                               int nci, int cj0, int ncj, cudaStream_t s) {
  using F = typename Types<PREC>::F;
  const long long n = (long long)nci * ncj * g.nk;
  if (n <= 0) return cudaSuccess;
  k_prepare_box<PREC><<<grid_for(n, 256), 256, 0, s>>>(g, (const F*)uu, (const F*)vv, (const F*)ww, (F*)uvw_d, ci0,
                                                       nci, cj0, ncj);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_traject_tol(const DGrid& g, const TrajArgs& a, double tol, int maxit, unsigned char* iters,
                               unsigned long long* stats, cudaStream_t s, const GuessStart& gs) {
#if ADZ_TOL_TILES
  const long long nb = (long long)((g.ni + 31) / 32) * ((g.nk - a.k00 + 1 + 3) / 4) * g.nj;
  if (nb > 0x7fffffffLL) return cudaErrorInvalidValue;
  k_traject_tol<PREC><<<(unsigned)nb, 128, 0, s>>>(g, a, tol, maxit, iters, stats, gs);
#else
  const long long n = (long long)g.ni * g.nj * (g.nk - a.k00 + 1);
  k_traject_tol<PREC><<<grid_for(n, 128, 1 << 30), 128, 0, s>>>(g, a, tol, maxit, iters, stats, gs);
#endif
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_tricub_set(const DGrid& g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                              const SetArgs& a, const FieldPtrs& fp, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  if (n <= 0) return cudaSuccess;
#if ADZ_SET_TILE_K > 1
  constexpr int TK = ADZ_SET_TILE_K, TI = 128 / TK;
  const long long nb = (long long)((nx + TI - 1) / TI) * ((nz + TK - 1) / TK) * ny;
  if (nb > 0x7fffffffLL) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)nb;
#else
  const int grid = grid_for(n, 128, 1 << 30);
#endif
  if (a.pert) k_tricub_set<PREC, true><<<grid, 128, 0, s>>>(g, set, i0, nx, j0, ny, k0, nz, a, fp);
  else k_tricub_set<PREC, false><<<grid, 128, 0, s>>>(g, set, i0, nx, j0, ny, k0, nz, a, fp);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_positions(const DGrid& g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                             const SetArgs& a, void* pos, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  if (n <= 0) return cudaSuccess;
  k_positions<PREC><<<grid_for(n, 256, 1 << 30), 256, 0, s>>>(g, set, i0, nx, j0, ny, k0, nz, a, pos);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_tricub_parts(const DGrid& g, const SetArgs& a, const SetParts& sp, cudaStream_t s) {
  if (sp.n < 1 || sp.n > kMaxParts) return cudaErrorInvalidValue;
  long long most = 0;  // blocks of the largest part
  for (int q = 0; q < sp.n; q++) {
#if ADZ_SET_TILE_K > 1
    constexpr int TK = ADZ_SET_TILE_K, TI = 128 / TK, TJ = ADZ_SET_TILE_J;
    const long long n = (long long)((sp.p[q].nx + TI - 1) / TI) * ((sp.p[q].nz + TK - 1) / TK) *
                        ((sp.p[q].ny + TJ - 1) / TJ) * 128;
#else
    const long long n = (long long)sp.p[q].nx * sp.p[q].ny * sp.p[q].nz;
#endif
    most = n > most ? n : most;
  }
  const long long blocks = (most + 127) / 128 * sp.n;
  if (blocks < 1) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
#if ADZ_SET_TILE_K > 1
  constexpr int threads = 128 * ADZ_SET_TILE_J;
#else
  constexpr int threads = 128;
#endif
  if (a.pert) k_tricub_parts<PREC, true><<<(unsigned)blocks, threads, 0, s>>>(g, a, sp);
  else k_tricub_parts<PREC, false><<<(unsigned)blocks, threads, 0, s>>>(g, a, sp);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_qv_set(const DGrid& g, int i0, int nx, int j0, int ny, int k0, int nz, const SetArgs& a,
                          const FieldPtrs& fp, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  if (n <= 0) return cudaSuccess;
#if ADZ_QV_TILES
  const long long nb = (long long)((nx + 31) / 32) * ((nz + 3) / 4) * ny;
  if (nb > 0x7fffffffLL) return cudaErrorInvalidValue;
  const unsigned grid = (unsigned)nb;
#else
  const int grid = grid_for(n, 128, 1 << 30);
#endif
  if (a.pert) k_qv_set<PREC, true><<<grid, 128, 0, s>>>(g, i0, nx, j0, ny, k0, nz, a, fp);
  else k_qv_set<PREC, false><<<grid, 128, 0, s>>>(g, i0, nx, j0, ny, k0, nz, a, fp);
  return cudaGetLastError();
}

template <int PREC>
cudaError_t launch_interp_pos(const DZtab& lv, int kind, int n, const void* pos, const FieldPtrs& fp,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int b = grid_for(n, 128, 1 << 30);
  if (kind == 0) k_interp_pos<PREC, 0><<<b, 128, 0, s>>>(lv, n, pos, fp);
  else if (kind == 1) k_interp_pos<PREC, 1><<<b, 128, 0, s>>>(lv, n, pos, fp);
  else k_interp_pos<PREC, 2><<<b, 128, 0, s>>>(lv, n, pos, fp);
  return cudaGetLastError();
}

// register-budget variants of the batch kernel (minimum resident blocks of
// 128 threads per SM handed to ptxas); FP64 needs about twice the registers
template <int PREC, int V>
struct BatchMinB {
  static constexpr int value = PREC == kFp64 ? 4 + V : (V == 0 ? 6 : V == 1 ? 7 : 9);
};

template <int PREC>
cudaError_t launch_batch(int variant, int grid, const BatchParams& P, const BDom* doms, const BItem* items,
                         long long nitems, const unsigned* need, unsigned long long* next, unsigned* done,
                         int* status, unsigned long long max_spins, cudaStream_t s) {
  if constexpr (PREC == kRef32) {
    return cudaErrorNotSupported;
  } else {
    if (variant == 1)
      k_batch<PREC, BatchMinB<PREC, 1>::value><<<grid, 128, 0, s>>>(P, doms, items, nitems, need, next, done, status, max_spins);
    else if (variant == 2)
      k_batch<PREC, BatchMinB<PREC, 2>::value><<<grid, 128, 0, s>>>(P, doms, items, nitems, need, next, done, status, max_spins);
    else
      k_batch<PREC, BatchMinB<PREC, 0>::value><<<grid, 128, 0, s>>>(P, doms, items, nitems, need, next, done, status, max_spins);
    return cudaGetLastError();
  }
}

template <int PREC>
cudaError_t launch_batch_phased(const int* grid, const BatchParams& P, const BDom* doms, const BItem* items,
                                const long long* pstart, unsigned long long* next, cudaStream_t s) {
  if constexpr (PREC == kRef32) {
    return cudaErrorNotSupported;
  } else {
    if (pstart[1] > pstart[0])
      k_batch_p0<PREC><<<grid[0], 128, 0, s>>>(P, doms, items + pstart[0], pstart[1] - pstart[0], next);
    if (pstart[2] > pstart[1])
      k_batch_p1<PREC><<<grid[1], 128, 0, s>>>(P, doms, items + pstart[1], pstart[2] - pstart[1], next + 1);
    if (pstart[3] > pstart[2])
      k_batch_p2<PREC><<<grid[2], 128, 0, s>>>(P, doms, items + pstart[2], pstart[3] - pstart[2], next + 2);
    return cudaGetLastError();
  }
}

template <int PREC>
int batch_phase_resident_blocks(int phase) {
  if constexpr (PREC == kRef32) {
    return 0;
  } else {
    const void* f = phase == 0 ? (const void*)k_batch_p0<PREC>
                    : phase == 1 ? (const void*)k_batch_p1<PREC>
                                 : (const void*)k_batch_p2<PREC>;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 128, 0) != cudaSuccess) return 0;
    return n;
  }
}

template <int PREC>
int batch_resident_blocks(int variant) {
  if constexpr (PREC == kRef32) {
    return 0;
  } else {
    const void* f = variant == 1   ? (const void*)k_batch<PREC, BatchMinB<PREC, 1>::value>
                    : variant == 2 ? (const void*)k_batch<PREC, BatchMinB<PREC, 2>::value>
                                   : (const void*)k_batch<PREC, BatchMinB<PREC, 0>::value>;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 128, 0) != cudaSuccess) return 0;
    return n;
  }
}

#define ADZ_INSTANTIATE(P)                                                                                         \
  template cudaError_t launch_prepare<P>(const DGrid&, const void*, const void*, const void*, void*, cudaStream_t); \
  template cudaError_t launch_inittraj<P>(const DGrid&, float*, double*, cudaStream_t);                            \
  template cudaError_t launch_traject<P>(const DGrid&, const TrajArgs&, cudaStream_t);                             \
  template cudaError_t launch_traject_box<P>(const DGrid&, const TrajArgs&, int, int, int, int, cudaStream_t);      \
  template cudaError_t launch_prepare_box<P>(const DGrid&, const void*, const void*, const void*, void*, int, int,  \
                                             int, int, cudaStream_t);                                               \
  template cudaError_t launch_traject_tol<P>(const DGrid&, const TrajArgs&, double, int, unsigned char*,           \
                                             unsigned long long*, cudaStream_t, const GuessStart&);                \
  template cudaError_t launch_tricub_set<P>(const DGrid&, int, int, int, int, int, int, int, const SetArgs&,       \
                                            const FieldPtrs&, cudaStream_t);                                       \
  template cudaError_t launch_interp_pos<P>(const DZtab&, int, int, const void*, const FieldPtrs&, cudaStream_t); \
  template cudaError_t launch_positions<P>(const DGrid&, int, int, int, int, int, int, int, const SetArgs&, void*, \
                                           cudaStream_t);                                                         \
  template cudaError_t launch_tricub_parts<P>(const DGrid&, const SetArgs&, const SetParts&, cudaStream_t);       \
  template cudaError_t launch_qv_set<P>(const DGrid&, int, int, int, int, int, int, const SetArgs&,               \
                                        const FieldPtrs&, cudaStream_t);                                          \
  template cudaError_t launch_batch<P>(int, int, const BatchParams&, const BDom*, const BItem*, long long,       \
                                       const unsigned*,                                                             \
                                       unsigned long long*, unsigned*, int*, unsigned long long, cudaStream_t);    \
  template int batch_resident_blocks<P>(int);                                                                   \
  template cudaError_t launch_batch_phased<P>(const int*, const BatchParams&, const BDom*, const BItem*,           \
                                              const long long*, unsigned long long*, cudaStream_t);                \
  template int batch_phase_resident_blocks<P>(int);

}  // namespace adz
