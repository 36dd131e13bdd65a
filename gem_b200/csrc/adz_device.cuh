// Device-side building blocks of the semi-Lagrangian advection kernels.
//
// Exact paths (REF32, FP64) follow the reference interpolator's production
// arithmetic order (src/gemdyn/src/base/turbo_tricublin.c, AVX2 branch) with
// explicit fma() and are compiled with -fmad=false, so every other
// multiply-add stays separately rounded as in the reference.  The MIXED path
// uses FP32 weights and packed FP32 FMAs (fma.rn.f32x2) and is compiled in its
// own translation unit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "adz_types.h"

namespace adz {

__device__ __forceinline__ void raise_status(int* st, int bits) {
  if (st) atomicOr(st, bits);
}

// ---------------------------------------------------------------------------
// cell selection and FP64 coefficients (turbo_tricublin.c:382-512)
// c[0..3] x, c[4..7] y, c[8..11] z (cubic or linear), c[12..19] linear
// ---------------------------------------------------------------------------
__device__ __forceinline__ int coef_cell(double* c, int& off, double px, double py, double dz, int ix, int iy, int iz,
                                         const DZtab& lv) {
  const double one = 1.0, two = 2.0;
  const double cp167 = 1.0 / 6.0, cm167 = -1.0 / 6.0, cp5 = 0.5, cm5 = -0.5;
  int ijk = ix - 2;
  c[12] = 0.0;
  c[13] = 1.0 - px;
  c[14] = px;
  c[15] = 0.0;
  ijk = ijk + (iy - 2) * lv.ni;
  c[16] = 1.0 - py;
  c[17] = py;
  ijk = ijk + (iz - 1) * lv.nij;
  c[18] = 1.0 - dz;
  c[19] = dz;
  iz--;
  const int zlinear = (iz < 1 || iz > lv.nk - 3) ? -1 : 0;
  if (!zlinear) ijk -= lv.nij;
  off = ijk;
  if (zlinear) {
    c[8] = 0.0;
    c[9] = 1.0 - dz;
    c[10] = dz;
    c[11] = 0.0;
  } else {
    const double* base = lv.ocz + 4 * iz;
    const double* pos = lv.z + iz;
    const double p0 = __ldg(pos), p1 = __ldg(pos + 1), pm1 = __ldg(pos - 1), p2 = __ldg(pos + 2);
    // the reference build fuses the first product of this line
    const double pz = fma(dz, p1, (1.0 - dz) * p0);
    const double zza = pz - pm1, zzb = pz - p0, zzc = pz - p1, zzd = pz - p2;
    const double zzab = zza * zzb, zzcd = zzc * zzd;
    c[8] = zzb * zzcd * __ldg(base);
    c[9] = zza * zzcd * __ldg(base + 1);
    c[10] = zzd * zzab * __ldg(base + 2);
    c[11] = zzc * zzab * __ldg(base + 3);
  }
  c[0] = cm167 * px * (px - one) * (px - two);
  c[1] = cp5 * (px + one) * (px - one) * (px - two);
  c[2] = cm5 * px * (px + one) * (px - two);
  c[3] = cp167 * px * (px + one) * (px - one);
  c[4] = cm167 * py * (py - one) * (py - two);
  c[5] = cp5 * (py + one) * (py - one) * (py - two);
  c[6] = cm5 * py * (py + one) * (py - two);
  c[7] = cp167 * py * (py + one) * (py - one);
  return zlinear;
}

// FP32 position (reference precision): truncate, offsets in FP64.
__device__ __forceinline__ int coef_f32pos(double* c, int& off, float pxf, float pyf, float pzf, const DZtab& lv) {
  double px = pxf, py = pyf, pz = pzf;
  int ix = __double2int_rz(px);
  px = px - ix;
  ix += lv.offi;
  int iy = __double2int_rz(py);
  py = py - iy;
  iy += lv.offj;
  int iz = __double2int_rz(pz);
  if (iz < 1) iz = 1;
  if (iz > lv.nk - 1) iz = lv.nk - 1;
  const double dz = pz - iz;
  return coef_cell(c, off, px, py, dz, ix, iy, iz, lv);
}

// The cell a FP64 position selects in the reference: its FP32 rounding,
// truncated.  Offsets stay FP64.
__device__ __forceinline__ void cell_of(double p, int& i) { i = __double2int_rz((double)__double2float_rn(p)); }

__device__ __forceinline__ int coef_f64pos(double* c, int& off, double px8, double py8, double pz8, const DZtab& lv) {
  int ix, iy, iz;
  cell_of(px8, ix);
  cell_of(py8, iy);
  cell_of(pz8, iz);
  const double px = px8 - ix, py = py8 - iy;
  ix += lv.offi;
  iy += lv.offj;
  if (iz < 1) iz = 1;
  if (iz > lv.nk - 1) iz = lv.nk - 1;
  const double dz = pz8 - iz;
  return coef_cell(c, off, px, py, dz, ix, iy, iz, lv);
}

// source loads: read-only path, or (COH) the coherent L1 path for data that
// the same launch wrote before an acquire (persistent batch kernel)
template <bool COH, typename T>
__device__ __forceinline__ T ldin(const T* p) {
  if (COH) return __ldca(p);
  return __ldg(p);
}

template <typename T, bool COH = false>
__device__ __forceinline__ double ldd(const T* p) {
  return (double)ldin<COH>(p);
}

// single field cubic, turbo_tricublin.c:551-615 (AVX2 order)
template <typename T>
__device__ __forceinline__ double interp1_exact(const T* __restrict__ f, const double* c, int ni, int ninj,
                                                int zlinear) {
  const int ninjl = zlinear ? 0 : ninj;
  double ya[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const T* s = f + r * ni;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const T* p0 = s + x;
      const T* p1 = p0 + ninjl;
      const T* p2 = p1 + ninj;
      const T* p3 = p2 + ninjl;
      double za = ldd(p0) * c[8];
      za = fma(ldd(p1), c[9], za);
      za = fma(ldd(p2), c[10], za);
      za = fma(ldd(p3), c[11], za);
      ya[x] = (r == 0) ? za * c[4] : fma(za, c[4 + r], ya[x]);
    }
  }
  return (ya[0] * c[0] + ya[2] * c[2]) + (ya[1] * c[1] + ya[3] * c[3]);
}

__device__ __forceinline__ double vmin(double a, double b) { return (a < b) ? a : b; }
__device__ __forceinline__ double vmax(double a, double b) { return (a > b) ? a : b; }

// cubic + trilinear + min/max, turbo_tricublin.c:869-997 (AVX2 box: x 1..2,
// y 0..3, z 1..2) or the scalar 2x2x2 box (:1017-1025) when box222.
template <typename T>
__device__ __forceinline__ void interp_mono_exact(const T* __restrict__ f, const double* c, int ni, int ninj,
                                                  int zlinear, bool box222, double& d, double& lin, double& mn,
                                                  double& mx) {
  const int ninjl = zlinear ? 0 : ninj;
  double ya[4], mi[4], ma[4], vyl[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const T* s = f + r * ni;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const T* p0 = s + x;
      const T* p1 = p0 + ninjl;
      const T* p2 = p1 + ninj;
      const T* p3 = p2 + ninjl;
      const double v0 = ldd(p0), v1 = ldd(p1), v2 = ldd(p2), v3 = ldd(p3);
      double za = v0 * c[8];
      if (r == 0) {
        mi[x] = v1;
        ma[x] = v1;
      } else {
        mi[x] = vmin(mi[x], v1);
        ma[x] = vmax(ma[x], v1);
      }
      za = fma(v1, c[9], za);
      mi[x] = vmin(mi[x], v2);
      ma[x] = vmax(ma[x], v2);
      za = fma(v2, c[10], za);
      za = fma(v3, c[11], za);
      ya[x] = (r == 0) ? za * c[4] : fma(za, c[4 + r], ya[x]);
      if (r == 1 || r == 2) {
        double vzl = v1 * c[18];
        vzl = fma(v2, c[19], vzl);
        vyl[x] = (r == 1) ? vzl * c[16] : fma(vzl, c[17], vyl[x]);
      }
    }
  }
  mn = vmin(mi[1], mi[2]);
  mx = vmax(ma[1], ma[2]);
  if (box222) {
    // scalar branch: start at point [1,1,1], rows 1..2, planes 1..2, x 1..2
    const int ninj2 = ninj + ninjl;
    double a = ldd(f + 1 + ni + ninjl), lo = a, hi = a;
#pragma unroll
    for (int i = 1; i < 3; i++) {
      const double e1 = ldd(f + i + ni + ninjl), e2 = ldd(f + i + ni + ninj2);
      const double e3 = ldd(f + i + 2 * ni + ninjl), e4 = ldd(f + i + 2 * ni + ninj2);
      hi = vmax(hi, e1); hi = vmax(hi, e2);
      lo = vmin(lo, e1); lo = vmin(lo, e2);
      hi = vmax(hi, e3); hi = vmax(hi, e4);
      lo = vmin(lo, e3); lo = vmin(lo, e4);
    }
    mn = lo;
    mx = hi;
  }
  const double l0 = vyl[0] * c[12], l1 = vyl[1] * c[13], l2 = vyl[2] * c[14], l3 = vyl[3] * c[15];
  lin = (l0 + l2) + (l1 + l3);
  d = (ya[0] * c[0] + ya[2] * c[2]) + (ya[1] * c[1] + ya[3] * c[3]);
}

// 3-component interleaved source, turbo_tricublin.c:1153-1272 (AVX2 order)
template <typename T, bool COH = false>
__device__ __forceinline__ void interp3_exact(const T* __restrict__ f, const double* c, int ni, int ninj, int zlinear,
                                              double* out) {
  const int n3 = 3 * ni, nn3 = 3 * ninj;
  const int ninjl = zlinear ? 0 : nn3;
  double ya[12];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const T* s = f + r * n3;
#pragma unroll
    for (int e = 0; e < 12; e++) {
      const T* p0 = s + e;
      const T* p1 = p0 + ninjl;
      const T* p2 = p1 + nn3;
      const T* p3 = p2 + ninjl;
      double za = ldd<T, COH>(p0) * c[8];
      za = fma(ldd<T, COH>(p1), c[9], za);
      za = fma(ldd<T, COH>(p2), c[10], za);
      za = fma(ldd<T, COH>(p3), c[11], za);
      ya[e] = (r == 0) ? za * c[4] : fma(za, c[4 + r], ya[e]);
    }
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    double x0 = ya[q] * c[0];
    x0 = fma(ya[3 + q], c[1], x0);
    x0 = fma(ya[6 + q], c[2], x0);
    x0 = fma(ya[9 + q], c[3], x0);
    out[q] = x0;
  }
}

// ---------------------------------------------------------------------------
// mixed precision: FP64 cell + offset, FP32 weights and sums
// ---------------------------------------------------------------------------
struct WF {
  float cx[4], cy[4], cz[4];
  float lx0, lx1, ly0, ly1, lz0, lz1;
  int off;  // corner offset relative to cell (1,1,1): xy + zb*nij
  int zl;
  int xy;   // corner offset within a plane, relative to cell (1,1)
  int zb;   // 0-based plane of the corner (iz0-1 cubic, iz0 linear)
};

__device__ __forceinline__ void cubic_w(float t, float* w) {
  // 4-point Lagrange weights on nodes -1, 0, 1, 2 at offset t
  const float tm1 = t - 1.0f, tm2 = t - 2.0f, tp1 = t + 1.0f;
  w[0] = (-1.0f / 6.0f) * t * tm1 * tm2;
  w[1] = 0.5f * tp1 * tm1 * tm2;
  w[2] = -0.5f * t * tp1 * tm2;
  w[3] = (1.0f / 6.0f) * t * tp1 * tm1;
}

__device__ __forceinline__ void coef_mixed(WF& w, double px8, double py8, double pz8, const DZtab& lv) {
  int ix, iy, iz;
  cell_of(px8, ix);
  cell_of(py8, iy);
  cell_of(pz8, iz);
  const float fx = (float)(px8 - ix), fy = (float)(py8 - iy);
  ix += lv.offi;
  iy += lv.offj;
  if (iz < 1) iz = 1;
  if (iz > lv.nk - 1) iz = lv.nk - 1;
  const double dz8 = pz8 - iz;
  const float dz = (float)dz8;
  const int xy = (ix - 2) + (iy - 2) * lv.ni;
  const int iz0 = iz - 1;
  const int zl = (iz0 < 1 || iz0 > lv.nk - 3);
  w.zb = zl ? iz0 : iz0 - 1;
  w.xy = xy;
  w.off = xy + w.zb * lv.nij;
  w.zl = zl;
  cubic_w(fx, w.cx);
  cubic_w(fy, w.cy);
  w.lx0 = 1.0f - fx;
  w.lx1 = fx;
  w.ly0 = 1.0f - fy;
  w.ly1 = fy;
  w.lz0 = 1.0f - dz;
  w.lz1 = dz;
  if (zl) {
    w.cz[0] = 0.0f;
    w.cz[1] = 1.0f - dz;
    w.cz[2] = dz;
    w.cz[3] = 0.0f;
  } else {
    const float4 a = __ldg(reinterpret_cast<const float4*>(lv.zn + 8 * iz0));
    const float2 b = __ldg(reinterpret_cast<const float2*>(lv.zn + 8 * iz0 + 4));
    const float um1 = a.x, u2 = a.y;
    const float t = dz;
    const float d0 = t - um1, d1 = t, d2 = t - 1.0f, d3 = t - u2;
    w.cz[0] = d1 * d2 * d3 * a.z;
    w.cz[1] = d0 * d2 * d3 * a.w;
    w.cz[2] = d0 * d1 * d3 * b.x;
    w.cz[3] = d0 * d1 * d2 * b.y;
  }
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// single field, FP32 sums with the two x-column pairs packed
template <bool COH = false>
__device__ __forceinline__ float interp1_mixed(const float* __restrict__ f, const WF& w, int ni, int ninj) {
  const int ninjl = w.zl ? 0 : ninj;
  const float2 cz0 = f2(w.cz[0], w.cz[0]), cz1 = f2(w.cz[1], w.cz[1]);
  const float2 cz2 = f2(w.cz[2], w.cz[2]), cz3 = f2(w.cz[3], w.cz[3]);
  float2 ya = f2(0.f, 0.f), yb = f2(0.f, 0.f);
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const float* s = f + r * ni;
    const float* p1 = s + ninjl;
    const float* p2 = p1 + ninj;
    const float* p3 = p2 + ninjl;
    float2 za = __fmul2_rn(f2(ldin<COH>(s), ldin<COH>(s + 1)), cz0);
    float2 zb = __fmul2_rn(f2(ldin<COH>(s + 2), ldin<COH>(s + 3)), cz0);
    za = __ffma2_rn(f2(ldin<COH>(p1), ldin<COH>(p1 + 1)), cz1, za);
    zb = __ffma2_rn(f2(ldin<COH>(p1 + 2), ldin<COH>(p1 + 3)), cz1, zb);
    za = __ffma2_rn(f2(ldin<COH>(p2), ldin<COH>(p2 + 1)), cz2, za);
    zb = __ffma2_rn(f2(ldin<COH>(p2 + 2), ldin<COH>(p2 + 3)), cz2, zb);
    za = __ffma2_rn(f2(ldin<COH>(p3), ldin<COH>(p3 + 1)), cz3, za);
    zb = __ffma2_rn(f2(ldin<COH>(p3 + 2), ldin<COH>(p3 + 3)), cz3, zb);
    const float2 cyr = f2(w.cy[r], w.cy[r]);
    ya = __ffma2_rn(za, cyr, ya);
    yb = __ffma2_rn(zb, cyr, yb);
  }
  float2 x = __fmul2_rn(ya, f2(w.cx[0], w.cx[1]));
  x = __ffma2_rn(yb, f2(w.cx[2], w.cx[3]), x);
  return x.x + x.y;
}

// mono: cubic, trilinear, min/max over the AVX2 box (x 1..2, y 0..3, z 1..2)
__device__ __forceinline__ void interp_mono_mixed(const float* __restrict__ f, const WF& w, int ni, int ninj,
                                                  float& d, float& lin, float& mn, float& mx) {
  const int ninjl = w.zl ? 0 : ninj;
  const float2 cz0 = f2(w.cz[0], w.cz[0]), cz1 = f2(w.cz[1], w.cz[1]);
  const float2 cz2 = f2(w.cz[2], w.cz[2]), cz3 = f2(w.cz[3], w.cz[3]);
  const float2 lz0 = f2(w.lz0, w.lz0), lz1 = f2(w.lz1, w.lz1);
  float2 ya = f2(0.f, 0.f), yb = f2(0.f, 0.f), yl = f2(0.f, 0.f);
  float lo = 3.402823466e38f, hi = -3.402823466e38f;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const float* s = f + r * ni;
    const float* p1 = s + ninjl;
    const float* p2 = p1 + ninj;
    const float* p3 = p2 + ninjl;
    const float2 a1 = f2(__ldg(p1), __ldg(p1 + 1)), b1 = f2(__ldg(p1 + 2), __ldg(p1 + 3));
    const float2 a2 = f2(__ldg(p2), __ldg(p2 + 1)), b2 = f2(__ldg(p2 + 2), __ldg(p2 + 3));
    float2 za = __fmul2_rn(f2(__ldg(s), __ldg(s + 1)), cz0);
    float2 zb = __fmul2_rn(f2(__ldg(s + 2), __ldg(s + 3)), cz0);
    za = __ffma2_rn(a1, cz1, za);
    zb = __ffma2_rn(b1, cz1, zb);
    za = __ffma2_rn(a2, cz2, za);
    zb = __ffma2_rn(b2, cz2, zb);
    za = __ffma2_rn(f2(__ldg(p3), __ldg(p3 + 1)), cz3, za);
    zb = __ffma2_rn(f2(__ldg(p3 + 2), __ldg(p3 + 3)), cz3, zb);
    const float2 cyr = f2(w.cy[r], w.cy[r]);
    ya = __ffma2_rn(za, cyr, ya);
    yb = __ffma2_rn(zb, cyr, yb);
    // bound box: columns 1 and 2 of planes 1 and 2
    lo = fminf(lo, fminf(fminf(a1.y, b1.x), fminf(a2.y, b2.x)));
    hi = fmaxf(hi, fmaxf(fmaxf(a1.y, b1.x), fmaxf(a2.y, b2.x)));
    if (r == 1 || r == 2) {
      // trilinear: columns 1,2 of planes 1,2 of rows 1,2
      const float2 zl = __ffma2_rn(f2(a2.y, b2.x), lz1, __fmul2_rn(f2(a1.y, b1.x), lz0));
      const float cyl = (r == 1) ? w.ly0 : w.ly1;
      yl = __ffma2_rn(zl, f2(cyl, cyl), yl);
    }
  }
  float2 x = __fmul2_rn(ya, f2(w.cx[0], w.cx[1]));
  x = __ffma2_rn(yb, f2(w.cx[2], w.cx[3]), x);
  d = x.x + x.y;
  lin = fmaf(yl.y, w.lx1, yl.x * w.lx0);
  mn = lo;
  mx = hi;
}

// 3-component interleaved source (departure winds), FP32 sums
template <bool COH = false>
__device__ __forceinline__ void interp3_mixed(const float* __restrict__ f, const WF& w, int ni, int ninj,
                                              float* out) {
  const int n3 = 3 * ni, nn3 = 3 * ninj;
  const int ninjl = w.zl ? 0 : nn3;
  float2 y[6];
#pragma unroll
  for (int e = 0; e < 6; e++) y[e] = f2(0.f, 0.f);
  const float2 cz0 = f2(w.cz[0], w.cz[0]), cz1 = f2(w.cz[1], w.cz[1]);
  const float2 cz2 = f2(w.cz[2], w.cz[2]), cz3 = f2(w.cz[3], w.cz[3]);
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const float* s = f + r * n3;
    const float* p1 = s + ninjl;
    const float* p2 = p1 + nn3;
    const float* p3 = p2 + ninjl;
    const float2 cyr = f2(w.cy[r], w.cy[r]);
#pragma unroll
    for (int e = 0; e < 6; e++) {
      float2 z = __fmul2_rn(f2(ldin<COH>(s + 2 * e), ldin<COH>(s + 2 * e + 1)), cz0);
      z = __ffma2_rn(f2(ldin<COH>(p1 + 2 * e), ldin<COH>(p1 + 2 * e + 1)), cz1, z);
      z = __ffma2_rn(f2(ldin<COH>(p2 + 2 * e), ldin<COH>(p2 + 2 * e + 1)), cz2, z);
      z = __ffma2_rn(f2(ldin<COH>(p3 + 2 * e), ldin<COH>(p3 + 2 * e + 1)), cz3, z);
      y[e] = __ffma2_rn(z, cyr, y[e]);
    }
  }
  // element e of the 12 is component e%3 of column e/3
  float v[12];
#pragma unroll
  for (int e = 0; e < 6; e++) {
    v[2 * e] = y[e].x;
    v[2 * e + 1] = y[e].y;
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    float x0 = v[q] * w.cx[0];
    x0 = fmaf(v[3 + q], w.cx[1], x0);
    x0 = fmaf(v[6 + q], w.cx[2], x0);
    x0 = fmaf(v[9 + q], w.cx[3], x0);
    out[q] = x0;
  }
}

}  // namespace adz
