// BICUBH_QV: bicubic horizontal, quintic vertical interpolation on thermo
// levels (cubic at levels 2 and nk-2, linear at the ends, linear everywhere
// in an autobarotropic run), with the trilinear
// value and min/max over the inner 2x2x2 box.
//   coefficients   B/bicubHQV_lin_mono.F90:66-147
//   sums, box      B/bicubHQV_lin_min_max_zyx.F90:20-83
//   denominators   B/adz_set.F90:286-311 (host, DGrid::qv_t)
// Exact modes (REF32, FP64) keep the reference's operation order: FP64
// weights and sums, each column sum rounded to the field type before the x
// sum.  MIXED computes the weights in FP64 and sums in FP32.
#pragma once
#include "adz_device.cuh"

namespace adz {

struct QvCoef {
  double cx[4], cy[4], qz[6], lx[2], ly[2], lz[2];
  long long off;  // ext offset of the stencil origin (column i-1, row j-1, first plane) from (1,1,1)
  int pl[6];      // plane of each of the six vertical terms, relative to the first plane
};

// PREC kRef32 takes FP32 positions (the reference's Adz_pt); the others FP64
// positions whose cell index is that of the FP32 rounding
template <int PREC>
__device__ __forceinline__ void qv_coef(const DGrid& g, double px, double py, double pz, QvCoef& c) {
  const int nk = g.nk;
  const double ov6 = 1.0 / 6.0, ov2 = 1.0 / 2.0;
  const int ii1 = (int)(float)px;
  double del = px - (double)ii1;
  double del12 = (del - 1.0) * (del - 2.0), del10 = (del + 1.0) * del;
  c.cx[0] = -(del * del12 * ov6);
  c.cx[1] = (del + 1.0) * del12 * ov2;
  c.cx[2] = -(del10 * (del - 2.0) * ov2);
  c.cx[3] = del10 * (del - 1.0) * ov6;
  c.lx[0] = 1.0 - del;
  c.lx[1] = del;
  const int jj1 = (int)(float)py;
  del = py - (double)jj1;
  del12 = (del - 1.0) * (del - 2.0);
  del10 = (del + 1.0) * del;
  c.cy[0] = -(del * del12 * ov6);
  c.cy[1] = (del + 1.0) * del12 * ov2;
  c.cy[2] = -(del10 * (del - 2.0) * ov2);
  c.cy[3] = del10 * (del - 1.0) * ov6;
  c.ly[0] = 1.0 - del;
  c.ly[1] = del;
  int kk1 = (int)(float)pz;
  // an autobarotropic run (Schm_autobar_L) interpolates linearly in z at every level
  const bool quintic = (kk1 >= 3) && (kk1 <= nk - 3) && !g.autobar;
  const bool cubic = ((kk1 == 2) || (kk1 == nk - 2)) && !g.autobar;
  if (!quintic && !cubic) kk1 = kk1 < 1 ? 1 : (kk1 > nk - 1 ? nk - 1 : kk1);
  const double* posz = g.zt;
  const double zt = __ldg(posz + kk1) + (pz - (double)kk1) * __ldg(g.delz_t + kk1);
  c.lz[1] = (zt - __ldg(posz + kk1)) * __ldg(g.odelz_t + kk1);
  c.lz[0] = 1.0 - c.lz[1];
  const double* q = g.qv_t + 10 * kk1;
  int kb;
  if (quintic) {
    kb = kk1 - 2;
    const double rx = __ldg(posz + kk1 - 2), ra = __ldg(posz + kk1 - 1), rb = __ldg(posz + kk1);
    const double rc = __ldg(posz + kk1 + 1), rd = __ldg(posz + kk1 + 2), re = __ldg(posz + kk1 + 3);
    const double dx = zt - rx, da = zt - ra, db = zt - rb, dc = zt - rc, dd = zt - rd, de = zt - re;
    c.qz[0] = da * db * dc * dd * de * __ldg(q + 4);
    c.qz[1] = dx * db * dc * dd * de * __ldg(q + 5);
    c.qz[2] = dx * da * dc * dd * de * __ldg(q + 6);
    c.qz[3] = dx * da * db * dd * de * __ldg(q + 7);
    c.qz[4] = dx * da * db * dc * de * __ldg(q + 8);
    c.qz[5] = dx * da * db * dc * dd * __ldg(q + 9);
  } else if (cubic) {
    kb = kk1 - 1;
    const double ra = __ldg(posz + kk1 - 1), rb = __ldg(posz + kk1), rc = __ldg(posz + kk1 + 1),
                 rd = __ldg(posz + kk1 + 2);
    const double da = zt - ra, db = zt - rb, dc = zt - rc, dd = zt - rd;
    c.qz[0] = 0.0;
    c.qz[1] = db * dc * dd * __ldg(q + 0);
    c.qz[2] = da * dc * dd * __ldg(q + 1);
    c.qz[3] = da * db * dd * __ldg(q + 2);
    c.qz[4] = da * db * dc * __ldg(q + 3);
    c.qz[5] = 0.0;
  } else {
    kb = kk1;
    c.qz[0] = 0.0;
    c.qz[1] = 0.0;
    c.qz[3] = (zt - __ldg(posz + kk1)) * __ldg(g.odelz_t + kk1);
    c.qz[2] = 1.0 - c.qz[3];
    c.qz[4] = 0.0;
    c.qz[5] = 0.0;
  }
  const int nc = quintic ? 1 : 0, nl = (quintic || cubic) ? 1 : 0;
  c.pl[0] = 0;
  c.pl[1] = nc;
  c.pl[2] = c.pl[1] + nl;
  c.pl[3] = c.pl[2] + 1;
  c.pl[4] = c.pl[3] + nl;
  c.pl[5] = c.pl[4] + nc;
  const int il = ii1 - (g.i0g - 1), jl = jj1 - (g.j0g - 1);
  c.off = (long long)(il - 2) + (long long)(jl - 2) * g.nit + (long long)(kb - 1) * g.nij;
}

// the stencil of a QV origin (4 x 4 columns, planes 0..pl[5]) inside the ext array
__device__ __forceinline__ bool qv_stencil_ok(const DGrid& g, const QvCoef& c) {
  const long long e = c.off + (long long)(1 - g.lminx) + (long long)(1 - g.lminy) * g.nit;
  if (e < 0) return false;
  const long long k = e / g.nij;
  const long long r = e - k * g.nij;
  const int j = (int)(r / g.nit), i = (int)(r - (long long)j * g.nit);
  return k + c.pl[5] <= g.nk - 1 && i + 3 < g.nit && j + 3 < g.njt;
}

template <typename F>
__device__ __forceinline__ void interp_qv_exact(const F* __restrict__ s, int ni, long long nij, const QvCoef& c,
                                                F& xyz, F& li, F& mi, F& ma) {
  const long long p1 = c.pl[1] * nij, p2 = c.pl[2] * nij, p3 = c.pl[3] * nij, p4 = c.pl[4] * nij,
                  p5 = c.pl[5] * nij;
  F dst[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double v[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const F* t = s + i + r * ni;
      v[r] = (double)__ldg(t) * c.qz[0] + (double)__ldg(t + p1) * c.qz[1] + (double)__ldg(t + p2) * c.qz[2] +
             (double)__ldg(t + p3) * c.qz[3] + (double)__ldg(t + p4) * c.qz[4] + (double)__ldg(t + p5) * c.qz[5];
    }
    dst[i] = (F)(v[0] * c.cy[0] + v[1] * c.cy[1] + v[2] * c.cy[2] + v[3] * c.cy[3]);
  }
  xyz = (F)((double)dst[0] * c.cx[0] + (double)dst[1] * c.cx[1] + (double)dst[2] * c.cx[2] +
            (double)dst[3] * c.cx[3]);
  F dsl[2];
  F hi = __ldg(s + 1 + ni + p2), lo = hi;
#pragma unroll
  for (int i = 1; i <= 2; i++) {
    const F b2 = __ldg(s + i + ni + p2), b3 = __ldg(s + i + ni + p3);
    const F c2 = __ldg(s + i + 2 * ni + p2), c3 = __ldg(s + i + 2 * ni + p3);
    const double vb = (double)b2 * c.lz[0] + (double)b3 * c.lz[1];
    const double vc = (double)c2 * c.lz[0] + (double)c3 * c.lz[1];
    dsl[i - 1] = (F)(vb * c.ly[0] + vc * c.ly[1]);
    hi = hi > b2 ? hi : b2;
    hi = hi > b3 ? hi : b3;
    lo = lo < b2 ? lo : b2;
    lo = lo < b3 ? lo : b3;
    hi = hi > c2 ? hi : c2;
    hi = hi > c3 ? hi : c3;
    lo = lo < c2 ? lo : c2;
    lo = lo < c3 ? lo : c3;
  }
  li = (F)((double)dsl[0] * c.lx[0] + (double)dsl[1] * c.lx[1]);
  mi = lo;
  ma = hi;
}

struct QvCoefF {
  float cx[4], cy[4], qz[6], lx[2], ly[2], lz[2];
};

__device__ __forceinline__ void qv_to_float(const QvCoef& c, QvCoefF& w) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    w.cx[q] = (float)c.cx[q];
    w.cy[q] = (float)c.cy[q];
  }
#pragma unroll
  for (int q = 0; q < 6; q++) w.qz[q] = (float)c.qz[q];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    w.lx[q] = (float)c.lx[q];
    w.ly[q] = (float)c.ly[q];
    w.lz[q] = (float)c.lz[q];
  }
}

__device__ __forceinline__ void interp_qv_mixed(const float* __restrict__ s, int ni, long long nij, const QvCoef& c,
                                                const QvCoefF& w, float& xyz, float& li, float& mi, float& ma) {
  const long long p1 = c.pl[1] * nij, p2 = c.pl[2] * nij, p3 = c.pl[3] * nij, p4 = c.pl[4] * nij,
                  p5 = c.pl[5] * nij;
  float dst[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float v[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const float* t = s + i + r * ni;
      float a = __ldg(t) * w.qz[0];
      a = fmaf(__ldg(t + p1), w.qz[1], a);
      a = fmaf(__ldg(t + p2), w.qz[2], a);
      a = fmaf(__ldg(t + p3), w.qz[3], a);
      a = fmaf(__ldg(t + p4), w.qz[4], a);
      v[r] = fmaf(__ldg(t + p5), w.qz[5], a);
    }
    dst[i] = fmaf(v[3], w.cy[3], fmaf(v[2], w.cy[2], fmaf(v[1], w.cy[1], v[0] * w.cy[0])));
  }
  xyz = fmaf(dst[3], w.cx[3], fmaf(dst[2], w.cx[2], fmaf(dst[1], w.cx[1], dst[0] * w.cx[0])));
  float dsl[2];
  float hi = __ldg(s + 1 + ni + p2), lo = hi;
#pragma unroll
  for (int i = 1; i <= 2; i++) {
    const float b2 = __ldg(s + i + ni + p2), b3 = __ldg(s + i + ni + p3);
    const float c2 = __ldg(s + i + 2 * ni + p2), c3 = __ldg(s + i + 2 * ni + p3);
    dsl[i - 1] = fmaf(fmaf(c3, w.lz[1], c2 * w.lz[0]), w.ly[1], fmaf(b3, w.lz[1], b2 * w.lz[0]) * w.ly[0]);
    hi = fmaxf(fmaxf(hi, b2), fmaxf(b3, fmaxf(c2, c3)));
    lo = fminf(fminf(lo, b2), fminf(b3, fminf(c2, c3)));
  }
  li = fmaf(dsl[1], w.lx[1], dsl[0] * w.lx[0]);
  mi = lo;
  ma = hi;
}

}  // namespace adz
