/*
 * ORACLE — test infrastructure only.  Nothing in the product links this file.
 *
 * CPU restatement of GEM's tricubic / trilinear interpolators
 * (src/gemdyn/src/base/turbo_tricublin.c).  It follows the reference's
 * production (AVX2) arithmetic order operation by operation, written as scalar
 * C with explicit fma() calls, so that with -ffp-contract=off it reproduces the
 * reference build bit for bit:
 *
 *   - level descriptor          turbo_tricublin.c:164-173, 252-257, 320-380
 *   - per-point coefficients    turbo_tricublin.c:382-512 (non-SIMD branch)
 *   - single-field cubic        turbo_tricublin.c:551-615  (AVX2 branch)
 *   - mono (cubic+lin+min/max)  turbo_tricublin.c:869-997  (AVX2 branch: min/max
 *                               over x in {1,2}, y in {0..3}, z in {1,2})
 *                               and :998-1025 (scalar branch: 2x2x2 box)
 *   - 3-component cubic         turbo_tricublin.c:1153-1272 (AVX2 branch)
 *
 * The FP64 variants (``*_f64``) are this project's double-field extension of the
 * same algorithm.  Their cell index comes from the FP32-rounded position, like
 * the reference (turbo_tricublin.c:395-399 receives float positions), while the
 * fractional offset is taken from the FP64 position.  They use the same
 * operation order, and serve as the bit-exact oracle of the FP64 GPU path and
 * as the FP64 accuracy reference of the mixed-precision path.
 *
 * Parity of this restatement is pinned against the reference file compiled
 * unchanged (oracle/_ref) and against its SELF_TEST known answers.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* Contraction of ``pz = dz*pos[1] + (1.0-dz)*pos[0]`` (turbo_tricublin.c:440)
 * as emitted by gcc -O2 -mavx2 -mfma for the reference file: the first product
 * is fused into the add.  Pinned by test_oracle_vs_reference. */
#ifndef ORC_PZ_FMA
#define ORC_PZ_FMA 1
#endif

static inline double denom_inv(double x, double a, double b, double c) {
  return 1.0 / ((x - a) * (x - b) * (x - c));
}

orc_ztab *orc_vsearch_setup_plus(const double *levels, int nk, int ni, int nj, int offi, int offj) {
  int nkl = nk > 4 ? nk : 4;
  orc_ztab *lv = (orc_ztab *)calloc(1, sizeof(orc_ztab));
  if (!lv) return NULL;
  lv->z = (double *)malloc(sizeof(double) * (nk > 0 ? nk : 1));
  lv->ocz = (double *)malloc(sizeof(double) * 4 * nkl);
  if (!lv->z || !lv->ocz) { free(lv->z); free(lv->ocz); free(lv); return NULL; }
  for (int i = 0; i < nk; i++) lv->z[i] = levels[i];
  if (nk >= 4) {
    /* intervals 0, nk-2 and nk-1 get the end stencils; they are only read in
     * the cubic branch, which never selects them */
    const double *t = levels;
    double *r = lv->ocz;
    r[0] = denom_inv(t[0], t[1], t[2], t[3]);
    r[1] = denom_inv(t[1], t[0], t[2], t[3]);
    r[2] = denom_inv(t[2], t[0], t[1], t[3]);
    r[3] = denom_inv(t[3], t[0], t[1], t[2]);
    for (int i = 1; i < nk - 2; i++) {
      double a = t[i - 1], b = t[i], c = t[i + 1], d = t[i + 2];
      r[4 * i + 0] = denom_inv(a, b, c, d);
      r[4 * i + 1] = denom_inv(b, a, c, d);
      r[4 * i + 2] = denom_inv(c, a, b, d);
      r[4 * i + 3] = denom_inv(d, a, b, c);
    }
    for (int e = nk - 2; e <= nk - 1; e++) {
      double a = t[nk - 4], b = t[nk - 3], c = t[nk - 2], d = t[nk - 1];
      r[4 * e + 0] = denom_inv(a, b, c, d);
      r[4 * e + 1] = denom_inv(b, a, c, d);
      r[4 * e + 2] = denom_inv(c, a, b, d);
      r[4 * e + 3] = denom_inv(d, a, b, c);
    }
  } else {
    for (int i = 0; i < 4 * nkl; i++) lv->ocz[i] = 1.0;
  }
  lv->ni = ni; lv->nj = nj; lv->nk = nk; lv->nij = ni * nj;
  lv->offi = offi; lv->offj = offj;
  return lv;
}

void orc_ztab_free(orc_ztab *lv) {
  if (!lv) return;
  free(lv->z); free(lv->ocz); free(lv);
}

/* Coefficients shared by all variants once the cell (ix,iy,iz) and the three
 * offsets are known.  c[0..3] x cubic, c[4..7] y cubic, c[8..11] z (cubic or
 * linear), c[12..19] the linear coefficients.  Returns zlinear (0 or -1). */
static inline int coef_from_cell(double *c, int *offset, double px, double py, double dz,
                                 int ix, int iy, int iz, const orc_ztab *lv) {
  const double one = 1.0, two = 2.0;
  const double cp167 = 1.0 / 6.0, cm167 = -1.0 / 6.0, cp5 = 0.5, cm5 = -0.5;
  int ijk = ix - 2;
  c[12] = 0.0; c[13] = 1.0 - px; c[14] = px; c[15] = 0.0;
  ijk = ijk + (iy - 2) * lv->ni;
  c[16] = 1.0 - py; c[17] = py;
  ijk = ijk + (iz - 1) * lv->nij;
  c[18] = 1.0 - dz; c[19] = dz;
  iz--;
  int zlinear = (iz < 1 || iz > lv->nk - 3) ? -1 : 0;
  if (!zlinear) ijk -= lv->nij;
  *offset = ijk;
  if (zlinear) {
    c[8] = 0.0; c[9] = 1.0 - dz; c[10] = dz; c[11] = 0.0;
  } else {
    const double *base = lv->ocz + 4 * iz;
    const double *pos = lv->z + iz;
#if ORC_PZ_FMA == 1
    double pz = fma(dz, pos[1], (1.0 - dz) * pos[0]);
#elif ORC_PZ_FMA == 2
    double pz = fma(1.0 - dz, pos[0], dz * pos[1]);
#else
    double pz = dz * pos[1] + (1.0 - dz) * pos[0];
#endif
    double zza = pz - pos[-1], zzb = pz - pos[0], zzc = pz - pos[1], zzd = pz - pos[2];
    double zzab = zza * zzb, zzcd = zzc * zzd;
    c[8] = zzb * zzcd * base[0];
    c[9] = zza * zzcd * base[1];
    c[10] = zzd * zzab * base[2];
    c[11] = zzc * zzab * base[3];
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

/* Reference precision: FP32 position -> cell by truncation, offsets in FP64
 * (turbo_tricublin.c:395-423). */
int orc_coef_f32pos(double *c, int *offset, float pxf, float pyf, float pzf, const orc_ztab *lv) {
  double px = pxf, py = pyf, pz = pzf;
  int ix = (int)px; px = px - ix; ix += lv->offi;
  int iy = (int)py; py = py - iy; iy += lv->offj;
  int iz = (int)pz;
  if (iz < 1) iz = 1;
  if (iz > lv->nk - 1) iz = lv->nk - 1;
  double dz = pz - iz;
  return coef_from_cell(c, offset, px, py, dz, ix, iy, iz, lv);
}

/* FP64 position: the cell is chosen from the FP32-rounded position exactly as
 * the reference does, the offset inside the cell is the FP64 difference. */
int orc_coef_f64pos(double *c, int *offset, double px8, double py8, double pz8, const orc_ztab *lv) {
  int ix = (int)(double)(float)px8;
  int iy = (int)(double)(float)py8;
  int iz = (int)(double)(float)pz8;
  double px = px8 - ix, py = py8 - iy;
  ix += lv->offi; iy += lv->offj;
  if (iz < 1) iz = 1;
  if (iz > lv->nk - 1) iz = lv->nk - 1;
  double dz = pz8 - iz;
  return coef_from_cell(c, offset, px, py, dz, ix, iy, iz, lv);
}

/* ---- single field cubic, AVX2 order (turbo_tricublin.c:551-615) ---- */
#define ZYX1_BODY(LOAD)                                                        \
  const double *px = c, *py = c + 4, *pz = c + 8;                              \
  long ni = lv->ni, ninj = lv->nij, ninjl = zlinear ? 0 : ninj;                \
  double ya[4];                                                                \
  for (int r = 0; r < 4; r++) {                                                \
    long s = r * ni;                                                           \
    for (int x = 0; x < 4; x++) {                                              \
      long p0 = s + x, p1 = p0 + ninjl, p2 = p1 + ninj, p3 = p2 + ninjl;       \
      double za = LOAD(p0) * pz[0];                                            \
      za = fma(LOAD(p1), pz[1], za);                                           \
      za = fma(LOAD(p2), pz[2], za);                                           \
      za = fma(LOAD(p3), pz[3], za);                                           \
      ya[x] = (r == 0) ? za * py[0] : fma(za, py[r], ya[x]);                   \
    }                                                                          \
  }                                                                            \
  double res = (ya[0] * px[0] + ya[2] * px[2]) + (ya[1] * px[1] + ya[3] * px[3]);

static inline float zyx1_f32(const float *f, const double *c, const orc_ztab *lv, int zlinear) {
#define LD(p) ((double)f[p])
  ZYX1_BODY(LD)
#undef LD
  return (float)res;
}

static inline double zyx1_f64(const double *f, const double *c, const orc_ztab *lv, int zlinear) {
#define LD(p) (f[p])
  ZYX1_BODY(LD)
#undef LD
  return res;
}

/* ---- mono: cubic + trilinear + min/max (turbo_tricublin.c:869-997 AVX2,
 * :998-1025 scalar box) ---- */
static inline double vmin(double a, double b) { return (a < b) ? a : b; } /* _mm_min_pd */
static inline double vmax(double a, double b) { return (a > b) ? a : b; } /* _mm_max_pd */

#define MONO_BODY(LOAD)                                                          \
  const double *px = c, *py = c + 4, *pz = c + 8;                                \
  long ni = lv->ni, ninj = lv->nij, ninjl = zlinear ? 0 : ninj;                  \
  double ya[4], mi[4], ma[4], vyl[4];                                            \
  for (int r = 0; r < 4; r++) {                                                  \
    long s = r * ni;                                                             \
    for (int x = 0; x < 4; x++) {                                                \
      long p0 = s + x, p1 = p0 + ninjl, p2 = p1 + ninj, p3 = p2 + ninjl;         \
      double v0 = LOAD(p0), v1 = LOAD(p1), v2 = LOAD(p2), v3 = LOAD(p3);         \
      double za = v0 * pz[0];                                                    \
      if (r == 0) { mi[x] = v1; ma[x] = v1; }                                    \
      else { mi[x] = vmin(mi[x], v1); ma[x] = vmax(ma[x], v1); }                 \
      za = fma(v1, pz[1], za);                                                   \
      mi[x] = vmin(mi[x], v2); ma[x] = vmax(ma[x], v2);                          \
      za = fma(v2, pz[2], za);                                                   \
      za = fma(v3, pz[3], za);                                                   \
      ya[x] = (r == 0) ? za * py[0] : fma(za, py[r], ya[x]);                     \
      if (r == 1 || r == 2) {                                                    \
        double vzl = v1 * c[18];                                                 \
        vzl = fma(v2, c[19], vzl);                                               \
        vyl[x] = (r == 1) ? vzl * c[16] : fma(vzl, c[17], vyl[x]);               \
      }                                                                          \
    }                                                                            \
  }                                                                              \
  double fmi = vmin(mi[1], mi[2]);                                               \
  double fma_ = vmax(ma[1], ma[2]);                                              \
  double l0 = vyl[0] * c[12], l1 = vyl[1] * c[13], l2 = vyl[2] * c[14], l3 = vyl[3] * c[15]; \
  double lin = (l0 + l2) + (l1 + l3);                                            \
  double res = (ya[0] * px[0] + ya[2] * px[2]) + (ya[1] * px[1] + ya[3] * px[3]);

static inline void mono_f32(float *d, float *l, float *mn, float *mx, const float *f,
                            const double *c, const orc_ztab *lv, int zlinear) {
#define LD(p) ((double)f[p])
  MONO_BODY(LD)
#undef LD
  *mn = (float)fmi; *mx = (float)fma_; *l = (float)lin; *d = (float)res;
}

static inline void mono_f64(double *d, double *l, double *mn, double *mx, const double *f,
                            const double *c, const orc_ztab *lv, int zlinear) {
#define LD(p) (f[p])
  MONO_BODY(LD)
#undef LD
  *mn = fmi; *mx = fma_; *l = lin; *d = res;
}

/* scalar-branch box (2x2x2) min/max, turbo_tricublin.c:1017-1025, offered as
 * an option next to the AVX2 box */
static inline void box222_f32(float *mn, float *mx, const float *f, const orc_ztab *lv, int zlinear) {
  long ni = lv->ni, ninj = lv->nij, ninjl = zlinear ? 0 : ninj, ninj2 = ninj + ninjl;
  float ma = f[1 + ni + ninjl], mi = ma;
  for (int i = 1; i < 3; i++) {
    float a = f[i + ni + ninjl], b = f[i + ni + ninj2], e = f[i + 2 * ni + ninjl], g = f[i + 2 * ni + ninj2];
    ma = (ma > a) ? ma : a; ma = (ma > b) ? ma : b;
    mi = (mi < a) ? mi : a; mi = (mi < b) ? mi : b;
    ma = (ma > e) ? ma : e; ma = (ma > g) ? ma : g;
    mi = (mi < e) ? mi : e; mi = (mi < g) ? mi : g;
  }
  *mn = mi; *mx = ma;
}

/* ---- 3-component cubic (turbo_tricublin.c:1153-1272, AVX2) ---- */
#define ZYX3_BODY(LOAD, OUT)                                                     \
  const double *px = c, *py = c + 4, *pz = c + 8;                                \
  long ni = 3L * lv->ni, ninj = 3L * lv->nij, ninjl = zlinear ? 0 : ninj;        \
  double ya[12];                                                                 \
  for (int r = 0; r < 4; r++) {                                                  \
    long s = r * ni;                                                             \
    for (int e = 0; e < 12; e++) {                                               \
      long p0 = s + e, p1 = p0 + ninjl, p2 = p1 + ninj, p3 = p2 + ninjl;         \
      double za = LOAD(p0) * pz[0];                                              \
      za = fma(LOAD(p1), pz[1], za);                                             \
      za = fma(LOAD(p2), pz[2], za);                                             \
      za = fma(LOAD(p3), pz[3], za);                                             \
      ya[e] = (r == 0) ? za * py[0] : fma(za, py[r], ya[e]);                     \
    }                                                                            \
  }                                                                              \
  for (int comp = 0; comp < 3; comp++) {                                         \
    double x0 = ya[comp] * px[0];                                                \
    x0 = fma(ya[3 + comp], px[1], x0);                                           \
    x0 = fma(ya[6 + comp], px[2], x0);                                           \
    x0 = fma(ya[9 + comp], px[3], x0);                                           \
    OUT[comp] = x0;                                                              \
  }

static inline void zyx3_f32(float *d, const float *f, const double *c, const orc_ztab *lv, int zlinear) {
  double o[3];
#define LD(p) ((double)f[p])
  ZYX3_BODY(LD, o)
#undef LD
  d[0] = (float)o[0]; d[1] = (float)o[1]; d[2] = (float)o[2];
}

static inline void zyx3_f64(double *d, const double *f, const double *c, const orc_ztab *lv, int zlinear) {
#define LD(p) (f[p])
  ZYX3_BODY(LD, d)
#undef LD
}

/* ================= exported entry points (reference call shapes) ================= */

/* Tricublin_zyx1_m_n: d[m][n] (turbo_tricublin.c:793-815) */
void orc_zyx1_m_n_f32(float *d, const float *const *fs, const float *pxyz, const orc_ztab *lv, int n, int m) {
  double c[24];
  int off;
  for (int j = 0; j < n; j++) {
    int zl = orc_coef_f32pos(c, &off, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
    for (int i = 0; i < m; i++) d[(long)i * n + j] = zyx1_f32(fs[i] + off, c, lv, zl);
  }
}

/* Tricublin_mono_zyx_m_n (turbo_tricublin.c:1080-1109); box: 0 = AVX2 2x4x2,
 * 1 = scalar-branch 2x2x2 */
void orc_mono_m_n_f32(float *d, float *l, float *mn, float *mx, const float *const *fs, const float *pxyz,
                      const orc_ztab *lv, int n, int m, int box) {
  double c[24];
  int off;
  for (int j = 0; j < n; j++) {
    int zl = orc_coef_f32pos(c, &off, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
    for (int i = 0; i < m; i++) {
      long o = (long)i * n + j;
      mono_f32(d + o, l + o, mn + o, mx + o, fs[i] + off, c, lv, zl);
      if (box == 1) box222_f32(mn + o, mx + o, fs[i] + off, lv, zl);
    }
  }
}

/* Tricublin_zyx3_n: d[n][3] (turbo_tricublin.c:1298-1312) */
void orc_zyx3_n_f32(float *d, const float *f3, const float *pxyz, const orc_ztab *lv, int n) {
  double c[24];
  int off;
  for (int j = 0; j < n; j++) {
    int zl = orc_coef_f32pos(c, &off, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
    zyx3_f32(d + 3 * j, f3 + 3L * off, c, lv, zl);
  }
}

/* FP64 extension: double fields, double positions (3 per point). */
void orc_zyx1_m_n_f64(double *d, const double *const *fs, const double *pxyz, const orc_ztab *lv, int n, int m) {
  double c[24];
  int off;
  for (int j = 0; j < n; j++) {
    int zl = orc_coef_f64pos(c, &off, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
    for (int i = 0; i < m; i++) d[(long)i * n + j] = zyx1_f64(fs[i] + off, c, lv, zl);
  }
}

void orc_mono_m_n_f64(double *d, double *l, double *mn, double *mx, const double *const *fs, const double *pxyz,
                      const orc_ztab *lv, int n, int m) {
  double c[24];
  int off;
  for (int j = 0; j < n; j++) {
    int zl = orc_coef_f64pos(c, &off, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
    for (int i = 0; i < m; i++) {
      long o = (long)i * n + j;
      mono_f64(d + o, l + o, mn + o, mx + o, fs[i] + off, c, lv, zl);
    }
  }
}

void orc_zyx3_n_f64(double *d, const double *f3, const double *pxyz, const orc_ztab *lv, int n) {
  double c[24];
  int off;
  for (int j = 0; j < n; j++) {
    int zl = orc_coef_f64pos(c, &off, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
    zyx3_f64(d + 3 * j, f3 + 3L * off, c, lv, zl);
  }
}

/* Cell selection only, for index-parity checks: returns the linear offset of
 * the stencil corner and the zlinear flag for FP32 and FP64 positions. */
void orc_cells_f32(int *off, int *zl, const float *pxyz, const orc_ztab *lv, int n) {
  double c[24];
  for (int j = 0; j < n; j++) zl[j] = orc_coef_f32pos(c, off + j, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
}

void orc_cells_f64(int *off, int *zl, const double *pxyz, const orc_ztab *lv, int n) {
  double c[24];
  for (int j = 0; j < n; j++) zl[j] = orc_coef_f64pos(c, off + j, pxyz[3 * j], pxyz[3 * j + 1], pxyz[3 * j + 2], lv);
}
