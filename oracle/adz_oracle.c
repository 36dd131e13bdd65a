/*
 * ORACLE — test infrastructure only (the checker and the timed CPU baseline;
 * never part of the product path).
 *
 * C restatement of GEM's semi-Lagrangian trajectory drivers, which are Fortran
 * in the reference and cannot be compiled here (no gfortran; rmn/rpncomm/vgrid
 * submodules absent).  Each function cites the Fortran it follows.  Operation
 * order is kept literally and the file is compiled with -ffp-contract=off, so
 * the FP64 arithmetic is what an IEEE Fortran build without FMA contraction
 * produces.  Trajectory parity is therefore pinned to this restatement, not to
 * a Fortran run.
 *
 * Built twice:
 *   liboracle.so            - calls the interpolators restated in tricublin_oracle.c
 *   _ref/libadz_ref.so      - -DORC_USE_REF: calls the reference's own
 *                             turbo_tricublin.c (compiled unchanged) for the FP32
 *                             path; this is the timed "reference" CPU baseline.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "oracle.h"

#ifdef ORC_USE_REF
/* reference symbols (src/gemdyn/src/base/turbo_tricublin.c) */
typedef struct { float px, py, pz; } pxpypz;
void *Vsearch_setup_plus(double *targets, int nk, int ni, int nj, int offseti, int offsetj);
void Tricublin_zyx3_n(float *d, float *f3, pxpypz *pxyz, void *lv, int n);
void Tricublin_zyx1_m_n(float *dm, float **fs, pxpypz *pxyz, void *lv, int n, int m);
void Tricublin_mono_zyx_m_n(float *dm, float *lm, float *mim, float *mam, float **fs, pxpypz *pxyz, void *lv, int n,
                            int m);
static void *ref_ztab_m_of(const orc_set *s);
static void *ref_ztab_t_of(const orc_set *s);
#endif

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
static int nthr(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline double dmax(double a, double b) { return a > b ? a : b; }

/* ---------------- adz_set (src/gemdyn/src/base/adz_set.F90) ---------------- */
static double lag3(double zz, double z1, double z2, double z3, double z4) { /* adz_set.F90:530-536 */
  return (((zz - z2) * (zz - z3) * (zz - z4)) / ((z1 - z2) * (z1 - z3) * (z1 - z4)));
}

static int build_search(const double *z, int nk, double sig, const double *delz, double *ovdz, int **tab) {
  /* adz_set.F90:193-215: smallest_dz and posz are REAL128 in the reference */
  __float128 smallest = (__float128)(sig * delz[1]);
  for (int k = 2; k <= nk; k++) {
    __float128 v = (__float128)(sig * delz[k]);
    if (v < smallest) smallest = v;
  }
  double ov = (double)((__float128)1.0 / smallest);
  double pz = 1.0 + sig * (z[nk + 1] - z[0]) * ov;
  int pnz = (int)lround(pz); /* nint */
  *ovdz = (double)((__float128)sig / smallest);
  int *t = (int *)malloc(sizeof(int) * (pnz > 0 ? pnz : 1));
  int k0 = 0;
  for (int k = 1; k <= pnz; k++) {
    __float128 posz = (__float128)(sig * z[0]) + (__float128)(double)(k - 1) * smallest;
    if (posz > (__float128)(sig * z[k0 + 1])) k0 = imin(nk + 1, k0 + 1);
    t[k - 1] = k0;
  }
  *tab = t;
  return pnz;
}

int orc_adz_set(const orc_grid *g, orc_set *s) {
  memset(s, 0, sizeof(*s));
  s->g = *g;
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const double EPS_8 = 2.e-5;
  const int BCS_BASE = 4, ext = 1;
  int maxcfl = imax(1, g->maxcfl); /* adz_set.F90:71-82 */
  s->halox = maxcfl + 1; s->haloy = s->halox;
  s->lminx = 1 - s->halox; s->lmaxx = ni + s->halox;
  s->lminy = 1 - s->haloy; s->lmaxy = nj + s->haloy;
  s->nit = s->lmaxx - s->lminx + 1; s->njt = s->lmaxy - s->lminy + 1; s->nij = s->nit * s->njt;
  s->niu = ni - (g->east ? 1 : 0); s->njv = nj - (g->north ? 1 : 0); /* domain_decomp.F90:64-67 */
  s->i0 = 1 + g->pil_w - (ext + 1) * g->west; /* adz_set.F90:94-114 */
  s->in = ni - g->pil_e + ext * g->east;
  s->j0 = 1 + g->pil_s - (ext + 1) * g->south;
  s->jn = nj - g->pil_n + ext * g->north;
  s->i0u = 1 + g->pil_w; s->j0v = 1 + g->pil_s;
  s->inu = s->niu - g->pil_e; s->jnv = s->njv - g->pil_n;
  s->k0 = g->lam_gbpil_t + 1;
  s->k0t = imax(1, g->lam_gbpil_t);
  s->k0m = imax(s->k0t - 2, 1);
  if (g->bc_lam_flux != 0) s->k0m = 1;
  /* clip bounds, adz_set.F90:132-160 */
  s->iminposx = g->i0g + s->lminx + EPS_8;
  s->imaxposx = g->i0g + s->lmaxx - 2 - EPS_8;
  s->iminposy = g->j0g + s->lminy + EPS_8;
  s->imaxposy = g->j0g + s->lmaxy - 2 - EPS_8;
  if (g->west) s->iminposx = g->i0g + BCS_BASE + EPS_8;
  if (g->east) s->imaxposx = g->i0g + ni - BCS_BASE - 1 - EPS_8;
  if (g->south) s->iminposy = g->j0g + BCS_BASE + EPS_8;
  if (g->north) s->imaxposy = g->j0g + nj - BCS_BASE - 1 - EPS_8;
  s->i0b = 1 + BCS_BASE * g->west; s->inb = ni - BCS_BASE * g->east;
  s->j0b = 1 + BCS_BASE * g->south; s->jnb = nj - BCS_BASE * g->north;

  const double *zm = g->zm, *zt = g->zt, *zx = g->zx;
  s->delz_m = (double *)malloc(sizeof(double) * (nk + 1));
  s->delz_t = (double *)malloc(sizeof(double) * (nk + 1));
  s->odelz_m = (double *)malloc(sizeof(double) * (nk + 1));
  s->odelz_t = (double *)malloc(sizeof(double) * (nk + 1));
  s->sig = (zm[nk] - zm[1]) / fabs(zm[nk] - zm[1]); /* adz_set.F90:178-179 */
  const float verysmall = 1.17549435e-38f * 1.e5f;  /* tiny(real)*1.e5 */
  for (int k = 0; k <= nk; k++) {                   /* adz_set.F90:181-191 */
    s->delz_m[k] = (double)9.e33f; s->delz_t[k] = (double)9.e33f;
    if (fabs(zm[k + 1] - zm[k]) > verysmall) s->delz_m[k] = zm[k + 1] - zm[k];
    if (fabs(zt[k + 1] - zt[k]) > verysmall) s->delz_t[k] = zt[k + 1] - zt[k];
    s->odelz_m[k] = 1.0 / s->delz_m[k];
    s->odelz_t[k] = 1.0 / s->delz_t[k];
  }
  s->pnz_m = build_search(zm, nk, s->sig, s->delz_m, &s->ovdzm, &s->search_m);
  s->pnz_t = build_search(zt, nk, s->sig, s->delz_t, &s->ovdzt, &s->search_t);

  s->cy = (double *)malloc(sizeof(double) * s->njt);
  for (int j = 0; j < s->njt; j++) s->cy[j] = g->cy[j];

  double **vw[8] = {&s->vw1m, &s->vw2m, &s->vw3m, &s->vw4m, &s->vw1t, &s->vw2t, &s->vw3t, &s->vw4t};
  for (int q = 0; q < 8; q++) *vw[q] = (double *)calloc(nk + 1, sizeof(double));
  for (int k = 2; k <= nk - 1; k++) { /* adz_set.F90:261-271 */
    double rx = zm[k], ra = zx[k - 2], rb = zx[k - 1], rc = zx[k], rd = zx[k + 1];
    s->vw1m[k] = lag3(rx, ra, rb, rc, rd);
    s->vw2m[k] = lag3(rx, rb, ra, rc, rd);
    s->vw3m[k] = lag3(rx, rc, ra, rb, rd);
    s->vw4m[k] = lag3(rx, rd, ra, rb, rc);
  }
  for (int k = 2; k <= nk - 2; k++) { /* adz_set.F90:272-281 */
    double rx = zt[k], ra = zm[k - 1], rb = zm[k], rc = zm[k + 1], rd = zm[k + 2];
    s->vw1t[k] = lag3(rx, ra, rb, rc, rd);
    s->vw2t[k] = lag3(rx, rb, ra, rc, rd);
    s->vw3t[k] = lag3(rx, rc, ra, rb, rd);
    s->vw4t[k] = lag3(rx, rd, ra, rb, rc);
  }
  /* BICUBH_QV denominators, adz_set.F90:286-311 (products left to right) */
  s->qv_t = (double *)calloc((size_t)(nk + 1) * 10, sizeof(double));
  for (int k = 2; k <= nk - 2; k++) {
    const double ra = zt[k - 1], rb = zt[k], rc = zt[k + 1], rd = zt[k + 2];
    double *q = s->qv_t + (size_t)k * 10;
    q[0] = 1.0 / ((ra - rb) * (ra - rc) * (ra - rd));
    q[1] = 1.0 / ((rb - ra) * (rb - rc) * (rb - rd));
    q[2] = 1.0 / ((rc - ra) * (rc - rb) * (rc - rd));
    q[3] = 1.0 / ((rd - ra) * (rd - rb) * (rd - rc));
  }
  for (int k = 3; k <= nk - 3; k++) {
    const double r[6] = {zt[k - 2], zt[k - 1], zt[k], zt[k + 1], zt[k + 2], zt[k + 3]};
    double *q = s->qv_t + (size_t)k * 10 + 4;
    for (int a = 0; a < 6; a++) { /* quiprod(r_a, the other five in order) */
      double p = 1.0;
      int first = 1;
      for (int b = 0; b < 6; b++) {
        if (b == a) continue;
        if (first) { p = r[a] - r[b]; first = 0; }
        else p = p * (r[a] - r[b]);
      }
      q[a] = 1.0 / p;
    }
  }
  s->vw5 = (zx[0] - zm[1]) / (zx[0] - zx[1]); /* adz_set.F90:282-284 */
  s->vw6 = (zm[nk] - zx[nk]) / (zx[nk - 1] - zx[nk]);
  /* adz_interp_traj.F90:41-43 */
  s->ww = g->wmstar_nk;
  s->wp = (zt[nk] - zm[nk - 1]) * g->idz_t_nkm1;
  s->wm = 1.0 - s->wp;
  /* ztabs, adz_set.F90:128-131: levels m(1:nk) / t(1:nk), offsets 1-l_i0, 1-l_j0 */
  s->ztab_m = orc_vsearch_setup_plus(zm + 1, nk, s->nit, s->njt, 1 - g->i0g, 1 - g->j0g);
  s->ztab_t = orc_vsearch_setup_plus(zt + 1, nk, s->nit, s->njt, 1 - g->i0g, 1 - g->j0g);
#ifdef ORC_USE_REF
  /* the reference's own descriptors (never freed: the reference has no destroy) */
  s->ref_m = Vsearch_setup_plus((double *)zm + 1, nk, s->nit, s->njt, 1 - g->i0g, 1 - g->j0g);
  s->ref_t = Vsearch_setup_plus((double *)zt + 1, nk, s->nit, s->njt, 1 - g->i0g, 1 - g->j0g);
#endif
  return 0;
}

void orc_adz_free(orc_set *s) {
  free(s->delz_m); free(s->delz_t); free(s->odelz_m); free(s->odelz_t);
  free(s->search_m); free(s->search_t); free(s->cy);
  free(s->vw1m); free(s->vw2m); free(s->vw3m); free(s->vw4m);
  free(s->vw1t); free(s->vw2t); free(s->vw3t); free(s->vw4t);
  free(s->qv_t);
  orc_ztab_free(s->ztab_m); orc_ztab_free(s->ztab_t);
  memset(s, 0, sizeof(*s));
}

long orc_set_npoints(const orc_set *s, int set) {
  int nk = s->g.nk;
  switch (set) {
    case 0: return (long)(s->in - s->i0 + 1) * (s->jn - s->j0 + 1) * (nk - s->k0 + 1);
    case 1: return (long)(s->inu - s->i0u + 1) * (s->jn - s->j0 + 1) * (nk - s->k0 + 1);
    case 2: return (long)(s->in - s->i0 + 1) * (s->jnv - s->j0v + 1) * (nk - s->k0 + 1);
    default: return (long)(s->in - s->i0 + 1) * (s->jn - s->j0 + 1) * (nk - s->k0t + 1);
  }
}

/* ranges of a position set: i0,in,j0,jn,k0 */
static void set_range(const orc_set *s, int set, int *r) {
  switch (set) {
    case 0: r[0] = s->i0; r[1] = s->in; r[2] = s->j0; r[3] = s->jn; r[4] = s->k0; break;
    case 1: r[0] = s->i0u; r[1] = s->inu; r[2] = s->j0; r[3] = s->jn; r[4] = s->k0; break;
    case 2: r[0] = s->i0; r[1] = s->in; r[2] = s->j0v; r[3] = s->jnv; r[4] = s->k0; break;
    case 4: r[0] = s->i0b; r[1] = s->inb; r[2] = s->j0b; r[3] = s->jnb; r[4] = 1; break; /* Adz_pb */
    default: r[0] = s->i0; r[1] = s->in; r[2] = s->j0; r[3] = s->jn; r[4] = s->k0t; break;
  }
}

#ifdef ORC_USE_REF
static void *ref_ztab_m_of(const orc_set *s) { return s->ref_m; }
static void *ref_ztab_t_of(const orc_set *s) { return s->ref_t; }
#endif

/* ------------- precision templates ------------- */
#define REAL float
#define SFX(name) name##_f32
#define IS_F32 1
#include "adz_oracle_impl.h"
#undef REAL
#undef SFX
#undef IS_F32

#define REAL double
#define SFX(name) name##_f64
#define IS_F32 0
#include "adz_oracle_impl.h"
#undef REAL
#undef SFX
#undef IS_F32
