/*
 * ORACLE — test infrastructure only.  Precision template of the driver
 * restatement, included by adz_oracle.c with REAL = float (the reference's
 * ``real`` storage) and REAL = double (this project's FP64 extension).
 * Where Fortran adds two ``real`` values before promoting (e.g.
 * adz_prepareWinds.F90:42-43, adz_interp_traj.F90:112), the sum is formed in
 * REAL, as the reference does.
 */

#define EXT(i, j, k) ((long)((i) - s->lminx) + (long)((j) - s->lminy) * s->nit + (long)((k) - 1) * s->nij)
#define ARR(i, j, k) ((long)((i) - 1) + (long)((j) - 1) * ni + (long)((k) - 1) * (long)ni * nj)
#define WP(i, j, k, c)                                                                     \
  ((long)((i) + 1) + (long)((j) + 1) * (ni + 4) + (long)((k) - 1) * (long)(ni + 4) * (nj + 4) + \
   (long)((c) - 1) * (long)(ni + 4) * (nj + 4) * nk)

static inline REAL SFX(rmin)(REAL a, REAL b) { return a < b ? a : b; }
static inline REAL SFX(rmax)(REAL a, REAL b) { return a > b ? a : b; }

/* adz_prepareWinds.F90:16-107 */
void SFX(orc_prepare_winds)(const orc_set *s, const REAL *uu_ext, const REAL *vv_ext, const REAL *ww_ext,
                            const REAL *ut0, const REAL *vt0, const REAL *zdt0, REAL *uvw_d, REAL *uu_arr,
                            REAL *vv_arr, REAL *ww_arr) {
  const int ni = s->g.ni, nj = s->g.nj, nk = s->g.nk;
  const double alpha1 = -1.0 / 16.0, alpha2 = 9.0 / 16.0, inv_rayt = s->g.inv_rayt;
  double *wx = (double *)calloc(nk + 1, sizeof(double));
  int *km2 = (int *)calloc(nk + 1, sizeof(int));
  for (int k = 3; k <= nk; k++) wx[k] = s->vw1m[k];
  for (int k = 2; k <= nk - 1; k++) km2[k] = imax(1, k - 2);
#pragma omp parallel for num_threads(nthr()) schedule(static)
  for (int k = 1; k <= nk; k++) {
    for (int j = s->lminy; j <= s->lmaxy; j++) {
      double cyj = s->cy[j - s->lminy];
      for (int i = s->lminx; i <= s->lmaxx; i++) {
        long e = EXT(i, j, k);
        uvw_d[3 * e + 0] = (REAL)(inv_rayt * uu_ext[e] * cyj);
        uvw_d[3 * e + 1] = (REAL)(inv_rayt * vv_ext[e]);
        double w;
        if (k == 1) w = s->vw5 * ww_ext[EXT(i, j, 1)];
        else if (k == nk) w = s->vw6 * ww_ext[EXT(i, j, nk - 1)];
        else
          w = wx[k] * ww_ext[EXT(i, j, km2[k])] + s->vw2m[k] * ww_ext[EXT(i, j, k - 1)] +
              s->vw3m[k] * ww_ext[EXT(i, j, k)] + s->vw4m[k] * ww_ext[EXT(i, j, k + 1)];
        uvw_d[3 * e + 2] = (REAL)w;
      }
    }
    for (int j = 1; j <= nj; j++) {
      double cyj = s->cy[j - s->lminy];
      for (int i = 1; i <= ni; i++) {
        long a = ARR(i, j, k);
        REAL u1 = ut0[EXT(i - 2, j, k)] + ut0[EXT(i + 1, j, k)];
        REAL u2 = ut0[EXT(i, j, k)] + ut0[EXT(i - 1, j, k)];
        uu_arr[a] = (REAL)((u1 * alpha1 + u2 * alpha2) * inv_rayt * cyj);
        REAL v1 = vt0[EXT(i, j - 2, k)] + vt0[EXT(i, j + 1, k)];
        REAL v2 = vt0[EXT(i, j, k)] + vt0[EXT(i, j - 1, k)];
        vv_arr[a] = (REAL)((v1 * alpha1 + v2 * alpha2) * inv_rayt);
        double w;
        if (k == 1) w = s->vw5 * zdt0[EXT(i, j, 1)];
        else if (k == nk) w = s->vw6 * zdt0[EXT(i, j, nk - 1)];
        else
          w = wx[k] * zdt0[EXT(i, j, km2[k])] + s->vw2m[k] * zdt0[EXT(i, j, k - 1)] +
              s->vw3m[k] * zdt0[EXT(i, j, k)] + s->vw4m[k] * zdt0[EXT(i, j, k + 1)];
        ww_arr[a] = (REAL)w;
      }
    }
  }
  free(wx);
  free(km2);
}

/* adz_inittraj.F90:25-37 (the caller also sets niter = max(6, itraj)) */
void SFX(orc_inittraj)(const orc_set *s, REAL *pxyzm, double *wpxyz) {
  const int ni = s->g.ni, nj = s->g.nj, nk = s->g.nk;
  for (int k = s->k0m; k <= nk; k++)
    for (int j = 1; j <= nj; j++)
      for (int i = 1; i <= ni; i++) {
        long a = ARR(i, j, k);
        pxyzm[3 * a + 0] = (REAL)(i + s->g.i0g - 1);
        wpxyz[WP(i, j, k, 1)] = pxyzm[3 * a + 0];
        pxyzm[3 * a + 1] = (REAL)(j + s->g.j0g - 1);
        wpxyz[WP(i, j, k, 2)] = pxyzm[3 * a + 1];
        pxyzm[3 * a + 2] = (REAL)k;
        wpxyz[WP(i, j, k, 3)] = pxyzm[3 * a + 2];
      }
}

static void SFX(dt_split)(const orc_set *s, double dt, double *dtA, double *dtzA, double *dtD, double *dtzD) {
  /* adz_traject.F90:38-59 */
  double a = 0.0, za = 0.0;
  int adv = s->g.schm_advec;
  if (adv == 1) { a = dt * 0.5; za = dt * 0.5; }
  if (adv == 2) { a = dt * s->g.bA_m; za = dt * s->g.bA; }
  if (adv == 3) { a = (1.0 - s->g.bA_m) * dt; za = (1.0 - s->g.bA) * dt; }
  *dtD = dt - a; *dtzD = dt - za; *dtA = a; *dtzA = za;
  if (adv == 0) { *dtA = 0.0; *dtD = 0.0; *dtzA = 0.0; *dtzD = 0.0; }
}

/* adz_traject.F90:63-108 (iterations) */
void SFX(orc_traject)(const orc_set *s, double dt, int niter, const REAL *uvw_d, const REAL *uu_arr,
                      const REAL *vv_arr, const REAL *ww_arr, REAL *uvw_dep, REAL *pxyzm, double *wpxyz) {
  const int ni = s->g.ni, nj = s->g.nj, nk = s->g.nk;
  double dtA, dtzA, dtD, dtzD;
  SFX(dt_split)(s, dt, &dtA, &dtzA, &dtD, &dtzD);
  int k00 = s->k0m;
  if (s->k0 > 1) k00 = 1;
  const double *zm = s->g.zm;
  const double sig = s->sig;
  const REAL *f3 = uvw_d + 3 * EXT(1, 1, 1);
  for (int iter = 1; iter <= niter; iter++) {
#pragma omp parallel for num_threads(nthr()) schedule(static)
    for (int k = k00; k <= nk; k++) {
      long a0 = ARR(1, 1, k);
#if IS_F32
#ifdef ORC_USE_REF
      Tricublin_zyx3_n(uvw_dep + 3 * a0, (float *)f3, (pxpypz *)(pxyzm + 3 * a0), ref_ztab_m_of(s), ni * nj);
#else
      orc_zyx3_n_f32(uvw_dep + 3 * a0, f3, pxyzm + 3 * a0, s->ztab_m, ni * nj);
#endif
#else
      orc_zyx3_n_f64(uvw_dep + 3 * a0, f3, pxyzm + 3 * a0, s->ztab_m, ni * nj);
#endif
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          long a = ARR(i, j, k);
          double xm = (double)(i + s->g.i0g - 1) - (dtD * uvw_dep[3 * a] + dtA * uu_arr[a]) * s->g.inv_hx;
          double ym = (double)(j + s->g.j0g - 1) - (dtD * uvw_dep[3 * a + 1] + dtA * vv_arr[a]) * s->g.inv_hy;
          double pos = zm[k] - dtzD * uvw_dep[3 * a + 2] - dtzA * ww_arr[a];
          double zmv = dmin(dmax(pos, s->g.zmin), s->g.zmax);
          int kk1 = (int)((zmv - zm[0]) * s->ovdzm + 1.0);
          kk1 = imin(imax(1, kk1), s->pnz_m);
          kk1 = s->search_m[kk1 - 1];
          if (sig * zmv > sig * zm[imin(kk1 + 1, nk + 1)]) kk1 = kk1 + 1;
          if (sig * zmv < sig * zm[kk1]) kk1 = kk1 - 1;
          wpxyz[WP(i, j, k, 1)] = xm;
          pxyzm[3 * a + 0] = (REAL)dmin(dmax(xm, s->iminposx), s->imaxposx);
          wpxyz[WP(i, j, k, 2)] = ym;
          pxyzm[3 * a + 1] = (REAL)dmin(dmax(ym, s->iminposy), s->imaxposy);
          kk1 = imin(nk + 1, imax(0, kk1));
          int nb = imax(imin(kk1, nk - 1), 1);
          double w3 = (zmv - zm[nb]) * s->odelz_m[nb] + (double)nb;
          wpxyz[WP(i, j, k, 3)] = w3;
          pxyzm[3 * a + 2] = (REAL)w3;
        }
    }
  }
}

/* zindx, adz_interp_traj.F90:189-204 */
static inline double SFX(zindx)(const orc_set *s, double posz) {
  const int nk = s->g.nk;
  const double *zt = s->g.zt;
  posz = dmin(dmax(posz, s->g.zmin), s->g.zmax);
  int kk1 = (int)((posz - zt[0]) * s->ovdzt + 1.0);
  kk1 = imin(imax(1, kk1), s->pnz_t);
  kk1 = s->search_t[kk1 - 1];
  if (s->sig * posz > s->sig * zt[imin(kk1 + 1, nk + 1)]) kk1 = kk1 + 1;
  if (s->sig * posz < s->sig * zt[kk1]) kk1 = kk1 - 1;
  kk1 = imin(nk + 1, imax(0, kk1));
  int nb = imax(imin(kk1, nk - 1), 1);
  return (posz - zt[nb]) * s->odelz_t[nb] + (double)nb;
}

/* Adz_pb (adz_interp_traj.F90:105-187) over (i0b:inb, j0b:jnb, 1:nk), point
 * (i, j, k) at pb + 3 * ((i - i0b) + (j - j0b) * bx + (k - 1) * bx * by);
 * levels below k00 are left as they are */
void SFX(orc_pb)(const orc_set *s, double dt, const double *wpxyz, const REAL *uvw_dep, const REAL *zdt0,
                 const REAL *uslt, const REAL *vslt, REAL *pb) {
  const int ni = s->g.ni, nj = s->g.nj, nk = s->g.nk;
  double dtA, dtzA, dtD, dtzD;
  SFX(dt_split)(s, dt, &dtA, &dtzA, &dtD, &dtzD);
  (void)dtA;
  (void)dtD;
  const double half = 0.5;
  const double *zt = s->g.zt;
  int k00 = imax(s->k0t - 1, 1);
  if (s->g.bc_lam_flux != 0 && s->k0 > 1) k00 = 1;
  const double imnx = s->iminposx, imxx = s->imaxposx, imny = s->iminposy, imxy = s->imaxposy;
  long bx = s->inb - s->i0b + 1, by = s->jnb - s->j0b + 1;
#define W(i, j, k, c) wpxyz[WP(i, j, k, c)]
#define UD3(i, j, k) uvw_dep[3 * ARR(i, j, k) + 2]
#define ZD(i, j, k) zdt0[EXT(i, j, k)]
#define PB(i, j, k) (pb + 3 * ((i - s->i0b) + (j - s->j0b) * bx + (long)((k) - 1) * bx * by))
#pragma omp parallel for num_threads(nthr()) schedule(static)
    for (int k = imax(k00, 2); k <= nk - 2; k++)
      for (int j = s->j0b; j <= s->jnb; j++)
        for (int i = s->i0b; i <= s->inb; i++) {
          double xt = s->vw1t[k] * W(i, j, k - 1, 1) + s->vw2t[k] * W(i, j, k, 1) + s->vw3t[k] * W(i, j, k + 1, 1) +
                      s->vw4t[k] * W(i, j, k + 2, 1);
          double yt = s->vw1t[k] * W(i, j, k - 1, 2) + s->vw2t[k] * W(i, j, k, 2) + s->vw3t[k] * W(i, j, k + 1, 2) +
                      s->vw4t[k] * W(i, j, k + 2, 2);
          double wdt = s->vw1t[k] * UD3(i, j, k - 1) + s->vw2t[k] * UD3(i, j, k) + s->vw3t[k] * UD3(i, j, k + 1) +
                       s->vw4t[k] * UD3(i, j, k + 2);
          double ztv = zt[k] - dtzD * wdt - dtzA * ZD(i, j, k);
          REAL *p = PB(i, j, k);
          p[0] = (REAL)dmin(dmax(xt, imnx), imxx);
          p[1] = (REAL)dmin(dmax(yt, imny), imxy);
          p[2] = (REAL)SFX(zindx)(s, ztv);
        }
    {
      int k = nk - 1;
      for (int j = s->j0b; j <= s->jnb; j++)
        for (int i = s->i0b; i <= s->inb; i++) {
          double xt = (W(i, j, k, 1) + W(i, j, k + 1, 1)) * half;
          double yt = (W(i, j, k, 2) + W(i, j, k + 1, 2)) * half;
          REAL ws = UD3(i, j, k) + UD3(i, j, k + 1);
          double wdt = ws * half;
          double ztv = zt[k] - dtzD * wdt - dtzA * ZD(i, j, k);
          REAL *p = PB(i, j, k);
          p[0] = (REAL)dmin(dmax(xt, imnx), imxx);
          p[1] = (REAL)dmin(dmax(yt, imny), imxy);
          p[2] = (REAL)SFX(zindx)(s, ztv);
        }
    }
    {
      int k = nk;
      for (int j = s->j0b; j <= s->jnb; j++)
        for (int i = s->i0b; i <= s->inb; i++) {
          double xt, yt;
          if (s->g.slt_winds && uslt && vslt) {
            long a2 = (i - 1) + (long)(j - 1) * ni;
            xt = (double)(i + s->g.i0g - 1) -
                 s->g.inv_rayt * dt * uslt[a2] * s->cy[j - s->lminy] * s->g.inv_hx;
            yt = (double)(j + s->g.j0g - 1) - s->g.inv_rayt * dt * vslt[a2] * s->g.inv_hy;
          } else {
            xt = s->wp * W(i, j, k, 1) + s->wm * W(i, j, k - 1, 1);
            yt = s->wp * W(i, j, k, 2) + s->wm * W(i, j, k - 1, 2);
          }
          REAL ws = UD3(i, j, k - 1) + UD3(i, j, k);
          double wdt = ws * half;
          double ztv = zt[k] - s->ww * (dtzD * wdt + dtzA * ZD(i, j, k - 1));
          REAL *p = PB(i, j, k);
          p[0] = (REAL)dmin(dmax(xt, imnx), imxx);
          p[1] = (REAL)dmin(dmax(yt, imny), imxy);
          p[2] = (REAL)SFX(zindx)(s, ztv);
        }
    }
    if (k00 == 1) {
      for (int j = s->j0b; j <= s->jnb; j++)
        for (int i = s->i0b; i <= s->inb; i++) {
          double xt = (W(i, j, 1, 1) + W(i, j, 2, 1)) * half;
          double yt = (W(i, j, 1, 2) + W(i, j, 2, 2)) * half;
          REAL ws = UD3(i, j, 1) + UD3(i, j, 2);
          double wdt = ws * half;
          double ztv = zt[1] - dtzD * wdt - dtzA * ZD(i, j, 1);
          REAL *p = PB(i, j, 1);
          p[0] = (REAL)dmin(dmax(xt, imnx), imxx);
          p[1] = (REAL)dmin(dmax(yt, imny), imxy);
          p[2] = (REAL)SFX(zindx)(s, ztv);
        }
    }
#undef PB
#undef W
#undef UD3
#undef ZD
}

/* adz_traject.F90:113-116 (Adz_pm) and adz_interp_traj.F90:16-187 */
void SFX(orc_interp_traj)(const orc_set *s, double dt, const double *wpxyz, const REAL *uvw_dep, const REAL *zdt0,
                          const REAL *pxyzm, const REAL *uslt, const REAL *vslt, REAL *pm, REAL *pmu, REAL *pmv,
                          REAL *pt) {
  const int ni = s->g.ni, nj = s->g.nj, nk = s->g.nk;
  double dtA, dtzA, dtD, dtzD;
  SFX(dt_split)(s, dt, &dtA, &dtzA, &dtD, &dtzD);
  const double half = 0.5, aa = -0.0625, bb = 0.5625;
  const double zmin_b = 0.0, zmax_b = (double)(nk + 1);
  const double *zt = s->g.zt;
  int k00 = imax(s->k0t - 1, 1);
  if (s->g.bc_lam_flux != 0 && s->k0 > 1) k00 = 1;
  const double imnx = s->iminposx, imxx = s->imaxposx, imny = s->iminposy, imxy = s->imaxposy;
#define W(i, j, k, c) wpxyz[WP(i, j, k, c)]
#define UD3(i, j, k) uvw_dep[3 * ARR(i, j, k) + 2]
#define ZD(i, j, k) zdt0[EXT(i, j, k)]
  if (pm) {
    long nx = s->in - s->i0 + 1, ny = s->jn - s->j0 + 1;
    for (int k = s->k0; k <= nk; k++)
      for (int j = s->j0; j <= s->jn; j++)
        for (int i = s->i0; i <= s->in; i++) {
          long o = (i - s->i0) + (j - s->j0) * nx + (long)(k - s->k0) * nx * ny;
          for (int c = 0; c < 3; c++) pm[3 * o + c] = pxyzm[3 * ARR(i, j, k) + c];
        }
  }
  if (pmu) {
    long nx = s->inu - s->i0u + 1, ny = s->jn - s->j0 + 1;
#pragma omp parallel for num_threads(nthr()) schedule(static)
    for (int k = s->k0; k <= nk; k++)
      for (int j = s->j0; j <= s->jn; j++)
        for (int i = s->i0u; i <= s->inu; i++) {
          double xt = aa * (W(i - 1, j, k, 1) + W(i + 2, j, k, 1)) + bb * (W(i, j, k, 1) + W(i + 1, j, k, 1)) - 0.5;
          double yt = aa * (W(i - 1, j, k, 2) + W(i + 2, j, k, 2)) + bb * (W(i, j, k, 2) + W(i + 1, j, k, 2));
          double ztv = aa * (W(i - 1, j, k, 3) + W(i + 2, j, k, 3)) + bb * (W(i, j, k, 3) + W(i + 1, j, k, 3));
          long o = (i - s->i0u) + (j - s->j0) * nx + (long)(k - s->k0) * nx * ny;
          pmu[3 * o + 0] = (REAL)dmin(dmax(xt, imnx), imxx);
          pmu[3 * o + 1] = (REAL)dmin(dmax(yt, imny), imxy);
          pmu[3 * o + 2] = (REAL)dmin(dmax(ztv, zmin_b), zmax_b);
        }
  }
  if (pmv) {
    long nx = s->in - s->i0 + 1, ny = s->jnv - s->j0v + 1;
#pragma omp parallel for num_threads(nthr()) schedule(static)
    for (int k = s->k0; k <= nk; k++)
      for (int j = s->j0v; j <= s->jnv; j++)
        for (int i = s->i0; i <= s->in; i++) {
          double xt = aa * (W(i, j - 1, k, 1) + W(i, j + 2, k, 1)) + bb * (W(i, j, k, 1) + W(i, j + 1, k, 1));
          double yt = aa * (W(i, j - 1, k, 2) + W(i, j + 2, k, 2)) + bb * (W(i, j, k, 2) + W(i, j + 1, k, 2)) - 0.5;
          double ztv = aa * (W(i, j - 1, k, 3) + W(i, j + 2, k, 3)) + bb * (W(i, j, k, 3) + W(i, j + 1, k, 3));
          long o = (i - s->i0) + (j - s->j0v) * nx + (long)(k - s->k0) * nx * ny;
          pmv[3 * o + 0] = (REAL)dmin(dmax(xt, imnx), imxx);
          pmv[3 * o + 1] = (REAL)dmin(dmax(yt, imny), imxy);
          pmv[3 * o + 2] = (REAL)dmin(dmax(ztv, zmin_b), zmax_b);
        }
  }
  if (pt) {
    /* pb over (i0b:inb, j0b:jnb, 1:nk) then pt = pb on the t range */
    long bx = s->inb - s->i0b + 1, by = s->jnb - s->j0b + 1;
    REAL *pb = (REAL *)malloc(sizeof(REAL) * 3 * bx * by * nk);
#define PB(i, j, k) (pb + 3 * ((i - s->i0b) + (j - s->j0b) * bx + (long)((k) - 1) * bx * by))
    SFX(orc_pb)(s, dt, wpxyz, uvw_dep, zdt0, uslt, vslt, pb);
    long nx = s->in - s->i0 + 1, ny = s->jn - s->j0 + 1;
    for (int k = s->k0t; k <= nk; k++)
      for (int j = s->j0; j <= s->jn; j++)
        for (int i = s->i0; i <= s->in; i++) {
          long o = (i - s->i0) + (j - s->j0) * nx + (long)(k - s->k0t) * nx * ny;
          REAL *p = PB(i, j, k);
          pt[3 * o + 0] = p[0]; pt[3 * o + 1] = p[1]; pt[3 * o + 2] = p[2];
        }
    free(pb);
#undef PB
  }
#undef W
#undef UD3
#undef ZD
}

/* adz_tricub_hlt (adz_interp_hlt.F90:98-182) plus the clip of
 * adz_post_tr.F90:81-94: one kernel call per k-plane of the set's range. */
static REAL SFX(rabs)(REAL x) { return IS_F32 ? (REAL)fabsf((float)x) : (REAL)fabs((double)x); }

/* pert: mcrhsint (element (1,1), rows ld apart) or NULL; when set, every
 * field takes the mono path for its trilinear value and dst = value +
 * mcrhsint(i,j) * abs(value - lin) in REAL, before the clip
 * (adz_interp_hlt.F90:99-100, 125-133) */
void SFX(orc_tricub_p)(const orc_set *s, int set, const REAL *pos, int m, const REAL *const *srcs,
                       REAL *const *dsts, int mono, int clip, REAL *const *lin, REAL *const *mn, REAL *const *mx,
                       const REAL *pert, int ld) {
  int r[5];
  set_range(s, set, r);
  const int nk = s->g.nk;
  const long nx = r[1] - r[0] + 1, ny = r[3] - r[2] + 1, np = nx * ny;
  if (np <= 0 || m <= 0) return;
  const long o111 = EXT(1, 1, 1);
#pragma omp parallel num_threads(nthr())
  {
    REAL **fs = (REAL **)malloc(sizeof(REAL *) * m);
    REAL *wrk = (REAL *)malloc(sizeof(REAL) * 4 * m * np);
    REAL *wl = wrk + m * np, *wmi = wrk + 2 * m * np, *wma = wrk + 3 * m * np;
    for (int q = 0; q < m; q++) fs[q] = (REAL *)srcs[q] + o111;
#pragma omp for schedule(static)
    for (int k = r[4]; k <= nk; k++) {
      const REAL *p = pos + 3 * (long)(k - r[4]) * np;
      const int linmima = mono || pert;
#if IS_F32
#ifdef ORC_USE_REF
      void *zt = (set >= 3) ? ref_ztab_t_of(s) : ref_ztab_m_of(s);
      if (linmima) Tricublin_mono_zyx_m_n(wrk, wl, wmi, wma, fs, (pxpypz *)p, zt, (int)np, m);
      else Tricublin_zyx1_m_n(wrk, fs, (pxpypz *)p, zt, (int)np, m);
#else
      const orc_ztab *zt = (set >= 3) ? s->ztab_t : s->ztab_m;
      if (linmima) orc_mono_m_n_f32(wrk, wl, wmi, wma, (const float *const *)fs, p, zt, (int)np, m, 0);
      else orc_zyx1_m_n_f32(wrk, (const float *const *)fs, p, zt, (int)np, m);
#endif
#else
      const orc_ztab *zt = (set >= 3) ? s->ztab_t : s->ztab_m;
      if (linmima) orc_mono_m_n_f64(wrk, wl, wmi, wma, (const double *const *)fs, p, zt, (int)np, m);
      else orc_zyx1_m_n_f64(wrk, (const double *const *)fs, p, zt, (int)np, m);
#endif
      for (int q = 0; q < m; q++)
        for (int j = r[2]; j <= r[3]; j++)
          for (int i = r[0]; i <= r[1]; i++) {
            long w = q * np + (i - r[0]) + (j - r[2]) * nx;
            long e = EXT(i, j, k);
            REAL d = wrk[w];
            if (pert) {
              const REAL pt = pert[(i - 1) + (long)(j - 1) * ld] * SFX(rabs)(d - wl[w]);
              d = d + pt;
            }
            if (mono) {
              REAL lo = wmi[w], hi = wma[w];
              if (lin && lin[q]) lin[q][e] = SFX(rmax)(lo, SFX(rmin)(hi, wl[w]));
              if (mn && mn[q]) mn[q][e] = lo;
              if (mx && mx[q]) mx[q][e] = hi;
              if (clip) d = SFX(rmax)(lo, SFX(rmin)(hi, d));
            }
            dsts[q][e] = d;
          }
    }
    free(fs);
    free(wrk);
  }
}

void SFX(orc_tricub)(const orc_set *s, int set, const REAL *pos, int m, const REAL *const *srcs, REAL *const *dsts,
                     int mono, int clip, REAL *const *lin, REAL *const *mn, REAL *const *mx) {
  SFX(orc_tricub_p)(s, set, pos, m, srcs, dsts, mono, clip, lin, mn, mx, NULL, 0);
}

/* BICUBH_QV at one position: bicubHQV_lin_mono.F90:66-147 (coefficients)
 * and bicubHQV_lin_min_max_zyx.F90:20-83 (sums, lin, min/max), operation
 * order as written.  The cell index of an FP64 position is that of its FP32
 * rounding, as for the tricubic interpolator.  Returns the 0-based ext offset
 * of the stencil origin (column i-1, row j-1, first plane) and the six plane
 * offsets in po[]. */
static long SFX(qv_coef)(const orc_set *s, REAL px, REAL py, REAL pz, double cx[4], double cy[4], double qz[6],
                         double lx[2], double ly[2], double lz[2], long po[6]) {
  const int nk = s->g.nk;
  const double ov6 = 1.0 / 6.0, ov2 = 1.0 / 2.0;
  const double *posz = s->g.zt, *dz = s->delz_t, *odz = s->odelz_t;
  int ii1 = (int)(float)px;
  double del = (double)px - (double)ii1;
  double del12 = (del - 1) * (del - 2), del10 = (del + 1) * del;
  cx[0] = -(del * del12 * ov6);
  cx[1] = (del + 1) * del12 * ov2;
  cx[2] = -(del10 * (del - 2) * ov2);
  cx[3] = del10 * (del - 1) * ov6;
  lx[0] = 1.0 - del;
  lx[1] = del;
  int jj1 = (int)(float)py;
  del = (double)py - (double)jj1;
  del12 = (del - 1) * (del - 2);
  del10 = (del + 1) * del;
  cy[0] = -(del * del12 * ov6);
  cy[1] = (del + 1) * del12 * ov2;
  cy[2] = -(del10 * (del - 2) * ov2);
  cy[3] = del10 * (del - 1) * ov6;
  ly[0] = 1.0 - del;
  ly[1] = del;
  int kk1 = (int)(float)pz;
  /* bicubHQV_lin_mono.F90:95-96: no quintic or cubic case with Schm_autobar_L */
  const int quintic = (kk1 >= 3) && (kk1 <= nk - 3) && !s->g.schm_autobar;
  const int cubic = ((kk1 == 2) || (kk1 == nk - 2)) && !s->g.schm_autobar;
  if (!quintic && !cubic) kk1 = kk1 < 1 ? 1 : (kk1 > nk - 1 ? nk - 1 : kk1);
  const double zt = posz[kk1] + ((double)pz - (double)kk1) * dz[kk1];
  lz[1] = (zt - posz[kk1]) * odz[kk1];
  lz[0] = 1.0 - lz[1];
  const double *q = s->qv_t + (size_t)kk1 * 10;
  int kb;
  if (quintic) {
    kb = kk1 - 2;
    const double rx = posz[kk1 - 2], ra = posz[kk1 - 1], rb = posz[kk1], rc = posz[kk1 + 1], rd = posz[kk1 + 2],
                 re = posz[kk1 + 3];
    qz[0] = (zt - ra) * (zt - rb) * (zt - rc) * (zt - rd) * (zt - re) * q[4];
    qz[1] = (zt - rx) * (zt - rb) * (zt - rc) * (zt - rd) * (zt - re) * q[5];
    qz[2] = (zt - rx) * (zt - ra) * (zt - rc) * (zt - rd) * (zt - re) * q[6];
    qz[3] = (zt - rx) * (zt - ra) * (zt - rb) * (zt - rd) * (zt - re) * q[7];
    qz[4] = (zt - rx) * (zt - ra) * (zt - rb) * (zt - rc) * (zt - re) * q[8];
    qz[5] = (zt - rx) * (zt - ra) * (zt - rb) * (zt - rc) * (zt - rd) * q[9];
  } else if (cubic) {
    kb = kk1 - 1;
    const double ra = posz[kk1 - 1], rb = posz[kk1], rc = posz[kk1 + 1], rd = posz[kk1 + 2];
    qz[0] = 0.0;
    qz[1] = (zt - rb) * (zt - rc) * (zt - rd) * q[0];
    qz[2] = (zt - ra) * (zt - rc) * (zt - rd) * q[1];
    qz[3] = (zt - ra) * (zt - rb) * (zt - rd) * q[2];
    qz[4] = (zt - ra) * (zt - rb) * (zt - rc) * q[3];
    qz[5] = 0.0;
  } else {
    kb = kk1;
    qz[0] = 0.0;
    qz[1] = 0.0;
    qz[3] = (zt - posz[kk1]) * odz[kk1];
    qz[2] = 1.0 - qz[3];
    qz[4] = 0.0;
    qz[5] = 0.0;
  }
  /* plane offsets of the zyx kernel: ninj1..ninj5 */
  const long nij = s->nij;
  const long ninjc = quintic ? nij : 0, ninjl = (quintic || cubic) ? nij : 0;
  po[0] = 0;
  po[1] = ninjc;
  po[2] = po[1] + ninjl;
  po[3] = po[2] + nij;
  po[4] = po[3] + ninjl;
  po[5] = po[4] + ninjc;
  const int il = ii1 - (s->g.i0g - 1), jl = jj1 - (s->g.j0g - 1);
  return EXT(il - 1, jl - 1, kb);
}

static void SFX(qv_point)(const REAL *src, long ni, const double cx[4], const double cy[4], const double qz[6],
                          const double lx[2], const double ly[2], const double lz[2], const long po[6], REAL *xyz,
                          REAL *li, REAL *mi, REAL *ma) {
  const long ni2 = ni + ni, ni3 = ni2 + ni;
  REAL dst[4], dsl[3];
  for (int i = 0; i < 4; i++) {
    const double va = src[i] * qz[0] + src[i + po[1]] * qz[1] + src[i + po[2]] * qz[2] + src[i + po[3]] * qz[3] +
                      src[i + po[4]] * qz[4] + src[i + po[5]] * qz[5];
    const double vb = src[i + ni] * qz[0] + src[i + ni + po[1]] * qz[1] + src[i + ni + po[2]] * qz[2] +
                      src[i + ni + po[3]] * qz[3] + src[i + ni + po[4]] * qz[4] + src[i + ni + po[5]] * qz[5];
    const double vc = src[i + ni2] * qz[0] + src[i + ni2 + po[1]] * qz[1] + src[i + ni2 + po[2]] * qz[2] +
                      src[i + ni2 + po[3]] * qz[3] + src[i + ni2 + po[4]] * qz[4] + src[i + ni2 + po[5]] * qz[5];
    const double vd = src[i + ni3] * qz[0] + src[i + ni3 + po[1]] * qz[1] + src[i + ni3 + po[2]] * qz[2] +
                      src[i + ni3 + po[3]] * qz[3] + src[i + ni3 + po[4]] * qz[4] + src[i + ni3 + po[5]] * qz[5];
    dst[i] = (REAL)(va * cy[0] + vb * cy[1] + vc * cy[2] + vd * cy[3]);
  }
  *xyz = (REAL)(dst[0] * cx[0] + dst[1] * cx[1] + dst[2] * cx[2] + dst[3] * cx[3]);
  for (int i = 1; i <= 2; i++) {
    const double vb = src[i + ni + po[2]] * lz[0] + src[i + ni + po[3]] * lz[1];
    const double vc = src[i + ni2 + po[2]] * lz[0] + src[i + ni2 + po[3]] * lz[1];
    dsl[i] = (REAL)(vb * ly[0] + vc * ly[1]);
  }
  *li = (REAL)(dsl[1] * lx[0] + dsl[2] * lx[1]);
  REAL hi = src[1 + ni + po[2]], lo = hi;
  for (int i = 1; i <= 2; i++) {
    const REAL v[4] = {src[i + ni + po[2]], src[i + ni + po[3]], src[i + ni2 + po[2]], src[i + ni2 + po[3]]};
    for (int q = 0; q < 4; q++) {
      hi = SFX(rmax)(hi, v[q]);
      lo = SFX(rmin)(lo, v[q]);
    }
  }
  *mi = lo;
  *ma = hi;
}

/* adz_tricub_hlt with F_QV_L (adz_interp_hlt.F90:113-116 and the scatter of
 * :119-158) on position set t, plus the clip of adz_post_tr.F90:81-94. */
void SFX(orc_tricub_qv_set_p)(const orc_set *s, int set, const REAL *pos, int m, const REAL *const *srcs,
                              REAL *const *dsts, int clip, REAL *const *lin, REAL *const *mn, REAL *const *mx,
                              const REAL *pert, int ld) {
  int r[5];
  set_range(s, set, r);
  const int nk = s->g.nk;
  const long nx = r[1] - r[0] + 1, ny = r[3] - r[2] + 1, np = nx * ny;
  if (np <= 0 || m <= 0) return;
#pragma omp parallel for schedule(static) num_threads(nthr())
  for (int k = r[4]; k <= nk; k++) {
    for (int j = r[2]; j <= r[3]; j++)
      for (int i = r[0]; i <= r[1]; i++) {
        const REAL *p = pos + 3 * ((long)(k - r[4]) * np + (i - r[0]) + (long)(j - r[2]) * nx);
        double cx[4], cy[4], qz[6], lx[2], ly[2], lz[2];
        long po[6];
        const long o = SFX(qv_coef)(s, p[0], p[1], p[2], cx, cy, qz, lx, ly, lz, po);
        const long e = EXT(i, j, k);
        for (int q = 0; q < m; q++) {
          REAL d, l, lo, hi;
          SFX(qv_point)(srcs[q] + o, s->nit, cx, cy, qz, lx, ly, lz, po, &d, &l, &lo, &hi);
          if (pert) {
            const REAL pt = pert[(i - 1) + (long)(j - 1) * ld] * SFX(rabs)(d - l);
            d = d + pt;
          }
          if (lin && lin[q]) lin[q][e] = SFX(rmax)(lo, SFX(rmin)(hi, l));
          if (mn && mn[q]) mn[q][e] = lo;
          if (mx && mx[q]) mx[q][e] = hi;
          if (clip) d = SFX(rmax)(lo, SFX(rmin)(hi, d));
          dsts[q][e] = d;
        }
      }
  }
}

void SFX(orc_tricub_qv_p)(const orc_set *s, const REAL *pos, int m, const REAL *const *srcs, REAL *const *dsts,
                          int clip, REAL *const *lin, REAL *const *mn, REAL *const *mx, const REAL *pert, int ld) {
  SFX(orc_tricub_qv_set_p)(s, 3, pos, m, srcs, dsts, clip, lin, mn, mx, pert, ld);
}

void SFX(orc_tricub_qv)(const orc_set *s, const REAL *pos, int m, const REAL *const *srcs, REAL *const *dsts,
                        int clip, REAL *const *lin, REAL *const *mn, REAL *const *mx) {
  SFX(orc_tricub_qv_p)(s, pos, m, srcs, dsts, clip, lin, mn, mx, NULL, 0);
}

/* adz_BC_LAM_zlf_hlt (adz_BC_LAM_zlf_hlt.F90:18-319): the four setups of the
 * Zerroukat-Shipway LAM treatment, written as the reference's loops over the
 * tile's interior (1..ni, 1..nj, 1..nk), with its pilot widths and edge flags.
 *   1: F1 = 0 outside [i0_e:in_e]x[j0_e:jn_e] (the core widened by
 *      ext = maxcfl + 1 on the LAM edges) and on levels 1..nint(k0/2)-1 inside;
 *   2: F2 = F1 outside [i0_c:in_c]x[j0_c:jn_c] and on levels 1..k0-1 inside;
 *   3: F1 = 0 outside the BCS_BASE extension [i0_b:in_b]x[j0_b:jn_b];
 *   4: F1 = F2 where setup 2 copies.  k0 = Adz_k0t. */
void SFX(orc_bc_lam_zlf)(const orc_set *s, int setup, REAL *F1, REAL *F2) {
  const orc_grid *g = &s->g;
  const int ni = g->ni, nj = g->nj, nk = g->nk, k0 = s->k0t;
  const int k0d2 = (int)lround(k0 / 2.0); /* nint: halves away from zero */
  const int west = g->west, east = g->east, south = g->south, north = g->north;
#define F1_(i, j, k) F1[EXT(i, j, k)]
#define F2_(i, j, k) F2[EXT(i, j, k)]
  if (setup == 1) {
    const int ext = g->maxcfl + 1;
    const int i0_e = 1 + g->pil_w - ext * west, in_e = ni - g->pil_e + ext * east;
    const int j0_e = 1 + g->pil_s - ext * south, jn_e = nj - g->pil_n + ext * north;
    if (west)
      for (int i = 1; i <= i0_e - 1; i++)
        for (int j = 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    if (east)
      for (int i = in_e + 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    if (south)
      for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= j0_e - 1; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    if (north)
      for (int i = 1; i <= ni; i++)
        for (int j = jn_e + 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    for (int i = i0_e; i <= in_e; i++)
      for (int j = j0_e; j <= jn_e; j++)
        for (int k = 1; k <= k0d2 - 1; k++) F1_(i, j, k) = 0;
  } else if (setup == 2 || setup == 4) {
    const int i0_c = 1 + g->pil_w, in_c = ni - g->pil_e, j0_c = 1 + g->pil_s, jn_c = nj - g->pil_n;
    REAL *dst = (setup == 2) ? F2 : F1;
    const REAL *src = (setup == 2) ? F1 : F2;
    if (west)
      for (int i = 1; i <= i0_c - 1; i++)
        for (int j = 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) dst[EXT(i, j, k)] = src[EXT(i, j, k)];
    if (east)
      for (int i = in_c + 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) dst[EXT(i, j, k)] = src[EXT(i, j, k)];
    if (south)
      for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= j0_c - 1; j++)
          for (int k = 1; k <= nk; k++) dst[EXT(i, j, k)] = src[EXT(i, j, k)];
    if (north)
      for (int i = 1; i <= ni; i++)
        for (int j = jn_c + 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) dst[EXT(i, j, k)] = src[EXT(i, j, k)];
    for (int i = i0_c; i <= in_c; i++)
      for (int j = j0_c; j <= jn_c; j++)
        for (int k = 1; k <= k0 - 1; k++) dst[EXT(i, j, k)] = src[EXT(i, j, k)];
  } else if (setup == 3) {
    const int BCS_BASE = 4;
    const int i0_b = 1 + BCS_BASE * west, in_b = ni - BCS_BASE * east;
    const int j0_b = 1 + BCS_BASE * south, jn_b = nj - BCS_BASE * north;
    if (west)
      for (int i = 1; i <= i0_b - 1; i++)
        for (int j = 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    if (east)
      for (int i = in_b + 1; i <= ni; i++)
        for (int j = 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    if (south)
      for (int i = 1; i <= ni; i++)
        for (int j = 1; j <= j0_b - 1; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
    if (north)
      for (int i = 1; i <= ni; i++)
        for (int j = jn_b + 1; j <= nj; j++)
          for (int k = 1; k <= nk; k++) F1_(i, j, k) = 0;
  }
#undef F1_
#undef F2_
}

/* LAM boundary fluxes of Aranami et al. (2015) (adz_BC_LAM_Aranami_hlt.F90:
 * 18-236, masks of adz_BC_LAM_setup.F90:18-92), for m tracers: the tracer
 * times mask_o (1 on the core: k0t..nk and the tile's span inside the pilot
 * zones of the LAM edges it touches) and times mask_i (1 on the rest of the
 * domain), both 0 outside the domain, interpolated at Adz_pb over
 * (i0b:inb, j0b:jnb, 1:nk) on thermo levels, then FLUX_out zeroed on the
 * core and FLUX_in on the pilot zones and above k0t.  fo, fi: ext layout. */
static int SFX(in_core)(const orc_set *s, int i, int j, int k) {
  const orc_grid *g = &s->g;
  const int cx = (!g->west || i >= 1 + g->pil_w) && (!g->east || i <= g->ni - g->pil_e);
  const int cy = (!g->south || j >= 1 + g->pil_s) && (!g->north || j <= g->nj - g->pil_n);
  return cx && cy && k >= s->k0t;
}
static int SFX(in_domain)(const orc_set *s, int i, int j) {
  const orc_grid *g = &s->g;
  return (!g->west || i >= 1) && (!g->east || i <= g->ni) && (!g->south || j >= 1) && (!g->north || j <= g->nj);
}

void SFX(orc_bc_lam_flux)(const orc_set *s, double dt, const double *wpxyz, const REAL *uvw_dep, const REAL *zdt0,
                          const REAL *uslt, const REAL *vslt, int m, const REAL *const *srcs, REAL *const *fo,
                          REAL *const *fi) {
  const orc_grid *g = &s->g;
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const long bx = s->inb - s->i0b + 1, by = s->jnb - s->j0b + 1, np = bx * by;
  const long next = (long)s->nit * s->njt * nk;
  REAL *pb = (REAL *)malloc(sizeof(REAL) * 3 * np * nk);
  SFX(orc_pb)(s, dt, wpxyz, uvw_dep, zdt0, uslt, vslt, pb);
  REAL *masked = (REAL *)malloc(sizeof(REAL) * 2 * next);
  REAL *wrk = (REAL *)malloc(sizeof(REAL) * 2 * np);
  const long o111 = EXT(1, 1, 1);
  for (int q = 0; q < m; q++) {
    REAL *mo = masked, *mi = masked + next;
    for (int k = 1; k <= nk; k++)
      for (int j = s->lminy; j < s->lminy + s->njt; j++)
        for (int i = s->lminx; i < s->lminx + s->nit; i++) {
          const long e = EXT(i, j, k);
          const int dom = SFX(in_domain)(s, i, j), core = dom && SFX(in_core)(s, i, j, k);
          const REAL v = srcs[q] ? srcs[q][e] : (REAL)1; /* no tracer: the masks (PSADJ, :84-101) */
          mo[e] = core ? v : (REAL)0;
          mi[e] = (dom && !core) ? v : (REAL)0;
        }
    REAL *fs[2] = {mo + o111, mi + o111};
    for (int k = 1; k <= nk; k++) {
      const REAL *p = pb + 3 * (long)(k - 1) * np;
#if IS_F32
#ifdef ORC_USE_REF
      Tricublin_zyx1_m_n(wrk, fs, (pxpypz *)p, ref_ztab_t_of(s), (int)np, 2);
#else
      orc_zyx1_m_n_f32(wrk, (const float *const *)fs, p, s->ztab_t, (int)np, 2);
#endif
#else
      orc_zyx1_m_n_f64(wrk, (const double *const *)fs, p, s->ztab_t, (int)np, 2);
#endif
      for (int j = s->j0b; j <= s->jnb; j++)
        for (int i = s->i0b; i <= s->inb; i++) {
          const long w = (i - s->i0b) + (j - s->j0b) * bx;
          fo[q][EXT(i, j, k)] = wrk[w];
          fi[q][EXT(i, j, k)] = wrk[np + w];
        }
    }
    /* zeroing (adz_BC_LAM_Aranami_hlt.F90:160-226) */
    for (int k = s->k0t; k <= nk; k++) {
      for (int j = 1 + g->pil_s; j <= nj - g->pil_n; j++)
        for (int i = 1 + g->pil_w; i <= ni - g->pil_e; i++) fo[q][EXT(i, j, k)] = 0;
      if (g->north)
        for (int j = nj - g->pil_n + 1; j <= nj; j++)
          for (int i = 1; i <= ni; i++) fi[q][EXT(i, j, k)] = 0;
      if (g->east)
        for (int j = 1; j <= nj; j++)
          for (int i = ni - g->pil_e + 1; i <= ni; i++) fi[q][EXT(i, j, k)] = 0;
      if (g->south)
        for (int j = 1; j <= g->pil_s; j++)
          for (int i = 1; i <= ni; i++) fi[q][EXT(i, j, k)] = 0;
      if (g->west)
        for (int j = 1; j <= nj; j++)
          for (int i = 1; i <= g->pil_w; i++) fi[q][EXT(i, j, k)] = 0;
    }
    for (int k = 1; k <= s->k0t - 1; k++)
      for (int j = s->j0b; j <= s->jnb; j++)
        for (int i = s->i0b; i <= s->inb; i++) fi[q][EXT(i, j, k)] = 0;
  }
  free(wrk);
  free(masked);
  free(pb);
}

/* almost_zero (modelutils almost_zero.F90:16-36), bit for bit, including its
 * 32-bit constant for negative values */
static int SFX(almost_zero)(double a) {
  long long bits;
  memcpy(&bits, &a, 8);
  if (bits < 0) bits = (long long)((unsigned long long)0x80000000ULL - (unsigned long long)bits);
  return bits >= -1 && bits <= 1;
}

static double SFX(fsign1)(double x) { return signbit(x) ? -1.0 : 1.0; } /* sign(ONE_8, x) */

/* sum over the core region of t * air * mask, the product t * air in REAL */
static double SFX(bc_mass)(const orc_set *s, const REAL *t, const REAL *air, const double *mask, int i0, int in,
                           int j0, int jn, int k0, int k1) {
  const int ni = s->g.ni;
  double c = 0.0;
  for (int k = k0; k <= k1; k++)
    for (int j = j0; j <= jn; j++)
      for (int i = i0; i <= in; i++) {
        const long e = EXT(i, j, k);
        const REAL ta = t[e] * air[e];
        c = c + ta * mask[(i - 1) + (long)(j - 1) * ni];
      }
  return c;
}

void SFX(orc_bermejo_conde)(const orc_set *s, const REAL *p, REAL *m, const REAL *lin, const REAL *mn,
                            const REAL *mx, const REAL *fo, const REAL *fi, const REAL *pkps, int weight,
                            double p_exp, int min_max, const REAL *airm_p, const REAL *airm_m, const double *mask,
                            double *deficit, double *diag) {
  const orc_grid *g = &s->g;
  const int nk = g->nk;
  /* adz_post_tr.F90:146-152: core limits, or range b at every level with
   * the Zerroukat-Shipway fluxes (Adz_BC_LAM_flux 2) */
  const int zlf = g->bc_lam_flux == 2;
  const int i0 = zlf ? s->i0b : 1 + (g->west ? g->pil_w : 0), in = zlf ? s->inb : g->ni - (g->east ? g->pil_e : 0);
  const int j0 = zlf ? s->j0b : 1 + (g->south ? g->pil_s : 0), jn = zlf ? s->jnb : g->nj - (g->north ? g->pil_n : 0);
  const int k0 = zlf ? 1 : s->k0t;
  /* mass_tr_PM */
  double mass_p = SFX(bc_mass)(s, p, airm_p, mask, i0, in, j0, jn, k0, nk);
  const double mass_m = SFX(bc_mass)(s, m, airm_m, mask, i0, in, j0, jn, k0, nk);
  double mass_fo = 0.0, mass_fi = 0.0;
  if (fo && fi) {
    mass_fo = SFX(bc_mass)(s, fo, airm_m, mask, s->i0b, s->inb, s->j0b, s->jnb, 1, nk);
    mass_fi = SFX(bc_mass)(s, fi, airm_m, mask, s->i0b, s->inb, s->j0b, s->jnb, 1, nk);
  }
  if (diag) { diag[0] = mass_p; diag[1] = mass_m; diag[2] = mass_fo; diag[3] = mass_fi; }
  /* Bermejo_Conde.F90:70-84 */
  const double mass_bflux = mass_fi - mass_fo;
  mass_p = mass_p - *deficit;
  const double mass_tot_p = mass_p + mass_bflux, mass_tot_m = mass_m;
  double def = mass_tot_m - mass_tot_p;
  const double sd = SFX(fsign1)(def);
  const int ni = g->ni, nj = g->nj;
  /* weights (Bermejo_Conde.F90:87-137), REAL storage; mass_tr_X kind 1 */
  REAL *w = (REAL *)calloc((size_t)s->nit * s->njt * nk, sizeof(REAL));
  for (int k = k0; k <= nk; k++)
    for (int j = j0; j <= jn; j++)
      for (int i = i0; i <= in; i++) {
        const long e = EXT(i, j, k);
        const double hml = (double)(REAL)(m[e] - lin[e]);
        REAL wv = 0;
        if ((int)sd == (int)SFX(fsign1)(hml)) {
          const double a = fabs(hml);
          const double pw = (p_exp == 1.0) ? a : pow(a, p_exp);
          if (weight == 1) wv = (REAL)(pw * sd);
          else if (weight == 2) wv = (REAL)(pw * sd * (double)(m[e] > (REAL)0 ? m[e] : (REAL)0));
          else wv = (REAL)(pw * sd * (double)pkps[e]);
        }
        w[e] = wv;
      }
  const double mass_wei = SFX(bc_mass)(s, w, airm_m, mask, i0, in, j0, jn, k0, nk);
  if (diag) diag[4] = mass_wei;
  (void)nj;
  if (SFX(almost_zero)(mass_wei)) { /* Bermejo_Conde.F90:150-158: tracer left as it is */
    if (diag) { diag[5] = 0.0; diag[6] = 0.0; diag[7] = 0.0; }
    free(w);
    return;
  }
  const double lambda = def / mass_wei;
  if (diag) diag[5] = lambda;
  for (int k = k0; k <= nk; k++)
    for (int j = j0; j <= jn; j++)
      for (int i = i0; i <= in; i++) {
        const long e = EXT(i, j, k);
        const double corr = lambda * (double)w[e];
        if (!min_max) {
          m[e] = (REAL)((double)m[e] - corr);
        } else {
          const REAL wrk = (REAL)((double)m[e] - corr);
          m[e] = wrk;
          if (corr > 0.0 && wrk < mn[e]) m[e] = mn[e];
          if (corr < 0.0 && wrk > mx[e]) m[e] = mx[e];
        }
      }
  free(w);
  if (min_max) { /* Bermejo_Conde.F90:203-222 */
    const double mass_bc_r = SFX(bc_mass)(s, m, airm_m, mask, i0, in, j0, jn, k0, nk);
    if (diag) diag[6] = mass_bc_r;
    const double prop = mass_tot_p / mass_bc_r;
    for (int k = k0; k <= nk; k++)
      for (int j = j0; j <= jn; j++)
        for (int i = i0; i <= in; i++) {
          const long e = EXT(i, j, k);
          m[e] = (REAL)(prop * (double)m[e]);
        }
  } else if (diag) {
    diag[6] = 0.0;
  }
  /* Bermejo_Conde.F90:225-243: epsilon for the next step */
  const double mass_bc = SFX(bc_mass)(s, m, airm_m, mask, i0, in, j0, jn, k0, nk);
  if (diag) diag[7] = mass_bc;
  *deficit = mass_bc - mass_tot_p;
}

/* neighbour shell of (i,j,k) at one sweep, in the order of the reference's
 * sweep_rd lists (ILMC_LAM.F90:118-169): jx, then kx, then ix */
static int SFX(ilmc_shell)(int i, int j, int k, int sweep, int il, int ir, int jl, int jr, int k0, int nk,
                           int *ix_out, int *jx_out, int *kx_out) {
  int n = 0;
  const int kxm = (k - sweep > k0) ? k - sweep : k0, kxp = (k + sweep < nk) ? k + sweep : nk;
  const int j1 = (j - sweep > jl) ? j - sweep : jl, j2 = (j + sweep < jr) ? j + sweep : jr;
  const int i1 = (i - sweep > il) ? i - sweep : il, i2 = (i + sweep < ir) ? i + sweep : ir;
  for (int jx = j1; jx <= j2; jx++)
    for (int kx = kxm; kx <= kxp; kx++) {
      const int limit_i = (jx != j - sweep && jx != j + sweep) && (kx > k - sweep && kx < k + sweep);
      for (int ix = i1; ix <= i2; ix++) {
        if (limit_i && ix != i - sweep && ix != i + sweep) continue;
        ix_out[n] = ix;
        jx_out[n] = jx;
        kx_out[n] = kx;
        n++;
      }
    }
  return n;
}

void SFX(orc_ilmc)(const orc_set *s, REAL *f, const REAL *mn, const REAL *mx, const REAL *air, int sweep_max,
                   int min_max) {
  const int nk = s->g.nk;
  const int il = s->i0, ir = s->in, jl = s->j0, jr = s->jn, k0 = s->k0t;
  int ixs[400], jxs[400], kxs[400];
  REAL cap[400];
  for (int k = k0; k <= nk; k++) /* ilmc_lam_loop.inc */
    for (int j = jl; j <= jr; j++)
      for (int i = il; i <= ir; i++) {
        const long e = EXT(i, j, k);
        REAL o_shoot = SFX(rmax)((REAL)0, f[e] - mx[e]);
        REAL u_shoot = SFX(rmax)((REAL)0, mn[e] - f[e]);
        if (o_shoot == (REAL)0 && u_shoot == (REAL)0) continue;
        for (int sweep = 1; sweep <= sweep_max; sweep++) {
          const int nc = SFX(ilmc_shell)(i, j, k, sweep, il, ir, jl, jr, k0, nk, ixs, jxs, kxs);
          REAL msum = 0;
          if (o_shoot > (REAL)0) {
            for (int q = 0; q < nc; q++) {
              const long r = EXT(ixs[q], jxs[q], kxs[q]);
              cap[q] = SFX(rmax)((REAL)0, mx[r] - f[r]);
              msum = cap[q] * air[r] + msum;
            }
            const REAL use = SFX(rmin)(msum, o_shoot * air[e]);
            if (use > (REAL)0) {
              f[e] = SFX(rmax)(f[e] - (REAL)(use / air[e]), mn[e]);
              o_shoot = SFX(rmax)((REAL)0, f[e] - mx[e]);
              const REAL ratio = use / msum;
              for (int q = 0; q < nc; q++)
                if (cap[q] > (REAL)0) {
                  const long r = EXT(ixs[q], jxs[q], kxs[q]);
                  f[r] = SFX(rmin)(f[r] + (REAL)(cap[q] * ratio), mx[r]);
                }
            }
          } else {
            for (int q = 0; q < nc; q++) {
              const long r = EXT(ixs[q], jxs[q], kxs[q]);
              cap[q] = SFX(rmax)((REAL)0, f[r] - mn[r]);
              msum = cap[q] * air[r] + msum;
            }
            const REAL use = SFX(rmin)(msum, u_shoot * air[e]);
            if (use > (REAL)0) {
              f[e] = SFX(rmin)(f[e] + (REAL)(use / air[e]), mx[e]);
              u_shoot = SFX(rmax)((REAL)0, mn[e] - f[e]);
              const REAL ratio = use / msum;
              for (int q = 0; q < nc; q++)
                if (cap[q] > (REAL)0) {
                  const long r = EXT(ixs[q], jxs[q], kxs[q]);
                  f[r] = SFX(rmax)(f[r] - (REAL)(cap[q] * ratio), mn[r]);
                }
            }
          }
        }
      }
  if (min_max) /* ILMC_LAM.F90:186-208 */
    for (int k = k0; k <= nk; k++)
      for (int j = jl; j <= jr; j++)
        for (int i = il; i <= ir; i++) {
          const long e = EXT(i, j, k);
          if (f[e] < mn[e]) f[e] = mn[e];
          if (f[e] > mx[e]) f[e] = mx[e];
        }
}

#undef EXT
#undef ARR
#undef WP
