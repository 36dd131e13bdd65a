/*
 * ORACLE — test infrastructure only (checker, never shipped or measured as the
 * product).  CPU restatement of GEM's semi-Lagrangian advection path:
 * interpolators (tricublin_oracle.c) and the Fortran drivers (adz_oracle.c).
 */
#ifndef ADZ_ORACLE_H
#define ADZ_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* level descriptor, same content as the reference ``ztab``
 * (src/gemdyn/src/base/turbo_tricublin.c:164-173) */
typedef struct {
  double *z;   /* nk levels */
  double *ocz; /* 4*max(nk,4) inverse Lagrange denominators */
  int ni, nj, nk, nij;
  int offi, offj;
} orc_ztab;

orc_ztab *orc_vsearch_setup_plus(const double *levels, int nk, int ni, int nj, int offi, int offj);
void orc_ztab_free(orc_ztab *lv);
int orc_coef_f32pos(double *c, int *offset, float px, float py, float pz, const orc_ztab *lv);
int orc_coef_f64pos(double *c, int *offset, double px, double py, double pz, const orc_ztab *lv);

void orc_zyx1_m_n_f32(float *d, const float *const *fs, const float *pxyz, const orc_ztab *lv, int n, int m);
void orc_mono_m_n_f32(float *d, float *l, float *mn, float *mx, const float *const *fs, const float *pxyz,
                      const orc_ztab *lv, int n, int m, int box);
void orc_zyx3_n_f32(float *d, const float *f3, const float *pxyz, const orc_ztab *lv, int n);
void orc_zyx1_m_n_f64(double *d, const double *const *fs, const double *pxyz, const orc_ztab *lv, int n, int m);
void orc_mono_m_n_f64(double *d, double *l, double *mn, double *mx, const double *const *fs, const double *pxyz,
                      const orc_ztab *lv, int n, int m);
void orc_zyx3_n_f64(double *d, const double *f3, const double *pxyz, const orc_ztab *lv, int n);
void orc_cells_f32(int *off, int *zl, const float *pxyz, const orc_ztab *lv, int n);
void orc_cells_f64(int *off, int *zl, const double *pxyz, const orc_ztab *lv, int n);

/* ---------------- driver restatement (adz_oracle.c) ---------------- */

/* Inputs of adz_set (src/gemdyn/src/base/adz_set.F90:16-538) for one tile. */
typedef struct {
  int ni, nj, nk;              /* l_ni, l_nj, l_nk (= G_nk) */
  int maxcfl;                  /* Grd_maxcfl -> halo = max(1,maxcfl)+1 */
  int i0g, j0g;                /* l_i0, l_j0 */
  int west, east, south, north;/* tile touches that LAM edge (0/1) */
  int pil_w, pil_e, pil_s, pil_n;
  int lam_gbpil_t;             /* Lam_gbpil_t */
  int bc_lam_flux;             /* adz_BC_LAM_flux */
  int schm_advec;              /* Schm_advec (0..3) */
  int itraj;                   /* Adz_itraj */
  int slt_winds;               /* Adz_slt_winds (needs uslt/vslt) */
  int schm_autobar;            /* Schm_autobar_L */
  double bA_m, bA;             /* Cstv_bA_m_8, Cstv_bA_8 */
  double inv_rayt;             /* Dcst_inv_rayt_8 */
  double inv_hx, inv_hy;       /* geomh_inv_hx_8, geomh_inv_hy_8 */
  const double *cy;            /* Adz_cy_8(1-haloy : nj+haloy) */
  const double *zm;            /* Ver_z_8%m(0:nk+1) */
  const double *zt;            /* Ver_z_8%t(0:nk+1) */
  const double *zx;            /* Ver_z_8%x(0:nk) */
  double zmin, zmax;           /* Ver_zmin_8, Ver_zmax_8 */
  double wmstar_nk;            /* Ver_wmstar_8(nk) */
  double idz_t_nkm1;           /* Ver_idz_8%t(nk-1) */
} orc_grid;

/* Everything adz_set derives, in C 0-based storage. */
typedef struct {
  orc_grid g;
  int halox, haloy, lminx, lmaxx, lminy, lmaxy, nit, njt, nij;
  int i0, in, j0, jn, i0u, inu, j0v, jnv, i0b, inb, j0b, jnb;
  int k0, k0t, k0m, niu, njv;
  double iminposx, imaxposx, iminposy, imaxposy;
  double sig, ovdzm, ovdzt;
  int pnz_m, pnz_t;
  int *search_m, *search_t;    /* 1-based contents, stored 0-based */
  double *delz_m, *delz_t, *odelz_m, *odelz_t; /* index 0..nk */
  double *vw1m, *vw2m, *vw3m, *vw4m, *vw1t, *vw2t, *vw3t, *vw4t; /* index 1..nk (slot 0 unused) */
  double vw5, vw6;
  double ww, wp, wm;           /* interp_traj end weights */
  double *cy;                  /* index j - lminy */
  orc_ztab *ztab_m, *ztab_t;
  void *ref_m, *ref_t;         /* reference ztab objects (reference-linked build only) */
  /* BICUBH_QV denominators on thermo levels, 10 per level k (slot k*10 + q):
   * q 0..3 cubic Adz_zabcd/zbacd/zcabd/zdabc_8%t (k = 2..nk-2),
   * q 4..9 quintic Adz_zxabcde..zexabcd_8%t (k = 3..nk-3), adz_set.F90:286-311 */
  double *qv_t;
} orc_set;

int orc_adz_set(const orc_grid *g, orc_set *s);
void orc_adz_free(orc_set *s);

/* Array conventions (all Fortran column-major, offsets handled by the caller):
 *   ext field  : (lminx:lmaxx, lminy:lmaxy, 1:nk)          nit*njt*nk
 *   uvw_d      : (3, lminx:lmaxx, lminy:lmaxy, 1:nk)
 *   arr fields : (1:ni, 1:nj, 1:nk)
 *   uvw_dep    : (3, 1:ni, 1:nj, 1:nk)
 *   pxyzm      : (3, 1:ni, 1:nj, 1:nk)        FP32 (ref) / FP64 (f64 oracle)
 *   wpxyz      : (-1:ni+2, -1:nj+2, 1:nk, 3)  FP64
 *   pos sets   : (3, npoints) for ranges u, v, q(=m), t
 * The FP32 driver calls the restated interpolator, or the reference's own one
 * in the -DORC_USE_REF build. */

/* number of threads used by the OpenMP loops (0 = runtime default) */
void orc_set_threads(int n);

/* reference precision (FP32 fields/winds/positions, FP64 trajectory math) */
void orc_prepare_winds_f32(const orc_set *s, const float *uu_ext, const float *vv_ext, const float *ww_ext,
                           const float *ut0, const float *vt0, const float *zdt0,
                           float *uvw_d, float *uu_arr, float *vv_arr, float *ww_arr);
void orc_inittraj_f32(const orc_set *s, float *pxyzm, double *wpxyz);
void orc_traject_f32(const orc_set *s, double dt, int niter, const float *uvw_d,
                     const float *uu_arr, const float *vv_arr, const float *ww_arr,
                     float *uvw_dep, float *pxyzm, double *wpxyz);
/* position sets: pm, pmu, pmv (k0..nk), pt (k0t..nk); any may be NULL */
void orc_interp_traj_f32(const orc_set *s, double dt, const double *wpxyz, const float *uvw_dep,
                         const float *zdt0, const float *pxyzm, const float *uslt, const float *vslt,
                         float *pm, float *pmu, float *pmv, float *pt);
/* adz_tricub_hlt: interpolate m extended sources at a position set into
 * dst (ext layout, range only).  mono != 0 -> also lin/min/max (ext layout,
 * may be NULL) and, when clip != 0, dst = max(min, min(max, dst)). */
void orc_tricub_f32(const orc_set *s, int set, const float *pos, int m, const float *const *srcs,
                    float *const *dsts, int mono, int clip, float *const *lin, float *const *mn, float *const *mx);

/* FP64 extension of the same driver (all arrays double) */
void orc_prepare_winds_f64(const orc_set *s, const double *uu_ext, const double *vv_ext, const double *ww_ext,
                           const double *ut0, const double *vt0, const double *zdt0,
                           double *uvw_d, double *uu_arr, double *vv_arr, double *ww_arr);
void orc_inittraj_f64(const orc_set *s, double *pxyzm, double *wpxyz);
void orc_traject_f64(const orc_set *s, double dt, int niter, const double *uvw_d,
                     const double *uu_arr, const double *vv_arr, const double *ww_arr,
                     double *uvw_dep, double *pxyzm, double *wpxyz);
void orc_interp_traj_f64(const orc_set *s, double dt, const double *wpxyz, const double *uvw_dep,
                         const double *zdt0, const double *pxyzm, const double *uslt, const double *vslt,
                         double *pm, double *pmu, double *pmv, double *pt);
void orc_tricub_f64(const orc_set *s, int set, const double *pos, int m, const double *const *srcs,
                    double *const *dsts, int mono, int clip, double *const *lin, double *const *mn,
                    double *const *mx);

/* BICUBH_QV (bicubHQV_lin_mono.F90:20-172 with bicubHQV_lin_min_max_zyx.F90):
 * bicubic horizontal, quintic vertical (cubic at levels 2 and nk-2, linear
 * at the ends) on thermo levels, at position set t; lin/min/max over the
 * inner 2x2x2 box.  Arguments as orc_tricub_* (always computes lin/min/max;
 * they may be NULL). */
void orc_tricub_qv_f32(const orc_set *s, const float *pos, int m, const float *const *srcs, float *const *dsts,
                       int clip, float *const *lin, float *const *mn, float *const *mx);
void orc_tricub_qv_f64(const orc_set *s, const double *pos, int m, const double *const *srcs, double *const *dsts,
                       int clip, double *const *lin, double *const *mn, double *const *mx);

/* LAM boundary fluxes (adz_BC_LAM_Aranami_hlt.F90) of m tracers into fo, fi
 * (ext layout, range b and the zeroed regions written) */
void orc_bc_lam_flux_f32(const orc_set *s, double dt, const double *wpxyz, const float *uvw_dep, const float *zdt0,
                         const float *uslt, const float *vslt, int m, const float *const *srcs, float *const *fo,
                         float *const *fi);
void orc_bc_lam_flux_f64(const orc_set *s, double dt, const double *wpxyz, const double *uvw_dep,
                         const double *zdt0, const double *uslt, const double *vslt, int m,
                         const double *const *srcs, double *const *fo, double *const *fi);

/* the same with the ensemble perturbation mcrhsint (element (1,1), rows ld
 * apart; NULL: none): dst = value + mcrhsint * abs(value - lin) before the
 * clip (adz_interp_hlt.F90:99-100, 125-133) */
void orc_tricub_p_f32(const orc_set *s, int set, const float *pos, int m, const float *const *srcs,
                      float *const *dsts, int mono, int clip, float *const *lin, float *const *mn, float *const *mx,
                      const float *pert, int ld);
void orc_tricub_p_f64(const orc_set *s, int set, const double *pos, int m, const double *const *srcs,
                      double *const *dsts, int mono, int clip, double *const *lin, double *const *mn,
                      double *const *mx, const double *pert, int ld);
void orc_tricub_qv_p_f32(const orc_set *s, const float *pos, int m, const float *const *srcs, float *const *dsts,
                         int clip, float *const *lin, float *const *mn, float *const *mx, const float *pert, int ld);
void orc_tricub_qv_p_f64(const orc_set *s, const double *pos, int m, const double *const *srcs,
                         double *const *dsts, int clip, double *const *lin, double *const *mn, double *const *mx,
                         const double *pert, int ld);

/* Bermejo-Conde mass fixer for one tracer (Bermejo_Conde.F90:16-251 with
 * mass_tr_PM.F90 and mass_tr_X.F90), single domain (the MPI_Allgather sums
 * of one rank).  Arrays in the ext layout; mask (ni, nj) is geomh_mask_8.
 * Core region: 1+pil_w..ni-pil_e, 1+pil_s..nj-pil_n (pilots of edge tiles),
 * levels k0t..nk.  fo/fi (may be NULL): LAM flux masses over the b range,
 * levels 1..nk.  weight 1/2/3, p_exp, min_max as adz_BC_weight,
 * adz_BC_pexp_list(n), adz_BC_min_max_L.  *deficit: in the previous step's
 * epsilon, out this step's.  diag[8] (may be NULL): mass_p, mass_m, mass_fo,
 * mass_fi, mass_wei, lambda, mass_bc_r, mass_bc. */
/* adz_BC_LAM_zlf_hlt (adz_BC_LAM_zlf_hlt.F90:18-319), setups 1-4, on one
 * ext-layout tracer (f2 for setups 2 and 4) */
void orc_bc_lam_zlf_f32(const orc_set *s, int setup, float *f1, float *f2);
void orc_bc_lam_zlf_f64(const orc_set *s, int setup, double *f1, double *f2);
/* BICUBH_QV over any set's range (3: Adz_pt, 4: Adz_pb over range b) */
void orc_tricub_qv_set_p_f32(const orc_set *s, int set, const float *pos, int m, const float *const *srcs,
                             float *const *dsts, int clip, float *const *lin, float *const *mn, float *const *mx,
                             const float *pert, int ld);
void orc_tricub_qv_set_p_f64(const orc_set *s, int set, const double *pos, int m, const double *const *srcs,
                             double *const *dsts, int clip, double *const *lin, double *const *mn,
                             double *const *mx, const double *pert, int ld);
void orc_bermejo_conde_f32(const orc_set *s, const float *p, float *m, const float *lin, const float *mn,
                           const float *mx, const float *fo, const float *fi, const float *pkps, int weight,
                           double p_exp, int min_max, const float *airm_p, const float *airm_m, const double *mask,
                           double *deficit, double *diag);
void orc_bermejo_conde_f64(const orc_set *s, const double *p, double *m, const double *lin, const double *mn,
                           const double *mx, const double *fo, const double *fi, const double *pkps, int weight,
                           double p_exp, int min_max, const double *airm_p, const double *airm_m,
                           const double *mask, double *deficit, double *diag);

/* ILMC shape-preserving filter (ILMC_LAM.F90:16-388 with ilmc_lam_loop.inc),
 * single LAM domain: points i0..in, j0..jn (the arrival range), levels
 * k0t..nk, in that loop order; sweeps 1..sweep_max (<= 4) of neighbour shells
 * enumerated as the reference's sweep_rd lists; then, if min_max, the clip
 * to [min, max].  f fixed in place (ext layout). */
void orc_ilmc_f32(const orc_set *s, float *f, const float *mn, const float *mx, const float *air, int sweep_max,
                  int min_max);
void orc_ilmc_f64(const orc_set *s, double *f, const double *mn, const double *mx, const double *air,
                  int sweep_max, int min_max);

/* number of points of a position set (0=q/pm, 1=u, 2=v, 3=t) */
long orc_set_npoints(const orc_set *s, int set);

#ifdef __cplusplus
}
#endif
#endif
