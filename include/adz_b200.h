/*
 * adz_b200 — B200 (sm_100a) implementation of GEM's semi-Lagrangian advection
 * hot path: departure-point trajectories, tricubic Lagrange interpolation of
 * momentum and tracers, and monotone clipping.
 *
 * Plain C ABI: pointers, sizes and an opaque handle; no C++ or torch types.
 * Reference paths below are relative to the GEM source tree
 * (src/gemdyn/src/base/ is abbreviated B/).
 *
 * Two levels:
 *   Level A  the reference interpolator ABI, same symbol names and argument
 *            meaning as B/turbo_tricublin.c (bound from Fortran by
 *            B/tricublin_f90.inc).  HOST pointers; each call stages its inputs
 *            on the GPU and copies results back.  A Fortran program linked
 *            against this library instead of turbo_tricublin.o runs unchanged.
 *   Level B  device-pointer entry points for the whole adz step (the work of
 *            B/adz_set.F90, B/adz_traject.F90, B/adz_interp_traj.F90,
 *            B/adz_interp_hlt.F90, B/adz_post_tr.F90:81-94), stream ordered,
 *            returning an int status.  This is the product path.
 *
 * Precisions (argument ``prec``):
 *   ADZC_REF32  the reference's own arithmetic: FP32 fields, winds and stored
 *               positions; FP64 coefficients and sums; results bit-identical
 *               to the reference's AVX2 build.
 *   ADZC_FP64   FP64 fields, winds and positions throughout (plain FP64 drop-in).
 *   ADZC_MIXED  FP32 fields and winds, FP64 positions, cell index and cell
 *               offset; FP32 stencil weights and sums.
 * In every precision the cell index of a position is the one the reference
 * selects: the position rounded to FP32 and truncated.
 */
#ifndef ADZ_B200_H
#define ADZ_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* status codes                                                              */
/* ------------------------------------------------------------------------ */
#define ADZC_OK             0
#define ADZC_ERR_ARG        1  /* NULL pointer, bad size, unknown enum          */
#define ADZC_ERR_CUDA       2  /* a CUDA runtime call failed                    */
#define ADZC_ERR_NK         3  /* fewer than 4 levels                          */
#define ADZC_ERR_HALO       4  /* a stencil would leave the extended array      */
#define ADZC_ERR_NONFINITE  5  /* NaN/Inf wind or position met by a kernel      */
#define ADZC_ERR_TIMEOUT    6  /* a bounded device wait gave up                 */
#define ADZC_ERR_ALLOC      7  /* device or host allocation failed              */
#define ADZC_ERR_NODEVICE   8  /* no usable CUDA device                         */
#define ADZC_ERR_SIZE       9  /* request larger than a fixed capacity          */
#define ADZC_ERR_IO        10  /* file missing, unreadable or not matching      */

#define ADZC_REF32 0
#define ADZC_FP64  1
#define ADZC_MIXED 2

/* position sets of B/adz_mem.F90:87-88 */
#define ADZC_SET_Q 0  /* Adz_pm : momentum levels, mass points               */
#define ADZC_SET_U 1  /* Adz_pmu: momentum levels, u points                  */
#define ADZC_SET_V 2  /* Adz_pmv: momentum levels, v points                  */
#define ADZC_SET_T 3  /* Adz_pt : thermodynamic levels, mass points          */
#define ADZC_SET_B 4  /* Adz_pb : the t-set positions over range b
                       * (Adz_i0b:inb, Adz_j0b:jnb, 1:nk), B/adz_set.F90:167-172;
                       * needs bc_lam_flux != 0 (the k00 = 1 positions)     */

/* ------------------------------------------------------------------------ */
/* Level A — reference interpolator ABI (host pointers)                      */
/* ------------------------------------------------------------------------ */
typedef struct { float px, py, pz; } pxpypz;  /* B/turbo_tricublin.c:157-162 */
typedef struct adzc_ztab ztab;                /* opaque (B/turbo_tricublin.c:164-173) */

/* B/turbo_tricublin.c:320 — levels(nk), row length ni, rows nj of the source */
ztab *Vsearch_setup(double *levels, int nk, int ni, int nj);
/* B/turbo_tricublin.c:370 — plus global-to-local offsets added to (int)px, (int)py */
ztab *Vsearch_setup_plus(double *levels, int nk, int ni, int nj, int offseti, int offsetj);
/* B/turbo_tricublin.c:752 — d[n] */
void Tricublin_zyx1_n(float *d, float *f1, pxpypz *pxyz, ztab *lv, int n);
/* B/turbo_tricublin.c:771 — d[n][m] */
void Tricublin_zyx1_n_m(float *d, float **fs, pxpypz *pxyz, ztab *lv, int n, int m);
/* B/turbo_tricublin.c:793 — d[m][n] */
void Tricublin_zyx1_m_n(float *dm, float **fs, pxpypz *pxyz, ztab *lv, int n, int m);
/* B/turbo_tricublin.c:821 — dp[m][n] through a pointer list */
void Tricublin_zyx1_p(float **dp, float **fs, pxpypz *pxyz, ztab *lv, int n, int m);
/* B/turbo_tricublin.c:1033 — cubic, trilinear, min, max of one field */
void Tricublin_mono_zyx_n(float *d, float *l, float *mi, float *ma, float *f, pxpypz *pxyz, ztab *lv, int n);
/* B/turbo_tricublin.c:1055 — outputs [n][m] */
void Tricublin_mono_zyx_n_m(float *d, float *l, float *mi, float *ma, float **fs, pxpypz *pxyz, ztab *lv, int n,
                            int m);
/* B/turbo_tricublin.c:1080 — outputs [m][n] */
void Tricublin_mono_zyx_m_n(float *d, float *l, float *mi, float *ma, float **fs, pxpypz *pxyz, ztab *lv, int n,
                            int m);
/* B/turbo_tricublin.c:1298 — 3-component interleaved source f3(3,ni,nj,nk), d[n][3] */
void Tricublin_zyx3_n(float *d, float *f3, pxpypz *pxyz, ztab *lv, int n);

/* ------------------------------------------------------------------------ */
/* Level B — device pointers                                                 */
/* ------------------------------------------------------------------------ */

/* status of the last failing call on this thread, and its text */
int adzc_last_error(void);
const char *adzc_error_string(int status);

/* Interpolators on device data (the Level A kernels with device pointers and
 * a CUDA stream, passed as void*).  ``fs`` and ``ds`` are HOST arrays holding
 * m DEVICE pointers.  Positions: pxpypz (REF32) or double[3] per point
 * (FP64, MIXED).  Fields: float (REF32, MIXED) or double (FP64).  Results
 * follow the source type.  d is [m][n].  box: 0 = min/max over the
 * reference's AVX2 box (x 1..2, y 0..3, z 1..2 of the 4x4x4 stencil),
 * 1 = the scalar-branch 2x2x2 inner box.  (B/turbo_tricublin.c:752-1312) */
int adzc_ztab_create(const double *levels, int nk, int ni, int nj, int offi, int offj, ztab **out);
int adzc_ztab_destroy(ztab *lv);
int adzc_tricublin_m_n(const ztab *lv, int prec, void *d, const void *const *fs, const void *pxyz, int n, int m,
                       void *stream);
int adzc_tricublin_mono_m_n(const ztab *lv, int prec, void *d, void *l, void *mi, void *ma, const void *const *fs,
                            const void *pxyz, int n, int m, int box, void *stream);
int adzc_tricublin_zyx3_n(const ztab *lv, int prec, void *d, const void *f3, const void *pxyz, int n, void *stream);

/* Per-tile inputs of adz_set (B/adz_set.F90:16-538).  Level arrays are host
 * pointers read during adzc_setup only. */
typedef struct {
  int ni, nj, nk;                 /* l_ni, l_nj, l_nk (= G_nk)                     */
  int maxcfl;                     /* Grd_maxcfl: halo = max(1,maxcfl)+1            */
  int i0g, j0g;                   /* l_i0, l_j0: global index of local (1,1)       */
  int west, east, south, north;   /* 1 when the tile touches that LAM edge         */
  int pil_w, pil_e, pil_s, pil_n; /* pilot zone widths (0 on interior edges)       */
  int lam_gbpil_t;                /* Lam_gbpil_t                                   */
  int bc_lam_flux;                /* Adz_BC_LAM_flux: 0 none, 1 Aranami, 2 ZLF      */
  int schm_advec;                 /* Schm_advec: 0 none, 1 traditional, 2, 3        */
  int itraj;                      /* Adz_itraj                                     */
  int slt_winds;                  /* Adz_slt_winds (surface-layer winds at k=nk)   */
  int schm_autobar;               /* Schm_autobar_L: BICUBH_QV linear in z         */
  double bA_m, bA;                /* Cstv_bA_m_8, Cstv_bA_8                        */
  double inv_rayt;                /* Dcst_inv_rayt_8                               */
  double inv_hx, inv_hy;          /* geomh_inv_hx_8, geomh_inv_hy_8                */
  const double *cy;               /* Adz_cy_8(1-halo : nj+halo)                    */
  const double *zm;               /* Ver_z_8%m(0:nk+1)                             */
  const double *zt;               /* Ver_z_8%t(0:nk+1)                             */
  const double *zx;               /* Ver_z_8%x(0:nk)                               */
  double zmin, zmax;              /* Ver_zmin_8, Ver_zmax_8                        */
  double wmstar_nk;               /* Ver_wmstar_8(nk)                              */
  double idz_t_nkm1;              /* Ver_idz_8%t(nk-1)                             */
} adzc_grid;

/* What adz_set derived (ranges are Fortran 1-based, inclusive). */
typedef struct {
  int halox, haloy, nit, njt;     /* extended extents: nit = ni+2*halox            */
  int i0, in, j0, jn;             /* Adz_i0.. (mass points)                        */
  int i0u, inu, j0v, jnv;         /* u and v point ranges                          */
  int i0b, inb, j0b, jnb;         /* Adz_pb range                                  */
  int k0, k0t, k0m;
  long long npts[4];              /* points of sets Q, U, V, T                     */
  double iminposx, imaxposx, iminposy, imaxposy;
  int pnz_m, pnz_t;
} adzc_info;

typedef struct adzc_handle adzc_handle;

/* adz_set: derive tables on the host and upload them to the current device.
 * The kernels address a stencil inside the extended array with 32-bit
 * offsets, so a tile whose extended volume (ni + 2 halo) x (nj + 2 halo) x nk
 * reaches 2^31 cells is refused with ADZC_ERR_SIZE; split it into tiles. */
int adzc_setup(const adzc_grid *g, adzc_handle **h);
int adzc_destroy(adzc_handle *h);
int adzc_query(const adzc_handle *h, adzc_info *info);

/* Array layouts (Fortran column-major; all device pointers):
 *   ext   (1-halox:ni+halox, 1-haloy:nj+haloy, 1:nk)  winds, sources, outputs
 *   pxyzm (3, ni, nj, nk) float                        REF32 warm start (Adz_pxyzm)
 *   wpxyz (-1:ni+2, -1:nj+2, nk, 3) double             Adz_wpxyz
 * Winds and sources are float (REF32, MIXED) or double (FP64).
 *
 * adz_inittraj (B/adz_inittraj.F90:25-37): positions := arrival points; the
 * next adzc_traject then runs max(6, itraj) iterations. */
int adzc_inittraj(adzc_handle *h, int prec, void *pxyzm, double *wpxyz, void *stream);

/* adz_prepareWinds + Adz_niter trajectory iterations (niter <= 0: the
 * handle's current count, as Adz_niter) + the per-point state the position
 * sets need.  pxyzm is used by REF32 only (NULL otherwise: FP64 and MIXED
 * restart from wpxyz).  The handle keeps wpxyz, pxyzm, zdt0 and its own
 * departure-wind scratch for the adzc_tricub calls that follow; they must stay
 * valid until then.  (B/adz_traject.F90:16-125, B/adz_prepareWinds.F90) */
int adzc_traject(adzc_handle *h, int prec, double dt, int niter, const void *uu_ext, const void *vv_ext,
                 const void *ww_ext, const void *ut0, const void *vt0, const void *zdt0, void *pxyzm,
                 double *wpxyz, void *stream);

/* adz_tricub_hlt on a position set of the last trajectory, positions derived
 * on the fly as adz_interp_traj does (B/adz_interp_traj.F90:45-187).
 * srcs/dsts: HOST arrays of nfields DEVICE pointers (ext layout; only the
 * set's arrival range of dsts is written).  mono: NULL or nfields flags,
 * 1 = clip to the bound box (B/adz_post_tr.F90:81-94), 2 = bounds only;
 * | ADZC_QV (set T only) interpolates that field with BICUBH_QV instead:
 * bicubic horizontal, quintic vertical (B/bicubHQV_lin_mono.F90:20-172, the
 * F_QV_L branch of B/adz_interp_hlt.F90:113), bounds over the inner 2x2x2
 * box.  lin/mn/mx: NULL or nfields device pointers (entries may be NULL)
 * receiving Adz_post lin (clipped), min, max for mono and QV fields
 * (B/adz_interp_hlt.F90:152-156). */
#define ADZC_QV 4
int adzc_tricub(adzc_handle *h, int prec, int set, int nfields, const void *const *srcs, void *const *dsts,
                const int *mono, void *const *lin, void *const *mn, void *const *mx, void *stream);

/* adz_interp_traj's position arrays (B/adz_interp_traj.F90:45-187): the
 * departure points of one position set of the last trajectory, as Adz_pm,
 * Adz_pmu, Adz_pmv or Adz_pt hold them: pos is a DEVICE array (3, nx, ny, nz)
 * over the set's arrival range (i fastest, levels from the set's k0), FP32
 * in REF32 (the reference's real arrays) and FP64 in ADZC_FP64 and
 * ADZC_MIXED.  adzc_tricub derives the same positions in registers and never
 * stores them; this call is for callers that read them (diagnostics, other
 * interpolators, tests). */
int adzc_interp_traj(adzc_handle *h, int prec, int set, void *pos, void *stream);

/* Adz_uslt, Adz_vslt: DEVICE arrays (ni, nj) of the field type holding the
 * surface-layer winds.  When the grid sets slt_winds, the top-level points
 * of set T (k = nk) take their horizontal positions from them
 * (B/adz_interp_traj.F90:123-133); without them (or with NULL, NULL) those
 * points use the wpxyz extrapolation, as the reference does when the
 * physics does not provide the fields (B/adz_set.F90:364-370).  Used by
 * the adzc_tricub*, adzc_step_noalloc and batch calls that follow. */
int adzc_slt_winds(adzc_handle *h, const void *uslt, const void *vslt);

/* mcrhsint, the ensemble perturbation pattern (B/ens_setmem.F90:47): a
 * DEVICE array of the field type, element (1,1) at mcrhsint, rows ld >= ni
 * elements apart.  While set, every interpolation of the handle (adzc_tricub*,
 * adzc_step_noalloc) writes value + mcrhsint(i,j) * |value - lin|
 * (lin the trilinear value of the inner box), before any clip, as
 * adz_tricub_hlt does when mcrhsint is associated (B/adz_interp_hlt.F90:99-133).
 * NULL clears it.  adzc_batch_create refuses a handle with a pattern set. */
int adzc_rhs_perturbation(adzc_handle *h, const void *mcrhsint, int ld);

/* Zerroukat-Shipway (ZLF) LAM boundary treatment for the Bermejo-Conde
 * fixer, the grid's bc_lam_flux 2 (Adz_BC_LAM_flux 2):
 * adz_BC_LAM_zlf_hlt (B/adz_BC_LAM_zlf_hlt.F90:18-319) on ntr tracers,
 * DEVICE ext arrays, the tile's interior only:
 *   setup 1  f1 = 0 outside the core widened by maxcfl+1 on the LAM edges the
 *            tile touches, and below level nint(k0t/2) inside it;
 *   setup 2  f2 = f1 outside the core and below level k0t inside it;
 *   setup 3  f1 = 0 outside the BCS_BASE (4) extension on the LAM edges;
 *   setup 4  f1 = f2 where setup 2 copies.
 * f1, f2: HOST arrays of ntr DEVICE pointers (f2 for setups 2 and 4 only).
 * The sequence of B/adz_tracers.F90:84-98, 155-174 for mass-fixed tracers:
 * setup 1 on the sources and setup 2 from the destinations (still holding the
 * piloting values) into a keep array; adzc_tricub on ADZC_SET_B with mono and
 * post arrays; setup 3 on the destinations; the post-processing (ILMC,
 * adzc_bermejo_conde, which then runs over range b at every level and takes
 * no flux arrays); setup 4 from the keep array. */
int adzc_bc_lam_zlf(adzc_handle *h, int prec, int setup, int ntr, void *const *f1, void *const *f2, void *stream);

/* LAM boundary fluxes of Aranami et al. (2015), adz_BC_LAM_Aranami_hlt
 * (B/adz_BC_LAM_Aranami_hlt.F90:18-236 with the masks of
 * B/adz_BC_LAM_setup.F90:18-92), for the tracers Bermejo-Conde fixes
 * (mass 1 or 111..139), after the last trajectory.  srcs: ext tracers; fo,
 * fi: ext arrays receiving FLUX_out and FLUX_in at Adz_pb over Adz_i0b:inb,
 * Adz_j0b:jnb, 1:nk, then zeroed as the reference does (FLUX_out on the
 * core, FLUX_in on the pilot zones and above k0t); the fo, fi fields of
 * adzc_bermejo_conde.  srcs[q] NULL interpolates the masks themselves, the
 * PSADJ branch (:84-101).  The grid must set bc_lam_flux 1. */
int adzc_bc_lam_flux(adzc_handle *h, int prec, int ntr, const void *const *srcs, void *const *fo, void *const *fi,
                     void *stream);

/* Every position set of the last trajectory in one call: nfields[4] fields
 * for sets Q, U, V, T, srcs/dsts/mono holding all sets' entries in that order
 * (HOST arrays of DEVICE pointers; mono may be NULL).  Same results as
 * adzc_tricub per set.  (B/adz_main.F90:35-60, B/adz_tracers.F90:74-99) */
int adzc_tricub_sets(adzc_handle *h, int prec, const int *nfields, const void *const *srcs, void *const *dsts,
                     const int *mono, void *stream);

/* The step in two parts, for a tile of a decomposed domain whose halo
 * exchanges should overlap its own computation (B/dynstep.F90:52-53 and
 * B/adz_traject.F90:121-122 exchange before the whole trajectory and before
 * the whole interpolation).  region 0 is the whole tile (adzc_traject,
 * adzc_tricub_sets); region 1 the interior: the points at least maxcfl+3
 * (trajectory) or 2 (position sets) from every side that has a neighbour
 * tile, which read no halo cell; region 2 the band around it.  A caller
 * starts the exchange of the winds and sources, runs region 1 of the
 * trajectory (it prepares the departure winds of every cell), completes the
 * exchange, runs region 2 (it prepares the halo cells again from the winds
 * that arrived); then starts the exchange of wpxyz, runs region 1 of the
 * sets, completes it and runs region 2.  Together the two regions give the
 * results of the whole-tile calls bit for bit.  adzc_traject_region 2 needs
 * region 1 of the same precision just before (ADZC_ERR_ARG otherwise). */
int adzc_traject_region(adzc_handle *h, int prec, double dt, int niter, const void *uu_ext, const void *vv_ext,
                        const void *ww_ext, const void *ut0, const void *vt0, const void *zdt0, void *pxyzm,
                        double *wpxyz, int region, void *stream);
int adzc_tricub_sets_region(adzc_handle *h, int prec, const int *nfields, const void *const *srcs,
                            void *const *dsts, const int *mono, int region, void *stream);

/* Sticky device status of the handle's kernels (ADZC_ERR_HALO,
 * ADZC_ERR_NONFINITE ...); synchronises the stream; clears it when reset. */
int adzc_status(adzc_handle *h, int reset, void *stream);

/* ------------------------------------------------------------------------ */
/* Batches of independent domains: one persistent launch per step            */
/* ------------------------------------------------------------------------ */
/* Each domain is a tile set up with adzc_setup and already past its cold
 * start (adzc_inittraj + one adzc_traject).  The batch steps every domain as
 * adzc_traject + adzc_tricub on each set would (B/adz_main.F90 and
 * B/adz_tracers.F90 for many limited-area domains at once) in ONE persistent
 * kernel launch, replayed from a CUDA graph.  ADZC_FP64 or ADZC_MIXED.
 * The autotuner may instead pick the phased plan: three persistent launches
 * per step in the same graph (departure winds, trajectories, interpolations
 * of every domain), each with the register budget of the per-domain kernel
 * of that phase. */
typedef struct {
  adzc_handle *h;
  double dt;
  int niter;                      /* 0: the handle's Adz_itraj                     */
  const void *uu_ext, *vv_ext, *ww_ext, *ut0, *vt0, *zdt0;
  double *wpxyz;
  int nfields[4];                 /* fields of sets Q, U, V, T                     */
  const void *const *srcs;        /* HOST arrays of DEVICE pointers, all sets      */
  void *const *dsts;              /* in set order; copied by adzc_batch_create    */
  const int *mono;                /* NULL or per field 0/1/2 as in adzc_tricub     */
} adzc_domain;

typedef struct adzc_batch adzc_batch;

#define ADZC_BATCH_MAX_DOMAINS 40  /* more: ADZC_ERR_SIZE */
int adzc_batch_create(int prec, int ndom, const adzc_domain *doms, adzc_batch **out);
/* autotuner: times candidate tile heights (rows per work item), register
 * budgets (resident blocks per SM) of the one-launch kernel and the phased
 * plan on these domains, keeps the fastest and re-captures the graph.  The
 * timed launches are real steps: they advance the domains' positions.  A
 * work item of a region that tiles of 32 i by 4 levels cover with at most
 * 10 % idle lanes holds the tiles of rows/4 such rows (at least one). */
int adzc_batch_tune(adzc_batch *b, void *stream);
int adzc_batch_step(adzc_batch *b, void *stream);
/* the plan in use; blocks_per_sm of the one-launch kernel (phased plan: of
 * its trajectory launch; 0 for the per-domain launches, which have no
 * persistent launch); phased: 1 for the phased plan, 2 for the per-domain
 * launches (may be NULL) */
int adzc_batch_query(const adzc_batch *b, int *rows_per_item, int *blocks_per_sm, long long *nitems);
int adzc_batch_plan(const adzc_batch *b, int *phased);
/* pin a plan instead of tuning: rows per work item, plan 0..2 = register
 * budget of the one-launch kernel, 3 = phased, 4 = every domain's own
 * launches (departure winds, trajectory, all field groups) in turn inside the
 * graph, 5 = the same launches spread over 4 concurrent branches of the graph
 * (rows unused by 4 and 5); re-captures the graph.  adzc_batch_plan reports
 * 0 (one launch), 1 (phased), 2 (per-domain in turn) or 3 (per-domain on
 * concurrent branches). */
#define ADZC_BATCH_PHASED 3
#define ADZC_BATCH_DOMAINS 4
#define ADZC_BATCH_DOMAINS_CONCURRENT 5
/* after adzc_batch_tune: the best time per step the tuner measured for each
 * plan family, ms[0] the one-launch kernel, ms[1] the phased plan, ms[2] the
 * per-domain launches, in turn or concurrent (-1: not timed) */
int adzc_batch_tuned(const adzc_batch *b, float ms[3]);
int adzc_batch_select(adzc_batch *b, int rows_per_item, int plan);
/* Fault injection for tests of the failure path, on the host (no GPU fault).
 * ADZC_INJECT_SPINS: bound of a dependency wait of the one-launch kernel, in
 * iterations of a 64 ns sleep (0: the default, >= 1 s).  ADZC_INJECT_NEED:
 * domain 0's trajectory items also wait for value departure-wind items that
 * do not exist, so their waits run out: the kernel skips them, raises
 * ADZC_ERR_TIMEOUT (adzc_batch_status) and completes (0 clears).  Both
 * re-capture the graph; the phased plan has no waits. */
#define ADZC_INJECT_SPINS 1
#define ADZC_INJECT_NEED 2
int adzc_batch_inject(adzc_batch *b, int what, long long value);
/* synchronises; ADZC_ERR_TIMEOUT when a dependency wait gave up, else the
 * first non-zero status of the domains' handles */
int adzc_batch_status(adzc_batch *b, int reset, void *stream);
int adzc_batch_destroy(adzc_batch *b);

/* ------------------------------------------------------------------------ */
/* Trajectory to a convergence tolerance, and a learned starting guess        */
/* ------------------------------------------------------------------------ */
/* The reference iterates the departure point a fixed number of times
 * (B/adz_traject.F90:66-110; max(6, itraj) on a cold start,
 * B/adz_inittraj.F90:25).  adzc_traject_tol runs the same update until no
 * coordinate of the departure point moves by more than tol grid indices
 * between two updates, at most maxit (1..127) times.
 *   start 0: from the arrival point (the reference's cold start);
 *   start 1: from the points in wpxyz, e.g. written by adzc_guess_apply.
 *            A point that has not converged after maxit updates restarts
 *            from the arrival point (fallback).
 * iters (NULL or ni*nj*nk bytes, arr layout): updates used per point, +128
 * where the fallback ran.  stats (NULL or 3 zeroed device counters, summed
 * into): updates, fallbacks, points not converged.  ADZC_FP64 or ADZC_MIXED;
 * adzc_tricub may follow as after adzc_traject. */
int adzc_traject_tol(adzc_handle *h, int prec, double dt, double tol, int maxit, int start, const void *uu_ext,
                     const void *vv_ext, const void *ww_ext, const void *ut0, const void *vt0, const void *zdt0,
                     double *wpxyz, unsigned char *iters, unsigned long long *stats, void *stream);

/* Learned starting guess (no counterpart in the reference): a network
 * 82 -> 128 -> 128 -> 3 with GELU predicts the departure displacement of
 * each arrival point (i, j, k >= k00, order k, j, i) from the departure winds
 * at the 27 surrounding points, as Courant numbers, and dt / 300 s.
 * params: HOST FP32 arrays W1 (128x82, row = output), b1 (128), W2 (128x128),
 * b2 (128), W3 (3x128), b3 (3).  Inference: BF16 weights and layer inputs,
 * FP32 accumulation on the tensor cores.  MIXED winds (FP32 fields). */
#define ADZC_GUESS_NFEAT 82
#define ADZC_GUESS_HIDDEN 128
#define ADZC_GUESS_NOUT 3
#define ADZC_GUESS_DT_SCALE 300.0
typedef struct adzc_guess adzc_guess;
int adzc_guess_create(const float *const *params, adzc_guess **out);
int adzc_guess_destroy(adzc_guess *net);
/* Fault injection for tests of the inference kernel's failure path, on the
 * host (no GPU fault); no counterpart in the reference.  ADZC_INJECT_SPINS:
 * bound of a wait between the kernel's roles, in polls (0: the default,
 * about 1 s).  ADZC_INJECT_WITHHOLD (value 1): the features of each CTA's
 * first tile never signal the MMA thread, so its wait runs out; the kernel
 * raises ADZC_ERR_TIMEOUT in the handle's status (adzc_status), frees its
 * tensor memory and returns (0 clears).  Applies to the calls that follow. */
#define ADZC_INJECT_WITHHOLD 3
int adzc_guess_inject(adzc_guess *net, int what, long long value);
/* arrival points of the trajectory (ni*nj*(nk-k00+1)), -1 on a bad handle */
long long adzc_guess_npoints(adzc_handle *h);
/* start points X - d, Y - d, k - d (vertical clipped to 1..nk) into wpxyz,
 * and/or the raw displacement d into disp (npoints x 3) */
int adzc_guess_apply(adzc_handle *h, const adzc_guess *net, double dt, const void *uu_ext, const void *vv_ext,
                     const void *ww_ext, double *wpxyz, float *disp, void *stream);
/* The network on a coarse grid only: every stride-th point in i and j
 * (nodes i = min(1 + stride*m, ni), likewise j) on every level, then the
 * start point of each arrival point from its displacement interpolated
 * bilinearly in (i, j) between the nodes around it; into wpxyz as
 * adzc_guess_apply writes it.  stride 1..ADZC_GUESS_MAX_STRIDE (1 is
 * adzc_guess_apply).  Uses the handle's auxiliary device buffer. */
#define ADZC_GUESS_MAX_STRIDE 16
int adzc_guess_apply_coarse(adzc_handle *h, const adzc_guess *net, double dt, const void *uu_ext,
                            const void *vv_ext, const void *ww_ext, int stride, double *wpxyz, void *stream);
/* The learned start and the iteration to a tolerance in one call (MIXED):
 * the departure winds prepared once, the network on the coarse grid of
 * stride (as adzc_guess_apply_coarse), then adzc_traject_tol from those
 * displacements, interpolated per point inside the iteration (no start
 * points stored), with the same fallback, counters and outputs as
 * adzc_traject_tol with start 1.  Uses the handle's auxiliary buffer. */
int adzc_traject_guess(adzc_handle *h, const adzc_guess *net, int stride, double dt, double tol, int maxit,
                       const void *uu_ext, const void *vv_ext, const void *ww_ext, const void *ut0, const void *vt0,
                       const void *zdt0, double *wpxyz, unsigned char *iters, unsigned long long *stats,
                       void *stream);
/* FP32 features (n x 82) of the points idx[0..n) (device; NULL: all points) */
int adzc_guess_features(adzc_handle *h, double dt, const void *uu_ext, const void *vv_ext, const void *ww_ext,
                        const long long *idx, long long n, float *features, void *stream);

/* Training of the guess network in FP32: mean over the batch of the squared
 * displacement error, Adam (b1 0.9, b2 0.999, eps 1e-8).  x (batch x 82) and
 * target (batch x 3) are DEVICE arrays. */
#define ADZC_MLP_NPARAM 27523
typedef struct adzc_mlp adzc_mlp;
int adzc_mlp_create(const float *params, int max_batch, adzc_mlp **out); /* HOST flat parameter vector */
int adzc_mlp_destroy(adzc_mlp *t);
int adzc_mlp_forward(adzc_mlp *t, const float *x, int batch, float *y, void *stream);
int adzc_mlp_grad(adzc_mlp *t, const float *x, const float *target, int batch, void *stream);
int adzc_mlp_adam(adzc_mlp *t, float lr, void *stream);
/* what 0: parameters, 1: gradients (ADZC_MLP_NPARAM floats), 2: loss of the
 * last adzc_mlp_grad (1 float); synchronises the stream */
int adzc_mlp_read(adzc_mlp *t, int what, float *host_out, void *stream);

/* ------------------------------------------------------------------------ */
/* Bermejo-Conde mass fixer                                                   */
/* ------------------------------------------------------------------------ */
/* After the interpolation of mass-conserving tracers (B/adz_post_tr.F90:140-236,
 * B/Bermejo_Conde.F90:16-251, B/mass_tr_PM.F90, B/mass_tr_X.F90): restores
 * each tracer's air-mass-weighted total over the core region (the tile minus
 * its pilot zones, levels k0t..nk; with the grid's bc_lam_flux 2, ZLF, range
 * b at every level, B/adz_post_tr.F90:145-152) to its value before advection,
 * plus the Aranami LAM boundary flux when given (fo, fi: bc_lam_flux 1 only),
 * by adding lambda * w where the high-order
 * value departs from the low-order one.  All arrays are DEVICE arrays in the
 * ext layout of the handle, of the precision's field type (double for
 * ADZC_FP64, float otherwise); mask is the (ni, nj) FP64 area mask
 * (geomh_mask_8).  deficit: DEVICE array of ntr epsilons carried between
 * steps (in: previous step, out: this step; start at 0).  diag: NULL or
 * DEVICE ntr x 8 doubles receiving mass_p, mass_m, mass_fo, mass_fi,
 * mass_wei, lambda, mass_bc_r, mass_bc.  Nothing synchronises the stream. */
typedef struct {
  const void *p;              /* tracer before advection (time P)                 */
  void *m;                    /* tracer after advection (time M), fixed in place  */
  const void *lin, *min, *max;/* Adz_post of m: adzc_tricub post arrays           */
  const void *fo, *fi;        /* NULL, or LAM flux out / in (Adz_BC_LAM_flux 1)   */
  const void *pkps;           /* weight 3 only                                    */
  int weight;                 /* 1 additive, 2 multiplicative, 3 additive * pkps  */
  double p_exp;               /* exponent of |high - low| (adz_BC_pexp_list)      */
} adzc_bc_tracer;
int adzc_bermejo_conde(adzc_handle *h, int prec, int ntr, const adzc_bc_tracer *tracers, const void *airm_p,
                       const void *airm_m, const double *mask, int min_max, double *deficit, double *diag,
                       void *stream);

/* ILMC shape-preserving filter (B/ILMC_LAM.F90:16-388, B/ilmc_lam_loop.inc)
 * of ntr tracers f[q] (DEVICE, ext layout, fixed in place) with bounds
 * mn[q]/mx[q] (the Adz_post min/max of adzc_tricub) and air mass air:
 * single LAM domain (the arrival range i0..in, j0..jn, levels k0t..nk),
 * sweeps 1..sweep_max (1-4, adz_ILMC_sweep_max), then the clip to the bounds
 * when min_max (adz_ILMC_min_max_L).  Bit-exact with the reference's
 * sequential loop order, run as wavefronts of row tiles whose neighbourhoods
 * never interact, all tracers (at most ADZC_ILMC_MAX_TRACERS) together;
 * rounds (may be NULL) receives the number of wavefronts.  Does not
 * synchronise the stream. */
#define ADZC_ILMC_MAX_TRACERS 32
int adzc_ilmc(adzc_handle *h, int prec, int ntr, void *const *f, const void *const *mn, const void *const *mx,
              const void *air, int sweep_max, int min_max, int *rounds, void *stream);

/* ------------------------------------------------------------------------ */
/* Diagnostics and restart state                                              */
/* ------------------------------------------------------------------------ */
/* adz_cfl / adz_courant (B/adz_cfl.F90:47-189): maximum Courant numbers of
 * the departure points in wpxyz over Adz_i0:in, j0:jn, k0:nk, bit-exact with
 * the reference (FP64, first point of equal maxima in k, j, i order).
 * DEVICE outputs: cfl[3] (horizontal, vertical, 3-D), idx[9] (global i, j, k
 * of each maximum, as cfl_i(1:3, 1:3)). */
int adzc_cfl(adzc_handle *h, const double *wpxyz, double *cfl, int *idx, void *stream);

/* Trajectory state for a restart: Adz_wpxyz, Adz_pxyzm (REF32) and the
 * handle's iteration state (cold start pending, Adz_niter), which the
 * reference keeps through its memory manager's restart flag
 * (B/adz_set.F90:343-360).  The file format is this library's own (a 64-byte
 * header, then the device arrays).  Load checks precision and dimensions
 * (ADZC_ERR_IO otherwise).  Both synchronise the device. */
int adzc_state_save(adzc_handle *h, int prec, const void *pxyzm, const double *wpxyz, const char *path);
int adzc_state_load(adzc_handle *h, int prec, void *pxyzm, double *wpxyz, const char *path);

/* ------------------------------------------------------------------------ */
/* Halo exchange between tiles                                                */
/* ------------------------------------------------------------------------ */
/* The rpn_comm_xch_halo calls of the path, non-periodic, in a 2-D tile
 * decomposition: the departure winds (B/dynstep.F90:52-53, width
 * Adz_halox), the tracer sources (B/adz_interp_hlt.F90:87-88, same width)
 * and Adz_wpxyz (B/adz_traject.F90:121-122, width 2, between the trajectory
 * and the position sets).  The library packs a tile's halo strips into one
 * buffer and unpacks the neighbours' strips from another, one launch each;
 * the caller moves the bytes (NCCL send/recv, MPI, a device copy).
 *
 * Neighbours sit in slots q = 3*(dy+1) + (dx+1), dx, dy in -1..1 (dx = +1:
 * larger i, dy = +1: larger j); slot 4 is the tile itself and is never used.
 * Segment q of the send buffer holds the strip of this tile's interior that
 * the neighbour in slot q needs; segment q of the receive buffer is filled
 * from that neighbour's send segment 8 - q.  Both buffers have the layout
 * adzc_halo_layout returns.  A strip spans i = 1-hx..0, 1..ni or
 * ni+1..ni+hx (receive) and 1..hx, 1..ni or ni-hx+1..ni (send) by dx, the
 * same in j by dy, every plane and every array; inside a segment the order is
 * array, plane, j, i (i fastest).  Corner strips come from the diagonal
 * neighbours in the same exchange; inside the global domain this gives what
 * the two-pass (x, then y) exchange gives.  Absent neighbours (domain edges)
 * have empty segments and leave the halo untouched. */
typedef struct {
  int minx, maxx, miny, maxy;     /* array bounds; the interior is 1..ni, 1..nj    */
  int ni, nj;
  long long nplanes;              /* product of the trailing extents (nk, 3*nk)    */
  int hx, hy;                     /* widths exchanged: 1..1-minx, 1..ni            */
  int elem;                       /* bytes per element: 4 or 8                     */
  int nbr[9];                     /* 1 when the neighbour in slot q exists         */
} adzc_halo;
#define ADZC_HALO_MAX_ARRAYS 64
/* off[10]: byte offset of each segment in a buffer, off[9] the total. */
int adzc_halo_layout(const adzc_halo *x, int narrays, long long *off);
/* arrays: HOST array of narrays DEVICE pointers (element (minx, miny, 1)). */
int adzc_halo_pack(const adzc_halo *x, int narrays, const void *const *arrays, void *sendbuf, void *stream);
int adzc_halo_unpack(const adzc_halo *x, int narrays, void *const *arrays, const void *recvbuf, void *stream);

/* One whole advection step that allocates no device memory.  No counterpart
 * in the reference (its Fortran drivers use automatic arrays).
 *
 * For callers that cannot call cudaMalloc while stepping: a host model whose
 * device memory belongs to its own pool (an OpenACC runtime, a caching
 * allocator that reserved the GPU at start-up), one held to a device-memory
 * budget fixed at start-up, or one that must not let the step synchronise the
 * device.  adzc_traject allocates its scratch on first use; this entry point
 * keeps the same scratch (departure winds, departure vertical wind) in one
 * static device array of ADZC_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until exit.  Tiles whose scratch does not fit
 * (3*nit*njt*nk + ni*nj*nk values of the field type, each part rounded up to
 * 256 bytes) are rejected with ADZC_ERR_SIZE before anything runs.
 *
 * Computes what adzc_traject followed by adzc_tricub on sets Q, U, V, T
 * computes: nfields[4] fields per set; srcs/dsts/mono hold all sets' entries
 * in that order (HOST arrays of DEVICE pointers; mono may be NULL).  mono
 * takes 0, 1 or 2 per field: BICUBH_QV fields (ADZC_QV) are not supported
 * here (ADZC_ERR_ARG).  A non-finite dt is refused (ADZC_ERR_ARG).
 * The step's positions stay in the caller's wpxyz and its departure vertical
 * wind in the shared array, so the handle keeps no record of this trajectory:
 * adzc_tricub and adzc_bc_lam_flux on the same handle return ADZC_ERR_ARG
 * until the next adzc_traject.  The first call in a device's context resolves
 * the array's device address (again after cudaDeviceReset, which gives the
 * device a new context and the array a new address), so make it before any
 * stream capture.  All calls share the array and it keeps the last call's
 * contents: calls that overlap on the GPU race. */
#define ADZC_NOALLOC_SCRATCH_BYTES (64u << 20)
int adzc_step_noalloc(adzc_handle *h, int prec, double dt, int niter, const void *uu_ext, const void *vv_ext,
                      const void *ww_ext, const void *ut0, const void *vt0, const void *zdt0, void *pxyzm,
                      double *wpxyz, const int *nfields, const void *const *srcs, void *const *dsts,
                      const int *mono, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* ADZ_B200_H */
