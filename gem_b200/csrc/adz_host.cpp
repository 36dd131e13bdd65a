// Host side of the adz_b200 C ABI (include/adz_b200.h).
//
// adzc_setup derives on the host what GEM's adz_set derives
// (src/gemdyn/src/base/adz_set.F90:71-311, abbreviated B/ below) and uploads
// it; the step entry points only validate arguments and launch kernels.  Level
// A keeps the reference interpolator's names and host-pointer calling
// convention (B/turbo_tricublin.c) on top of the device kernels.
//
// Built with -ffp-contract=off: the level tables use the reference's operation
// order without fused multiply-adds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace {

thread_local int g_last_status = ADZC_OK;

int fail(int st) {
  g_last_status = st;
  return st;
}

#define ADZ_CK(x)                                  \
  do {                                             \
    if ((x) != cudaSuccess) return fail(ADZC_ERR_CUDA); \
  } while (0)

template <int P>
struct Sz;

size_t field_bytes(int prec) { return prec == ADZC_FP64 ? sizeof(double) : sizeof(float); }
size_t pos_bytes(int prec) { return prec == ADZC_REF32 ? sizeof(float) : sizeof(double); }

cudaError_t dispatch_prepare(int prec, const adz::DGrid& g, const void* uu, const void* vv, const void* ww, void* o,
                             cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_prepare<adz::kRef32>(g, uu, vv, ww, o, s);
    case ADZC_FP64: return adz::launch_prepare<adz::kFp64>(g, uu, vv, ww, o, s);
    default: return adz::launch_prepare<adz::kMixed>(g, uu, vv, ww, o, s);
  }
}
cudaError_t dispatch_traject(int prec, const adz::DGrid& g, const adz::TrajArgs& a, cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_traject<adz::kRef32>(g, a, s);
    case ADZC_FP64: return adz::launch_traject<adz::kFp64>(g, a, s);
    default: return adz::launch_traject<adz::kMixed>(g, a, s);
  }
}
cudaError_t dispatch_qv(int prec, const adz::DGrid& g, int i0, int nx, int j0, int ny, int k0, int nz,
                        const adz::SetArgs& a, const adz::FieldPtrs& fp, cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_qv_set<adz::kRef32>(g, i0, nx, j0, ny, k0, nz, a, fp, s);
    case ADZC_FP64: return adz::launch_qv_set<adz::kFp64>(g, i0, nx, j0, ny, k0, nz, a, fp, s);
    default: return adz::launch_qv_set<adz::kMixed>(g, i0, nx, j0, ny, k0, nz, a, fp, s);
  }
}
cudaError_t dispatch_set(int prec, const adz::DGrid& g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                         const adz::SetArgs& a, const adz::FieldPtrs& fp, cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_tricub_set<adz::kRef32>(g, set, i0, nx, j0, ny, k0, nz, a, fp, s);
    case ADZC_FP64: return adz::launch_tricub_set<adz::kFp64>(g, set, i0, nx, j0, ny, k0, nz, a, fp, s);
    default: return adz::launch_tricub_set<adz::kMixed>(g, set, i0, nx, j0, ny, k0, nz, a, fp, s);
  }
}
cudaError_t dispatch_parts(int prec, const adz::DGrid& g, const adz::SetArgs& a, const adz::SetParts& sp,
                           cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_tricub_parts<adz::kRef32>(g, a, sp, s);
    case ADZC_FP64: return adz::launch_tricub_parts<adz::kFp64>(g, a, sp, s);
    default: return adz::launch_tricub_parts<adz::kMixed>(g, a, sp, s);
  }
}
cudaError_t dispatch_pos(int prec, const adz::DZtab& lv, int kind, int n, const void* pos, const adz::FieldPtrs& fp,
                         cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_interp_pos<adz::kRef32>(lv, kind, n, pos, fp, s);
    case ADZC_FP64: return adz::launch_interp_pos<adz::kFp64>(lv, kind, n, pos, fp, s);
    default: return adz::launch_interp_pos<adz::kMixed>(lv, kind, n, pos, fp, s);
  }
}
cudaError_t dispatch_init(int prec, const adz::DGrid& g, float* pxyzm, double* wpxyz, cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_inittraj<adz::kRef32>(g, pxyzm, wpxyz, s);
    case ADZC_FP64: return adz::launch_inittraj<adz::kFp64>(g, pxyzm, wpxyz, s);
    default: return adz::launch_inittraj<adz::kMixed>(g, pxyzm, wpxyz, s);
  }
}

double triprd_inv(double x, double a, double b, double c) { return 1.0 / ((x - a) * (x - b) * (x - c)); }

}  // namespace

// ---------------------------------------------------------------------------
// level descriptor (B/turbo_tricublin.c:164-173, 252-257, 320-380)
// ---------------------------------------------------------------------------
struct adzc_ztab {
  std::vector<double> z, ocz;
  std::vector<float> zn;
  int ni = 0, nj = 0, nk = 0, offi = 0, offj = 0;
  int device = 0;
  double* d_z = nullptr;
  double* d_ocz = nullptr;
  float* d_zn = nullptr;
  adz::DZtab dev() const {
    adz::DZtab t;
    t.z = d_z;
    t.ocz = d_ocz;
    t.zn = d_zn;
    t.ni = ni;
    t.nj = nj;
    t.nk = nk;
    t.nij = ni * nj;
    t.offi = offi;
    t.offj = offj;
    return t;
  }
};

static void build_ztab_host(adzc_ztab* lv, const double* levels, int nk, int ni, int nj, int offi, int offj) {
  const int nkl = std::max(nk, 4);
  lv->z.assign(levels, levels + nk);
  lv->ocz.assign(4 * nkl, 1.0);
  if (nk >= 4) {
    const double* t = levels;
    auto den = [&](int e, double a, double b, double c, double d) {
      lv->ocz[4 * e + 0] = triprd_inv(a, b, c, d);
      lv->ocz[4 * e + 1] = triprd_inv(b, a, c, d);
      lv->ocz[4 * e + 2] = triprd_inv(c, a, b, d);
      lv->ocz[4 * e + 3] = triprd_inv(d, a, b, c);
    };
    den(0, t[0], t[1], t[2], t[3]);
    for (int i = 1; i < nk - 2; i++) den(i, t[i - 1], t[i], t[i + 1], t[i + 2]);
    den(nk - 2, t[nk - 4], t[nk - 3], t[nk - 2], t[nk - 1]);
    den(nk - 1, t[nk - 4], t[nk - 3], t[nk - 2], t[nk - 1]);
  }
  // FP32 per-interval table of the mixed path (normalised Lagrange nodes)
  lv->zn.assign(8 * nkl, 0.0f);
  for (int iz = 1; iz + 2 < nk; iz++) {
    const double z0 = levels[iz], h = levels[iz + 1] - z0;
    const double u[4] = {(levels[iz - 1] - z0) / h, 0.0, 1.0, (levels[iz + 2] - z0) / h};
    lv->zn[8 * iz + 0] = (float)u[0];
    lv->zn[8 * iz + 1] = (float)u[3];
    for (int c = 0; c < 4; c++) {
      double p = 1.0;
      for (int d = 0; d < 4; d++)
        if (d != c) p *= (u[c] - u[d]);
      lv->zn[8 * iz + 2 + c] = (float)(1.0 / p);
    }
  }
  lv->ni = ni;
  lv->nj = nj;
  lv->nk = nk;
  lv->offi = offi;
  lv->offj = offj;
}

static int upload_ztab(adzc_ztab* lv) {
  ADZ_CK(cudaGetDevice(&lv->device));
  ADZ_CK(cudaMalloc(&lv->d_z, sizeof(double) * lv->z.size()));
  ADZ_CK(cudaMalloc(&lv->d_ocz, sizeof(double) * lv->ocz.size()));
  ADZ_CK(cudaMalloc(&lv->d_zn, sizeof(float) * lv->zn.size()));
  ADZ_CK(cudaMemcpy(lv->d_z, lv->z.data(), sizeof(double) * lv->z.size(), cudaMemcpyHostToDevice));
  ADZ_CK(cudaMemcpy(lv->d_ocz, lv->ocz.data(), sizeof(double) * lv->ocz.size(), cudaMemcpyHostToDevice));
  ADZ_CK(cudaMemcpy(lv->d_zn, lv->zn.data(), sizeof(float) * lv->zn.size(), cudaMemcpyHostToDevice));
  return ADZC_OK;
}

extern "C" int adzc_ztab_create(const double* levels, int nk, int ni, int nj, int offi, int offj, ztab** out) {
  if (!levels || !out || nk < 1 || ni < 1 || nj < 1) return fail(ADZC_ERR_ARG);
  if (nk < 4) return fail(ADZC_ERR_NK);
  auto* lv = new (std::nothrow) adzc_ztab();
  if (!lv) return fail(ADZC_ERR_ALLOC);
  build_ztab_host(lv, levels, nk, ni, nj, offi, offj);
  int st = upload_ztab(lv);
  if (st != ADZC_OK) {
    adzc_ztab_destroy(lv);
    return st;
  }
  *out = lv;
  return ADZC_OK;
}

extern "C" int adzc_ztab_destroy(ztab* lv) {
  if (!lv) return ADZC_OK;
  cudaFree(lv->d_z);
  cudaFree(lv->d_ocz);
  cudaFree(lv->d_zn);
  delete lv;
  return ADZC_OK;
}

extern "C" int adzc_last_error(void) { return g_last_status; }

extern "C" const char* adzc_error_string(int st) {
  switch (st) {
    case ADZC_OK: return "ok";
    case ADZC_ERR_ARG: return "invalid argument";
    case ADZC_ERR_CUDA: return "CUDA runtime error";
    case ADZC_ERR_NK: return "fewer than 4 levels";
    case ADZC_ERR_HALO: return "stencil outside the extended array";
    case ADZC_ERR_NONFINITE: return "non-finite wind or position";
    case ADZC_ERR_TIMEOUT: return "bounded device wait expired";
    case ADZC_ERR_ALLOC: return "allocation failed";
    case ADZC_ERR_NODEVICE: return "no CUDA device";
    case ADZC_ERR_SIZE: return "size above capacity";
    case ADZC_ERR_IO: return "file missing, unreadable or not matching";
    default: return "unknown status";
  }
}

// ---------------------------------------------------------------------------
// Level B interpolators on device data
// ---------------------------------------------------------------------------
static int check_prec(int prec) { return (prec == ADZC_REF32 || prec == ADZC_FP64 || prec == ADZC_MIXED); }

static int run_interp(const ztab* lv, int prec, int kind, void* d, void* l, void* mi, void* ma,
                      const void* const* fs, const void* pxyz, int n, int m, int box, cudaStream_t s) {
  if (!lv || !check_prec(prec) || n < 0 || m < 0 || (n > 0 && (!d || !pxyz || !fs))) return fail(ADZC_ERR_ARG);
  if (n == 0) return ADZC_OK;
  const size_t fb = field_bytes(prec);
  const adz::DZtab t = lv->dev();
  if (kind == 2) {
    adz::FieldPtrs fp{};
    fp.src[0] = fs[0];
    fp.dst[0] = d;
    fp.nf = 1;
    fp.ostride = 3;
    ADZ_CK(dispatch_pos(prec, t, 2, n, pxyz, fp, s));
    return ADZC_OK;
  }
  for (int q0 = 0; q0 < m; q0 += adz::kMaxFields) {
    adz::FieldPtrs fp{};
    fp.nf = std::min(adz::kMaxFields, m - q0);
    fp.ostride = 1;
    fp.box222 = box;
    for (int q = 0; q < fp.nf; q++) {
      if (!fs[q0 + q]) return fail(ADZC_ERR_ARG);
      fp.src[q] = fs[q0 + q];
      const size_t o = (size_t)(q0 + q) * n * fb;
      fp.dst[q] = (char*)d + o;
      if (kind == 1) {
        if (!l || !mi || !ma) return fail(ADZC_ERR_ARG);
        fp.lin[q] = (char*)l + o;
        fp.mn[q] = (char*)mi + o;
        fp.mx[q] = (char*)ma + o;
      }
    }
    ADZ_CK(dispatch_pos(prec, t, kind, n, pxyz, fp, s));
  }
  return ADZC_OK;
}

extern "C" int adzc_tricublin_m_n(const ztab* lv, int prec, void* d, const void* const* fs, const void* pxyz, int n,
                                  int m, void* stream) {
  AdzRange nvtx_range("TRICUBLIN");
  return run_interp(lv, prec, 0, d, nullptr, nullptr, nullptr, fs, pxyz, n, m, 0, (cudaStream_t)stream);
}

extern "C" int adzc_tricublin_mono_m_n(const ztab* lv, int prec, void* d, void* l, void* mi, void* ma,
                                       const void* const* fs, const void* pxyz, int n, int m, int box, void* stream) {
  AdzRange nvtx_range("TRICUBLIN mono");
  return run_interp(lv, prec, 1, d, l, mi, ma, fs, pxyz, n, m, box, (cudaStream_t)stream);
}

extern "C" int adzc_tricublin_zyx3_n(const ztab* lv, int prec, void* d, const void* f3, const void* pxyz, int n,
                                     void* stream) {
  AdzRange nvtx_range("TRICUBLIN zyx3");
  const void* fs[1] = {f3};
  if (!f3) return fail(ADZC_ERR_ARG);
  return run_interp(lv, prec, 2, d, nullptr, nullptr, nullptr, fs, pxyz, n, 1, 0, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// adz_set and the step (Level B)
// ---------------------------------------------------------------------------
struct adzc_handle {
  adzc_grid g{};
  adzc_info info{};
  adz::DGrid dg{};
  int device = 0;
  int niter = 1;
  int cold = 0;
  // host copies of the derived tables
  std::vector<double> zm, zt, odelz_m, odelz_t, vw, cy, delz_t, qv_t;
  std::vector<int> search_m, search_t;
  double ovdzm = 0, ovdzt = 0, sig = 0;
  adzc_ztab* tab_m = nullptr;
  adzc_ztab* tab_t = nullptr;
  void* d_tables = nullptr;
  int* d_status = nullptr;
  // scratch owned by the handle: departure winds (3 x ext) and departure w
  void* d_uvw = nullptr;
  size_t uvw_bytes = 0;
  void* d_wdep = nullptr;
  void* d_aux = nullptr;  // mass-fixer scratch
  size_t aux_bytes = 0;
  size_t wdep_bytes = 0;
  // last trajectory, read by adzc_tricub
  int last_prec = -1;
  const double* wpxyz = nullptr;
  const float* pxyzm = nullptr;
  const void* zdt0 = nullptr;
  adz::DtSplit dt{};
  // Adz_uslt, Adz_vslt (ni, nj): surface-layer winds of the top-level pt
  // positions when the grid's slt_winds is set (adzc_slt_winds)
  const void* uslt = nullptr;
  const void* vslt = nullptr;
  // mcrhsint (field type, element (1,1), row stride pert_ld): the ensemble
  // perturbation of every interpolation while set (adzc_rhs_perturbation)
  const void* pert = nullptr;
  int pert_ld = 0;
  // a trajectory split into interior and band (adzc_traject_region): the
  // iteration state its first part ran with, -1 when none is pending
  int pending_prec = -1;
  int pending_niter = 0;
  int pending_cold = 0;
};

static int build_search(const std::vector<double>& z, int nk, double sig, const std::vector<double>& delz,
                        double* ovdz, std::vector<int>* tab) {
  // B/adz_set.F90:193-215; smallest_dz and posz are REAL128 there
  __float128 smallest = (__float128)(sig * delz[1]);
  for (int k = 2; k <= nk; k++) {
    __float128 v = (__float128)(sig * delz[k]);
    if (v < smallest) smallest = v;
  }
  const double ov = (double)((__float128)1.0 / smallest);
  const double pz = 1.0 + sig * (z[nk + 1] - z[0]) * ov;
  const int pnz = (int)std::lround(pz);
  if (pnz < 1 || pnz > (1 << 24)) return ADZC_ERR_ARG;
  *ovdz = (double)((__float128)sig / smallest);
  tab->assign(pnz, 0);
  int k0 = 0;
  for (int k = 1; k <= pnz; k++) {
    __float128 posz = (__float128)(sig * z[0]) + (__float128)(double)(k - 1) * smallest;
    if (posz > (__float128)(sig * z[k0 + 1])) k0 = std::min(nk + 1, k0 + 1);
    (*tab)[k - 1] = k0;
  }
  return ADZC_OK;
}

static double lag3(double zz, double z1, double z2, double z3, double z4) {  // B/adz_set.F90:530-536
  return (((zz - z2) * (zz - z3) * (zz - z4)) / ((z1 - z2) * (z1 - z3) * (z1 - z4)));
}

extern "C" int adzc_setup(const adzc_grid* gin, adzc_handle** out) {
  if (!gin || !out || !gin->zm || !gin->zt || !gin->zx || !gin->cy) return fail(ADZC_ERR_ARG);
  const adzc_grid& g = *gin;
  if (g.ni < 1 || g.nj < 1 || g.bc_lam_flux < 0 || g.bc_lam_flux > 2 || g.schm_autobar < 0 || g.schm_autobar > 1)
    return fail(ADZC_ERR_ARG);
  if (g.nk < 4) return fail(ADZC_ERR_NK);
  {  // stencil offsets inside the extended array are 32-bit in the kernels
    const long long hx = std::max(1, g.maxcfl) + 1;
    if (((long long)g.ni + 2 * hx) * ((long long)g.nj + 2 * hx) * g.nk > 0x7fffffffLL) return fail(ADZC_ERR_SIZE);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(ADZC_ERR_NODEVICE);
  auto* h = new (std::nothrow) adzc_handle();
  if (!h) return fail(ADZC_ERR_ALLOC);
  h->g = g;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const double EPS_8 = 2.e-5;
  const int BCS_BASE = 4, ext = 1;
  adzc_info& I = h->info;
  const int maxcfl = std::max(1, g.maxcfl);  // B/adz_set.F90:71-82
  I.halox = I.haloy = maxcfl + 1;
  const int lminx = 1 - I.halox, lmaxx = ni + I.halox, lminy = 1 - I.haloy, lmaxy = nj + I.haloy;
  I.nit = lmaxx - lminx + 1;
  I.njt = lmaxy - lminy + 1;
  const int niu = ni - (g.east ? 1 : 0), njv = nj - (g.north ? 1 : 0);
  I.i0 = 1 + g.pil_w - (ext + 1) * g.west;  // B/adz_set.F90:94-114
  I.in = ni - g.pil_e + ext * g.east;
  I.j0 = 1 + g.pil_s - (ext + 1) * g.south;
  I.jn = nj - g.pil_n + ext * g.north;
  I.i0u = 1 + g.pil_w;
  I.j0v = 1 + g.pil_s;
  I.inu = niu - g.pil_e;
  I.jnv = njv - g.pil_n;
  I.k0 = g.lam_gbpil_t + 1;
  I.k0t = std::max(1, g.lam_gbpil_t);
  I.k0m = std::max(I.k0t - 2, 1);
  if (g.bc_lam_flux != 0) I.k0m = 1;
  I.iminposx = g.i0g + lminx + EPS_8;  // B/adz_set.F90:132-160
  I.imaxposx = g.i0g + lmaxx - 2 - EPS_8;
  I.iminposy = g.j0g + lminy + EPS_8;
  I.imaxposy = g.j0g + lmaxy - 2 - EPS_8;
  if (g.west) I.iminposx = g.i0g + BCS_BASE + EPS_8;
  if (g.east) I.imaxposx = g.i0g + ni - BCS_BASE - 1 - EPS_8;
  if (g.south) I.iminposy = g.j0g + BCS_BASE + EPS_8;
  if (g.north) I.imaxposy = g.j0g + nj - BCS_BASE - 1 - EPS_8;
  I.i0b = 1 + BCS_BASE * g.west;
  I.inb = ni - BCS_BASE * g.east;
  I.j0b = 1 + BCS_BASE * g.south;
  I.jnb = nj - BCS_BASE * g.north;
  auto np = [&](int a, int b, int c, int d, int k) {
    return (long long)std::max(0, b - a + 1) * std::max(0, d - c + 1) * std::max(0, nk - k + 1);
  };
  I.npts[0] = np(I.i0, I.in, I.j0, I.jn, I.k0);
  I.npts[1] = np(I.i0u, I.inu, I.j0, I.jn, I.k0);
  I.npts[2] = np(I.i0, I.in, I.j0v, I.jnv, I.k0);
  I.npts[3] = np(I.i0, I.in, I.j0, I.jn, I.k0t);

  h->zm.assign(g.zm, g.zm + nk + 2);
  h->zt.assign(g.zt, g.zt + nk + 2);
  std::vector<double> zx(g.zx, g.zx + nk + 1);
  const auto& zm = h->zm;
  const auto& zt = h->zt;
  h->sig = (zm[nk] - zm[1]) / std::fabs(zm[nk] - zm[1]);  // B/adz_set.F90:178-179
  std::vector<double> delz_m(nk + 1), delz_t(nk + 1);
  h->odelz_m.assign(nk + 1, 0.0);
  h->odelz_t.assign(nk + 1, 0.0);
  const float verysmall = 1.17549435e-38f * 1.e5f;  // tiny(real)*1.e5
  for (int k = 0; k <= nk; k++) {                   // B/adz_set.F90:181-191
    delz_m[k] = (double)9.e33f;
    delz_t[k] = (double)9.e33f;
    if (std::fabs(zm[k + 1] - zm[k]) > verysmall) delz_m[k] = zm[k + 1] - zm[k];
    if (std::fabs(zt[k + 1] - zt[k]) > verysmall) delz_t[k] = zt[k + 1] - zt[k];
    h->odelz_m[k] = 1.0 / delz_m[k];
    h->odelz_t[k] = 1.0 / delz_t[k];
  }
  if (build_search(zm, nk, h->sig, delz_m, &h->ovdzm, &h->search_m) != ADZC_OK ||
      build_search(zt, nk, h->sig, delz_t, &h->ovdzt, &h->search_t) != ADZC_OK) {
    delete h;
    return fail(ADZC_ERR_ARG);
  }
  I.pnz_m = (int)h->search_m.size();
  I.pnz_t = (int)h->search_t.size();
  h->vw.assign(8 * (nk + 1), 0.0);
  double* vw = h->vw.data();
  for (int k = 2; k <= nk - 1; k++) {  // B/adz_set.F90:261-271
    const double rx = zm[k], ra = zx[k - 2], rb = zx[k - 1], rc = zx[k], rd = zx[k + 1];
    vw[0 * (nk + 1) + k] = lag3(rx, ra, rb, rc, rd);
    vw[1 * (nk + 1) + k] = lag3(rx, rb, ra, rc, rd);
    vw[2 * (nk + 1) + k] = lag3(rx, rc, ra, rb, rd);
    vw[3 * (nk + 1) + k] = lag3(rx, rd, ra, rb, rc);
  }
  for (int k = 2; k <= nk - 2; k++) {  // B/adz_set.F90:272-281
    const double rx = zt[k], ra = zm[k - 1], rb = zm[k], rc = zm[k + 1], rd = zm[k + 2];
    vw[4 * (nk + 1) + k] = lag3(rx, ra, rb, rc, rd);
    vw[5 * (nk + 1) + k] = lag3(rx, rb, ra, rc, rd);
    vw[6 * (nk + 1) + k] = lag3(rx, rc, ra, rb, rd);
    vw[7 * (nk + 1) + k] = lag3(rx, rd, ra, rb, rc);
  }
  // BICUBH_QV denominators on thermo levels (B/adz_set.F90:286-311), products left to right
  h->qv_t.assign(10 * (nk + 1), 0.0);
  for (int k = 2; k <= nk - 2; k++) {
    const double ra = zt[k - 1], rb = zt[k], rc = zt[k + 1], rd = zt[k + 2];
    double* q = h->qv_t.data() + 10 * k;
    q[0] = 1.0 / ((ra - rb) * (ra - rc) * (ra - rd));
    q[1] = 1.0 / ((rb - ra) * (rb - rc) * (rb - rd));
    q[2] = 1.0 / ((rc - ra) * (rc - rb) * (rc - rd));
    q[3] = 1.0 / ((rd - ra) * (rd - rb) * (rd - rc));
  }
  for (int k = 3; k <= nk - 3; k++) {
    const double r[6] = {zt[k - 2], zt[k - 1], zt[k], zt[k + 1], zt[k + 2], zt[k + 3]};
    double* q = h->qv_t.data() + 10 * k + 4;
    for (int a = 0; a < 6; a++) {  // product over the other five nodes, in order
      double prod = 0.0;
      bool first = true;
      for (int b = 0; b < 6; b++) {
        if (b == a) continue;
        prod = first ? (r[a] - r[b]) : prod * (r[a] - r[b]);
        first = false;
      }
      q[a] = 1.0 / prod;
    }
  }
  h->delz_t = delz_t;
  h->cy.assign(g.cy, g.cy + I.njt);
  h->niter = std::max(1, g.itraj);

  int st;
  if ((st = adzc_ztab_create(zm.data() + 1, nk, I.nit, I.njt, 1 - g.i0g, 1 - g.j0g, &h->tab_m)) != ADZC_OK ||
      (st = adzc_ztab_create(zt.data() + 1, nk, I.nit, I.njt, 1 - g.i0g, 1 - g.j0g, &h->tab_t)) != ADZC_OK) {
    adzc_destroy(h);
    return fail(st);
  }
  // one device block for every table
  const size_t nd = zm.size() + zt.size() + h->odelz_m.size() + h->odelz_t.size() + h->vw.size() + h->cy.size() +
                    h->delz_t.size() + h->qv_t.size();
  const size_t ni_ = h->search_m.size() + h->search_t.size() + 1;
  if (cudaGetDevice(&h->device) != cudaSuccess || cudaMalloc(&h->d_tables, nd * sizeof(double) + ni_ * sizeof(int)) !=
                                                      cudaSuccess) {
    adzc_destroy(h);
    return fail(ADZC_ERR_CUDA);
  }
  std::vector<char> blob(nd * sizeof(double) + ni_ * sizeof(int), 0);
  double* dp = (double*)blob.data();
  size_t o = 0;
  auto put = [&](const std::vector<double>& v) {
    std::memcpy(dp + o, v.data(), v.size() * sizeof(double));
    const double* dev = (const double*)h->d_tables + o;
    o += v.size();
    return dev;
  };
  adz::DGrid& D = h->dg;
  D.zm = put(zm);
  D.zt = put(zt);
  D.odelz_m = put(h->odelz_m);
  D.odelz_t = put(h->odelz_t);
  D.vw = put(h->vw);
  D.cy = put(h->cy);
  D.delz_t = put(h->delz_t);
  D.qv_t = put(h->qv_t);
  int* ip = (int*)(dp + nd);
  int* dip = (int*)((double*)h->d_tables + nd);
  std::memcpy(ip, h->search_m.data(), h->search_m.size() * sizeof(int));
  D.search_m = dip;
  std::memcpy(ip + h->search_m.size(), h->search_t.data(), h->search_t.size() * sizeof(int));
  D.search_t = dip + h->search_m.size();
  h->d_status = dip + h->search_m.size() + h->search_t.size();
  if (cudaMemcpy(h->d_tables, blob.data(), blob.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    adzc_destroy(h);
    return fail(ADZC_ERR_CUDA);
  }
  D.ni = ni; D.nj = nj; D.nk = nk;
  D.halox = I.halox; D.haloy = I.haloy;
  D.lminx = lminx; D.lminy = lminy;
  D.nit = I.nit; D.njt = I.njt;
  D.nij = (long long)I.nit * I.njt;
  D.i0g = g.i0g; D.j0g = g.j0g;
  D.i0 = I.i0; D.in = I.in; D.j0 = I.j0; D.jn = I.jn;
  D.i0u = I.i0u; D.inu = I.inu; D.j0v = I.j0v; D.jnv = I.jnv;
  D.i0b = I.i0b; D.inb = I.inb; D.j0b = I.j0b; D.jnb = I.jnb;
  D.k0 = I.k0; D.k0t = I.k0t; D.k0m = I.k0m;
  D.pnz_m = I.pnz_m; D.pnz_t = I.pnz_t;
  D.slt_winds = g.slt_winds;
  D.autobar = g.schm_autobar;
  D.imnx = I.iminposx; D.imxx = I.imaxposx; D.imny = I.iminposy; D.imxy = I.imaxposy;
  D.sig = h->sig; D.ovdzm = h->ovdzm; D.ovdzt = h->ovdzt;
  D.zmin = g.zmin; D.zmax = g.zmax;
  D.inv_rayt = g.inv_rayt; D.inv_hx = g.inv_hx; D.inv_hy = g.inv_hy;
  D.vw5 = (zx[0] - zm[1]) / (zx[0] - zx[1]);  // B/adz_set.F90:282-284
  D.vw6 = (zm[nk] - zx[nk]) / (zx[nk - 1] - zx[nk]);
  D.ww = g.wmstar_nk;  // B/adz_interp_traj.F90:41-43
  D.wp = (zt[nk] - zm[nk - 1]) * g.idz_t_nkm1;
  D.wm = 1.0 - D.wp;
  D.tab_m = h->tab_m->dev();
  D.tab_t = h->tab_t->dev();
  D.status = h->d_status;
  *out = h;
  return ADZC_OK;
}

extern "C" int adzc_destroy(adzc_handle* h) {
  if (!h) return ADZC_OK;
  adzc_ztab_destroy(h->tab_m);
  adzc_ztab_destroy(h->tab_t);
  cudaFree(h->d_tables);
  cudaFree(h->d_uvw);
  cudaFree(h->d_wdep);
  cudaFree(h->d_aux);
  delete h;
  return ADZC_OK;
}

extern "C" int adzc_query(const adzc_handle* h, adzc_info* info) {
  if (!h || !info) return fail(ADZC_ERR_ARG);
  *info = h->info;
  return ADZC_OK;
}

static adz::DtSplit dt_split(const adzc_grid& g, double dt) {  // B/adz_traject.F90:38-59
  adz::DtSplit s{};
  double a = 0.0, za = 0.0;
  if (g.schm_advec == 1) { a = dt * 0.5; za = dt * 0.5; }
  if (g.schm_advec == 2) { a = dt * g.bA_m; za = dt * g.bA; }
  if (g.schm_advec == 3) { a = (1.0 - g.bA_m) * dt; za = (1.0 - g.bA) * dt; }
  s.dtD = dt - a; s.dtzD = dt - za; s.dtA = a; s.dtzA = za;
  if (g.schm_advec == 0) { s.dtA = s.dtD = s.dtzA = s.dtzD = 0.0; }
  s.dt = dt;
  return s;
}

static int ensure(void** p, size_t* have, size_t need) {
  if (*have >= need) return ADZC_OK;
  cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMalloc(p, need) != cudaSuccess) return ADZC_ERR_ALLOC;
  *have = need;
  return ADZC_OK;
}

extern "C" int adzc_inittraj(adzc_handle* h, int prec, void* pxyzm, double* wpxyz, void* stream) {
  AdzRange nvtx_range("adz_inittraj");
  if (!h || !check_prec(prec) || !wpxyz || (prec == ADZC_REF32 && !pxyzm)) return fail(ADZC_ERR_ARG);
  ADZ_CK(dispatch_init(prec, h->dg, (float*)pxyzm, wpxyz, (cudaStream_t)stream));
  h->niter = std::max(6, h->g.itraj);  // B/adz_inittraj.F90:25
  h->cold = 1;
  return ADZC_OK;
}

extern "C" int adzc_traject(adzc_handle* h, int prec, double dt, int niter, const void* uu_ext, const void* vv_ext,
                            const void* ww_ext, const void* ut0, const void* vt0, const void* zdt0, void* pxyzm,
                            double* wpxyz, void* stream) {
  AdzRange nvtx_range("adz_traject");
  if (!h || !check_prec(prec) || !uu_ext || !vv_ext || !ww_ext || !ut0 || !vt0 || !zdt0 || !wpxyz ||
      (prec == ADZC_REF32 && !pxyzm))
    return fail(ADZC_ERR_ARG);
  if (!std::isfinite(dt)) return fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  const adz::DGrid& D = h->dg;
  const size_t fb = field_bytes(prec);
  if (ensure(&h->d_uvw, &h->uvw_bytes, adz::uvw_values(prec) * fb * (size_t)D.nij * D.nk) != ADZC_OK ||
      ensure(&h->d_wdep, &h->wdep_bytes, fb * (size_t)D.ni * D.nj * D.nk) != ADZC_OK)
    return fail(ADZC_ERR_ALLOC);
  ADZ_CK(dispatch_prepare(prec, D, uu_ext, vv_ext, ww_ext, h->d_uvw, s));
  adz::TrajArgs a{};
  a.uvw_d = h->d_uvw;
  a.ut0 = ut0;
  a.vt0 = vt0;
  a.zdt0 = zdt0;
  a.pxyzm = (float*)pxyzm;
  a.wpxyz = wpxyz;
  a.wdep = h->d_wdep;
  a.niter = niter > 0 ? niter : h->niter;
  a.cold = h->cold;
  a.k00 = (D.k0 > 1) ? 1 : D.k0m;  // B/adz_traject.F90:63-64
  a.dt = dt_split(h->g, dt);
  ADZ_CK(dispatch_traject(prec, D, a, s));
  h->niter = std::max(1, h->g.itraj);  // B/adz_traject.F90:120
  h->cold = 0;
  h->last_prec = prec;
  h->wpxyz = wpxyz;
  h->pxyzm = (const float*)pxyzm;
  h->zdt0 = zdt0;
  h->dt = a.dt;
  return ADZC_OK;
}

namespace {

// arrival points of a position set (B/adz_set.F90:94-114, 167-172); set B is
// range b, all levels, at the t-set positions (Adz_pb)
void set_box(const adzc_handle* h, int set, int& i0, int& nx, int& j0, int& ny, int& k0, int& nz) {
  const adzc_info& I = h->info;
  int i1, j1;
  switch (set) {
    case ADZC_SET_Q: i0 = I.i0; i1 = I.in; j0 = I.j0; j1 = I.jn; k0 = I.k0; break;
    case ADZC_SET_U: i0 = I.i0u; i1 = I.inu; j0 = I.j0; j1 = I.jn; k0 = I.k0; break;
    case ADZC_SET_V: i0 = I.i0; i1 = I.in; j0 = I.j0v; j1 = I.jnv; k0 = I.k0; break;
    case ADZC_SET_B: i0 = I.i0b; i1 = I.inb; j0 = I.j0b; j1 = I.jnb; k0 = 1; break;
    default: i0 = I.i0; i1 = I.in; j0 = I.j0; j1 = I.jn; k0 = I.k0t; break;
  }
  nx = i1 - i0 + 1;
  ny = j1 - j0 + 1;
  nz = h->dg.nk - k0 + 1;
}

adz::SetArgs set_args(const adzc_handle* h) {
  const adzc_info& I = h->info;
  adz::SetArgs a{};
  a.wpxyz = h->wpxyz;
  a.pxyzm = h->pxyzm;
  a.wdep = h->d_wdep;
  a.zdt0 = h->zdt0;
  a.dt = h->dt;
  a.k00 = std::max(I.k0t - 1, 1);  // B/adz_interp_traj.F90:39-40
  if (h->g.bc_lam_flux != 0 && I.k0 > 1) a.k00 = 1;
  a.uslt = h->uslt;
  a.vslt = h->vslt;
  a.pert = h->pert;
  a.pert_ld = h->pert_ld;
  return a;
}

// a mono flag of adzc_tricub: 0..2, | ADZC_QV on the thermo sets T and B only
bool mono_ok(int mv, int set) {
  if ((mv & ~(3 | ADZC_QV)) != 0 || (mv & 3) == 3) return false;
  return !((mv & ADZC_QV) && set != ADZC_SET_T && set != ADZC_SET_B);
}

// the position set a kernel derives: set B is range b of the t set
int kernel_set(int set) { return set == ADZC_SET_B ? ADZC_SET_T : set; }

}  // namespace

extern "C" int adzc_slt_winds(adzc_handle* h, const void* uslt, const void* vslt) {
  if (!h || (!uslt) != (!vslt)) return fail(ADZC_ERR_ARG);
  h->uslt = uslt;
  h->vslt = vslt;
  return ADZC_OK;
}

extern "C" int adzc_rhs_perturbation(adzc_handle* h, const void* mcrhsint, int ld) {
  if (!h || (mcrhsint && ld < h->g.ni)) return fail(ADZC_ERR_ARG);
  h->pert = mcrhsint;
  h->pert_ld = mcrhsint ? ld : 0;
  return ADZC_OK;
}

extern "C" int adzc_tricub(adzc_handle* h, int prec, int set, int nfields, const void* const* srcs, void* const* dsts,
                           const int* mono, void* const* lin, void* const* mn, void* const* mx, void* stream) {
  AdzRange nvtx_range("adz_tricub_hlt");
  if (!h || !check_prec(prec) || set < 0 || set > ADZC_SET_B || nfields < 0 || (nfields > 0 && (!srcs || !dsts)))
    return fail(ADZC_ERR_ARG);
  if (h->last_prec != prec || !h->wpxyz) return fail(ADZC_ERR_ARG);
  if (set == ADZC_SET_B && h->g.bc_lam_flux == 0) return fail(ADZC_ERR_ARG);  // range b needs k00 = 1
  const adz::DGrid& D = h->dg;
  int i0, nx, j0, ny, k0, nz;
  set_box(h, set, i0, nx, j0, ny, k0, nz);
  if (nx <= 0 || ny <= 0 || nz <= 0 || nfields == 0) return ADZC_OK;
  const adz::SetArgs a = set_args(h);
  // tricubic fields, then BICUBH_QV fields (set t only), in groups of kMaxFields
  std::vector<int> groups[2];
  for (int f = 0; f < nfields; f++) {
    const int mv = mono ? mono[f] : 0;
    if (!mono_ok(mv, set)) return fail(ADZC_ERR_ARG);
    if (!srcs[f] || !dsts[f]) return fail(ADZC_ERR_ARG);
    groups[(mv & ADZC_QV) ? 1 : 0].push_back(f);
  }
  for (int kind = 0; kind < 2; kind++) {
    const std::vector<int>& fl = groups[kind];
    for (size_t q0 = 0; q0 < fl.size(); q0 += adz::kMaxFields) {
      adz::FieldPtrs fp{};
      fp.nf = (int)std::min<size_t>(adz::kMaxFields, fl.size() - q0);
      for (int q = 0; q < fp.nf; q++) {
        const int f = fl[q0 + q];
        fp.src[q] = srcs[f];
        fp.dst[q] = dsts[f];
        const int mv = (mono ? mono[f] : 0) & 3;
        if (mv != 0) fp.mono_mask |= 1u << q;
        if (mv == 1) fp.clip_mask |= 1u << q;
        fp.lin[q] = lin ? lin[f] : nullptr;
        fp.mn[q] = mn ? mn[f] : nullptr;
        fp.mx[q] = mx ? mx[f] : nullptr;
      }
      if (kind == 0) {
        ADZ_CK(dispatch_set(prec, D, kernel_set(set), i0, nx, j0, ny, k0, nz, a, fp, (cudaStream_t)stream));
      } else {
        ADZ_CK(dispatch_qv(prec, D, i0, nx, j0, ny, k0, nz, a, fp, (cudaStream_t)stream));
      }
    }
  }
  return ADZC_OK;
}

namespace {

struct Box {
  int i0, nx, j0, ny;
};

// the interior of a tile (points at least m from every side that has a
// neighbour tile, i.e. is not a LAM edge) and the band around it, as boxes
// in local point indices; a box is skipped when empty
int region_boxes(const adzc_handle* h, int region, int m, Box* out) {
  const adzc_grid& g = h->g;
  const int ni = g.ni, nj = g.nj;
  const int mw = g.west ? 0 : m, me = g.east ? 0 : m, ms = g.south ? 0 : m, mn = g.north ? 0 : m;
  int n = 0;
  auto add = [&](int i0, int i1, int j0, int j1) {
    if (i1 >= i0 && j1 >= j0) out[n++] = Box{i0, i1 - i0 + 1, j0, j1 - j0 + 1};
  };
  if (region == 1) {
    add(1 + mw, ni - me, 1 + ms, nj - mn);
    return n;
  }
  // band: west and east strips over every row, south and north strips between them
  const int xw1 = std::min(mw, ni), xe0 = std::max(mw + 1, ni - me + 1);
  add(1, xw1, 1, nj);
  add(xe0, ni, 1, nj);
  const int ys1 = std::min(ms, nj), yn0 = std::max(ms + 1, nj - mn + 1);
  add(xw1 + 1, xe0 - 1, 1, ys1);
  add(xw1 + 1, xe0 - 1, yn0, nj);
  return n;
}

// a box intersected with a horizontal range (i0..i1, j0..j1)
bool clip_box(const Box& b, int i0, int i1, int j0, int j1, Box* out) {
  const int a0 = std::max(b.i0, i0), a1 = std::min(b.i0 + b.nx - 1, i1);
  const int c0 = std::max(b.j0, j0), c1 = std::min(b.j0 + b.ny - 1, j1);
  if (a1 < a0 || c1 < c0) return false;
  *out = Box{a0, a1 - a0 + 1, c0, c1 - c0 + 1};
  return true;
}

cudaError_t dispatch_traject_box(int prec, const adz::DGrid& g, const adz::TrajArgs& a, const Box& b,
                                 cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_traject_box<adz::kRef32>(g, a, b.i0, b.nx, b.j0, b.ny, s);
    case ADZC_FP64: return adz::launch_traject_box<adz::kFp64>(g, a, b.i0, b.nx, b.j0, b.ny, s);
    default: return adz::launch_traject_box<adz::kMixed>(g, a, b.i0, b.nx, b.j0, b.ny, s);
  }
}
cudaError_t dispatch_prepare_box(int prec, const adz::DGrid& g, const void* uu, const void* vv, const void* ww,
                                 void* o, int ci0, int nci, int cj0, int ncj, cudaStream_t s) {
  switch (prec) {
    case ADZC_REF32: return adz::launch_prepare_box<adz::kRef32>(g, uu, vv, ww, o, ci0, nci, cj0, ncj, s);
    case ADZC_FP64: return adz::launch_prepare_box<adz::kFp64>(g, uu, vv, ww, o, ci0, nci, cj0, ncj, s);
    default: return adz::launch_prepare_box<adz::kMixed>(g, uu, vv, ww, o, ci0, nci, cj0, ncj, s);
  }
}

}  // namespace

extern "C" int adzc_traject_region(adzc_handle* h, int prec, double dt, int niter, const void* uu_ext,
                                   const void* vv_ext, const void* ww_ext, const void* ut0, const void* vt0,
                                   const void* zdt0, void* pxyzm, double* wpxyz, int region, void* stream) {
  if (region == 0)
    return adzc_traject(h, prec, dt, niter, uu_ext, vv_ext, ww_ext, ut0, vt0, zdt0, pxyzm, wpxyz, stream);
  AdzRange nvtx_range(region == 1 ? "adz_traject interior" : "adz_traject band");
  if (!h || !check_prec(prec) || !uu_ext || !vv_ext || !ww_ext || !ut0 || !vt0 || !zdt0 || !wpxyz ||
      (prec == ADZC_REF32 && !pxyzm) || (region != 1 && region != 2) || !std::isfinite(dt))
    return fail(ADZC_ERR_ARG);
  if (region == 2 && h->pending_prec != prec) return fail(ADZC_ERR_ARG);  // the interior first
  const cudaStream_t s = (cudaStream_t)stream;
  const adz::DGrid& D = h->dg;
  const size_t fb = field_bytes(prec);
  if (ensure(&h->d_uvw, &h->uvw_bytes, adz::uvw_values(prec) * fb * (size_t)D.nij * D.nk) != ADZC_OK ||
      ensure(&h->d_wdep, &h->wdep_bytes, fb * (size_t)D.ni * D.nj * D.nk) != ADZC_OK)
    return fail(ADZC_ERR_ALLOC);
  if (region == 1) {
    // every cell; the halo cells are prepared again once their winds arrive
    ADZ_CK(dispatch_prepare(prec, D, uu_ext, vv_ext, ww_ext, h->d_uvw, s));
    h->pending_prec = prec;
    h->pending_niter = niter > 0 ? niter : h->niter;
    h->pending_cold = h->cold;
  } else {
    // the halo frame of the extended array: columns outside 1..ni, rows outside 1..nj
    const int hx = h->info.halox, hy = h->info.haloy, nit = D.nit, njt = D.njt;
    ADZ_CK(dispatch_prepare_box(prec, D, uu_ext, vv_ext, ww_ext, h->d_uvw, 0, nit, 0, hy, s));
    ADZ_CK(dispatch_prepare_box(prec, D, uu_ext, vv_ext, ww_ext, h->d_uvw, 0, nit, njt - hy, hy, s));
    ADZ_CK(dispatch_prepare_box(prec, D, uu_ext, vv_ext, ww_ext, h->d_uvw, 0, hx, hy, njt - 2 * hy, s));
    ADZ_CK(dispatch_prepare_box(prec, D, uu_ext, vv_ext, ww_ext, h->d_uvw, nit - hx, hx, hy, njt - 2 * hy, s));
  }
  adz::TrajArgs a{};
  a.uvw_d = h->d_uvw;
  a.ut0 = ut0;
  a.vt0 = vt0;
  a.zdt0 = zdt0;
  a.pxyzm = (float*)pxyzm;
  a.wpxyz = wpxyz;
  a.wdep = h->d_wdep;
  a.niter = h->pending_niter;
  a.cold = h->pending_cold;
  a.k00 = (D.k0 > 1) ? 1 : D.k0m;  // B/adz_traject.F90:63-64
  a.dt = dt_split(h->g, dt);
  // a departure stencil reaches maxcfl + 1 cells, the arrival winds' averaging 2
  Box boxes[4];
  const int nb = region_boxes(h, region, std::max(1, h->g.maxcfl) + 3, boxes);
  for (int q = 0; q < nb; q++) ADZ_CK(dispatch_traject_box(prec, D, a, boxes[q], s));
  if (region == 2) {
    h->pending_prec = -1;
    h->niter = std::max(1, h->g.itraj);  // B/adz_traject.F90:120
    h->cold = 0;
    h->last_prec = prec;
    h->wpxyz = wpxyz;
    h->pxyzm = (const float*)pxyzm;
    h->zdt0 = zdt0;
    h->dt = a.dt;
  }
  return ADZC_OK;
}

extern "C" int adzc_interp_traj(adzc_handle* h, int prec, int set, void* pos, void* stream) {
  AdzRange nvtx_range("adz_interp_traj");
  if (!h || !check_prec(prec) || set < 0 || set > ADZC_SET_B || !pos) return fail(ADZC_ERR_ARG);
  if (h->last_prec != prec || !h->wpxyz) return fail(ADZC_ERR_ARG);
  if (set == ADZC_SET_B && h->g.bc_lam_flux == 0) return fail(ADZC_ERR_ARG);  // range b needs k00 = 1
  int i0, nx, j0, ny, k0, nz;
  set_box(h, set, i0, nx, j0, ny, k0, nz);
  if (nx <= 0 || ny <= 0 || nz <= 0) return ADZC_OK;
  const adz::SetArgs a = set_args(h);
  const adz::DGrid& D = h->dg;
  const cudaStream_t s = (cudaStream_t)stream;
  const int ks = kernel_set(set);
  switch (prec) {
    case ADZC_REF32: ADZ_CK(adz::launch_positions<adz::kRef32>(D, ks, i0, nx, j0, ny, k0, nz, a, pos, s)); break;
    case ADZC_FP64: ADZ_CK(adz::launch_positions<adz::kFp64>(D, ks, i0, nx, j0, ny, k0, nz, a, pos, s)); break;
    default: ADZ_CK(adz::launch_positions<adz::kMixed>(D, ks, i0, nx, j0, ny, k0, nz, a, pos, s)); break;
  }
  return ADZC_OK;
}

extern "C" int adzc_bc_lam_flux(adzc_handle* h, int prec, int ntr, const void* const* srcs, void* const* fo,
                                void* const* fi, void* stream) {
  AdzRange nvtx_range("adz_BC_LAM_Aranami_hlt");
  if (!h || !check_prec(prec) || ntr < 0 || (ntr > 0 && (!srcs || !fo || !fi))) return fail(ADZC_ERR_ARG);
  if (h->last_prec != prec || !h->wpxyz) return fail(ADZC_ERR_ARG);
  if (h->g.bc_lam_flux != 1) return fail(ADZC_ERR_ARG);  // Aranami fluxes (adz_BC_LAM_flux 1) only
  if (!srcs) return fail(ADZC_ERR_ARG);
  for (int q = 0; q < ntr; q++)  // srcs[q] NULL: the masks alone (PSADJ)
    if (!fo[q] || !fi[q]) return fail(ADZC_ERR_ARG);
  if (ntr == 0) return ADZC_OK;
  const adzc_info& I = h->info;
  const adz::DGrid& D = h->dg;
  adz::BcMask m{D.lminx, D.lminy, D.nit, D.njt, D.nk, D.ni, D.nj, h->g.west, h->g.east, h->g.south, h->g.north,
                h->g.pil_w, h->g.pil_e, h->g.pil_s, h->g.pil_n, I.k0t, I.i0b, I.inb, I.j0b, I.jnb, h->g.maxcfl + 1};
  const int nxb = I.inb - I.i0b + 1, nyb = I.jnb - I.j0b + 1;
  if (nxb <= 0 || nyb <= 0) return ADZC_OK;
  const size_t fb = prec == ADZC_FP64 ? sizeof(double) : sizeof(float);
  const size_t ext = (size_t)D.nij * D.nk * fb;
  constexpr int kChunk = adz::kMaxFields / 2;  // tracers per interpolation launch (out and in fields)
  void* scratch = nullptr;
  if (adz_internal_aux(h, 2 * std::min(kChunk, ntr) * ext, &scratch) != ADZC_OK) return fail(ADZC_ERR_ALLOC);
  adz::SetArgs a = set_args(h);
  a.pert = nullptr;  // the fluxes are plain interpolations (tricublin_zyx1_m_n)
  const cudaStream_t s = (cudaStream_t)stream;
  for (int q0 = 0; q0 < ntr; q0 += kChunk) {
    const int nf = std::min(kChunk, ntr - q0);
    adz::FieldPtrs fp{};
    fp.nf = 2 * nf;
    for (int q = 0; q < nf; q++) {
      char* mo = (char*)scratch + (size_t)(2 * q) * ext;
      char* mi = (char*)scratch + (size_t)(2 * q + 1) * ext;
      ADZ_CK(prec == ADZC_FP64 ? adz::launch_bc_mask<double>(m, srcs[q0 + q], mo, mi, s)
                               : adz::launch_bc_mask<float>(m, srcs[q0 + q], mo, mi, s));
      fp.src[2 * q] = mo;
      fp.src[2 * q + 1] = mi;
      fp.dst[2 * q] = fo[q0 + q];
      fp.dst[2 * q + 1] = fi[q0 + q];
    }
    // Adz_pb over (i0b:inb, j0b:jnb, 1:nk): the set-t positions of those points
    ADZ_CK(dispatch_set(prec, D, ADZC_SET_T, I.i0b, nxb, I.j0b, nyb, 1, D.nk, a, fp, s));
    for (int q = 0; q < nf; q++)
      ADZ_CK(prec == ADZC_FP64 ? adz::launch_bc_zero<double>(m, fo[q0 + q], fi[q0 + q], s)
                               : adz::launch_bc_zero<float>(m, fo[q0 + q], fi[q0 + q], s));
  }
  return ADZC_OK;
}

extern "C" int adzc_bc_lam_zlf(adzc_handle* h, int prec, int setup, int ntr, void* const* f1, void* const* f2,
                               void* stream) {
  AdzRange nvtx_range("ZLF_0");
  if (!h || !check_prec(prec) || setup < 1 || setup > 4 || ntr < 0 || (ntr > 0 && !f1)) return fail(ADZC_ERR_ARG);
  if (h->g.bc_lam_flux != 2) return fail(ADZC_ERR_ARG);  // Adz_BC_LAM_flux 2: Zerroukat-Shipway
  const bool two = setup == 2 || setup == 4;
  if (ntr > 0 && two && !f2) return fail(ADZC_ERR_ARG);
  for (int q = 0; q < ntr; q++)
    if (!f1[q] || (two && !f2[q])) return fail(ADZC_ERR_ARG);
  const adzc_info& I = h->info;
  const adz::DGrid& D = h->dg;
  const adz::BcMask m{D.lminx, D.lminy, D.nit, D.njt, D.nk, D.ni, D.nj, h->g.west, h->g.east, h->g.south,
                      h->g.north, h->g.pil_w, h->g.pil_e, h->g.pil_s, h->g.pil_n, I.k0t, I.i0b, I.inb, I.j0b,
                      I.jnb, h->g.maxcfl + 1};
  const cudaStream_t s = (cudaStream_t)stream;
  for (int q0 = 0; q0 < ntr; q0 += adz::kMaxFields) {
    adz::ZlfPtrs fp{};
    fp.n = std::min(adz::kMaxFields, ntr - q0);
    for (int q = 0; q < fp.n; q++) {
      fp.f1[q] = f1[q0 + q];
      fp.f2[q] = two ? f2[q0 + q] : nullptr;
    }
    ADZ_CK(prec == ADZC_FP64 ? adz::launch_bc_zlf<double>(m, setup, fp, s) : adz::launch_bc_zlf<float>(m, setup, fp, s));
  }
  return ADZC_OK;
}

extern "C" int adzc_tricub_sets_region(adzc_handle* h, int prec, const int* nfields, const void* const* srcs,
                                       void* const* dsts, const int* mono, int region, void* stream) {
  if (region == 0) return adzc_tricub_sets(h, prec, nfields, srcs, dsts, mono, stream);
  AdzRange nvtx_range(region == 1 ? "ADZ_MAIN sets interior" : "ADZ_MAIN sets band");
  if (!h || !check_prec(prec) || !nfields || (region != 1 && region != 2)) return fail(ADZC_ERR_ARG);
  if (h->last_prec != prec || !h->wpxyz) return fail(ADZC_ERR_ARG);
  int ntot = 0;
  for (int q = 0; q < 4; q++) {
    if (nfields[q] < 0) return fail(ADZC_ERR_ARG);
    ntot += nfields[q];
  }
  if (ntot == 0) return ADZC_OK;
  if (!srcs || !dsts) return fail(ADZC_ERR_ARG);
  for (int f = 0, set = 0, left = nfields[0]; f < ntot; f++, left--) {
    while (left == 0) left = nfields[++set];
    if (!srcs[f] || !dsts[f] || !mono_ok(mono ? mono[f] : 0, set)) return fail(ADZC_ERR_ARG);
  }
  // the position sets read Adz_wpxyz up to 2 points away (Adz_pmu, Adz_pmv)
  Box rb[4];
  const int nb = region_boxes(h, region, 2, rb);
  const adz::SetArgs a = set_args(h);
  const adz::DGrid& D = h->dg;
  const cudaStream_t s = (cudaStream_t)stream;
  adz::SetParts sp{};
  int f0 = 0;
  for (int set = 0; set < 4; set++) {
    const int nf = nfields[set];
    int i0, nx, j0, ny, k0, nz;
    set_box(h, set, i0, nx, j0, ny, k0, nz);
    for (int q = 0; q < nb && nf > 0 && nx > 0 && ny > 0 && nz > 0; q++) {
      Box c;
      if (!clip_box(rb[q], i0, i0 + nx - 1, j0, j0 + ny - 1, &c)) continue;
      for (int qv = 0; qv < 2; qv++) {  // tricubic field groups, then BICUBH_QV ones
        adz::FieldPtrs fp{};
        for (int f = f0; f < f0 + nf; f++) {
          const int mv = mono ? mono[f] : 0;
          if (((mv & ADZC_QV) != 0) != (qv == 1)) continue;
          const int k = fp.nf++;
          fp.src[k] = srcs[f];
          fp.dst[k] = dsts[f];
          if ((mv & 3) != 0) fp.mono_mask |= 1u << k;
          if ((mv & 3) == 1) fp.clip_mask |= 1u << k;
          const bool last = f == f0 + nf - 1;
          if (fp.nf < adz::kMaxFields && !last) continue;
          if (qv) {
            ADZ_CK(dispatch_qv(prec, D, c.i0, c.nx, c.j0, c.ny, k0, nz, a, fp, s));
          } else {
            if (sp.n == adz::kMaxParts) {
              ADZ_CK(dispatch_parts(prec, D, a, sp, s));
              sp = adz::SetParts{};
            }
            adz::SetPart& P = sp.p[sp.n++];
            P.fp = fp;
            P.set = set;
            P.i0 = c.i0; P.nx = c.nx; P.j0 = c.j0; P.ny = c.ny; P.k0 = k0; P.nz = nz;
          }
          fp = adz::FieldPtrs{};
        }
        if (fp.nf > 0) {  // a group closed by a field of the other kind
          if (qv) {
            ADZ_CK(dispatch_qv(prec, D, c.i0, c.nx, c.j0, c.ny, k0, nz, a, fp, s));
          } else {
            if (sp.n == adz::kMaxParts) {
              ADZ_CK(dispatch_parts(prec, D, a, sp, s));
              sp = adz::SetParts{};
            }
            adz::SetPart& P = sp.p[sp.n++];
            P.fp = fp;
            P.set = set;
            P.i0 = c.i0; P.nx = c.nx; P.j0 = c.j0; P.ny = c.ny; P.k0 = k0; P.nz = nz;
          }
        }
      }
    }
    f0 += nf;
  }
  if (sp.n > 0) ADZ_CK(dispatch_parts(prec, D, a, sp, s));
  return ADZC_OK;
}

extern "C" int adzc_tricub_sets(adzc_handle* h, int prec, const int* nfields, const void* const* srcs,
                                void* const* dsts, const int* mono, void* stream) {
  AdzRange nvtx_range("ADZ_MAIN sets");
  if (!h || !check_prec(prec) || !nfields) return fail(ADZC_ERR_ARG);
  if (h->last_prec != prec || !h->wpxyz) return fail(ADZC_ERR_ARG);
  int ntot = 0;
  for (int q = 0; q < 4; q++) {
    if (nfields[q] < 0) return fail(ADZC_ERR_ARG);
    ntot += nfields[q];
  }
  if (ntot == 0) return ADZC_OK;
  if (!srcs || !dsts) return fail(ADZC_ERR_ARG);
  for (int f = 0, set = 0, left = nfields[0]; f < ntot; f++, left--) {
    while (left == 0) left = nfields[++set];
    if (!srcs[f] || !dsts[f] || !mono_ok(mono ? mono[f] : 0, set)) return fail(ADZC_ERR_ARG);
  }
  // every tricubic field group of every set in one interleaved launch
  // (k_tricub_parts); BICUBH_QV fields of set t after it
  const adz::SetArgs a = set_args(h);
  const cudaStream_t s = (cudaStream_t)stream;
  adz::SetParts sp{};
  std::vector<const void*> qv_src;
  std::vector<void*> qv_dst;
  std::vector<int> qv_mono;
  int f0 = 0;
  for (int set = 0; set < 4; set++) {
    const int nf = nfields[set];
    int i0, nx, j0, ny, k0, nz;
    set_box(h, set, i0, nx, j0, ny, k0, nz);
    const bool empty = nx <= 0 || ny <= 0 || nz <= 0;
    adz::SetPart* part = nullptr;
    for (int f = f0; f < f0 + nf && !empty; f++) {
      const int mv = mono ? mono[f] : 0;
      if (mv & ADZC_QV) {
        qv_src.push_back(srcs[f]);
        qv_dst.push_back(dsts[f]);
        qv_mono.push_back(mv);
        continue;
      }
      if (!part || part->fp.nf == adz::kMaxFields) {
        if (sp.n == adz::kMaxParts) {
          ADZ_CK(dispatch_parts(prec, h->dg, a, sp, s));
          sp = adz::SetParts{};
        }
        part = &sp.p[sp.n++];
        part->set = set;
        part->i0 = i0; part->nx = nx; part->j0 = j0; part->ny = ny; part->k0 = k0; part->nz = nz;
      }
      adz::FieldPtrs& fp = part->fp;
      const int q = fp.nf++;
      fp.src[q] = srcs[f];
      fp.dst[q] = dsts[f];
      if ((mv & 3) != 0) fp.mono_mask |= 1u << q;
      if ((mv & 3) == 1) fp.clip_mask |= 1u << q;
    }
    f0 += nf;
  }
  if (sp.n > 0) ADZ_CK(dispatch_parts(prec, h->dg, a, sp, s));
  if (!qv_src.empty())
    return adzc_tricub(h, prec, ADZC_SET_T, (int)qv_src.size(), qv_src.data(), qv_dst.data(), qv_mono.data(),
                       nullptr, nullptr, nullptr, stream);
  return ADZC_OK;
}

extern "C" int adzc_status(adzc_handle* h, int reset, void* stream) {
  if (!h) return fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  ADZ_CK(cudaStreamSynchronize(s));
  int bits = 0;
  ADZ_CK(cudaMemcpy(&bits, h->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) ADZ_CK(cudaMemset(h->d_status, 0, sizeof(int)));
  if (bits & adz::kErrHalo) return ADZC_ERR_HALO;
  if (bits & adz::kErrNonFinite) return ADZC_ERR_NONFINITE;
  if (bits & adz::kErrTimeout) return ADZC_ERR_TIMEOUT;
  return ADZC_OK;
}

// ---------------------------------------------------------------------------
// Level A: the reference ABI with host pointers
// ---------------------------------------------------------------------------
namespace {

// The reference calls its interpolators from every OpenMP thread, one plane
// each.  A Level A call takes one of kSlots staging slots (a stream, a device
// buffer and a pinned buffer for the transposed layout), so calls from
// different threads overlap their copies and kernels.  A thread whose slot is
// busy takes the next free one, and waits for its own when all are busy.
//
// Host arrays are the caller's pageable memory.  Copies go through a ring of
// pinned chunks per slot: the calling thread copies chunk c into pinned
// memory while the DMA of chunk c-1 runs (and the other way round for the
// results), which moves the bytes several times faster than pageable copies.
constexpr int kSlots = 16;
constexpr size_t kChunk = (size_t)8 << 20;
constexpr int kRing = 4;
struct Staging {
  std::mutex mu;
  cudaStream_t stream = nullptr;
  int device = -1;
  void* buf = nullptr;
  size_t cap = 0;
  float* pinned = nullptr;
  size_t pinned_cap = 0;
  char* ring = nullptr;  // kRing chunks of pinned memory
  cudaEvent_t ev[kRing] = {};
  unsigned next = 0;
};

// chunk r of the ring, once the copy that last used it has finished
char* ring_chunk(Staging& S, unsigned r) {
  return cudaEventSynchronize(S.ev[r]) == cudaSuccess ? S.ring + (size_t)r * kChunk : nullptr;
}

bool ring_h2d(Staging& S, void* dst, const void* src, size_t bytes) {
  for (size_t off = 0; off < bytes; off += kChunk) {
    const size_t len = std::min(kChunk, bytes - off);
    const unsigned r = S.next++ % kRing;
    char* c = ring_chunk(S, r);
    if (!c) return false;
    std::memcpy(c, (const char*)src + off, len);
    if (cudaMemcpyAsync((char*)dst + off, c, len, cudaMemcpyHostToDevice, S.stream) != cudaSuccess ||
        cudaEventRecord(S.ev[r], S.stream) != cudaSuccess)
      return false;
  }
  return true;
}

// device -> caller's memory, up to kRing chunks in flight ahead of the
// thread's copy out of the ring
bool ring_d2h(Staging& S, void* dst, const void* src, size_t bytes) {
  const size_t nch = (bytes + kChunk - 1) / kChunk;
  const unsigned first = S.next;
  size_t issued = 0;
  for (size_t c = 0; c < nch; c++) {
    for (; issued < nch && issued < c + kRing; issued++) {
      const unsigned r = (first + (unsigned)issued) % kRing;
      char* h = ring_chunk(S, r);
      const size_t len = std::min(kChunk, bytes - issued * kChunk);
      if (!h || cudaMemcpyAsync(h, (const char*)src + issued * kChunk, len, cudaMemcpyDeviceToHost, S.stream) !=
                    cudaSuccess ||
          cudaEventRecord(S.ev[r], S.stream) != cudaSuccess)
        return false;
    }
    const unsigned r = (first + (unsigned)c) % kRing;
    char* h = ring_chunk(S, r);
    if (!h) return false;
    std::memcpy((char*)dst + c * kChunk, h, std::min(kChunk, bytes - c * kChunk));
  }
  S.next = first + (unsigned)nch;
  return true;
}
Staging& acquire_slot(std::unique_lock<std::mutex>* lock) {
  static Staging slots[kSlots];
  const size_t h = std::hash<std::thread::id>{}(std::this_thread::get_id());
  for (int t = 0; t < kSlots; t++) {
    Staging& s = slots[(h + t) % kSlots];
    std::unique_lock<std::mutex> l(s.mu, std::try_to_lock);
    if (l.owns_lock()) {
      *lock = std::move(l);
      return s;
    }
  }
  Staging& s = slots[h % kSlots];
  *lock = std::unique_lock<std::mutex>(s.mu);
  return s;
}

// corner offset the kernel will use for an FP32 position (same arithmetic as
// the device coef_f32pos) and the stencil extent beyond it
void corner_f32(const adzc_ztab* lv, const pxpypz& p, long long* lo, long long* hi) {
  const double px = p.px, py = p.py, pz = p.pz;
  int ix = (int)px + lv->offi;
  int iy = (int)py + lv->offj;
  int iz = (int)pz;
  if (iz < 1) iz = 1;
  if (iz > lv->nk - 1) iz = lv->nk - 1;
  long long ijk = (long long)(ix - 2) + (long long)(iy - 2) * lv->ni + (long long)(iz - 1) * lv->ni * lv->nj;
  const int iz0 = iz - 1;
  const bool zl = (iz0 < 1 || iz0 > lv->nk - 3);
  const long long nij = (long long)lv->ni * lv->nj;
  if (!zl) ijk -= nij;
  *lo = ijk;
  *hi = ijk + 3 + 3LL * lv->ni + (zl ? nij : 3 * nij);
}

// Stage the touched part of each source (elements [lo, hi] per field, in
// units of ``comp`` floats) plus positions; returns device base pointers
// already shifted so that base[off] addresses what f[off] addresses.
int stage_inputs(Staging& S, const adzc_ztab* lv, int comp, const float* const* fs, int m, const pxpypz* pos, int n,
                 size_t out_floats, std::vector<const void*>* dbase, void** dpos, float** dout) {
  int dev = 0;
  ADZ_CK(cudaGetDevice(&dev));
  if (S.stream == nullptr || S.device != dev) {
    if (S.stream) cudaStreamDestroy(S.stream);
    cudaFree(S.buf);
    cudaFreeHost(S.pinned);
    cudaFreeHost(S.ring);
    for (cudaEvent_t& e : S.ev) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    S.buf = nullptr;
    S.cap = 0;
    S.pinned = nullptr;
    S.pinned_cap = 0;
    S.ring = nullptr;
    S.device = -1;
    ADZ_CK(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking));
    ADZ_CK(cudaMallocHost(&S.ring, kRing * kChunk));
    for (cudaEvent_t& e : S.ev) ADZ_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    S.device = dev;
  }
  long long lo = (1LL << 62), hi = -(1LL << 62);
  for (int j = 0; j < n; j++) {
    // the reference takes positions already clipped to the array; a
    // non-finite or huge one would be truncated differently here and on the
    // device, so the staged range would not cover what the kernel reads
    const pxpypz& q = pos[j];
    if (!(std::fabs(q.px) < 1.0e9f && std::fabs(q.py) < 1.0e9f && std::fabs(q.pz) < 1.0e9f)) return fail(ADZC_ERR_ARG);
    long long a, b;
    corner_f32(lv, q, &a, &b);
    lo = std::min(lo, a);
    hi = std::max(hi, b);
  }
  const size_t span = (size_t)(hi - lo + 1) * comp;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t need = al(sizeof(pxpypz) * n) + m * al(sizeof(float) * span) + al(sizeof(float) * out_floats);
  if (S.cap < need) {
    cudaFree(S.buf);
    S.buf = nullptr;
    S.cap = 0;
    if (cudaMalloc(&S.buf, need) != cudaSuccess) return fail(ADZC_ERR_ALLOC);
    S.cap = need;
  }
  char* p = (char*)S.buf;
  *dpos = p;
  if (!ring_h2d(S, p, pos, sizeof(pxpypz) * n)) return fail(ADZC_ERR_CUDA);
  p += al(sizeof(pxpypz) * n);
  dbase->clear();
  for (int q = 0; q < m; q++) {
    if (!ring_h2d(S, p, fs[q] + lo * comp, sizeof(float) * span)) return fail(ADZC_ERR_CUDA);
    dbase->push_back((const float*)p - lo * comp);
    p += al(sizeof(float) * span);
  }
  *dout = (float*)p;
  return ADZC_OK;
}

void level_a(int kind, float* d, float* l, float* mi, float* ma, float** dp, const float* const* fs, pxpypz* pxyz,
             ztab* lv, int n, int m, int layout /*0 m_n, 1 n_m, 2 p*/) {
  if (!lv || n <= 0 || m <= 0 || !fs || !pxyz) {
    if (n > 0) fail(ADZC_ERR_ARG);
    return;
  }
  std::unique_lock<std::mutex> lock;
  Staging& S = acquire_slot(&lock);
  const int comp = (kind == 2) ? 3 : 1;
  const int nout = (kind == 1) ? 4 : 1;
  const size_t out_floats = (size_t)nout * m * n * comp;
  std::vector<const void*> base;
  void* dpos = nullptr;
  float* dout = nullptr;
  if (stage_inputs(S, lv, comp, fs, (kind == 2) ? 1 : m, pxyz, n, out_floats, &base, &dpos, &dout) != ADZC_OK)
    return;
  const adz::DZtab t = lv->dev();
  int st;
  if (kind == 2) {
    adz::FieldPtrs fp{};
    fp.src[0] = base[0];
    fp.dst[0] = dout;
    fp.nf = 1;
    fp.ostride = 3;
    st = dispatch_pos(ADZC_REF32, t, 2, n, dpos, fp, S.stream) == cudaSuccess ? ADZC_OK : ADZC_ERR_CUDA;
  } else {
    st = run_interp(lv, ADZC_REF32, kind, dout, dout + (size_t)m * n, dout + 2 * (size_t)m * n,
                    dout + 3 * (size_t)m * n, base.data(), dpos, n, m, 0, S.stream);
  }
  if (st != ADZC_OK) {
    fail(st);
    return;
  }
  // results go straight into the caller's arrays where the layouts agree
  float* outs[4] = {d, l, mi, ma};
  bool ok = true;
  if (kind == 2) {
    ok = ring_d2h(S, d, dout, sizeof(float) * 3 * n);
  } else if (layout == 0) {
    for (int o = 0; o < nout && ok; o++) ok = ring_d2h(S, outs[o], dout + (size_t)o * m * n, sizeof(float) * m * n);
  } else if (layout == 2) {
    for (int q = 0; q < m && ok; q++) ok = ring_d2h(S, dp[q], dout + (size_t)q * n, sizeof(float) * n);
  } else {  // n_m: through the slot's pinned buffer, transposed on the host
    if (S.pinned_cap < out_floats) {
      cudaFreeHost(S.pinned);
      S.pinned = nullptr;
      S.pinned_cap = 0;
      if (cudaMallocHost(&S.pinned, sizeof(float) * out_floats) != cudaSuccess) {
        fail(ADZC_ERR_ALLOC);
        return;
      }
      S.pinned_cap = out_floats;
    }
    ok = cudaMemcpyAsync(S.pinned, dout, sizeof(float) * out_floats, cudaMemcpyDeviceToHost, S.stream) ==
         cudaSuccess;
  }
  if (!ok || cudaStreamSynchronize(S.stream) != cudaSuccess) {
    fail(ADZC_ERR_CUDA);
    return;
  }
  if (kind != 2 && layout == 1) {
    for (int o = 0; o < nout; o++)
      for (int q = 0; q < m; q++) {
        const float* row = S.pinned + ((size_t)o * m + q) * n;
        float* dst = outs[o];
        for (int j = 0; j < n; j++) dst[(size_t)j * m + q] = row[j];
      }
  }
}

}  // namespace

extern "C" ztab* Vsearch_setup_plus(double* levels, int nk, int ni, int nj, int offseti, int offsetj) {
  ztab* lv = nullptr;
  if (adzc_ztab_create(levels, nk, ni, nj, offseti, offsetj, &lv) != ADZC_OK) return nullptr;
  return lv;
}

extern "C" ztab* Vsearch_setup(double* levels, int nk, int ni, int nj) {
  return Vsearch_setup_plus(levels, nk, ni, nj, 0, 0);
}

extern "C" void Tricublin_zyx1_n(float* d, float* f1, pxpypz* pxyz, ztab* lv, int n) {
  const float* fs[1] = {f1};
  level_a(0, d, nullptr, nullptr, nullptr, nullptr, fs, pxyz, lv, n, 1, 0);
}
extern "C" void Tricublin_zyx1_n_m(float* d, float** fs, pxpypz* pxyz, ztab* lv, int n, int m) {
  level_a(0, d, nullptr, nullptr, nullptr, nullptr, fs, pxyz, lv, n, m, 1);
}
extern "C" void Tricublin_zyx1_m_n(float* dm, float** fs, pxpypz* pxyz, ztab* lv, int n, int m) {
  level_a(0, dm, nullptr, nullptr, nullptr, nullptr, fs, pxyz, lv, n, m, 0);
}
extern "C" void Tricublin_zyx1_p(float** dp, float** fs, pxpypz* pxyz, ztab* lv, int n, int m) {
  level_a(0, nullptr, nullptr, nullptr, nullptr, dp, fs, pxyz, lv, n, m, 2);
}
extern "C" void Tricublin_mono_zyx_n(float* d, float* l, float* mi, float* ma, float* f, pxpypz* pxyz, ztab* lv,
                                     int n) {
  const float* fs[1] = {f};
  level_a(1, d, l, mi, ma, nullptr, fs, pxyz, lv, n, 1, 0);
}
extern "C" void Tricublin_mono_zyx_n_m(float* d, float* l, float* mi, float* ma, float** fs, pxpypz* pxyz, ztab* lv,
                                       int n, int m) {
  level_a(1, d, l, mi, ma, nullptr, fs, pxyz, lv, n, m, 1);
}
extern "C" void Tricublin_mono_zyx_m_n(float* d, float* l, float* mi, float* ma, float** fs, pxpypz* pxyz, ztab* lv,
                                       int n, int m) {
  level_a(1, d, l, mi, ma, nullptr, fs, pxyz, lv, n, m, 0);
}
extern "C" void Tricublin_zyx3_n(float* d, float* f3, pxpypz* pxyz, ztab* lv, int n) {
  const float* fs[1] = {f3};
  level_a(2, d, nullptr, nullptr, nullptr, nullptr, fs, pxyz, lv, n, 1, 0);
}

// ---------------------------------------------------------------------------
// accessors used by the no-allocation entry point (adz_noalloc.cu)
// ---------------------------------------------------------------------------

int adz_internal_view(const adzc_handle* h, adz::DGrid* dg, adzc_info* info, adzc_grid* g, int* niter, int* cold) {
  if (!h) return ADZC_ERR_ARG;
  *dg = h->dg;
  *info = h->info;
  *g = h->g;
  *niter = h->niter;
  *cold = h->cold;
  return ADZC_OK;
}

int adz_internal_warm(const adzc_handle* h) { return h && !h->cold && h->wpxyz != nullptr; }

void adz_internal_after_traject(adzc_handle* h) {
  h->niter = std::max(1, h->g.itraj);
  h->cold = 0;
}

void adz_internal_forget_positions(adzc_handle* h) {
  h->last_prec = -1;
  h->wpxyz = nullptr;
  h->pxyzm = nullptr;
  h->zdt0 = nullptr;
}

adz::DtSplit adz_internal_dt_split(const adzc_grid& g, double dt) { return dt_split(g, dt); }

void adz_internal_set_inputs(const adzc_handle* h, adz::SetArgs* a) {
  a->uslt = h ? h->uslt : nullptr;
  a->vslt = h ? h->vslt : nullptr;
  a->pert = h ? h->pert : nullptr;
  a->pert_ld = h ? h->pert_ld : 0;
}

void adz_internal_record_positions(adzc_handle* h, int prec, double* wpxyz, const void* zdt0, const adz::DtSplit& dt) {
  adz_internal_after_traject(h);
  h->last_prec = prec;
  h->wpxyz = wpxyz;
  h->pxyzm = nullptr;
  h->zdt0 = zdt0;
  h->dt = dt;
}

int adz_internal_fail(int status) { return fail(status); }

int adz_internal_scratch(adzc_handle* h, int prec, void** uvw, void** wdep) {
  if (!h || !uvw || !wdep) return ADZC_ERR_ARG;
  const adz::DGrid& D = h->dg;
  const size_t fb = field_bytes(prec);
  if (ensure(&h->d_uvw, &h->uvw_bytes, adz::uvw_values(prec) * fb * (size_t)D.nij * D.nk) != ADZC_OK ||
      ensure(&h->d_wdep, &h->wdep_bytes, fb * (size_t)D.ni * D.nj * D.nk) != ADZC_OK)
    return ADZC_ERR_ALLOC;
  *uvw = h->d_uvw;
  *wdep = h->d_wdep;
  return ADZC_OK;
}

int adz_internal_aux(adzc_handle* h, size_t bytes, void** p) {
  if (!h || !p) return ADZC_ERR_ARG;
  if (ensure(&h->d_aux, &h->aux_bytes, bytes) != ADZC_OK) return ADZC_ERR_ALLOC;
  *p = h->d_aux;
  return ADZC_OK;
}

void adz_internal_set_iteration(adzc_handle* h, int cold, int niter) {
  h->cold = cold ? 1 : 0;
  h->niter = niter > 0 ? niter : std::max(1, h->g.itraj);
}
