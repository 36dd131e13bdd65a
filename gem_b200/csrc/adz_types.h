// Plain data structures shared by the kernels and the host C-ABI code
// (no device code here, so g++ can compile the host side).
#pragma once
#include "../../include/adz_b200.h"
#include <cuda_runtime.h>
#include <stdint.h>

namespace adz {

constexpr int kMaxFields = 16;  // fields per launch (more are split in chunks)

enum : int { kRef32 = 0, kFp64 = 1, kMixed = 2 };
enum : int { kErrHalo = 1 << 0, kErrNonFinite = 1 << 1, kErrTimeout = 1 << 2 };

// Level descriptor (turbo_tricublin.c:164-173) plus the per-interval FP32
// table of the mixed path: for interval iz the normalised nodes
// u = {(z[iz-1]-z[iz])/h, 0, 1, (z[iz+2]-z[iz])/h}, h = z[iz+1]-z[iz],
// stored as {u[0], u[3], 1/prod(u0-ud), ..., 1/prod(u3-ud), 0, 0}.
struct DZtab {
  const double* z;
  const double* ocz;
  const float* zn;
  int ni, nj, nk, nij, offi, offj;
};

// Everything adz_set derives, as the kernels read it.
struct DGrid {
  int ni, nj, nk, halox, haloy, lminx, lminy, nit, njt;
  long long nij;
  int i0g, j0g;
  int i0, in, j0, jn, i0u, inu, j0v, jnv, i0b, inb, j0b, jnb, k0, k0t, k0m;
  int pnz_m, pnz_t, slt_winds, autobar;
  double imnx, imxx, imny, imxy, sig, ovdzm, ovdzt, zmin, zmax;
  double inv_rayt, inv_hx, inv_hy, vw5, vw6, ww, wp, wm;
  const int* search_m;
  const int* search_t;
  const double* zm;       // Ver_z_8%m(0:nk+1)
  const double* zt;       // Ver_z_8%t(0:nk+1)
  const double* odelz_m;  // 0..nk
  const double* odelz_t;
  const double* vw;       // 8 x (nk+1): vw1m vw2m vw3m vw4m vw1t vw2t vw3t vw4t
  const double* cy;       // index j - lminy
  const double* delz_t;   // 0..nk
  const double* qv_t;     // BICUBH_QV denominators, 10 per level (B/adz_set.F90:286-311)
  DZtab tab_m, tab_t;
  int* status;
};

struct DtSplit {
  double dtA, dtD, dtzA, dtzD, dt;
};

template <int PREC>
struct Types;
template <>
struct Types<kRef32> {
  using F = float;   // fields and winds
  using P = float;   // stored positions
};
template <>
struct Types<kFp64> {
  using F = double;
  using P = double;
};
template <>
struct Types<kMixed> {
  using F = float;
  using P = double;
};

struct FieldPtrs {
  const void* src[kMaxFields];
  void* dst[kMaxFields];
  void* lin[kMaxFields];
  void* mn[kMaxFields];
  void* mx[kMaxFields];
  int nf;
  unsigned mono_mask;  // bit q: field q gets bounds (and clip if clip_mask)
  unsigned clip_mask;
  int box222;
  long long ostride;   // explicit-position kernels: output element stride per point
};

// the tricubic field groups of several position sets in one launch
struct SetPart {
  FieldPtrs fp;
  int set, i0, nx, j0, ny, k0, nz, pad;
};
constexpr int kMaxParts = 8;
struct SetParts {
  SetPart p[kMaxParts];
  int n;
};

struct TrajArgs {
  const void* uvw_d;  // ext, 3 interleaved
  const void* ut0;
  const void* vt0;
  const void* zdt0;
  float* pxyzm;       // REF32 state
  double* wpxyz;
  void* wdep;         // (ni,nj,nk) departure vertical wind of the last iteration
  int niter, cold, k00;
  DtSplit dt;
};

// start of the tolerance iteration from displacements given on a coarse grid
// (nodes i = min(1 + stride*m, ni), likewise j, every level from k00; 3
// floats per node), interpolated bilinearly in (i, j); d NULL: from the
// arrival point (cold) or from wpxyz
struct GuessStart {
  const float* d;
  int stride, nxc, nyc;
};

struct SetArgs {
  const double* wpxyz;
  const float* pxyzm;  // REF32 only
  const void* wdep;
  const void* zdt0;
  const void* uslt;    // optional surface-layer winds (ni,nj)
  const void* vslt;
  const void* pert;    // optional mcrhsint (field type, element (1,1), row stride pert_ld)
  DtSplit dt;
  int k00;             // interp_traj k00
  int pert_ld;
};


// values per cell of the departure-wind scratch (u, v, w interleaved)
inline int uvw_values(int prec) {
  (void)prec;
  return 3;
}

template <int PREC>
cudaError_t launch_prepare(const DGrid& g, const void* uu, const void* vv, const void* ww, void* uvw_d,
                           cudaStream_t s);
template <int PREC>
cudaError_t launch_traject_box(const DGrid& g, const TrajArgs& a, int i0, int nx, int j0, int ny, cudaStream_t s);
template <int PREC>
cudaError_t launch_prepare_box(const DGrid& g, const void* uu, const void* vv, const void* ww, void* uvw_d, int ci0,
                               int nci, int cj0, int ncj, cudaStream_t s);
template <int PREC>
cudaError_t launch_positions(const DGrid& g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                             const SetArgs& a, void* pos, cudaStream_t s);
template <int PREC>
cudaError_t launch_inittraj(const DGrid& g, float* pxyzm, double* wpxyz, cudaStream_t s);
template <int PREC>
cudaError_t launch_traject(const DGrid& g, const TrajArgs& a, cudaStream_t s);
template <int PREC>
cudaError_t launch_traject_tol(const DGrid& g, const TrajArgs& a, double tol, int maxit, unsigned char* iters,
                               unsigned long long* stats, cudaStream_t s, const GuessStart& gs = GuessStart{});
template <int PREC>
cudaError_t launch_tricub_set(const DGrid& g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                              const SetArgs& a, const FieldPtrs& fp, cudaStream_t s);
template <int PREC>
cudaError_t launch_qv_set(const DGrid& g, int i0, int nx, int j0, int ny, int k0, int nz, const SetArgs& a,
                          const FieldPtrs& fp, cudaStream_t s);
template <int PREC>
cudaError_t launch_interp_pos(const DZtab& lv, int kind, int n, const void* pos, const FieldPtrs& fp,
                              cudaStream_t s);

// ---- batches of domains in one persistent launch (adz_batch.cu) ----
constexpr int kMaxGroups = 8;  // field groups per domain (a set may need several)

struct BDom {
  DGrid g;
  const void* uu;  // departure winds (ext layout) read by phase 0
  const void* vv;
  const void* ww;
  TrajArgs ta;
  SetArgs sa;
  int ngroups;
  int gset[kMaxGroups];        // position set of each group
  int grange[kMaxGroups][5];   // i0, nx, j0, ny, k0 of each group's set
  FieldPtrs gfp[kMaxGroups];
};

// per-domain descriptors of the batch kernel, passed as one grid-constant
// kernel parameter (read from the constant bank, never aliased by stores)
struct BDomC {
  DGrid g;
  const void* uu;
  const void* vv;
  const void* ww;
  TrajArgs ta;
  SetArgs sa;
};
constexpr int kBatchMaxDomains = ADZC_BATCH_MAX_DOMAINS;
struct BatchParams {
  BDomC d[kBatchMaxDomains];
};
static_assert(sizeof(BatchParams) <= 32000, "kernel parameter limit");

struct BItem {
  int dom, phase, group;
  int tiles;  // phases 1 and 2: 1 when start/count count tiles of kBatchTileI x kBatchTileK, 0 points
  long long start, count;
};

constexpr int kBatchVariants = 3;  // register budgets of the batch kernel
constexpr int kBatchLanes = 4;     // concurrent graph branches of the per-domain plan
// trajectory items of the batch are runs of tiles of kBatchTileI consecutive
// i by kBatchTileK consecutive levels (one warp row per level, a block of 128
// threads per tile), as the per-domain trajectory kernel walks its points
constexpr int kBatchTileI = 32, kBatchTileK = 4;
// a region walks tiles when they leave at most 10 % of their lanes idle,
// else rows of consecutive i (narrow and shallow domains)
inline bool batch_use_tiles(long long nx, long long nz) {
  const long long nic = (nx + kBatchTileI - 1) / kBatchTileI, nkg = (nz + kBatchTileK - 1) / kBatchTileK;
  return nx > 0 && nz > 0 && nic * kBatchTileI * nkg * kBatchTileK * 10 <= nx * nz * 11;
}
static_assert(kBatchTileI * kBatchTileK == 128, "a batch trajectory tile is one block of 128 threads");
template <int PREC>
cudaError_t launch_tricub_parts(const DGrid& g, const SetArgs& a, const SetParts& sp, cudaStream_t s);
// the tile geometry of the LAM boundary-flux masks (adz_bcflux.cu)
struct BcMask {
  int lminx, lminy, nit, njt, nk, ni, nj;
  int west, east, south, north, pil_w, pil_e, pil_s, pil_n, k0t;
  int i0b, inb, j0b, jnb;
  int ext;  // Grd_maxcfl + 1: the ZLF extension of the core
};
// the Zerroukat-Shipway (ZLF) setups of adz_BC_LAM_zlf_hlt on up to
// kMaxFields tracers at once: f1[q] (and f2[q] for setups 2 and 4)
struct ZlfPtrs {
  void* f1[kMaxFields];
  void* f2[kMaxFields];
  int n;
};
template <typename T>
cudaError_t launch_bc_zlf(const BcMask& m, int setup, const ZlfPtrs& f, cudaStream_t s);
template <typename T>
cudaError_t launch_bc_mask(const BcMask& m, const void* src, void* mo, void* mi, cudaStream_t s);
template <typename T>
cudaError_t launch_bc_zero(const BcMask& m, void* fo, void* fi, cudaStream_t s);

// bound of a dependency wait of the batch kernel: >= 1 s of 64 ns sleeps
constexpr unsigned long long kDepSpins = 1ull << 24;
template <int PREC>
cudaError_t launch_batch(int variant, int grid, const BatchParams& P, const BDom* doms, const BItem* items,
                         long long nitems,
                         const unsigned* need, unsigned long long* next, unsigned* done, int* status,
                         unsigned long long max_spins, cudaStream_t s);
template <int PREC>
int batch_resident_blocks(int variant);  // blocks of 128 threads resident per SM
// the phased plan: one persistent launch per phase (items[pstart[p], pstart[p+1])),
// each with the register budget of the per-domain kernel of that phase;
// next[3] are the phases' queue counters
template <int PREC>
cudaError_t launch_batch_phased(const int* grid, const BatchParams& P, const BDom* doms, const BItem* items,
                                const long long* pstart, unsigned long long* next, cudaStream_t s);
template <int PREC>
int batch_phase_resident_blocks(int phase);

}  // namespace adz
