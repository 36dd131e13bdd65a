// Trajectory diagnostics and state I/O.
//
// adzc_cfl: the maximum Courant numbers of the last trajectory
// (B/adz_cfl.F90:47-189, adz_courant): horizontal |(dx, dy)|, vertical |dz|
// and 3-D, with the grid point of each maximum.  Values are formed in FP64
// in the reference's operation order (IEEE square roots), and ties go to the
// first point in the reference's loop order (k, then j, then i), so the
// result is bit-for-bit the reference's.  Two passes: per-block best, then
// one block over the block bests in index order.
//
// adzc_state_save / adzc_state_load: the trajectory state a restart needs,
// Adz_wpxyz and (REF32) Adz_pxyzm, which the reference registers with its
// memory manager's restart flag (B/adz_set.F90:343-360), plus the iteration
// state of the handle (cold start pending, Adz_niter).  The file is this
// library's own: a 64-byte header, then the arrays as stored on the device.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace adz {
namespace diag {

constexpr int kBlocks = 296;
constexpr int kThreads = 256;

struct Best {
  double v[3];
  long long t[3];  // linear index in loop order, -1 = none
};

// a thread visits its points in increasing loop order, so keeping only a
// strictly larger value keeps the first of equal maxima, as the reference does
__device__ __forceinline__ void take(double& bv, long long& bt, double v, long long t) {
  if (v > bv) {
    bv = v;
    bt = t;
  }
}

__global__ void __launch_bounds__(kThreads) k_cfl_part(const double* __restrict__ wp, int i0, int nx, int j0,
                                                       int ny, int k0, int nz, int ni, int nj, int nk, int l_i0,
                                                       int l_j0, Best* __restrict__ part) {
  const long long n = (long long)nx * ny * nz;
  const long long wnx = ni + 4, wny = nj + 4, plane = wnx * wny, comp = plane * nk;
  double bv[3] = {0.0, 0.0, 0.0};
  long long bt[3] = {-1, -1, -1};
  for (long long t = blockIdx.x * (long long)kThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kThreads) {
    // the tile's volume is below 2^31 cells (adzc_setup refuses larger tiles)
    const int ti = (int)t, nxy = nx * ny;
    const int i = i0 + ti % nx, j = j0 + (ti / nx) % ny, k = k0 + ti / nxy;
    const long long e = (long long)(i + 1) + (long long)(j + 1) * wnx + (long long)(k - 1) * plane;
    const double x = fabs(wp[e] - (double)l_i0 + 1.0 - (double)i);
    const double y = fabs(wp[e + comp] - (double)l_j0 + 1.0 - (double)j);
    const double z = fabs(wp[e + 2 * comp] - (double)k);
    // explicit roundings: no contraction into FMA, as the reference computes them
    const double x2 = __dmul_rn(x, x), y2 = __dmul_rn(y, y), z2 = __dmul_rn(z, z);
    const double xy = sqrt(__dadd_rn(x2, y2));
    const double xyz = sqrt(__dadd_rn(__dadd_rn(x2, y2), z2));
    take(bv[0], bt[0], xy, t);
    take(bv[1], bt[1], z, t);
    take(bv[2], bt[2], xyz, t);
  }
  __shared__ double sv[3][kThreads];
  __shared__ long long st[3][kThreads];
  for (int q = 0; q < 3; q++) {
    sv[q][threadIdx.x] = bv[q];
    st[q][threadIdx.x] = bt[q];
  }
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 3; q++) {
        const double v = sv[q][threadIdx.x + o];
        const long long t = st[q][threadIdx.x + o];
        if (t >= 0 && (st[q][threadIdx.x] < 0 || v > sv[q][threadIdx.x] ||
                       (v == sv[q][threadIdx.x] && t < st[q][threadIdx.x]))) {
          sv[q][threadIdx.x] = v;
          st[q][threadIdx.x] = t;
        }
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) {
      part[blockIdx.x].v[q] = sv[q][0];
      part[blockIdx.x].t[q] = st[q][0];
    }
}

__global__ void k_cfl_final(const Best* __restrict__ part, int nblk, int i0, int nx, int j0, int ny, int k0,
                            int l_i0, int l_j0, double* __restrict__ cfl, int* __restrict__ idx) {
  if (threadIdx.x != 0) return;
  for (int q = 0; q < 3; q++) {
    double bv = 0.0;
    long long bt = -1;
    for (int b = 0; b < nblk; b++) {
      const double v = part[b].v[q];
      const long long t = part[b].t[q];
      if (t >= 0 && v > 0.0 && (v > bv || (v == bv && (bt < 0 || t < bt)))) {
        bv = v;
        bt = t;
      }
    }
    // no point above 0: the reference reports index 0 (+ offset)
    int i = 0, j = 0, k = 0;
    if (bt >= 0) {
      i = i0 + (int)(bt % nx);
      j = j0 + (int)((bt / nx) % ny);
      k = k0 + (int)(bt / ((long long)nx * ny));
    }
    cfl[q] = bv;
    idx[3 * q + 0] = i + l_i0 - 1;
    idx[3 * q + 1] = j + l_j0 - 1;
    idx[3 * q + 2] = k;
  }
}

}  // namespace diag
}  // namespace adz

extern "C" int adzc_cfl(adzc_handle* h, const double* wpxyz, double* cfl, int* idx, void* stream) {
  AdzRange nvtx_range("adz_cfl");
  using namespace adz::diag;
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int niter = 0, cold = 0;
  if (!h || !wpxyz || !cfl || !idx || adz_internal_view(h, &D, &I, &G, &niter, &cold) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  // scope of adz_cfl: Adz_i0:Adz_in, Adz_j0:Adz_jn, Adz_k0:l_nk
  const int nx = I.in - I.i0 + 1, ny = I.jn - I.j0 + 1, nz = D.nk - I.k0 + 1;
  if (nx <= 0 || ny <= 0 || nz <= 0) return adz_internal_fail(ADZC_ERR_ARG);
  void* scratch = nullptr;
  if (adz_internal_aux(h, kBlocks * sizeof(Best), &scratch) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ALLOC);
  const cudaStream_t s = (cudaStream_t)stream;
  k_cfl_part<<<kBlocks, kThreads, 0, s>>>(wpxyz, I.i0, nx, I.j0, ny, I.k0, nz, D.ni, D.nj, D.nk, G.i0g, G.j0g,
                                          (Best*)scratch);
  k_cfl_final<<<1, 32, 0, s>>>((const Best*)scratch, kBlocks, I.i0, nx, I.j0, ny, I.k0, G.i0g, G.j0g, cfl, idx);
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

namespace {

struct StateHeader {
  char magic[8];   // "ADZSTATE"
  int version, prec, ni, nj, nk, k0m, cold, niter;
  long long wp_bytes, px_bytes;
  char pad[8];
};
static_assert(sizeof(StateHeader) == 64, "state header size");

// pxyzm as the handle stores it: (3, ni, nj, nk) FP32, REF32 only
size_t px_bytes_of(const adz::DGrid& D, int prec) {
  return prec == ADZC_REF32 ? (size_t)3 * D.ni * D.nj * D.nk * sizeof(float) : 0;
}

}  // namespace

extern "C" int adzc_state_save(adzc_handle* h, int prec, const void* pxyzm, const double* wpxyz, const char* path) {
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int niter = 0, cold = 0;
  if (!h || !wpxyz || !path || (prec == ADZC_REF32 && !pxyzm) ||
      (prec != ADZC_REF32 && prec != ADZC_FP64 && prec != ADZC_MIXED) ||
      adz_internal_view(h, &D, &I, &G, &niter, &cold) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  StateHeader hd{};
  std::memcpy(hd.magic, "ADZSTATE", 8);
  hd.version = 1;
  hd.prec = prec;
  hd.ni = D.ni;
  hd.nj = D.nj;
  hd.nk = D.nk;
  hd.k0m = D.k0m;
  hd.cold = cold;
  hd.niter = niter;
  hd.wp_bytes = (long long)(D.ni + 4) * (D.nj + 4) * D.nk * 3 * sizeof(double);
  hd.px_bytes = (long long)px_bytes_of(D, prec);
  std::vector<char> buf(hd.wp_bytes + hd.px_bytes);
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(buf.data(), wpxyz, hd.wp_bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
      (hd.px_bytes && cudaMemcpy(buf.data() + hd.wp_bytes, pxyzm, hd.px_bytes, cudaMemcpyDeviceToHost) != cudaSuccess))
    return adz_internal_fail(ADZC_ERR_CUDA);
  FILE* f = std::fopen(path, "wb");
  if (!f) return adz_internal_fail(ADZC_ERR_IO);
  const bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  if (std::fclose(f) != 0 || !ok) return adz_internal_fail(ADZC_ERR_IO);
  return ADZC_OK;
}

extern "C" int adzc_state_load(adzc_handle* h, int prec, void* pxyzm, double* wpxyz, const char* path) {
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int niter = 0, cold = 0;
  if (!h || !wpxyz || !path || (prec == ADZC_REF32 && !pxyzm) ||
      adz_internal_view(h, &D, &I, &G, &niter, &cold) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  FILE* f = std::fopen(path, "rb");
  if (!f) return adz_internal_fail(ADZC_ERR_IO);
  StateHeader hd{};
  bool ok = std::fread(&hd, sizeof(hd), 1, f) == 1 && std::memcmp(hd.magic, "ADZSTATE", 8) == 0 && hd.version == 1;
  ok = ok && hd.prec == prec && hd.ni == D.ni && hd.nj == D.nj && hd.nk == D.nk && hd.k0m == D.k0m &&
       hd.wp_bytes == (long long)(D.ni + 4) * (D.nj + 4) * D.nk * 3 * (long long)sizeof(double) &&
       hd.px_bytes == (long long)px_bytes_of(D, prec);
  std::vector<char> buf;
  if (ok) {
    buf.resize(hd.wp_bytes + hd.px_bytes);
    ok = std::fread(buf.data(), 1, buf.size(), f) == buf.size();
  }
  std::fclose(f);
  if (!ok) return adz_internal_fail(ADZC_ERR_IO);
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(wpxyz, buf.data(), hd.wp_bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      (hd.px_bytes && cudaMemcpy(pxyzm, buf.data() + hd.wp_bytes, hd.px_bytes, cudaMemcpyHostToDevice) != cudaSuccess))
    return adz_internal_fail(ADZC_ERR_CUDA);
  adz_internal_set_iteration(h, hd.cold, hd.niter);
  return ADZC_OK;
}
