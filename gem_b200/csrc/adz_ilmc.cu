// ILMC shape-preserving filter (B/ILMC_LAM.F90:16-388 with
// B/ilmc_lam_loop.inc): each point outside its [min, max] bounds moves its
// excess (or deficit) of air-mass-weighted tracer into the room its
// neighbours have, shell by shell (sweeps), then an optional clip.
//
// The reference visits the points in loop order (k, then j, then i) and
// every visit changes the point's neighbourhood, so later visits see earlier
// results.  This file keeps that order exactly and still runs in parallel:
// a point's visit reads and writes only the cube of radius sweep_max around
// it, so two visits commute unless the points are within 2 * sweep_max of
// each other (Chebyshev).  Work runs in rounds; in each round every pending
// point with no earlier pending point within 2 * sweep_max is visited (their
// cubes are disjoint), then those points leave the pending set.  The earliest
// pending point is always ready, so every round makes progress, and the
// result is bit-for-bit the sequential one.  Only points outside their bounds
// at the start are pending: a visit never pushes a neighbour out of its
// bounds (the reference clamps every neighbour update), so no other point can
// become one.  Built with -fmad=false: the REAL arithmetic is the
// reference's, without contraction.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace adz {
namespace ilmc {

constexpr int kMaxShell = 400;  // sweep_max <= 4 (the reference's sweep_max(400))

struct Box {
  int il, ir, jl, jr, k0, nk;
  int lminx, lminy, nit;
  long long nij;
  __host__ __device__ int bx() const { return ir - il + 1; }
  __host__ __device__ int by() const { return jr - jl + 1; }
  __host__ __device__ long long n() const { return (long long)bx() * by() * (nk - k0 + 1); }
};

__device__ __forceinline__ long long ext(const Box& b, int i, int j, int k) {
  return (long long)(i - b.lminx) + (long long)(j - b.lminy) * b.nit + (long long)(k - 1) * b.nij;
}

__device__ __forceinline__ void coords(const Box& b, long long o, int& i, int& j, int& k) {
  i = b.il + (int)(o % b.bx());
  j = b.jl + (int)((o / b.bx()) % b.by());
  k = b.k0 + (int)(o / ((long long)b.bx() * b.by()));
}

template <typename T>
__device__ __forceinline__ T rmax(T a, T b) { return a > b ? a : b; }
template <typename T>
__device__ __forceinline__ T rmin(T a, T b) { return a < b ? a : b; }

// the neighbour shell of one sweep, in the order of the reference's sweep_rd
// lists (B/ILMC_LAM.F90:118-169): jx, then kx, then ix
template <typename Fn>
__device__ __forceinline__ void shell(const Box& b, int i, int j, int k, int sweep, Fn fn) {
  const int kxm = max(k - sweep, b.k0), kxp = min(k + sweep, b.nk);
  const int j1 = max(j - sweep, b.jl), j2 = min(j + sweep, b.jr);
  const int i1 = max(i - sweep, b.il), i2 = min(i + sweep, b.ir);
  int q = 0;
  for (int jx = j1; jx <= j2; jx++)
    for (int kx = kxm; kx <= kxp; kx++) {
      const bool limit_i = (jx != j - sweep && jx != j + sweep) && (kx > k - sweep && kx < k + sweep);
      for (int ix = i1; ix <= i2; ix++) {
        if (limit_i && ix != i - sweep && ix != i + sweep) continue;
        fn(q++, ext(b, ix, jx, kx));
      }
    }
}

// one visit of B/ilmc_lam_loop.inc
template <typename T>
__device__ void visit(const Box& b, T* f, const T* mn, const T* mx, const T* air, int sweep_max, int i, int j,
                      int k) {
  const long long e = ext(b, i, j, k);
  T o_shoot = rmax((T)0, f[e] - mx[e]);
  T u_shoot = rmax((T)0, mn[e] - f[e]);
  if (o_shoot == (T)0 && u_shoot == (T)0) return;
  T cap[kMaxShell];
  const bool over = o_shoot > (T)0;
  for (int sweep = 1; sweep <= sweep_max; sweep++) {
    T msum = 0;
    shell(b, i, j, k, sweep, [&](int q, long long r) {
      cap[q] = over ? rmax((T)0, mx[r] - f[r]) : rmax((T)0, f[r] - mn[r]);
      msum = cap[q] * air[r] + msum;
    });
    const T use = rmin(msum, (over ? o_shoot : u_shoot) * air[e]);
    if (use > (T)0) {
      if (over) {
        f[e] = rmax(f[e] - (T)(use / air[e]), mn[e]);
        o_shoot = rmax((T)0, f[e] - mx[e]);
      } else {
        f[e] = rmin(f[e] + (T)(use / air[e]), mx[e]);
        u_shoot = rmax((T)0, mn[e] - f[e]);
      }
      const T ratio = use / msum;
      shell(b, i, j, k, sweep, [&](int q, long long r) {
        if (cap[q] > (T)0) f[r] = over ? rmin(f[r] + (T)(cap[q] * ratio), mx[r]) : rmax(f[r] - (T)(cap[q] * ratio), mn[r]);
      });
    }
  }
}

// pending points: outside their bounds at the start
template <typename T>
__global__ void __launch_bounds__(256) k_mark(Box b, const T* __restrict__ f, const T* __restrict__ mn,
                                              const T* __restrict__ mx, unsigned char* __restrict__ pend,
                                              int* __restrict__ list, unsigned* __restrict__ count) {
  const long long n = b.n();
  for (long long o = blockIdx.x * 256LL + threadIdx.x; o < n; o += (long long)gridDim.x * 256) {
    int i, j, k;
    coords(b, o, i, j, k);
    const long long e = ext(b, i, j, k);
    const bool v = rmax((T)0, f[e] - mx[e]) != (T)0 || rmax((T)0, mn[e] - f[e]) != (T)0;
    pend[o] = v ? 1 : 0;
    if (v) list[atomicAdd(count, 1u)] = (int)o;
  }
}

// ready: pending, and no earlier pending point within 2 sweep_max
__global__ void __launch_bounds__(256) k_ready(Box b, int sweep_max, const unsigned char* __restrict__ pend,
                                               const int* __restrict__ list, unsigned nlist,
                                               unsigned char* __restrict__ ready) {
  const unsigned q = blockIdx.x * 256u + threadIdx.x;
  if (q >= nlist) return;
  const long long o = list[q];
  if (!pend[o]) {
    ready[q] = 0;
    return;
  }
  int i, j, k;
  coords(b, o, i, j, k);
  const int R = 2 * sweep_max, bx = b.bx(), by = b.by();
  bool ok = true;
  for (int kx = max(k - R, b.k0); kx <= k && ok; kx++)
    for (int jx = max(j - R, b.jl); jx <= min(j + R, b.jr) && ok; jx++) {
      if (kx == k && jx > j) break;
      const int iend = (kx == k && jx == j) ? i - 1 : min(i + R, b.ir);
      const long long row = (long long)(jx - b.jl) * bx + (long long)(kx - b.k0) * bx * by - b.il;
      for (int ix = max(i - R, b.il); ix <= iend; ix++)
        if (pend[row + ix]) {
          ok = false;
          break;
        }
    }
  ready[q] = ok ? 1 : 0;
}

template <typename T>
__global__ void __launch_bounds__(128) k_visit(Box b, T* f, const T* __restrict__ mn, const T* __restrict__ mx,
                                               const T* __restrict__ air, int sweep_max,
                                               const int* __restrict__ list, unsigned nlist,
                                               const unsigned char* __restrict__ ready) {
  const unsigned q = blockIdx.x * 128u + threadIdx.x;
  if (q >= nlist || !ready[q]) return;
  int i, j, k;
  coords(b, list[q], i, j, k);
  visit<T>(b, f, mn, mx, air, sweep_max, i, j, k);
}

__global__ void __launch_bounds__(256) k_retire(unsigned char* __restrict__ pend, const int* __restrict__ list,
                                                unsigned nlist, const unsigned char* __restrict__ ready,
                                                unsigned* __restrict__ remaining) {
  const unsigned q = blockIdx.x * 256u + threadIdx.x;
  if (q >= nlist) return;
  if (ready[q]) pend[list[q]] = 0;
  else if (pend[list[q]]) atomicAdd(remaining, 1u);
}

// the rest in loop order on one thread (only after the round limit)
template <typename T>
__global__ void k_sequential(Box b, T* f, const T* mn, const T* mx, const T* air, int sweep_max,
                             const unsigned char* pend) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const long long n = b.n();
  for (long long o = 0; o < n; o++)
    if (pend[o]) {
      int i, j, k;
      coords(b, o, i, j, k);
      visit<T>(b, f, mn, mx, air, sweep_max, i, j, k);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_clip(Box b, T* __restrict__ f, const T* __restrict__ mn,
                                              const T* __restrict__ mx) {
  const long long n = b.n();
  for (long long o = blockIdx.x * 256LL + threadIdx.x; o < n; o += (long long)gridDim.x * 256) {
    int i, j, k;
    coords(b, o, i, j, k);
    const long long e = ext(b, i, j, k);
    T v = f[e];
    if (v < mn[e]) v = mn[e];
    if (v > mx[e]) v = mx[e];
    f[e] = v;
  }
}

}  // namespace ilmc
}  // namespace adz

namespace {

using namespace adz::ilmc;

constexpr int kMaxRounds = 4096;

template <typename T>
int run_ilmc(const Box& b, T* f, const T* mn, const T* mx, const T* air, int sweep_max, int min_max, char* scratch,
             int* rounds, cudaStream_t s) {
  const long long n = b.n();
  unsigned char* pend = (unsigned char*)scratch;
  int* list = (int*)(scratch + ((n + 255) & ~255LL));
  unsigned char* ready = (unsigned char*)(list + ((n + 63) & ~63LL));
  unsigned* counters = (unsigned*)(ready + ((n + 255) & ~255LL));  // [0] list length, [1] remaining
  const int gb = (int)std::min<long long>((n + 255) / 256, 148LL * 32);
  if (cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned), s) != cudaSuccess) return ADZC_ERR_CUDA;
  k_mark<T><<<gb, 256, 0, s>>>(b, f, mn, mx, pend, list, counters);
  unsigned nlist = 0;
  if (cudaMemcpyAsync(&nlist, counters, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return ADZC_ERR_CUDA;
  int r = 0;
  unsigned remaining = nlist;
  while (remaining > 0 && r < kMaxRounds) {
    const unsigned g = (nlist + 255) / 256;
    k_ready<<<g, 256, 0, s>>>(b, sweep_max, pend, list, nlist, ready);
    k_visit<T><<<(nlist + 127) / 128, 128, 0, s>>>(b, f, mn, mx, air, sweep_max, list, nlist, ready);
    if (cudaMemsetAsync(counters + 1, 0, sizeof(unsigned), s) != cudaSuccess) return ADZC_ERR_CUDA;
    k_retire<<<g, 256, 0, s>>>(pend, list, nlist, ready, counters + 1);
    if (cudaMemcpyAsync(&remaining, counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return ADZC_ERR_CUDA;
    r++;
  }
  if (remaining > 0) k_sequential<T><<<1, 1, 0, s>>>(b, f, mn, mx, air, sweep_max, pend);
  if (min_max) k_clip<T><<<gb, 256, 0, s>>>(b, f, mn, mx);
  if (rounds) *rounds = r + (remaining > 0 ? 1 : 0);
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : ADZC_ERR_CUDA;
}

}  // namespace

extern "C" int adzc_ilmc(adzc_handle* h, int prec, int ntr, void* const* f, const void* const* mn,
                         const void* const* mx, const void* air, int sweep_max, int min_max, int* rounds,
                         void* stream) {
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int niter = 0, cold = 0;
  if (!h || (prec != ADZC_REF32 && prec != ADZC_MIXED && prec != ADZC_FP64) || ntr < 0 || (ntr > 0 && (!f || !mn || !mx)) ||
      !air || sweep_max < 1 || sweep_max > 4 || adz_internal_view(h, &D, &I, &G, &niter, &cold) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  for (int q = 0; q < ntr; q++)
    if (!f[q] || !mn[q] || !mx[q]) return adz_internal_fail(ADZC_ERR_ARG);
  // single LAM domain: il..ir, jl..jr = Adz_i0..Adz_in, Adz_j0..Adz_jn (B/ILMC_LAM.F90:57-63), levels k0t..nk
  Box b{I.i0, I.in, I.j0, I.jn, I.k0t, D.nk, D.lminx, D.lminy, D.nit, D.nij};
  const long long n = b.n();
  if (n <= 0 || n > (1LL << 31) - 1) return adz_internal_fail(ADZC_ERR_SIZE);
  const size_t bytes = ((n + 255) & ~255LL) + 4 * ((n + 63) & ~63LL) + ((n + 255) & ~255LL) + 256;
  void* scratch = nullptr;
  if (adz_internal_aux(h, bytes, &scratch) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ALLOC);
  const cudaStream_t s = (cudaStream_t)stream;
  int total = 0;
  for (int q = 0; q < ntr; q++) {
    int r = 0;
    const int st = prec == ADZC_FP64
                       ? run_ilmc<double>(b, (double*)f[q], (const double*)mn[q], (const double*)mx[q],
                                          (const double*)air, sweep_max, min_max, (char*)scratch, &r, s)
                       : run_ilmc<float>(b, (float*)f[q], (const float*)mn[q], (const float*)mx[q],
                                         (const float*)air, sweep_max, min_max, (char*)scratch, &r, s);
    if (st != ADZC_OK) return adz_internal_fail(st);
    total = std::max(total, r);
  }
  if (rounds) *rounds = total;
  return ADZC_OK;
}
