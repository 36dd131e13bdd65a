// ILMC shape-preserving filter (B/ILMC_LAM.F90:16-388 with
// B/ilmc_lam_loop.inc): each point outside its [min, max] bounds moves its
// excess (or deficit) of air-mass-weighted tracer into the room its
// neighbours have, shell by shell (sweeps), then an optional clip.
//
// The reference visits the points in loop order (k, then j, then i) and
// every visit changes the point's neighbourhood, so later visits see earlier
// results.  This file keeps that order exactly and still runs in parallel.
// A visit reads and writes only the cube of radius S = sweep_max around its
// point, so a visit can depend only on earlier points within R = 2 S
// (Chebyshev).  The region is cut into tiles of one row and R columns,
// numbered (k, j, it); every earlier point within R of a
// tile's point lies in the same tile (handled in order by one thread) or in a
// tile of strictly smaller wavefront number
//     t = (2 R + 2) k + 2 j + it
// (a level below: at most R rows and one tile column away; the same level: an
// earlier row, at most one tile column away; the same row: the tile before).
// Tiles of one wavefront therefore never interact, and running the wavefronts
// in increasing t, each tile by one warp in loop order, reproduces the
// sequential result bit for bit.  Within a visit the lanes split the shell's
// loads and updates; lane 0 forms the capacity sum in the reference's order.
//
// A visit moves a neighbour only toward its bounds (it gains up to its max or
// loses down to its min) and its own point into them, so a point inside its
// bounds when the filter starts stays inside, and the reference's visit of it
// does nothing.  Candidate tiles (a point outside its bounds at the start)
// are therefore listed per wavefront once (count, scan, scatter), each wave
// launch visits only its listed tiles, and a warp loads a tile's 8 points at
// once and visits, in order, only those that were outside.
// Built with -fmad=false: the REAL arithmetic is the reference's, without
// contraction.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace adz {
namespace ilmc {


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

constexpr int kWarps = 4;   // tiles (warps) per block of k_wave
// columns per tile: R = 2 sweep_max, the narrowest width the wavefront order
// allows (a tile's visits are sequential, so narrow tiles shorten each wave)
inline int tile_width(int sweep_max) { return 2 * sweep_max; }

template <typename T>
struct Fields {
  T* f[ADZC_ILMC_MAX_TRACERS];
  const T* mn[ADZC_ILMC_MAX_TRACERS];
  const T* mx[ADZC_ILMC_MAX_TRACERS];
};

// the unclipped shells of sweeps 1..4 in the order of the reference's
// sweep_rd lists (jx, then kx, then ix; offsets di, dj, dk), concatenated;
// a shell clipped to the region is this list filtered to the region, in the
// same order (the inclusion test of a cell depends only on its offsets)
constexpr int kShellTotal = 26 + 98 + 218 + 386;
__constant__ signed char c_shell[kShellTotal][3];
__constant__ int c_shell_start[5];

// one visit by a warp: lane l owns the cells l, l + 32, ... of each shell;
// lane 0 forms the capacity sum in the reference's order (bit-exact)
template <typename T>
__device__ void visit_warp(const Box& b, T* f, const T* mn, const T* mx, const T* air, int sweep_max, int i, int j,
                           int k, int lane, T* cap, T* prod, long long* cell) {
  const long long e = ext(b, i, j, k);
  T o_shoot = rmax((T)0, f[e] - mx[e]);
  T u_shoot = rmax((T)0, mn[e] - f[e]);
  if (o_shoot == (T)0 && u_shoot == (T)0) return;
  const bool over = o_shoot > (T)0;
  for (int sweep = 1; sweep <= sweep_max; sweep++) {
    const int q0 = c_shell_start[sweep - 1], nq = c_shell_start[sweep] - q0;
    for (int q = lane; q < nq; q += 32) {
      const int ix = i + c_shell[q0 + q][0], jx = j + c_shell[q0 + q][1], kx = k + c_shell[q0 + q][2];
      const bool in = ix >= b.il && ix <= b.ir && jx >= b.jl && jx <= b.jr && kx >= b.k0 && kx <= b.nk;
      long long r = -1;
      T c = 0, pr = 0;
      if (in) {
        r = ext(b, ix, jx, kx);
        c = over ? rmax((T)0, mx[r] - f[r]) : rmax((T)0, f[r] - mn[r]);
        pr = c * air[r];
      }
      cell[q] = r;
      cap[q] = c;
      prod[q] = pr;
    }
    __syncwarp();
    T ratio = 0;
    int go = 0;
    if (lane == 0) {
      // the reference skips cells outside the region; their prod is +0 and
      // msum >= +0, so adding it leaves msum unchanged bit for bit
      T msum = 0;
#pragma unroll 8
      for (int q = 0; q < nq; q++) msum = prod[q] + msum;
      const T use = rmin(msum, (over ? o_shoot : u_shoot) * air[e]);
      if (use > (T)0) {
        if (over) {
          f[e] = rmax(f[e] - (T)(use / air[e]), mn[e]);
          o_shoot = rmax((T)0, f[e] - mx[e]);
        } else {
          f[e] = rmin(f[e] + (T)(use / air[e]), mx[e]);
          u_shoot = rmax((T)0, mn[e] - f[e]);
        }
        ratio = use / msum;
        go = 1;
      }
    }
    go = __shfl_sync(0xffffffffu, go, 0);
    ratio = __shfl_sync(0xffffffffu, ratio, 0);
    o_shoot = __shfl_sync(0xffffffffu, o_shoot, 0);
    u_shoot = __shfl_sync(0xffffffffu, u_shoot, 0);
    if (go)
      for (int q = lane; q < nq; q += 32) {
        const long long r = cell[q];
        if (r >= 0 && cap[q] > (T)0)
          f[r] = over ? rmin(f[r] + (T)(cap[q] * ratio), mx[r]) : rmax(f[r] - (T)(cap[q] * ratio), mn[r]);
      }
    __syncwarp();
  }
}

// tile id (tracer, level, tile column) and the row it has in wavefront t
__device__ __forceinline__ int tile_row(int t, int c1, int kk, int it) { return (t - c1 * kk - it) >> 1; }

// candidate tiles per wavefront.  pass 0 counts them, pass 1 lists their ids
// (order inside a wave is free: its tiles never interact)
template <typename T, int PASS>
__global__ void __launch_bounds__(256) k_candidates(Box b, Fields<T> fl, int ntr, int c1, int ntile, int tw,
                                                    int* __restrict__ count, const int* __restrict__ wstart,
                                                    int* __restrict__ list) {
  const int nz = b.nk - b.k0 + 1, ny = b.by();
  const long long n = (long long)ntr * nz * ny * ntile;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int it = (int)(g % ntile);
    const int jr = (int)((g / ntile) % ny);
    const long long rest = g / ((long long)ntile * ny);
    const int kk = (int)(rest % nz), tr = (int)(rest / nz);
    const int j = b.jl + jr, k = b.k0 + kk;
    const int i0 = b.il + it * tw, i1 = min(i0 + tw - 1, b.ir);
    const T* f = fl.f[tr];
    const T* mn = fl.mn[tr];
    const T* mx = fl.mx[tr];
    bool any = false;
    for (int i = i0; i <= i1; i++) {
      const long long e = ext(b, i, j, k);
      const T v = f[e];
      any |= (v > mx[e]) || (v < mn[e]);
    }
    if (!any) continue;
    const int t = c1 * kk + 2 * jr + it;
    if (PASS == 0) {
      atomicAdd(count + t, 1);
    } else {
      list[wstart[t] + atomicAdd(count + t, 1)] = (tr * nz + kk) * ntile + it;
    }
  }
}

// exclusive scan of the per-wave counts (one block): wstart[0..n]
__global__ void __launch_bounds__(1024) k_scan(const int* __restrict__ count, int n, int* __restrict__ wstart) {
  __shared__ int part[1024];
  const int per = (n + 1023) / 1024, a = threadIdx.x * per, z = min(a + per, n);
  int sum = 0;
  for (int q = a; q < z; q++) sum += count[q];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // inclusive Hillis-Steele
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - sum;
  for (int q = a; q < z; q++) {
    wstart[q] = run;
    run += count[q];
  }
  if (threadIdx.x == 1023) wstart[n] = part[1023];
}

// one wavefront t: a warp per listed tile, its points in loop order
template <typename T>
__global__ void __launch_bounds__(32 * kWarps) k_wave(Box b, Fields<T> fl, const T* __restrict__ air, int sweep_max,
                                                      int t, int c1, int ntile, int tw, int nshell,
                                                      const int* __restrict__ wstart, const int* __restrict__ list) {
  // dynamic shared memory: cell[kWarps][nshell] (8 B), then cap and prod
  // [kWarps][2][nshell] (T)
  extern __shared__ long long s_dyn[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long* s_cell = s_dyn + (size_t)w * nshell;
  T* s_cap = reinterpret_cast<T*>(s_dyn + (size_t)kWarps * nshell) + (size_t)w * 2 * nshell;
  T* s_prod = s_cap + nshell;
  const int nz = b.nk - b.k0 + 1;
  const int beg = wstart[t], end = wstart[t + 1];
  for (int q = beg + blockIdx.x * kWarps + w; q < end; q += gridDim.x * kWarps) {
    const int id = list[q];
    const int it = id % ntile, kk = (id / ntile) % nz, tr = id / (ntile * nz);
    const int j = b.jl + tile_row(t, c1, kk, it), k = b.k0 + kk;
    const int i0 = b.il + it * tw, i1 = min(i0 + tw - 1, b.ir);
    T* f = fl.f[tr];
    const T* mn = fl.mn[tr];
    const T* mx = fl.mx[tr];
    bool out = false;
    if (lane < tw && i0 + lane <= i1) {
      const long long e = ext(b, i0 + lane, j, k);
      const T v = f[e];
      out = (v > mx[e]) || (v < mn[e]);
    }
    unsigned todo = __ballot_sync(0xffffffffu, out);
    while (todo) {
      const int l = __ffs(todo) - 1;
      todo &= todo - 1;
      visit_warp<T>(b, f, mn, mx, air, sweep_max, i0 + l, j, k, lane, s_cap, s_prod, s_cell);
      __syncwarp();
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_clip(Box b, T* __restrict__ f, const T* __restrict__ mn,
                                              const T* __restrict__ mx) {
  const int by = b.by();
  for (long long row = blockIdx.x; row < (long long)by * (b.nk - b.k0 + 1); row += gridDim.x) {
    const int j = b.jl + (int)(row % by), k = b.k0 + (int)(row / by);
    for (int i = b.il + threadIdx.x; i <= b.ir; i += blockDim.x) {
      const long long e = ext(b, i, j, k);
      T v = f[e];
      if (v < mn[e]) v = mn[e];
      if (v > mx[e]) v = mx[e];
      f[e] = v;
    }
  }
}

}  // namespace ilmc
}  // namespace adz

namespace {

using namespace adz::ilmc;

// the reference's sweep_rd order for an unclipped point (B/ILMC_LAM.F90:118-169)
struct ShellTable {
  signed char off[kShellTotal][3];
  int start[5];
  ShellTable() {
    int n = 0;
    start[0] = 0;
    for (int sw = 1; sw <= 4; sw++) {
      for (int dj = -sw; dj <= sw; dj++)
        for (int dk = -sw; dk <= sw; dk++) {
          const bool limit_i = (dj != -sw && dj != sw) && (dk > -sw && dk < sw);
          for (int di = -sw; di <= sw; di++) {
            if (limit_i && di != -sw && di != sw) continue;
            off[n][0] = (signed char)di;
            off[n][1] = (signed char)dj;
            off[n][2] = (signed char)dk;
            n++;
          }
        }
      start[sw] = n;
    }
  }
};

// largest shell of sweeps 1..sweep_max (the reference's sweep counts)
int c_shell_len(int sweep_max) {
  int m = 0;
  for (int sw = 1; sw <= sweep_max; sw++) {
    const int side = 2 * sw + 1, inner = 2 * sw - 1;
    m = std::max(m, side * side * side - inner * inner * inner);
  }
  return m;
}

int upload_shells(cudaStream_t s) {
  static const ShellTable tab;
  if (cudaMemcpyToSymbolAsync(c_shell, tab.off, sizeof(tab.off), 0, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyToSymbolAsync(c_shell_start, tab.start, sizeof(tab.start), 0, cudaMemcpyHostToDevice, s) !=
          cudaSuccess)
    return ADZC_ERR_CUDA;
  return ADZC_OK;
}

template <typename T>
int run_ilmc(adzc_handle* h, const Box& b, int ntr, void* const* f, const void* const* mn, const void* const* mx,
             const T* air, int sweep_max, int min_max, int* waves, cudaStream_t s) {
  if (upload_shells(s) != ADZC_OK) return ADZC_ERR_CUDA;
  Fields<T> fl{};
  for (int q = 0; q < ntr; q++) {
    fl.f[q] = (T*)f[q];
    fl.mn[q] = (const T*)mn[q];
    fl.mx[q] = (const T*)mx[q];
  }
  const int R = 2 * sweep_max, c1 = 2 * R + 2;
  const int tw = tile_width(sweep_max);
  const int nz = b.nk - b.k0 + 1, ny = b.by(), ntile = (b.bx() + tw - 1) / tw;
  const int nwave = c1 * (nz - 1) + 2 * (ny - 1) + (ntile - 1) + 1;
  const long long ntiles = (long long)ntr * nz * ny * ntile;
  if ((long long)ntr * nz * ntile > (1LL << 31) - 1 || ntiles > (1LL << 31) - 1) return ADZC_ERR_SIZE;
  // scratch: count[nwave], wstart[nwave + 1], list[ntiles] (ints)
  void* scratch = nullptr;
  const size_t nint = (size_t)nwave * 2 + 1 + (size_t)ntiles;
  if (adz_internal_aux(h, nint * sizeof(int), &scratch) != ADZC_OK) return ADZC_ERR_ALLOC;
  int* count = (int*)scratch;
  int* wstart = count + nwave;
  int* list = wstart + nwave + 1;
  const int gc = (int)std::max<long long>(1, std::min<long long>((ntiles + 255) / 256, 148LL * 16));
  if (cudaMemsetAsync(count, 0, (size_t)nwave * sizeof(int), s) != cudaSuccess) return ADZC_ERR_CUDA;
  k_candidates<T, 0><<<gc, 256, 0, s>>>(b, fl, ntr, c1, ntile, tw, count, nullptr, nullptr);
  k_scan<<<1, 1024, 0, s>>>(count, nwave, wstart);
  if (cudaMemsetAsync(count, 0, (size_t)nwave * sizeof(int), s) != cudaSuccess) return ADZC_ERR_CUDA;
  k_candidates<T, 1><<<gc, 256, 0, s>>>(b, fl, ntr, c1, ntile, tw, count, wstart, list);
  const int nshell = c_shell_len(sweep_max);
  const size_t smem = (size_t)kWarps * nshell * (sizeof(long long) + 2 * sizeof(T));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<T>, 32 * kWarps, smem) != cudaSuccess ||
      per_sm < 1)
    return ADZC_ERR_CUDA;
  const int grid = per_sm * 148;
  for (int t = 0; t < nwave; t++)
    k_wave<T><<<grid, 32 * kWarps, smem, s>>>(b, fl, air, sweep_max, t, c1, ntile, tw, nshell, wstart, list);
  if (min_max) {
    const long long rows = (long long)ny * nz;
    const int gr = (int)std::min<long long>(rows, 148LL * 16);
    for (int q = 0; q < ntr; q++) k_clip<T><<<gr, 256, 0, s>>>(b, fl.f[q], fl.mn[q], fl.mx[q]);
  }
  if (waves) *waves = nwave;
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : ADZC_ERR_CUDA;
}

}  // namespace

extern "C" int adzc_ilmc(adzc_handle* h, int prec, int ntr, void* const* f, const void* const* mn,
                         const void* const* mx, const void* air, int sweep_max, int min_max, int* rounds,
                         void* stream) {
  AdzRange nvtx_range("ILMC_LAM");
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int niter = 0, cold = 0;
  if (!h || (prec != ADZC_REF32 && prec != ADZC_MIXED && prec != ADZC_FP64) || ntr < 0 ||
      ntr > ADZC_ILMC_MAX_TRACERS || (ntr > 0 && (!f || !mn || !mx)) || !air || sweep_max < 1 || sweep_max > 4 ||
      adz_internal_view(h, &D, &I, &G, &niter, &cold) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  for (int q = 0; q < ntr; q++)
    if (!f[q] || !mn[q] || !mx[q]) return adz_internal_fail(ADZC_ERR_ARG);
  if (rounds) *rounds = 0;
  if (ntr == 0) return ADZC_OK;
  // single LAM domain: il..ir, jl..jr = Adz_i0..Adz_in, Adz_j0..Adz_jn (B/ILMC_LAM.F90:57-63), levels k0t..nk
  Box b{I.i0, I.in, I.j0, I.jn, I.k0t, D.nk, D.lminx, D.lminy, D.nit, D.nij};
  if (b.n() <= 0) return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  const int st = prec == ADZC_FP64 ? run_ilmc<double>(h, b, ntr, f, mn, mx, (const double*)air, sweep_max,
                                                      min_max, rounds, s)
                                   : run_ilmc<float>(h, b, ntr, f, mn, mx, (const float*)air, sweep_max, min_max,
                                                     rounds, s);
  return st == ADZC_OK ? ADZC_OK : adz_internal_fail(st);
}
