// Bermejo-Conde mass fixer (B/Bermejo_Conde.F90:16-251, B/mass_tr_PM.F90,
// B/mass_tr_X.F90, driven as B/adz_post_tr.F90:140-236 does) for a group of
// tracers, device-resident from start to end: no host synchronisation, the
// per-tracer scalars (masses, deficit, lambda, proportion) live in device
// memory between the launches.
//
// Every mass is an FP64 sum of (field * air mass) * area mask over the core
// region, the first product in the field type as the reference forms it.
// Sums are deterministic: each block reduces a fixed slice in a fixed tree
// order, then one thread per tracer adds the block partials in index order.
// The order differs from the reference's sequential loop, so masses agree to
// rounding (about 1e-15 relative), not bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace adz {
namespace mass {

constexpr int kBlocks = 1024;  // blocks per tracer in every pass (each owns a fixed slice of rows)
constexpr int kThreads = 256;

template <typename T>
struct Tr {
  const T* p;
  T* m;
  const T* lin;
  const T* mn;
  const T* mx;
  const T* fo;
  const T* fi;
  const T* pkps;
  int weight;
  double p_exp;
};

struct State {
  double mass_p, mass_m, fo, fi, tot_p, def, wei, lambda, bc_r, prop, bc, wei_pos, wei_neg;
  int skip;
};

struct Region {
  int i0, nx, j0, ny, k0, nz;
  __host__ __device__ long long n() const { return (long long)nx * ny * nz; }
};

struct Geo {
  int lminx, lminy, nit, ni;
  long long nij;
  const double* mask;  // (ni, nj)
};

__device__ __forceinline__ long long ext(const Geo& g, int i, int j, int k) {
  return (long long)(i - g.lminx) + (long long)(j - g.lminy) * g.nit + (long long)(k - 1) * g.nij;
}

__device__ __forceinline__ double sign1(double x) { return signbit(x) ? -1.0 : 1.0; }

// weight of Bermejo_Conde.F90:87-137 (stored as T by the reference) from the
// point's values m, lin and (weight 3) pkps
template <typename T>
__device__ __forceinline__ T bc_weight_v(const Tr<T>& tr, T m, T lin, T pk, double sd) {
  const T hmlt = m - lin;
  const double hml = (double)hmlt;
  if ((int)sd != (int)sign1(hml)) return (T)0;
  const double a = fabs(hml);
  const double pw = (tr.p_exp == 1.0) ? a : pow(a, tr.p_exp);
  if (tr.weight == 1) return (T)(pw * sd);
  if (tr.weight == 2) return (T)(pw * sd * (double)(m > (T)0 ? m : (T)0));
  return (T)(pw * sd * (double)pk);
}
template <typename T>
__device__ __forceinline__ T bc_weight(const Tr<T>& tr, long long e, double sd) {
  return bc_weight_v<T>(tr, tr.m[e], tr.lin[e], tr.weight == 3 ? tr.pkps[e] : (T)0, sd);
}

// FP32 fields four cells at a time: every array and every row start of the
// region is 16-byte aligned (checked on the host), the region's x extent a
// multiple of 4, the mask's row start 16-byte aligned
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float c4(const float4& v, int u) { return u == 0 ? v.x : u == 1 ? v.y : u == 2 ? v.z : v.w; }
__device__ __forceinline__ void mask4(const double* p, double* mk) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p + 2));
  mk[0] = a.x; mk[1] = a.y; mk[2] = b.x; mk[3] = b.y;
}

enum Mode { kPMW = 0, kFlux = 1 };
constexpr int kSums = 4;  // partial sums per block

// block-wide tree sum of up to kSums values per thread (fixed order), into
// part[(q * kBlocks + block) * kSums + c]
__device__ __forceinline__ void block_sums(const double* v, int nv, int q, double* __restrict__ part) {
  __shared__ double red[kSums][kThreads];
  for (int c = 0; c < nv; c++) red[c][threadIdx.x] = v[c];
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < nv; c++) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < nv; c++) part[((long long)q * kBlocks + blockIdx.x) * kSums + c] = red[c][0];
}

// the rows (j, k) a block owns in every pass, so each sum keeps its order
__device__ __forceinline__ void block_rows(const Region& r, long long& r0, long long& r1) {
  const long long rows = (long long)r.ny * r.nz;
  const long long chunk = (rows + kBlocks - 1) / kBlocks;
  r0 = blockIdx.x * chunk;
  r1 = min(rows, r0 + chunk);
}

// cell t of a block's rows (row-major from row r0, x fastest) as (i, j, k),
// advanced kThreads cells at a time without divisions
struct Walk {
  int i, j, k;
};
__device__ __forceinline__ Walk walk_start(const Region& r, int r0, int t) {
  const int rr = t / r.nx, row = r0 + rr;
  return Walk{r.i0 + (t - rr * r.nx), r.j0 + row % r.ny, r.k0 + row / r.ny};
}
__device__ __forceinline__ void walk_step(const Region& r, Walk& w) {
  w.i += kThreads;
  while (w.i >= r.i0 + r.nx) {
    w.i -= r.nx;
    if (++w.j == r.j0 + r.ny) {
      w.j = r.j0;
      ++w.k;
    }
  }
}

// every cell of the block's rows, each thread's cells in row order.  FP64
// walks the flattened rows (no idle threads at the end of a row); FP32 takes
// one row at a time, so that the four unrolled cells of a row load together
template <typename T, typename F>
__device__ __forceinline__ void for_cells(const Region& r, long long r0, long long r1, F&& f) {
  if constexpr (sizeof(T) == 8) {
    const int nt = (int)(r1 - r0) * r.nx;
    Walk w = walk_start(r, (int)r0, threadIdx.x);
#pragma unroll 4
    for (int t = threadIdx.x; t < nt; t += kThreads, walk_step(r, w)) f(w.i, w.j, w.k);
  } else {
    for (long long row = r0; row < r1; row++) {
      const int j = r.j0 + (int)(row % r.ny), k = r.k0 + (int)(row / r.ny);
#pragma unroll 4
      for (int i = r.i0 + threadIdx.x; i < r.i0 + r.nx; i += kThreads) f(i, j, k);
    }
  }
}

// masses before the correction and the weight sums of both deficit signs in
// one read of the fields (kPMW), or the boundary fluxes (kFlux); blockIdx.y
// = tracer.  A point's weight is non-zero for one sign only, and its value is
// the one bc_weight gives for that sign.
template <typename T, int MODE, bool VEC>
__global__ void __launch_bounds__(kThreads, VEC ? 3 : 0) k_reduce(const Tr<T>* __restrict__ trs, Region r, Geo g,
                                                     const T* __restrict__ air_p, const T* __restrict__ air_m,
                                                     double* __restrict__ part) {
  const int q = blockIdx.y;
  const Tr<T> tr = trs[q];
  long long r0, r1;
  block_rows(r, r0, r1);
  double v[kSums] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (VEC && std::is_same<T, float>::value) {
    if (!(MODE == kFlux && (!tr.fo || !tr.fi)) && r.nx > 0) {
      const int nx4 = r.nx >> 2, n4 = (int)(r1 - r0) * nx4;
      for (int t = threadIdx.x; t < n4; t += kThreads) {  // the block's (row, 4-cell chunk) pairs
        const int rr = t / nx4, c = t - rr * nx4;
        const int row = (int)r0 + rr;
        const int j = r.j0 + row % r.ny, k = r.k0 + row / r.ny;
        const long long e = ext(g, r.i0, j, k) + 4 * c;
        double mk[4];
        mask4(g.mask + (r.i0 - 1) + (long long)(j - 1) * g.ni + 4 * c, mk);
        {
          if (MODE == kPMW) {
            const float4 p4 = ld4(tr.p + e), ap4 = ld4(air_p + e), m4 = ld4(tr.m + e), am4 = ld4(air_m + e);
            const float4 l4 = ld4(tr.lin + e);
            const float4 k4 = tr.weight == 3 ? ld4(tr.pkps + e) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int u = 0; u < 4; u++) {
              const float mu = c4(m4, u), lu = c4(l4, u), amu = c4(am4, u);
              const float a = c4(p4, u) * c4(ap4, u);
              const float b = mu * amu;
              v[0] += (double)a * mk[u];
              v[1] += (double)b * mk[u];
              const double sd = sign1((double)(float)(mu - lu));
              const float w = bc_weight_v<float>(tr, mu, lu, c4(k4, u), sd) * amu;
              if (sd > 0.0) v[2] += (double)w * mk[u];
              else v[3] += (double)w * mk[u];
            }
          } else {
            const float4 o4 = ld4(tr.fo + e), i4 = ld4(tr.fi + e), am4 = ld4(air_m + e);
#pragma unroll
            for (int u = 0; u < 4; u++) {
              const float a = c4(o4, u) * c4(am4, u);
              const float b = c4(i4, u) * c4(am4, u);
              v[0] += (double)a * mk[u];
              v[1] += (double)b * mk[u];
            }
          }
        }
      }
    }
  } else if (!(MODE == kFlux && (!tr.fo || !tr.fi)) && r.nx > 0) {
    for_cells<T>(r, r0, r1, [&](int i, int j, int k) {
      const long long e = ext(g, i, j, k);
      const double mk = __ldg(g.mask + (i - 1) + (long long)(j - 1) * g.ni);
      if (MODE == kPMW) {
        const T a = tr.p[e] * air_p[e];
        const T b = tr.m[e] * air_m[e];
        v[0] += (double)a * mk;
        v[1] += (double)b * mk;
        const double sd = sign1((double)(T)(tr.m[e] - tr.lin[e]));
        const T w = bc_weight<T>(tr, e, sd) * air_m[e];
        if (sd > 0.0) v[2] += (double)w * mk;
        else v[3] += (double)w * mk;
      } else {
        const T a = tr.fo[e] * air_m[e];
        const T b = tr.fi[e] * air_m[e];
        v[0] += (double)a * mk;
        v[1] += (double)b * mk;
      }
        });
  }
  block_sums(v, MODE == kPMW ? 4 : 2, q, part);
}

// almost_zero (modelutils almost_zero.F90:16-36), bit for bit
__device__ __forceinline__ bool almost_zero(double a) {
  long long bits = __double_as_longlong(a);
  if (bits < 0) bits = (long long)(0x80000000ULL - (unsigned long long)bits);
  return bits >= -1 && bits <= 1;
}

enum Stage { kAfterPMW = 0, kAfterFlux = 1, kAfterBcR = 2, kAfterBc = 3 };

// one thread per tracer: partials in index order, then the scalar formulas
template <int STAGE>
__global__ void k_finish(const double* __restrict__ part, State* __restrict__ st, int ntr,
                         double* __restrict__ deficit, double* __restrict__ diag) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ntr) return;
  double s[kSums] = {0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < kBlocks; b++)
    for (int c = 0; c < kSums; c++) s[c] += part[((long long)q * kBlocks + b) * kSums + c];
  State& S = st[q];
  if (STAGE == kAfterPMW) {
    S = State{};
    S.mass_p = s[0];
    S.mass_m = s[1];
    S.wei_pos = s[2];
    S.wei_neg = s[3];
  } else if (STAGE == kAfterFlux) {  // Bermejo_Conde.F90:70-84, then the weight sum of the deficit's sign
    S.fo = s[0];
    S.fi = s[1];
    const double bflux = S.fi - S.fo;
    const double mp = S.mass_p - deficit[q];
    S.tot_p = mp + bflux;
    S.def = S.mass_m - S.tot_p;
    S.wei = sign1(S.def) > 0.0 ? S.wei_pos : S.wei_neg;
    S.skip = almost_zero(S.wei) ? 1 : 0;
    S.lambda = S.skip ? 0.0 : S.def / S.wei;
  } else if (STAGE == kAfterBcR) {
    if (!S.skip) {
      S.bc_r = s[0];
      S.prop = S.tot_p / s[0];
    }
  } else {
    if (!S.skip) {
      S.bc = s[0];
      deficit[q] = s[0] - S.tot_p;  // Bermejo_Conde.F90:225-243
    }
    if (diag) {
      double* d = diag + 8 * q;
      d[0] = S.mass_p; d[1] = S.mass_m; d[2] = S.fo; d[3] = S.fi;
      d[4] = S.wei; d[5] = S.lambda; d[6] = S.bc_r; d[7] = S.bc;
    }
  }
}

// m - lambda w, clipped to the bound box when min_max (Bermejo_Conde.F90:163-199),
// and the mass of the corrected field in the same pass
template <typename T, bool VEC>
__global__ void __launch_bounds__(kThreads, VEC ? 3 : 0) k_correct(const Tr<T>* __restrict__ trs, const State* __restrict__ st,
                                                      Region r, Geo g, const T* __restrict__ air_m, int min_max,
                                                      double* __restrict__ part) {
  const int q = blockIdx.y;
  const Tr<T> tr = trs[q];
  const bool skip = st[q].skip;
  const double lambda = st[q].lambda, sd = sign1(st[q].def);
  long long r0, r1;
  block_rows(r, r0, r1);
  double v = 0.0;
  if constexpr (VEC && std::is_same<T, float>::value) {
    if (!skip && r.nx > 0) {
      const int nx4 = r.nx >> 2, n4 = (int)(r1 - r0) * nx4;
      for (int t = threadIdx.x; t < n4; t += kThreads) {  // the block's (row, 4-cell chunk) pairs
        const int rr = t / nx4, c = t - rr * nx4;
        const int row = (int)r0 + rr;
        const int j = r.j0 + row % r.ny, k = r.k0 + row / r.ny;
        const long long e = ext(g, r.i0, j, k) + 4 * c;
        double mk[4];
        mask4(g.mask + (r.i0 - 1) + (long long)(j - 1) * g.ni + 4 * c, mk);
        {
          const float4 m4 = ld4(tr.m + e), l4 = ld4(tr.lin + e), am4 = ld4(air_m + e);
          const float4 k4 = tr.weight == 3 ? ld4(tr.pkps + e) : make_float4(0.f, 0.f, 0.f, 0.f);
          const float4 n4 = min_max ? ld4(tr.mn + e) : make_float4(0.f, 0.f, 0.f, 0.f);
          const float4 x4 = min_max ? ld4(tr.mx + e) : make_float4(0.f, 0.f, 0.f, 0.f);
          float out[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const float mu = c4(m4, u);
            const double corr = lambda * (double)bc_weight_v<float>(tr, mu, c4(l4, u), c4(k4, u), sd);
            float nv;
            if (!min_max) {
              nv = (float)((double)mu - corr);
            } else {
              const float wrk = (float)((double)mu - corr);
              nv = wrk;
              if (corr > 0.0 && wrk < c4(n4, u)) nv = c4(n4, u);
              if (corr < 0.0 && wrk > c4(x4, u)) nv = c4(x4, u);
            }
            out[u] = nv;
            const float a = nv * c4(am4, u);
            v += (double)a * mk[u];
          }
          *reinterpret_cast<float4*>(tr.m + e) = make_float4(out[0], out[1], out[2], out[3]);
        }
      }
    }
  } else if (!skip && r.nx > 0) {
    for_cells<T>(r, r0, r1, [&](int i, int j, int k) {
      const long long e = ext(g, i, j, k);
      const double corr = lambda * (double)bc_weight<T>(tr, e, sd);
      T nv;
      if (!min_max) {
        nv = (T)((double)tr.m[e] - corr);
      } else {
        const T wrk = (T)((double)tr.m[e] - corr);
        nv = wrk;
        if (corr > 0.0 && wrk < tr.mn[e]) nv = tr.mn[e];
        if (corr < 0.0 && wrk > tr.mx[e]) nv = tr.mx[e];
      }
      tr.m[e] = nv;
      const T a = nv * air_m[e];
      v += (double)a * __ldg(g.mask + (i - 1) + (long long)(j - 1) * g.ni);
        });
  }
  block_sums(&v, 1, q, part);
}

// proportional rescale after the clipped correction (Bermejo_Conde.F90:203-222),
// and the final mass in the same pass
template <typename T, bool VEC>
__global__ void __launch_bounds__(kThreads) k_scale(const Tr<T>* __restrict__ trs, const State* __restrict__ st,
                                                    Region r, Geo g, const T* __restrict__ air_m,
                                                    double* __restrict__ part) {
  const int q = blockIdx.y;
  T* m = trs[q].m;
  const bool skip = st[q].skip;
  const double prop = st[q].prop;
  long long r0, r1;
  block_rows(r, r0, r1);
  double v = 0.0;
  if constexpr (VEC && std::is_same<T, float>::value) {
    if (!skip && r.nx > 0) {
      const int nx4 = r.nx >> 2, n4 = (int)(r1 - r0) * nx4;
      for (int t = threadIdx.x; t < n4; t += kThreads) {  // the block's (row, 4-cell chunk) pairs
        const int rr = t / nx4, c = t - rr * nx4;
        const int row = (int)r0 + rr;
        const int j = r.j0 + row % r.ny, k = r.k0 + row / r.ny;
        const long long e = ext(g, r.i0, j, k) + 4 * c;
        double mk[4];
        mask4(g.mask + (r.i0 - 1) + (long long)(j - 1) * g.ni + 4 * c, mk);
        {
          const float4 m4 = ld4(m + e), am4 = ld4(air_m + e);
          float out[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const float nv = (float)(prop * (double)c4(m4, u));
            out[u] = nv;
            const float a = nv * c4(am4, u);
            v += (double)a * mk[u];
          }
          *reinterpret_cast<float4*>(m + e) = make_float4(out[0], out[1], out[2], out[3]);
        }
      }
    }
  } else if (!skip && r.nx > 0) {
    for_cells<T>(r, r0, r1, [&](int i, int j, int k) {
      const long long e = ext(g, i, j, k);
      const T nv = (T)(prop * (double)m[e]);
      m[e] = nv;
      const T a = nv * air_m[e];
      v += (double)a * __ldg(g.mask + (i - 1) + (long long)(j - 1) * g.ni);
        });
  }
  block_sums(&v, 1, q, part);
}

}  // namespace mass
}  // namespace adz

namespace {

using namespace adz::mass;

bool al16(const void* p) { return p == nullptr || ((uintptr_t)p & 15) == 0; }

// the four-cell path applies: FP32, every array 16-byte aligned, every row
// start of the region at a multiple of 4 cells, the mask's rows likewise
template <typename T>
bool vec_ok(int ntr, const adzc_bc_tracer* in, const void* ap, const void* am, const double* mask, const Region& r,
            const Geo& g) {
  if (sizeof(T) != 4 || !al16(ap) || !al16(am) || !al16(mask)) return false;
  if (r.nx % 4 || (r.i0 - g.lminx) % 4 || g.nit % 4 || g.nij % 4 || (r.i0 - 1) % 2 || g.ni % 2) return false;
  for (int q = 0; q < ntr; q++) {
    const adzc_bc_tracer& t = in[q];
    if (!al16(t.p) || !al16(t.m) || !al16(t.lin) || !al16(t.min) || !al16(t.max) || !al16(t.fo) || !al16(t.fi) ||
        !al16(t.pkps))
      return false;
  }
  return true;
}

template <typename T>
int run_bc(int ntr, const adzc_bc_tracer* in, const void* airm_p, const void* airm_m, const double* mask,
           int min_max, double* deficit, double* diag, const Region& core, const Region& brange, const Geo& g,
           void* scratch, cudaStream_t s) {
  // scratch: tracer descriptors | states | partials
  Tr<T>* d_tr = (Tr<T>*)scratch;
  State* d_st = (State*)((char*)scratch + ((ntr * sizeof(Tr<T>) + 255) & ~size_t(255)));
  double* d_part =
      (double*)((char*)d_st + ((ntr * sizeof(State) + 255) & ~size_t(255)));
  std::vector<Tr<T>> h(ntr);
  for (int q = 0; q < ntr; q++) {
    h[q].p = (const T*)in[q].p;
    h[q].m = (T*)in[q].m;
    h[q].lin = (const T*)in[q].lin;
    h[q].mn = (const T*)in[q].min;
    h[q].mx = (const T*)in[q].max;
    h[q].fo = (const T*)in[q].fo;
    h[q].fi = (const T*)in[q].fi;
    h[q].pkps = (const T*)in[q].pkps;
    h[q].weight = in[q].weight;
    h[q].p_exp = in[q].p_exp;
  }
  if (cudaMemcpyAsync(d_tr, h.data(), ntr * sizeof(Tr<T>), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return ADZC_ERR_CUDA;
  const dim3 rg(kBlocks, ntr);
  const T* ap = (const T*)airm_p;
  const T* am = (const T*)airm_m;
  const int fb = (ntr + 127) / 128;
  Geo gm = g;
  gm.mask = mask;
  // four passes over the fields: masses and weights; fluxes (boundary only);
  // correction with its mass; rescale with the final mass (clipped only)
  const bool vc = vec_ok<T>(ntr, in, ap, am, mask, core, gm);
  const bool vb = vec_ok<T>(ntr, in, ap, am, mask, brange, gm);
  if (vc) k_reduce<T, kPMW, true><<<rg, kThreads, 0, s>>>(d_tr, core, gm, ap, am, d_part);
  else k_reduce<T, kPMW, false><<<rg, kThreads, 0, s>>>(d_tr, core, gm, ap, am, d_part);
  k_finish<kAfterPMW><<<fb, 128, 0, s>>>(d_part, d_st, ntr, deficit, diag);
  if (vb) k_reduce<T, kFlux, true><<<rg, kThreads, 0, s>>>(d_tr, brange, gm, ap, am, d_part);
  else k_reduce<T, kFlux, false><<<rg, kThreads, 0, s>>>(d_tr, brange, gm, ap, am, d_part);
  k_finish<kAfterFlux><<<fb, 128, 0, s>>>(d_part, d_st, ntr, deficit, diag);
  if (vc) k_correct<T, true><<<rg, kThreads, 0, s>>>(d_tr, d_st, core, gm, am, min_max, d_part);
  else k_correct<T, false><<<rg, kThreads, 0, s>>>(d_tr, d_st, core, gm, am, min_max, d_part);
  if (min_max) {
    k_finish<kAfterBcR><<<fb, 128, 0, s>>>(d_part, d_st, ntr, deficit, diag);
    if (vc) k_scale<T, true><<<rg, kThreads, 0, s>>>(d_tr, d_st, core, gm, am, d_part);
    else k_scale<T, false><<<rg, kThreads, 0, s>>>(d_tr, d_st, core, gm, am, d_part);
  }
  k_finish<kAfterBc><<<fb, 128, 0, s>>>(d_part, d_st, ntr, deficit, diag);
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : ADZC_ERR_CUDA;
}

}  // namespace

extern "C" int adzc_bermejo_conde(adzc_handle* h, int prec, int ntr, const adzc_bc_tracer* tracers,
                                  const void* airm_p, const void* airm_m, const double* mask, int min_max,
                                  double* deficit, double* diag, void* stream) {
  AdzRange nvtx_range("Bermejo_Conde");
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int niter = 0, cold = 0;
  if (!h || (prec != ADZC_REF32 && prec != ADZC_MIXED && prec != ADZC_FP64) || ntr < 1 || !tracers || !airm_p ||
      !airm_m || !mask || !deficit || adz_internal_view(h, &D, &I, &G, &niter, &cold) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  const bool zlf = G.bc_lam_flux == 2;
  for (int q = 0; q < ntr; q++) {
    const adzc_bc_tracer& t = tracers[q];
    if (!t.p || !t.m || !t.lin || (min_max && (!t.min || !t.max)) || t.weight < 1 || t.weight > 3 ||
        (t.weight == 3 && !t.pkps) || (!t.fo) != (!t.fi) || (zlf && t.fo) || !std::isfinite(t.p_exp))
      return adz_internal_fail(ADZC_ERR_ARG);
  }
  // core region (B/adz_post_tr.F90:146-152) and the LAM flux range (b set, all levels)
  Region core{1 + (G.west ? G.pil_w : 0), 0, 1 + (G.south ? G.pil_s : 0), 0, I.k0t, 0};
  core.nx = D.ni - (G.east ? G.pil_e : 0) - core.i0 + 1;
  core.ny = D.nj - (G.north ? G.pil_n : 0) - core.j0 + 1;
  core.nz = D.nk - I.k0t + 1;
  Region br{I.i0b, I.inb - I.i0b + 1, I.j0b, I.jnb - I.j0b + 1, 1, D.nk};
  // Zerroukat-Shipway fluxes (Adz_BC_LAM_flux 2): the fixer runs over range b,
  // every level (B/adz_post_tr.F90:145-152), and reads no flux arrays
  if (zlf) core = br;
  if (core.nx <= 0 || core.ny <= 0 || core.nz <= 0) return adz_internal_fail(ADZC_ERR_ARG);
  Geo g{D.lminx, D.lminy, D.nit, D.ni, D.nij, mask};
  const size_t ts = prec == ADZC_FP64 ? sizeof(Tr<double>) : sizeof(Tr<float>);
  const size_t bytes = ((ntr * ts + 255) & ~size_t(255)) + ((ntr * sizeof(State) + 255) & ~size_t(255)) +
                       (size_t)ntr * kBlocks * kSums * sizeof(double);
  void* scratch = nullptr;
  if (adz_internal_aux(h, bytes, &scratch) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ALLOC);
  const int st = prec == ADZC_FP64 ? run_bc<double>(ntr, tracers, airm_p, airm_m, mask, min_max, deficit, diag, core,
                                                     br, g, scratch, (cudaStream_t)stream)
                                   : run_bc<float>(ntr, tracers, airm_p, airm_m, mask, min_max, deficit, diag, core,
                                                   br, g, scratch, (cudaStream_t)stream);
  return st == ADZC_OK ? ADZC_OK : adz_internal_fail(st);
}
