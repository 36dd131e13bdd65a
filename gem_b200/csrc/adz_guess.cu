// Learned starting guess for the departure-point iteration, and the
// iteration run to a convergence tolerance.
//
// The reference starts the fixed-point iteration of adz_traject.F90 from the
// arrival point on a cold start (adz_inittraj.F90) and runs a fixed number of
// updates.  Here a small network, 82 -> 128 -> 128 -> 3 with GELU, predicts the
// departure displacement of every arrival point from the departure winds
// around it; the plain iteration then finishes from that guess to a stated
// tolerance (k_traject_tol), falling back to the plain start where the guess
// does not converge.
//
// Inference runs on the 5th-generation tensor cores: a persistent kernel, one
// CTA per SM, keeps the BF16 weights in shared memory and four 128-point
// tiles in flight.  Gather warps write the features of a tile into a BF16
// tile, one thread issues tcgen05.mma for each layer with the FP32
// accumulator in tensor memory, and epilogue warps (tcgen05.ld, bias, GELU
// with the hardware tanh on BF16 pairs, BF16) write the next layer's input
// tile in place; mbarriers hand each tile from one role to the next, so the
// gathers and epilogues of some tiles overlap the MMAs of others.  Operands
// use the K-major no-swizzle layout of 8x16-byte core matrices (K chunks of a
// row group adjacent).  Every wait is bounded: on expiry the CTA raises
// kErrTimeout in the handle's status, waits (bounded) for its MMAs in
// flight, frees its tensor memory and stops.
//
// Feature definition, network and training: oracle/guess_oracle.py restates
// them; the training kernels are in adz_train.cu.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace adz {
namespace guess {

constexpr int kFeat = ADZC_GUESS_NFEAT;  // 82
constexpr int kK1 = 96;                  // features padded to the MMA K step
constexpr int kHid = ADZC_GUESS_HIDDEN;  // 128
constexpr int kN3 = 16;                  // 3 outputs padded to the smallest N
constexpr int kRows = 128;               // arrival points per tile (MMA M)

// weight image: core-matrix layouts of W1 (128x96), W2 (128x128), W3 (16x128),
// then FP32 biases b1 (128), b2 (128), b3 (16); copied verbatim to shared memory
constexpr int kW1 = 0;
constexpr int kW2 = kW1 + kHid * kK1 * 2;
constexpr int kW3 = kW2 + kHid * kHid * 2;
constexpr int kB1 = kW3 + kN3 * kHid * 2;
constexpr int kB2 = kB1 + kHid * 4;
constexpr int kB3 = kB2 + kHid * 4;
constexpr int kNetBytes = kB3 + kN3 * 4;  // 62528
static_assert(kB1 % 16 == 0 && kB2 % 16 == 0, "biases read as 16-byte vectors");
constexpr unsigned kWaitPolls = 1u << 20;
static_assert(kNetBytes % 16 == 0, "weight image copied in 16-byte words");

// byte offset of element (r, k) of a K-major BF16 operand with row length
// KC stored as 8-row x 16-byte core matrices: the K chunks of a row group
// adjacent (LBO = 128 B), row groups KC * 16 B apart (SBO).  With this
// arrangement every byte an MMA addresses stays inside the operand whichever
// way round the two strides are read.
__host__ __device__ constexpr int core_off(int r, int k, int KC) {
  return (r >> 3) * (KC * 16) + ((k >> 3) << 7) + ((r & 7) << 4) + ((k & 7) << 1);
}

// shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1,
// no swizzle
__device__ __forceinline__ unsigned long long smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  const unsigned long long lo = ((addr >> 4) & 0x3FFFu) | (((lbo >> 4) & 0x3FFFu) << 16);
  const unsigned long long hi = ((sbo >> 4) & 0x3FFFu) | (1u << 14);
  return lo | (hi << 32);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M x N
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (unsigned n = 0; n < kWaitPolls; n++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, unsigned long long a, unsigned long long b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; q++) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// tanh form of GELU (Hendrycks and Gimpel, 2016) of a pair, packed to BF16:
// u = c h (1 + 0.044715 h^2) on an FP32 pair, the tanh by the hardware
// approximation on a BF16 pair, then h (0.5 + 0.5 tanh u) on BF16 pairs
__device__ __forceinline__ uint32_t gelu_bf16x2(float2 h) {
  const float c = 0.7978845608028654f;
  const float2 p = __ffma2_rn(__fmul2_rn(h, h), make_float2(0.044715f * c, 0.044715f * c), make_float2(c, c));
  const float2 u = __fmul2_rn(h, p);
  uint32_t t, sh, g;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(pack_bf16(u.x, u.y)));
  asm("fma.rn.bf16x2 %0, %1, %2, %2;" : "=r"(sh) : "r"(t), "r"(0x3F003F00u));  // 0.5 t + 0.5
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(g) : "r"(pack_bf16(h.x, h.y)), "r"(sh));
  return g;
}

struct Args {
  DGrid g;
  const float* uvw;  // prepared departure winds, three component planes (MIXED scratch)
  double* wpxyz;     // start positions out
  float* disp;       // optional displacement out (npts x 3)
  float* feat;       // features out (training data), npts x 82
  const long long* idx;  // features of these points only (NULL: all)
  const unsigned char* net;
  long long npts;    // points the network runs on (the coarse nodes when stride > 1)
  int k00;
  double dt;
  // coarse evaluation: the network runs on the nodes i = min(1 + stride*m, ni),
  // j likewise (nxc x nyc nodes per level, every level); stride 1 is every point
  int stride, nxc, nyc;
  // failure-path tests (adzc_guess_inject): bound of a pipeline wait in polls
  // (0: kWaitPolls), and whether each CTA's first gather withholds its signal
  unsigned polls;
  int withhold;
};

__device__ __forceinline__ long long wp_at(const DGrid& g, int i, int j, int k, int c) {
  const long long nx = g.ni + 4, ny = g.nj + 4;
  return (long long)(i + 1) + (long long)(j + 1) * nx + (long long)(k - 1) * nx * ny +
         (long long)(c - 1) * nx * ny * g.nk;
}

__device__ __forceinline__ void point_of(const DGrid& g, int k00, long long t, int& i, int& j, int& k) {
  const long long plane = (long long)g.ni * g.nj;
  i = (int)(t % g.ni) + 1;
  j = (int)((t / g.ni) % g.nj) + 1;
  k = (int)(t / plane) + k00;
}

// node t of the network's grid (every point when stride is 1)
__device__ __forceinline__ void node_of(const Args& a, long long t, int& i, int& j, int& k) {
  const long long plane = (long long)a.nxc * a.nyc;
  const int ic = (int)(t % a.nxc), jc = (int)((t / a.nxc) % a.nyc);
  i = 1 + a.stride * ic;
  j = 1 + a.stride * jc;
  i = i > a.g.ni ? a.g.ni : i;
  j = j > a.g.nj ? a.g.nj : j;
  k = (int)(t / plane) + a.k00;
}

// start point from a displacement: X - dx, Y - dy, k - dz with the level
// clipped to 1..nk
__device__ __forceinline__ void put_start(const Args& a, int i, int j, int k, float dx, float dy, float dz) {
  const DGrid& g = a.g;
  const double X = (double)(i + g.i0g - 1), Y = (double)(j + g.j0g - 1);
  double pz = (double)k - (double)dz;
  pz = pz < 1.0 ? 1.0 : (pz > (double)g.nk ? (double)g.nk : pz);
  a.wpxyz[wp_at(g, i, j, k, 1)] = X - (double)dx;
  a.wpxyz[wp_at(g, i, j, k, 2)] = Y - (double)dy;
  a.wpxyz[wp_at(g, i, j, k, 3)] = pz;
}

// bracketing nodes and weight of coordinate i along an axis of n points with
// nodes at min(1 + s m, n), m = 0..nc-1
__device__ __forceinline__ void bracket(int i, int s, int n, int nc, int& m0, float& w) {
  if (nc < 2) {
    m0 = 0;
    w = 0.0f;
    return;
  }
  m0 = (i - 1) / s;
  m0 = m0 > nc - 2 ? nc - 2 : m0;
  const int x0 = 1 + s * m0, x1r = 1 + s * (m0 + 1), x1 = x1r > n ? n : x1r;
  w = (float)(i - x0) / (float)(x1 - x0);
}

// start points of every arrival point from the network's displacements on the
// coarse nodes, bilinear in (i, j) on each level
__global__ void __launch_bounds__(256) k_guess_interp(Args a, const float* __restrict__ cd) {
  const DGrid& g = a.g;
  const long long plane = (long long)g.ni * g.nj, n = plane * (g.nk - a.k00 + 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    point_of(g, a.k00, t, i, j, k);
    int mx, my;
    float wx, wy;
    bracket(i, a.stride, g.ni, a.nxc, mx, wx);
    bracket(j, a.stride, g.nj, a.nyc, my, wy);
    const int mx1 = a.nxc > 1 ? mx + 1 : mx, my1 = a.nyc > 1 ? my + 1 : my;
    const long long base = (long long)(k - a.k00) * a.nxc * a.nyc;
    const float* c00 = cd + 3 * (base + (long long)my * a.nxc + mx);
    const float* c10 = cd + 3 * (base + (long long)my * a.nxc + mx1);
    const float* c01 = cd + 3 * (base + (long long)my1 * a.nxc + mx);
    const float* c11 = cd + 3 * (base + (long long)my1 * a.nxc + mx1);
    float d[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      // (1 - w) a + w b: exact at both nodes
      const float lo = fmaf(wx, __ldg(c10 + q), (1.0f - wx) * __ldg(c00 + q));
      const float hi = fmaf(wx, __ldg(c11 + q), (1.0f - wx) * __ldg(c01 + q));
      d[q] = fmaf(wy, hi, (1.0f - wy) * lo);
    }
    put_start(a, i, j, k, d[0], d[1], d[2]);
  }
}

// the 27 neighbourhood rows of an arrival point: row (dk, dj) starts at
// column i - 1 of plane k + dk (clamped to 1..nk), row j + dj; components are
// ncell apart.  Scales turn winds into Courant numbers.
struct Nbr {
  const float* row[9];
  long long ncell;
  float sx, sy, sz, dts;
};

__device__ __forceinline__ void neighbourhood(const DGrid& g, const float* uvw, int i, int j, int k, double dt,
                                              Nbr& nb) {
  nb.ncell = g.nij * g.nk;
  const long long r0 = (long long)(i - 1 - g.lminx) + (long long)(j - g.lminy) * g.nit;
#pragma unroll
  for (int dk = 0; dk < 3; dk++) {
    int kq = k + dk - 1;
    kq = kq < 1 ? 1 : (kq > g.nk ? g.nk : kq);
#pragma unroll
    for (int dj = 0; dj < 3; dj++) nb.row[dk * 3 + dj] = uvw + (long long)(kq - 1) * g.nij + r0 + (long long)(dj - 1) * g.nit;
  }
  const int kb = k < 1 ? 1 : (k > g.nk - 1 ? g.nk - 1 : k);
  nb.sx = (float)(dt * g.inv_hx);
  nb.sy = (float)(dt * g.inv_hy);
  nb.sz = (float)(dt * __ldg(g.odelz_m + kb));
  nb.dts = (float)(dt / ADZC_GUESS_DT_SCALE);
}

// feature q (0..81) of arrival point (i,j,k): oracle/guess_oracle.py:features
template <int Q>
__device__ __forceinline__ float feature(const Nbr& nb) {
  if (Q >= kFeat) return 0.0f;
  if (Q == kFeat - 1) return nb.dts;
  constexpr int n = Q / 3, c = Q % 3;
  constexpr int dk = n / 9, dj = (n / 3) % 3, di = n % 3;
  const float v = __ldg(nb.row[dk * 3 + dj] + c * nb.ncell + di);
  return v * (c == 0 ? nb.sx : c == 1 ? nb.sy : nb.sz);
}

template <int Q0>
__device__ __forceinline__ void features8(const Nbr& nb, float* f) {
  f[0] = feature<Q0 + 0>(nb);
  f[1] = feature<Q0 + 1>(nb);
  f[2] = feature<Q0 + 2>(nb);
  f[3] = feature<Q0 + 3>(nb);
  f[4] = feature<Q0 + 4>(nb);
  f[5] = feature<Q0 + 5>(nb);
  f[6] = feature<Q0 + 6>(nb);
  f[7] = feature<Q0 + 7>(nb);
}

// training features: FP32, all 82 per point
__global__ void __launch_bounds__(128) k_features(Args a, long long n) {
  const DGrid& g = a.g;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const long long t = a.idx ? a.idx[s] : s;
    if (t < 0 || t >= a.npts) continue;
    int i, j, k;
    point_of(g, a.k00, t, i, j, k);
    Nbr nb;
    neighbourhood(g, a.uvw, i, j, k, a.dt, nb);
    float* o = a.feat + s * kFeat;
    float f[8];
#define ADZ_FEAT_CHUNK(KC)                                    \
  features8<KC * 8>(nb, f);                                   \
  for (int q = 0; q < 8 && KC * 8 + q < kFeat; q++) o[KC * 8 + q] = f[q];
    ADZ_FEAT_CHUNK(0) ADZ_FEAT_CHUNK(1) ADZ_FEAT_CHUNK(2) ADZ_FEAT_CHUNK(3) ADZ_FEAT_CHUNK(4)
    ADZ_FEAT_CHUNK(5) ADZ_FEAT_CHUNK(6) ADZ_FEAT_CHUNK(7) ADZ_FEAT_CHUNK(8) ADZ_FEAT_CHUNK(9)
    ADZ_FEAT_CHUNK(10)
#undef ADZ_FEAT_CHUNK
  }
}

// epilogue of a hidden layer: this thread's part (NCOLS columns) of the accumulator
// columns of its row,
// + bias, GELU, BF16, written as the next layer's K-major input row
template <int NCOLS>
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem_row, const float* bias, unsigned char* A, int r,
                                                int part) {
#pragma unroll
  for (int c0 = part * NCOLS; c0 < (part + 1) * NCOLS; c0 += 32) {
    float v[32];
    tmem_ld32(tmem_row + c0, v);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint4 w;
      const int c = c0 + 8 * q;
      // the biases are 16-byte aligned in shared memory (c is a multiple of 8)
      const float4 b0 = *reinterpret_cast<const float4*>(bias + c), b1 = *reinterpret_cast<const float4*>(bias + c + 4);
      const float2 h01 = __fadd2_rn(make_float2(v[8 * q + 0], v[8 * q + 1]), make_float2(b0.x, b0.y));
      const float2 h23 = __fadd2_rn(make_float2(v[8 * q + 2], v[8 * q + 3]), make_float2(b0.z, b0.w));
      const float2 h45 = __fadd2_rn(make_float2(v[8 * q + 4], v[8 * q + 5]), make_float2(b1.x, b1.y));
      const float2 h67 = __fadd2_rn(make_float2(v[8 * q + 6], v[8 * q + 7]), make_float2(b1.z, b1.w));
      w.x = gelu_bf16x2(h01);
      w.y = gelu_bf16x2(h23);
      w.z = gelu_bf16x2(h45);
      w.w = gelu_bf16x2(h67);
      *reinterpret_cast<uint4*>(A + core_off(r, c, kHid)) = w;
    }
  }
}

// ---------------------------------------------------------------------------
// The inference kernel: one CTA per SM, warp-specialised, kStages tiles in
// flight.  Tile n (of this CTA) lives in stage n mod kStages: one 128-row
// activation tile in shared memory and one 128-column FP32 accumulator in
// tensor memory.
//   gather warps (8)     features of tile n's 128 arrival points -> tile
//                        (two threads per point, as the K chunks split);
//   MMA thread (1)       a fixed schedule: step n issues layer 3 of tile
//                        n-2, layer 2 of tile n-1 and layer 1 of tile n
//                        (8, 8 and 6 K steps), each committed to its stage's
//                        done barrier (of the six orders, the one a model of
//                        the roles' measured durations puts first);
//   epilogue groups (2 x 8 warps)  group e takes the tiles n = e mod 2 in
//                        the same order: the 3 outputs + bias of tile n-2,
//                        then bias, GELU and BF16 of the two hidden layers of
//                        tile n, written into the same tile as the next
//                        layer's input.
// So the gathers and epilogues of some tiles overlap the MMAs of others, and
// the MMA thread never polls.  Per stage barriers: full (gather -> MMA), hid
// (epilogue -> MMA, twice per tile), done (MMA commit -> epilogue, three
// times per tile) and empty (last epilogue -> gather).  Every wait is
// bounded: on expiry a role sets the CTA's abort flag and raises
// kErrTimeout; the others see the flag and stop, and the MMA thread waits
// (bounded) for its last commits before the tensor memory is freed.
constexpr int kStages = 4;
#ifndef ADZ_GUESS_GATHER_GROUPS
#define ADZ_GUESS_GATHER_GROUPS 1
#endif
// gather groups of 8 warps; group q gathers the tiles n = q mod groups
constexpr int kGatherGroups = ADZ_GUESS_GATHER_GROUPS;
#ifndef ADZ_GUESS_EPI_WARPS
#define ADZ_GUESS_EPI_WARPS 8
#endif
#ifndef ADZ_GUESS_EPI_GROUPS
#define ADZ_GUESS_EPI_GROUPS 2
#endif
// epilogue groups: group e serves the stages st = e mod groups, so that the
// groups' epilogues of different tiles run side by side.  A group's warps
// are 4 row quarters (the TMEM lanes a warp may read) times kEpiWarps / 4
// column parts of kEpiCols columns
constexpr int kEpiGroups = ADZ_GUESS_EPI_GROUPS;
constexpr int kEpiGroupWarps = ADZ_GUESS_EPI_WARPS, kEpiWarps = kEpiGroupWarps * kEpiGroups;
constexpr int kEpiCols = kHid / (kEpiGroupWarps / 4);
constexpr int kGroupWarps = 8, kGatherWarps = kGroupWarps * kGatherGroups;
static_assert(kEpiGroupWarps % 4 == 0 && kEpiCols % 32 == 0, "epilogue column parts of 32-column loads");
constexpr int kPipeThreads = (kEpiWarps + kGatherWarps + 1) * 32;
constexpr int kStageBytes = kRows * kHid * 2;
constexpr int kPA = (kNetBytes + 1023) / 1024 * 1024;
constexpr int kPBar = kPA + kStages * kStageBytes;  // full[S], hid[S], done[S], empty[S]
constexpr int kPTaddr = kPBar + 4 * kStages * 8;
constexpr int kPAbort = kPTaddr + 4;
constexpr int kPSmem = kPAbort + 4 + 1024;  // + alignment slack
constexpr int kPTmemCols = kStages * kHid;  // 512: the whole of an SM's tensor memory
static_assert(kPSmem <= 227 * 1024, "pipelined inference shared memory");

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__global__ void __launch_bounds__(kPipeThreads, 1) k_guess(Args a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const DGrid& g = a.g;
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.net);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (int q = tid; q < kNetBytes / 16; q += blockDim.x) dst[q] = src[q];
  }
  fence_async_smem();  // the weights are read by the MMAs (async proxy)
  const uint32_t s_base = smem_u32(sm);
  const uint32_t bar0 = s_base + kPBar;
  auto full_bar = [&](int st) { return bar0 + 8u * st; };
  auto hid_bar = [&](int st) { return bar0 + 8u * (kStages + st); };
  auto done_bar = [&](int st) { return bar0 + 8u * (2 * kStages + st); };
  auto empty_bar = [&](int st) { return bar0 + 8u * (3 * kStages + st); };
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + kPAbort);
  if (tid == 0) {
    for (int st = 0; st < kStages; st++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(full_bar(st)), "r"(kGroupWarps) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(hid_bar(st)), "r"(kEpiGroupWarps) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(done_bar(st)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty_bar(st)), "r"(kEpiGroupWarps) : "memory");
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_base + kPTaddr),
                 "r"(kPTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kPTaddr);
  const long long ntiles = (a.npts + kRows - 1) / kRows;
  // tiles of this CTA: blockIdx.x + n * gridDim.x, n = 0 .. nt-1, stage n % kStages
  const long long nt = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const unsigned polls = a.polls ? a.polls : kWaitPolls;
  auto wait_or_abort = [&](uint32_t bar, uint32_t parity) {
    for (unsigned q = 0; q < polls; q++) {
      if (mbar_try_wait(bar, parity)) return true;
      if (*abort_flag) return false;
    }
    return false;
  };
  auto give_up = [&]() {
    *abort_flag = 1;
    atomicOr(g.status, kErrTimeout);
  };

  if (warp >= kEpiWarps && warp < kEpiWarps + kGatherWarps) {
    // ---- gather: tile n into stage n % kStages once its previous tile left
    const int gq = (warp - kEpiWarps) / kGroupWarps;
    const int gt = tid - (kEpiWarps + gq * kGroupWarps) * 32, row = gt & (kRows - 1), half = gt / kRows;
    for (long long n = gq; n < nt; n += kGatherGroups) {
      const int st = (int)(n % kStages);
      const long long use = n / kStages;
      if (use > 0) {
        // lane 0 polls, then every lane acquires the completed phase
        const uint32_t par = (uint32_t)((use - 1) & 1);
        int ok = 0;
        if (lane == 0)
          for (unsigned q = 0; q < polls && !ok; q++) {
            ok = mbar_try_wait(empty_bar(st), par);
            if (!ok && *abort_flag) break;
          }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) ok = __all_sync(0xffffffffu, mbar_wait_bounded(empty_bar(st), par));
        if (!ok) {
          if (lane == 0 && !*abort_flag) give_up();
          break;
        }
      }
      const long long t = (blockIdx.x + n * gridDim.x) * kRows + row;
      const bool valid = t < a.npts;
      int i = 1, j = 1, k = 1;
      if (valid) node_of(a, t, i, j, k);
      Nbr nb;
      neighbourhood(g, a.uvw, i, j, k, a.dt, nb);
      unsigned char* A = sm + kPA + st * kStageBytes;
      // every load of the thread's 6 K chunks first, so that they are all in
      // flight at once, then the BF16 stores
      float f[48];
      if (half == 0) {
        features8<0>(nb, f);
        features8<8>(nb, f + 8);
        features8<16>(nb, f + 16);
        features8<24>(nb, f + 24);
        features8<32>(nb, f + 32);
        features8<40>(nb, f + 40);
      } else {
        features8<48>(nb, f);
        features8<56>(nb, f + 8);
        features8<64>(nb, f + 16);
        features8<72>(nb, f + 24);
        features8<80>(nb, f + 32);
        features8<88>(nb, f + 40);
      }
#pragma unroll
      for (int c = 0; c < 6; c++) {
        uint4 w = make_uint4(0u, 0u, 0u, 0u);
        if (valid) {
          w.x = pack_bf16(f[8 * c + 0], f[8 * c + 1]);
          w.y = pack_bf16(f[8 * c + 2], f[8 * c + 3]);
          w.z = pack_bf16(f[8 * c + 4], f[8 * c + 5]);
          w.w = pack_bf16(f[8 * c + 6], f[8 * c + 7]);
        }
        *reinterpret_cast<uint4*>(A + core_off(row, (half * 6 + c) * 8, kHid)) = w;
      }
      fence_async_smem();
      __syncwarp();
      if (lane == 0 && !(a.withhold && n == 0)) mbar_arrive(full_bar(st));
    }
  } else if (warp == kEpiWarps + kGatherWarps) {
    // ---- MMA issue, one thread, on a fixed schedule: step n issues layer
    // 3 of tile n-2, layer 2 of tile n-1, then layer 1 of tile n, each once
    // its input is ready (one bounded wait each)
    if (lane == 0) {
      const uint32_t id_hid = instr_desc(kRows, kHid), id_out = instr_desc(kRows, kN3);
      // descriptors of K step 0; a K step of 16 is 256 bytes further (16 in
      // the descriptor's address field)
      const unsigned long long dw1 = smem_desc(s_base + kW1, 128, kK1 * 16);
      const unsigned long long dw2 = smem_desc(s_base + kW2, 128, kHid * 16);
      const unsigned long long dw3 = smem_desc(s_base + kW3, 128, kHid * 16);
      const unsigned long long da0 = smem_desc(s_base + kPA, 128, kHid * 16);
      unsigned commits[kStages] = {};
      bool ok = true;
      auto issue = [&](long long n, int layer) {
        const int st = (int)(n % kStages);
        const long long u = n / kStages;  // earlier tiles of this stage
        const bool ready = layer == 0 ? wait_or_abort(full_bar(st), (uint32_t)(u & 1))
                                      : wait_or_abort(hid_bar(st), (uint32_t)(layer - 1));
        if (!ready) return false;
        fence_after();
        const unsigned long long da = da0 + (unsigned long long)((st * kStageBytes) >> 4);
        const unsigned long long db = layer == 0 ? dw1 : layer == 1 ? dw2 : dw3;
        const uint32_t idesc = layer == 2 ? id_out : id_hid, acc = tmem + st * kHid;
        const int ksteps = layer == 0 ? kK1 / 16 : kHid / 16;
        for (int q = 0; q < ksteps; q++) mma_bf16(acc, da + 16ull * q, db + 16ull * q, idesc, q > 0 ? 1u : 0u);
        mma_commit(done_bar(st));
        commits[st]++;
        return true;
      };
      for (long long n = 0; n < nt + 2 && ok; n++) {
        if (n >= 2) ok = issue(n - 2, 2);
        if (ok && n >= 1 && n - 1 < nt) ok = issue(n - 1, 1);
        if (ok && n < nt) ok = issue(n, 0);
      }
      if (!ok) {
        if (!*abort_flag) give_up();
        // let the MMAs in flight finish before the memory is freed
        for (int st = 0; st < kStages; st++)
          if (commits[st] > 0) mbar_wait_bounded(done_bar(st), (commits[st] - 1) & 1u);
      }
    }
  } else {
    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows),
    // column part w / 4 of each hidden layer.  Group e takes the tiles
    // n = e mod kEpiGroups in the MMA thread's order: the outputs of tile
    // n-2, then the first and the second hidden layer of tile n.
    const int egrp = warp / kEpiGroupWarps, ew = warp % kEpiGroupWarps;
    const int quarter = ew & 3, part = ew >> 2, row = quarter * 32 + lane;
    const float* b1 = reinterpret_cast<const float*>(sm + kB1);
    const float* b2 = reinterpret_cast<const float*>(sm + kB2);
    const float* b3 = reinterpret_cast<const float*>(sm + kB3);
    // wait for commit c (0, 1, 2: layer) of tile n's stage; every lane acquires
    auto await = [&](long long n, int c) {
      const uint32_t par = (uint32_t)((3 * (n / kStages) + c) & 1);
      const bool ok = __all_sync(0xffffffffu, wait_or_abort(done_bar((int)(n % kStages)), par));
      if (ok) fence_after();
      return ok;
    };
    auto hidden = [&](long long n, int layer) {
      const int st = (int)(n % kStages);
      const uint32_t taddr = tmem + st * kHid + ((uint32_t)(quarter * 32) << 16);
      hidden_epilogue<kEpiCols>(taddr, layer == 0 ? b1 : b2, sm + kPA + st * kStageBytes, row, part);
      fence_async_smem();
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(hid_bar(st));
    };
    auto outputs = [&](long long n) {
      const int st = (int)(n % kStages);
      if (part == 0) {
        float v[32];
        tmem_ld32(tmem + st * kHid + ((uint32_t)(quarter * 32) << 16), v);  // the first 3 columns are the outputs
        const long long t = (blockIdx.x + n * gridDim.x) * kRows + row;
        if (t < a.npts) {
          const float y0 = v[0] + b3[0], y1 = v[1] + b3[1], y2 = v[2] + b3[2];
          if (a.disp) {
            a.disp[3 * t + 0] = y0;
            a.disp[3 * t + 1] = y1;
            a.disp[3 * t + 2] = y2;
          }
          if (a.wpxyz) {
            int i, j, k;
            node_of(a, t, i, j, k);
            put_start(a, i, j, k, y0, y1, y2);
          }
        }
      }
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(empty_bar(st));
    };
    bool ok = true;
    for (long long n = egrp; n - 2 < nt && ok; n += kEpiGroups) {
      if (n >= 2) {
        if (!(ok = await(n - 2, 2))) break;
        outputs(n - 2);
      }
      if (n < nt) {
        if (!(ok = await(n, 0))) break;
        hidden(n, 0);
        if (!(ok = await(n, 1))) break;
        hidden(n, 1);
      }
    }
    if (!ok && lane == 0 && !*abort_flag) give_up();
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPTmemCols) : "memory");
}

// launch of the inference kernel: one CTA per SM
inline cudaError_t launch_guess(const Args& a, cudaStream_t s) {
  if (a.npts <= 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_guess, cudaFuncAttributeMaxDynamicSharedMemorySize, kPSmem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long ntiles = (a.npts + kRows - 1) / kRows;
  k_guess<<<(int)std::min<long long>(ntiles, sms), kPipeThreads, kPSmem, s>>>(a);
  return cudaGetLastError();
}

// BF16 round to nearest even on the host
inline uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x7FFFFFu)) return (uint16_t)((u >> 16) | 0x40);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

}  // namespace guess
}  // namespace adz

struct adzc_guess {
  unsigned char* d_net = nullptr;
  int device = 0;
  unsigned polls = 0;  // adzc_guess_inject
  int withhold = 0;
};

namespace {

using adz::guess::Args;

int check_handle(adzc_handle* h, adz::DGrid* dg, adzc_info* info, adzc_grid* gr) {
  int niter = 0, cold = 0;
  return adz_internal_view(h, dg, info, gr, &niter, &cold);
}

// departure winds of the MIXED path into the handle's scratch
int prepare_mixed(adzc_handle* h, const adz::DGrid& D, const void* uu, const void* vv, const void* ww, void** uvw,
                  void** wdep, cudaStream_t s) {
  if (adz_internal_scratch(h, ADZC_MIXED, uvw, wdep) != ADZC_OK) return ADZC_ERR_ALLOC;
  if (adz::launch_prepare<adz::kMixed>(D, uu, vv, ww, *uvw, s) != cudaSuccess) return ADZC_ERR_CUDA;
  return ADZC_OK;
}

int k00_of(const adz::DGrid& D) { return (D.k0 > 1) ? 1 : D.k0m; }  // B/adz_traject.F90:63-64

}  // namespace

extern "C" int adzc_guess_create(const float* const* params, adzc_guess** out) {
  using namespace adz::guess;
  if (!params || !out) return adz_internal_fail(ADZC_ERR_ARG);
  for (int q = 0; q < 6; q++)
    if (!params[q]) return adz_internal_fail(ADZC_ERR_ARG);
  std::vector<unsigned char> img(kNetBytes, 0);
  auto put = [&](int base, int kcap, const float* W, int n, int kdim) {  // rows beyond n and K beyond kdim stay 0
    for (int r = 0; r < n; r++)
      for (int k = 0; k < kdim; k++) {
        const uint16_t b = bf16_bits(W[(size_t)r * kdim + k]);
        std::memcpy(&img[base + core_off(r, k, kcap)], &b, 2);
      }
  };
  put(kW1, kK1, params[0], kHid, kFeat);
  put(kW2, kHid, params[2], kHid, kHid);
  put(kW3, kHid, params[4], ADZC_GUESS_NOUT, kHid);
  std::memcpy(&img[kB1], params[1], kHid * 4);
  std::memcpy(&img[kB2], params[3], kHid * 4);
  std::memcpy(&img[kB3], params[5], ADZC_GUESS_NOUT * 4);
  auto* net = new (std::nothrow) adzc_guess();
  if (!net) return adz_internal_fail(ADZC_ERR_ALLOC);
  cudaGetDevice(&net->device);
  if (cudaMalloc(&net->d_net, kNetBytes) != cudaSuccess) {
    delete net;
    return adz_internal_fail(ADZC_ERR_ALLOC);
  }
  if (cudaMemcpy(net->d_net, img.data(), kNetBytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(net->d_net);
    delete net;
    return adz_internal_fail(ADZC_ERR_CUDA);
  }
  *out = net;
  return ADZC_OK;
}

extern "C" int adzc_guess_inject(adzc_guess* net, int what, long long value) {
  if (!net || value < 0) return adz_internal_fail(ADZC_ERR_ARG);
  if (what == ADZC_INJECT_SPINS && value <= 0x7fffffffLL) {
    net->polls = (unsigned)value;
  } else if (what == ADZC_INJECT_WITHHOLD && value <= 1) {
    net->withhold = (int)value;
  } else {
    return adz_internal_fail(ADZC_ERR_ARG);
  }
  return ADZC_OK;
}

extern "C" int adzc_guess_destroy(adzc_guess* net) {
  if (!net) return ADZC_OK;
  cudaFree(net->d_net);
  delete net;
  return ADZC_OK;
}

extern "C" long long adzc_guess_npoints(adzc_handle* h) {
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  if (!h || check_handle(h, &D, &I, &G) != ADZC_OK) return -1;
  return (long long)D.ni * D.nj * (D.nk - k00_of(D) + 1);
}

extern "C" int adzc_guess_features(adzc_handle* h, double dt, const void* uu_ext, const void* vv_ext,
                                   const void* ww_ext, const long long* idx, long long n, float* features,
                                   void* stream) {
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  if (!h || !uu_ext || !vv_ext || !ww_ext || !features || n < 0 || !std::isfinite(dt) ||
      check_handle(h, &D, &I, &G) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  void *uvw = nullptr, *wdep = nullptr;
  int st = prepare_mixed(h, D, uu_ext, vv_ext, ww_ext, &uvw, &wdep, s);
  if (st != ADZC_OK) return adz_internal_fail(st);
  Args a{};
  a.g = D;
  a.uvw = (const float*)uvw;
  a.feat = features;
  a.idx = idx;
  a.k00 = k00_of(D);
  a.npts = (long long)D.ni * D.nj * (D.nk - a.k00 + 1);
  a.dt = dt;
  if (!idx) n = a.npts;
  if (n == 0) return ADZC_OK;
  const long long blocks = std::min<long long>((n + 127) / 128, 148LL * 64);
  adz::guess::k_features<<<(int)blocks, 128, 0, s>>>(a, n);
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

extern "C" int adzc_guess_apply(adzc_handle* h, const adzc_guess* net, double dt, const void* uu_ext,
                                const void* vv_ext, const void* ww_ext, double* wpxyz, float* disp, void* stream) {
  AdzRange nvtx_range("adz guess");
  using namespace adz::guess;
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  if (!h || !net || !uu_ext || !vv_ext || !ww_ext || (!wpxyz && !disp) || !std::isfinite(dt) ||
      check_handle(h, &D, &I, &G) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  void *uvw = nullptr, *wdep = nullptr;
  int st = prepare_mixed(h, D, uu_ext, vv_ext, ww_ext, &uvw, &wdep, s);
  if (st != ADZC_OK) return adz_internal_fail(st);
  Args a{};
  a.g = D;
  a.uvw = (const float*)uvw;
  a.wpxyz = wpxyz;
  a.disp = disp;
  a.net = net->d_net;
  a.polls = net->polls;
  a.withhold = net->withhold;
  a.k00 = k00_of(D);
  a.npts = (long long)D.ni * D.nj * (D.nk - a.k00 + 1);
  a.dt = dt;
  a.stride = 1;
  a.nxc = D.ni;
  a.nyc = D.nj;
  return launch_guess(a, s) == cudaSuccess ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

extern "C" int adzc_guess_apply_coarse(adzc_handle* h, const adzc_guess* net, double dt, const void* uu_ext,
                                       const void* vv_ext, const void* ww_ext, int stride, double* wpxyz,
                                       void* stream) {
  AdzRange nvtx_range("adz guess coarse");
  using namespace adz::guess;
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  if (!h || !net || !uu_ext || !vv_ext || !ww_ext || !wpxyz || stride < 1 || stride > ADZC_GUESS_MAX_STRIDE ||
      !std::isfinite(dt) || check_handle(h, &D, &I, &G) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  if (stride == 1) return adzc_guess_apply(h, net, dt, uu_ext, vv_ext, ww_ext, wpxyz, nullptr, stream);
  const cudaStream_t s = (cudaStream_t)stream;
  Args a{};
  a.g = D;
  a.net = net->d_net;
  a.polls = net->polls;
  a.withhold = net->withhold;
  a.k00 = k00_of(D);
  a.dt = dt;
  a.stride = stride;
  a.nxc = (D.ni - 1 + stride - 1) / stride + 1;
  a.nyc = (D.nj - 1 + stride - 1) / stride + 1;
  const long long nkp = D.nk - a.k00 + 1;
  a.npts = (long long)a.nxc * a.nyc * nkp;
  if (nkp <= 0) return ADZC_OK;
  // the coarse displacements live in the handle's auxiliary buffer
  void* cd = nullptr;
  if (adz_internal_aux(h, (size_t)a.npts * 3 * sizeof(float), &cd) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ALLOC);
  void *uvw = nullptr, *wdep = nullptr;
  int st = prepare_mixed(h, D, uu_ext, vv_ext, ww_ext, &uvw, &wdep, s);
  if (st != ADZC_OK) return adz_internal_fail(st);
  a.uvw = (const float*)uvw;
  a.disp = (float*)cd;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (launch_guess(a, s) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  a.wpxyz = wpxyz;
  const long long n = (long long)D.ni * D.nj * nkp;
  const long long blocks = std::min<long long>((n + 255) / 256, (long long)sms * 16);
  k_guess_interp<<<(int)blocks, 256, 0, s>>>(a, (const float*)cd);
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

extern "C" int adzc_traject_guess(adzc_handle* h, const adzc_guess* net, int stride, double dt, double tol,
                                  int maxit, const void* uu_ext, const void* vv_ext, const void* ww_ext,
                                  const void* ut0, const void* vt0, const void* zdt0, double* wpxyz,
                                  unsigned char* iters, unsigned long long* stats, void* stream) {
  AdzRange nvtx_range("adz_traject guess");
  using namespace adz::guess;
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  if (!h || !net || !uu_ext || !vv_ext || !ww_ext || !ut0 || !vt0 || !zdt0 || !wpxyz || stride < 1 ||
      stride > ADZC_GUESS_MAX_STRIDE || maxit < 1 || maxit > 127 || !(tol >= 0.0) || !std::isfinite(dt) ||
      check_handle(h, &D, &I, &G) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  Args a{};
  a.g = D;
  a.net = net->d_net;
  a.polls = net->polls;
  a.withhold = net->withhold;
  a.k00 = k00_of(D);
  a.dt = dt;
  a.stride = stride;
  a.nxc = (D.ni - 1 + stride - 1) / stride + 1;
  a.nyc = (D.nj - 1 + stride - 1) / stride + 1;
  const long long nkp = D.nk - a.k00 + 1;
  a.npts = (long long)a.nxc * a.nyc * nkp;
  if (nkp <= 0) return ADZC_OK;
  void* cd = nullptr;
  if (adz_internal_aux(h, (size_t)a.npts * 3 * sizeof(float), &cd) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ALLOC);
  // the departure winds are prepared once, for the network and the iteration
  void *uvw = nullptr, *wdep = nullptr;
  int st = prepare_mixed(h, D, uu_ext, vv_ext, ww_ext, &uvw, &wdep, s);
  if (st != ADZC_OK) return adz_internal_fail(st);
  a.uvw = (const float*)uvw;
  a.disp = (float*)cd;
  if (launch_guess(a, s) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  adz::TrajArgs t{};
  t.uvw_d = uvw;
  t.ut0 = ut0;
  t.vt0 = vt0;
  t.zdt0 = zdt0;
  t.wpxyz = wpxyz;
  t.wdep = wdep;
  t.niter = maxit;
  t.cold = 0;
  t.k00 = a.k00;
  t.dt = adz_internal_dt_split(G, dt);
  const adz::GuessStart gs{(const float*)cd, stride, a.nxc, a.nyc};
  if (adz::launch_traject_tol<adz::kMixed>(D, t, tol, maxit, iters, stats, s, gs) != cudaSuccess)
    return adz_internal_fail(ADZC_ERR_CUDA);
  adz_internal_record_positions(h, ADZC_MIXED, wpxyz, zdt0, t.dt);
  return ADZC_OK;
}

extern "C" int adzc_traject_tol(adzc_handle* h, int prec, double dt, double tol, int maxit, int start,
                                const void* uu_ext, const void* vv_ext, const void* ww_ext, const void* ut0,
                                const void* vt0, const void* zdt0, double* wpxyz, unsigned char* iters,
                                unsigned long long* stats, void* stream) {
  AdzRange nvtx_range("adz_traject tol");
  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  if (!h || (prec != ADZC_MIXED && prec != ADZC_FP64) || !uu_ext || !vv_ext || !ww_ext || !ut0 || !vt0 || !zdt0 ||
      !wpxyz || maxit < 1 || maxit > 127 || !(tol >= 0.0) || (start != 0 && start != 1) || !std::isfinite(dt) ||
      check_handle(h, &D, &I, &G) != ADZC_OK)
    return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  void *uvw = nullptr, *wdep = nullptr;
  if (adz_internal_scratch(h, prec, &uvw, &wdep) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ALLOC);
  const cudaError_t pe = prec == ADZC_FP64 ? adz::launch_prepare<adz::kFp64>(D, uu_ext, vv_ext, ww_ext, uvw, s)
                                           : adz::launch_prepare<adz::kMixed>(D, uu_ext, vv_ext, ww_ext, uvw, s);
  if (pe != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  adz::TrajArgs a{};
  a.uvw_d = uvw;
  a.ut0 = ut0;
  a.vt0 = vt0;
  a.zdt0 = zdt0;
  a.wpxyz = wpxyz;
  a.wdep = wdep;
  a.niter = maxit;
  a.cold = start == 0 ? 1 : 0;
  a.k00 = k00_of(D);
  a.dt = adz_internal_dt_split(G, dt);
  const cudaError_t te = prec == ADZC_FP64 ? adz::launch_traject_tol<adz::kFp64>(D, a, tol, maxit, iters, stats, s)
                                           : adz::launch_traject_tol<adz::kMixed>(D, a, tol, maxit, iters, stats, s);
  if (te != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  adz_internal_record_positions(h, prec, wpxyz, zdt0, a.dt);
  return ADZC_OK;
}
