// Halo strips of a tile: pack into one send buffer, unpack from one receive
// buffer, one launch each, for the rpn_comm_xch_halo calls of the path
// (B/dynstep.F90:52-53, B/adz_interp_hlt.F90:87-88, B/adz_traject.F90:121-122).
//
// Work is split into slabs: one strip (neighbour slot) of one plane of one
// array, w x h elements with i fastest, the same order as the buffer.  Blocks
// stride over slabs and threads over a slab's elements, so the buffer side is
// written (or read) contiguously and the array side row by row.
#include <cuda_runtime.h>

#include "../../include/adz_b200.h"
#include "adz_internal.h"

namespace adz {
namespace halo {

constexpr int kThreads = 256;

struct Args {
  void* arr[ADZC_HALO_MAX_ARRAYS];
  long long seg[9];     // element offset of each present segment in the buffer
  int x0[9], y0[9];     // first i, j of the strip in the array (send or receive side)
  int w[9], h[9];
  int slot[9];          // present slots in buffer order
  int nseg, narrays;
  long long nplanes, row, plane;  // array strides in elements
  int minx, miny;
};

template <typename T, bool PACK>
__global__ void __launch_bounds__(kThreads) k_halo(Args a, T* __restrict__ buf) {
  const long long per_seg = (long long)a.narrays * a.nplanes;
  const long long nslab = per_seg * a.nseg;
  for (long long s = blockIdx.x; s < nslab; s += gridDim.x) {
    const int q = a.slot[s / per_seg];
    const long long r = s % per_seg;
    const int arr = (int)(r / a.nplanes);
    const long long p = r % a.nplanes;
    const int w = a.w[q], n = w * a.h[q];
    T* __restrict__ b = buf + a.seg[q] + r * n;
    T* __restrict__ f = (T*)a.arr[arr] + p * a.plane + (long long)(a.x0[q] - a.minx) + (long long)(a.y0[q] - a.miny) * a.row;
    for (int u = threadIdx.x; u < n; u += kThreads) {
      const int y = u / w, x = u - y * w;
      if (PACK) b[u] = f[x + (long long)y * a.row];
      else f[x + (long long)y * a.row] = b[u];
    }
  }
}

bool valid(const adzc_halo* x, int narrays) {
  return x && narrays >= 1 && narrays <= ADZC_HALO_MAX_ARRAYS && (x->elem == 4 || x->elem == 8) && x->ni >= 1 &&
         x->nj >= 1 && x->nplanes >= 1 && x->hx >= 1 && x->hy >= 1 && x->hx <= x->ni && x->hy <= x->nj &&
         x->minx <= 1 - x->hx && x->maxx >= x->ni + x->hx && x->miny <= 1 - x->hy && x->maxy >= x->nj + x->hy;
}

// strip of slot q along one axis: send (interior) or receive (halo) start, width
void strip(int d, int n, int hw, bool send, int& s0, int& len) {
  if (d == 0) {
    s0 = 1;
    len = n;
  } else if (d < 0) {
    s0 = send ? 1 : 1 - hw;
    len = hw;
  } else {
    s0 = send ? n - hw + 1 : n + 1;
    len = hw;
  }
}

// element offsets of the segments (absent slots: empty) and the total
void layout(const adzc_halo* x, int narrays, long long* off) {
  long long o = 0;
  for (int q = 0; q < 9; q++) {
    off[q] = o;
    if (q == 4 || !x->nbr[q]) continue;
    int s0, w, h;
    strip(q % 3 - 1, x->ni, x->hx, true, s0, w);
    strip(q / 3 - 1, x->nj, x->hy, true, s0, h);
    o += (long long)w * h * x->nplanes * narrays;
  }
  off[9] = o;
}

int run(const adzc_halo* x, int narrays, const void* const* arrays, void* buf, bool pack, void* stream) {
  if (!valid(x, narrays) || !arrays || !buf) return adz_internal_fail(ADZC_ERR_ARG);
  Args a{};
  long long off[10];
  layout(x, narrays, off);
  if (off[9] == 0) return ADZC_OK;  // no neighbour
  for (int k = 0; k < narrays; k++) {
    if (!arrays[k]) return adz_internal_fail(ADZC_ERR_ARG);
    a.arr[k] = const_cast<void*>(arrays[k]);
  }
  a.narrays = narrays;
  a.nplanes = x->nplanes;
  a.row = (long long)x->maxx - x->minx + 1;
  a.plane = a.row * ((long long)x->maxy - x->miny + 1);
  a.minx = x->minx;
  a.miny = x->miny;
  for (int q = 0; q < 9; q++) {
    if (q == 4 || !x->nbr[q]) continue;
    strip(q % 3 - 1, x->ni, x->hx, pack, a.x0[q], a.w[q]);
    strip(q / 3 - 1, x->nj, x->hy, pack, a.y0[q], a.h[q]);
    a.seg[q] = off[q];
    a.slot[a.nseg++] = q;
  }
  const long long nslab = (long long)a.nseg * narrays * x->nplanes;
  const int grid = (int)(nslab < 148LL * 16 ? nslab : 148LL * 16);
  const cudaStream_t s = (cudaStream_t)stream;
  if (x->elem == 4) {
    if (pack) k_halo<float, true><<<grid, kThreads, 0, s>>>(a, (float*)buf);
    else k_halo<float, false><<<grid, kThreads, 0, s>>>(a, (float*)buf);
  } else {
    if (pack) k_halo<double, true><<<grid, kThreads, 0, s>>>(a, (double*)buf);
    else k_halo<double, false><<<grid, kThreads, 0, s>>>(a, (double*)buf);
  }
  return cudaGetLastError() == cudaSuccess ? ADZC_OK : adz_internal_fail(ADZC_ERR_CUDA);
}

}  // namespace halo
}  // namespace adz

extern "C" int adzc_halo_layout(const adzc_halo* x, int narrays, long long* off) {
  if (!adz::halo::valid(x, narrays) || !off) return adz_internal_fail(ADZC_ERR_ARG);
  adz::halo::layout(x, narrays, off);
  for (int q = 0; q < 10; q++) off[q] *= x->elem;
  return ADZC_OK;
}

extern "C" int adzc_halo_pack(const adzc_halo* x, int narrays, const void* const* arrays, void* sendbuf,
                              void* stream) {
  AdzRange nvtx_range("rpn_comm_xch_halo pack");
  return adz::halo::run(x, narrays, arrays, sendbuf, true, stream);
}

extern "C" int adzc_halo_unpack(const adzc_halo* x, int narrays, void* const* arrays, const void* recvbuf,
                                void* stream) {
  AdzRange nvtx_range("rpn_comm_xch_halo unpack");
  return adz::halo::run(x, narrays, (const void* const*)arrays, const_cast<void*>(recvbuf), false, stream);
}
