// adzc_step_noalloc: one advection step that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they step the model: a host model
// whose device memory is handed out by its own pool (an OpenACC runtime, a
// framework's caching allocator that reserved the GPU at start-up), one that
// runs under a device-memory budget fixed at start-up, or one that must not
// let the step synchronise the device (cudaMalloc and cudaFree can).  The
// regular path, adzc_traject, allocates its departure-wind scratch with
// cudaMalloc on first use.  This entry point keeps that scratch (departure
// winds and the departure vertical wind) in a file-scope static device array
// of ADZC_NOALLOC_SCRATCH_BYTES instead; every GPU that loads the library
// holds the array until the process exits.
//
// The array's name is a host-side stand-in in host code, not a device
// address.  Its device address is resolved here with cudaGetSymbolAddress,
// once per device context, with that device current, by the first call made
// in the context; that first call should therefore come before any stream
// capture.  A new primary context (after cudaDeviceReset) reloads the module
// and moves the array, so the address is resolved again there.
// All calls share the one array and it keeps the last call's contents, so
// calls that overlap on the GPU (two streams, two threads, two handles) race.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <mutex>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[ADZC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};
unsigned long long g_ctx_id[kMaxDevices] = {};

// unique id of the calling thread's current context (0: none yet, or not
// available), through the runtime's entry-point lookup (no link to libcuda)
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent)p;
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetId)p;
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// device address of the static array in the current device's context: looked
// up once per context (the array moves when a reset gives the device a new
// primary context); without a context id it is looked up on every call
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ADZC_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  const unsigned long long id = current_context_id();
  if (!g_addr[dev] || id == 0 || id != g_ctx_id[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ADZC_ERR_CUDA;
    g_addr[dev] = p;
    g_ctx_id[dev] = current_context_id();  // the lookup created the context if there was none
  }
  *out = g_addr[dev];
  return ADZC_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

cudaError_t prepare(int prec, const adz::DGrid& g, const void* uu, const void* vv, const void* ww, void* o,
                    cudaStream_t s) {
  if (prec == ADZC_REF32) return adz::launch_prepare<adz::kRef32>(g, uu, vv, ww, o, s);
  if (prec == ADZC_FP64) return adz::launch_prepare<adz::kFp64>(g, uu, vv, ww, o, s);
  return adz::launch_prepare<adz::kMixed>(g, uu, vv, ww, o, s);
}
cudaError_t traject(int prec, const adz::DGrid& g, const adz::TrajArgs& a, cudaStream_t s) {
  if (prec == ADZC_REF32) return adz::launch_traject<adz::kRef32>(g, a, s);
  if (prec == ADZC_FP64) return adz::launch_traject<adz::kFp64>(g, a, s);
  return adz::launch_traject<adz::kMixed>(g, a, s);
}
cudaError_t tricub(int prec, const adz::DGrid& g, int set, int i0, int nx, int j0, int ny, int k0, int nz,
                   const adz::SetArgs& a, const adz::FieldPtrs& fp, cudaStream_t s) {
  if (prec == ADZC_REF32) return adz::launch_tricub_set<adz::kRef32>(g, set, i0, nx, j0, ny, k0, nz, a, fp, s);
  if (prec == ADZC_FP64) return adz::launch_tricub_set<adz::kFp64>(g, set, i0, nx, j0, ny, k0, nz, a, fp, s);
  return adz::launch_tricub_set<adz::kMixed>(g, set, i0, nx, j0, ny, k0, nz, a, fp, s);
}

}  // namespace

extern "C" int adzc_step_noalloc(adzc_handle* h, int prec, double dt, int niter, const void* uu_ext,
                                 const void* vv_ext, const void* ww_ext, const void* ut0, const void* vt0,
                                 const void* zdt0, void* pxyzm, double* wpxyz, const int* nfields,
                                 const void* const* srcs, void* const* dsts, const int* mono, void* stream) {
  AdzRange nvtx_range("ADZ_MAIN");
  if (!h || (prec != ADZC_REF32 && prec != ADZC_FP64 && prec != ADZC_MIXED) || !uu_ext || !vv_ext || !ww_ext ||
      !ut0 || !vt0 || !zdt0 || !wpxyz || (prec == ADZC_REF32 && !pxyzm) || !nfields || !std::isfinite(dt))
    return adz_internal_fail(ADZC_ERR_ARG);
  long long total = 0;
  for (int s = 0; s < 4; s++) {
    if (nfields[s] < 0) return adz_internal_fail(ADZC_ERR_ARG);
    total += nfields[s];
  }
  if (total > INT_MAX / 2) return adz_internal_fail(ADZC_ERR_ARG);
  const int ntot = (int)total;
  if (ntot > 0 && (!srcs || !dsts)) return adz_internal_fail(ADZC_ERR_ARG);
  for (int f = 0; f < ntot; f++)
    if (!srcs[f] || !dsts[f]) return adz_internal_fail(ADZC_ERR_ARG);
  for (int f = 0; mono && f < ntot; f++)  // tricubic fields only: mono 0, 1 or 2
    if (mono[f] < 0 || mono[f] > 2) return adz_internal_fail(ADZC_ERR_ARG);

  adz::DGrid D;
  adzc_info I;
  adzc_grid G;
  int hn = 1, cold = 0;
  if (adz_internal_view(h, &D, &I, &G, &hn, &cold) != ADZC_OK) return adz_internal_fail(ADZC_ERR_ARG);
  // scratch: departure winds (3 values per extended cell) then departure w (ni*nj*nk)
  const size_t fb = (prec == ADZC_FP64) ? sizeof(double) : sizeof(float);
  const size_t uvw_bytes = align256(adz::uvw_values(prec) * fb * (size_t)D.nij * D.nk);
  const size_t wdep_bytes = align256(fb * (size_t)D.ni * D.nj * D.nk);
  if (uvw_bytes + wdep_bytes > (size_t)ADZC_NOALLOC_SCRATCH_BYTES) return adz_internal_fail(ADZC_ERR_SIZE);
  void* base = nullptr;
  const int st = scratch_address(&base);
  if (st != ADZC_OK) return adz_internal_fail(st);
  void* uvw = base;
  void* wdep = (char*)base + uvw_bytes;
  const cudaStream_t s = (cudaStream_t)stream;

  // points the kernels skip (a stencil outside the array) must read zero, not
  // what the previous call left
  if (cudaMemsetAsync(wdep, 0, wdep_bytes, s) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  if (prepare(prec, D, uu_ext, vv_ext, ww_ext, uvw, s) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  adz::TrajArgs a{};
  a.uvw_d = uvw;
  a.ut0 = ut0;
  a.vt0 = vt0;
  a.zdt0 = zdt0;
  a.pxyzm = (float*)pxyzm;
  a.wpxyz = wpxyz;
  a.wdep = wdep;
  a.niter = niter > 0 ? niter : hn;
  a.cold = cold;
  a.k00 = (D.k0 > 1) ? 1 : D.k0m;
  a.dt = adz_internal_dt_split(G, dt);
  // the positions and departure w of this step live in the caller's wpxyz
  // and the shared array, not in the handle: follow-on calls that read the
  // handle's last trajectory (adzc_tricub, adzc_bc_lam_flux) refuse until the
  // next adzc_traject
  adz_internal_forget_positions(h);
  if (traject(prec, D, a, s) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  adz_internal_after_traject(h);

  adz::SetArgs sa{};
  sa.wpxyz = wpxyz;
  sa.pxyzm = (const float*)pxyzm;
  sa.wdep = wdep;
  sa.zdt0 = zdt0;
  sa.dt = a.dt;
  sa.k00 = std::max(I.k0t - 1, 1);
  if (G.bc_lam_flux != 0 && I.k0 > 1) sa.k00 = 1;
  adz_internal_set_inputs(h, &sa);
  int f0 = 0;
  for (int set = 0; set < 4; set++) {
    const int nf = nfields[set];
    int i0, i1, j0, j1, k0;
    switch (set) {
      case ADZC_SET_Q: i0 = I.i0; i1 = I.in; j0 = I.j0; j1 = I.jn; k0 = I.k0; break;
      case ADZC_SET_U: i0 = I.i0u; i1 = I.inu; j0 = I.j0; j1 = I.jn; k0 = I.k0; break;
      case ADZC_SET_V: i0 = I.i0; i1 = I.in; j0 = I.j0v; j1 = I.jnv; k0 = I.k0; break;
      default: i0 = I.i0; i1 = I.in; j0 = I.j0; j1 = I.jn; k0 = I.k0t; break;
    }
    const int nx = i1 - i0 + 1, ny = j1 - j0 + 1, nz = D.nk - k0 + 1;
    for (int q0 = 0; q0 < nf && nx > 0 && ny > 0 && nz > 0; q0 += adz::kMaxFields) {
      adz::FieldPtrs fp{};
      fp.nf = std::min(adz::kMaxFields, nf - q0);
      for (int q = 0; q < fp.nf; q++) {
        const int f = f0 + q0 + q;
        fp.src[q] = srcs[f];
        fp.dst[q] = dsts[f];
        const int mv = mono ? mono[f] : 0;
        if (mv != 0) fp.mono_mask |= 1u << q;
        if (mv == 1) fp.clip_mask |= 1u << q;
      }
      if (tricub(prec, D, set, i0, nx, j0, ny, k0, nz, sa, fp, s) != cudaSuccess)
        return adz_internal_fail(ADZC_ERR_CUDA);
    }
    f0 += nf;
  }
  return ADZC_OK;
}
