// Batches of independent limited-area domains stepped by ONE persistent launch.
//
// Work items (domain, phase, group, first point, count) are laid out phase by
// phase: every departure-wind item (phase 0) of every domain, then every
// trajectory item (phase 1), then every interpolation item (phase 2, one
// field group of one position set).  Blocks take items from an atomic queue.
// An item of phase p>0 first waits until all items of phase p-1 of its own
// domain have completed (per-domain counters).  Every such item was taken by
// a block that is running and never waits on anything later in the queue, so
// the wait always ends; it is bounded anyway (kErrTimeout, item skipped).
// Counters are released with a device-scope fence by every writer thread and
// read with acquire semantics; positions written in the same launch are read
// around L1.
//
// The tile of an item is ``rows`` consecutive rows of one level band
// (rows * row length points; trajectory and interpolation items of regions
// that tiles of 32 i by 4 levels cover with few idle lanes are the tiles that
// cover rows / 4 such rows, as the per-domain kernels walk their points);
// adzc_batch_tune times candidate row counts and
// resident block counts and keeps the fastest.  The tuned launch is captured
// in a CUDA graph (counter reset + persistent kernel) and replayed per step.
//
// The phased plan runs the same items as three persistent launches in the
// graph, one per phase, each kernel with the register budget of the
// per-domain kernel of its phase; launch order replaces the dependency waits.
// The per-domain plan replays every domain's own launches in turn: departure
// winds, trajectory and all field groups in one k_tricub_parts launch, as the
// per-domain entry points run them.  The tuner weighs the phased and
// per-domain plans against the one-launch kernel's budgets.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/adz_b200.h"
#include "adz_internal.h"
#include "adz_types.h"


// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct adzc_batch {
  int prec = 0, ndom = 0;
  std::vector<adz::BDom> doms;
  adz::BatchParams* params = nullptr;  // the domains' grid-constant descriptors
  std::vector<adzc_handle*> handles;
  adz::BDom* d_doms = nullptr;
  adz::BItem* d_items = nullptr;
  size_t items_cap = 0;
  long long nitems = 0;
  unsigned* d_need = nullptr;
  unsigned long long* d_next = nullptr;
  unsigned* d_done = nullptr;
  int* d_status = nullptr;
  int rows = 8, bps = 4, sms = 148, variant = 0;
  int phased = 0;           // 1: the phased plan (one launch per phase); 2: the per-domain launches
  unsigned long long spins = adz::kDepSpins;  // bound of a dependency wait
  long long inject_need = 0;  // fault injection: extra items domain 0's trajectory waits for
  long long pstart[4] = {}; // first item of each phase, total
  int pgrid[3] = {};        // persistent grid of each phased launch
  float tuned_ms[3] = {-1.f, -1.f, -1.f};  // tuner: best ms per step of each plan family (one launch, phased, per-domain)
  cudaStream_t cap = nullptr;
  // the per-domain plan on concurrent branches: lanes streams (lane 0 is the
  // caller's), a fork event and one join event per lane
  int lanes = 1;
  cudaStream_t lane_s[adz::kBatchLanes] = {};
  cudaEvent_t fork = nullptr, join[adz::kBatchLanes] = {};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

int build_items(adzc_batch* b, int rows) {
  std::vector<adz::BItem> items;
  std::vector<unsigned> need(2 * b->ndom, 0);
  for (int phase = 0; phase < 3; phase++) {
    b->pstart[phase] = (long long)items.size();
    for (int d = 0; d < b->ndom; d++) {
      const adz::BDom& D = b->doms[d];
      auto push = [&](int group, long long n, long long chunk, int tiles = 0) {
        for (long long s = 0; s < n; s += chunk) {
          adz::BItem it{};
          it.dom = d;
          it.phase = phase;
          it.group = group;
          it.tiles = tiles;
          it.start = s;
          it.count = std::min(chunk, n - s);
          items.push_back(it);
          if (phase < 2) need[2 * d + phase]++;
        }
      };
      if (phase == 0) push(0, D.g.nij * D.g.nk, (long long)rows * D.g.nit);
      // a region of nx i by nz levels by ny rows: tiles of kBatchTileI i by
      // kBatchTileK levels (rows / kBatchTileK tile rows an item) where they
      // leave few lanes idle, else points in (i, k, j) order (rows rows)
      auto region = [&](int group, long long nx, long long nz, long long ny) {
        if (adz::batch_use_tiles(nx, nz)) {
          const long long nic = (nx + adz::kBatchTileI - 1) / adz::kBatchTileI;
          const long long nkg = (nz + adz::kBatchTileK - 1) / adz::kBatchTileK;
          push(group, nic * nkg * ny, std::max(1, rows / adz::kBatchTileK) * nic, 1);
        } else {
          push(group, nx * nz * ny, (long long)rows * nx, 0);
        }
      };
      if (phase == 1) region(0, D.g.ni, D.g.nk - D.ta.k00 + 1, D.g.nj);
      if (phase == 2)
        for (int q = 0; q < D.ngroups; q++) {
          const int* r = D.grange[q];
          region(q, r[1], D.g.nk - r[4] + 1, r[3]);
        }
    }
  }
  need[0] += (unsigned)b->inject_need;  // fault injection (adzc_batch_inject): items that never come
  if (items.size() > b->items_cap) {
    cudaFree(b->d_items);
    b->d_items = nullptr;
    if (cudaMalloc(&b->d_items, items.size() * sizeof(adz::BItem)) != cudaSuccess) return ADZC_ERR_ALLOC;
    b->items_cap = items.size();
  }
  if (cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(adz::BItem), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_need, need.data(), need.size() * sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess)
    return ADZC_ERR_CUDA;
  b->nitems = (long long)items.size();
  b->pstart[3] = b->nitems;
  b->rows = rows;
  return ADZC_OK;
}

// one domain's own launches: departure winds, trajectory and all field
// groups in one k_tricub_parts launch
template <int PREC>
cudaError_t enqueue_domain(const adz::BDom& D, cudaStream_t s) {
  cudaError_t e = adz::launch_prepare<PREC>(D.g, D.uu, D.vv, D.ww, const_cast<void*>(D.ta.uvw_d), s);
  if (e == cudaSuccess) e = adz::launch_traject<PREC>(D.g, D.ta, s);
  adz::SetParts sp{};
  for (int q = 0; q < D.ngroups && e == cudaSuccess; q++) {
    adz::SetPart& P = sp.p[sp.n++];
    P.fp = D.gfp[q];
    P.set = D.gset[q];
    P.i0 = D.grange[q][0];
    P.nx = D.grange[q][1];
    P.j0 = D.grange[q][2];
    P.ny = D.grange[q][3];
    P.k0 = D.grange[q][4];
    P.nz = D.g.nk - P.k0 + 1;
    if (P.nx <= 0 || P.ny <= 0 || P.nz <= 0) sp.n--;
    if (sp.n == adz::kMaxParts || (q == D.ngroups - 1 && sp.n > 0)) {
      e = adz::launch_tricub_parts<PREC>(D.g, D.sa, sp, s);
      sp = adz::SetParts{};
    }
  }
  return e;
}

// the per-domain plan: every domain's own launches in turn, or spread over
// b->lanes concurrent branches (a fork and a join event; domains assigned
// largest first to the least loaded branch), so that one domain's launch
// tails and its memory-bound departure winds overlap another's gathers
template <int PREC>
cudaError_t enqueue_domains(const adzc_batch* b, cudaStream_t s) {
  if (b->lanes <= 1) {
    for (int d = 0; d < b->ndom; d++) {
      const cudaError_t e = enqueue_domain<PREC>(b->doms[d], s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::vector<std::pair<double, int>> cost(b->ndom);
  for (int d = 0; d < b->ndom; d++) {
    const adz::BDom& D = b->doms[d];
    double c = (double)D.g.nij * D.g.nk;  // winds and trajectory
    for (int q = 0; q < D.ngroups; q++)
      c += (double)D.grange[q][1] * D.grange[q][3] * (D.g.nk - D.grange[q][4] + 1) * (0.5 + 0.5 * D.gfp[q].nf);
    cost[d] = {c, d};
  }
  std::sort(cost.begin(), cost.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  std::vector<double> load(b->lanes, 0.0);
  std::vector<std::vector<int>> lane_doms(b->lanes);
  for (const auto& c : cost) {
    const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[l] += c.first;
    lane_doms[l].push_back(c.second);
  }
  cudaError_t e = cudaEventRecord(b->fork, s);
  for (int l = 1; l < b->lanes && e == cudaSuccess; l++) e = cudaStreamWaitEvent(b->lane_s[l], b->fork, 0);
  for (int l = 0; l < b->lanes && e == cudaSuccess; l++)
    for (int d : lane_doms[l]) {
      e = enqueue_domain<PREC>(b->doms[d], l == 0 ? s : b->lane_s[l]);
      if (e != cudaSuccess) break;
    }
  for (int l = 1; l < b->lanes; l++) {  // join every branch even after an error
    const cudaError_t r = cudaEventRecord(b->join[l], b->lane_s[l]);
    const cudaError_t w = cudaStreamWaitEvent(s, b->join[l], 0);
    if (e == cudaSuccess) e = r != cudaSuccess ? r : w;
  }
  return e;
}

cudaError_t enqueue(adzc_batch* b, cudaStream_t s) {
  cudaError_t e;
  if (b->phased == 2)
    return b->prec == ADZC_FP64 ? enqueue_domains<adz::kFp64>(b, s) : enqueue_domains<adz::kMixed>(b, s);
  if (b->phased) {
    if ((e = cudaMemsetAsync(b->d_next + 1, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
    if (b->prec == ADZC_FP64)
      return adz::launch_batch_phased<adz::kFp64>(b->pgrid, *b->params, b->d_doms, b->d_items, b->pstart,
                                                  b->d_next + 1, s);
    return adz::launch_batch_phased<adz::kMixed>(b->pgrid, *b->params, b->d_doms, b->d_items, b->pstart,
                                                 b->d_next + 1, s);
  }
  if ((e = cudaMemsetAsync(b->d_next, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(b->d_done, 0, 2 * b->ndom * sizeof(unsigned), s)) != cudaSuccess) return e;
  const int grid = b->bps * b->sms;
  if (b->prec == ADZC_FP64)
    return adz::launch_batch<adz::kFp64>(b->variant, grid, *b->params, b->d_doms, b->d_items, b->nitems, b->d_need,
                                         b->d_next, b->d_done, b->d_status, b->spins, s);
  return adz::launch_batch<adz::kMixed>(b->variant, grid, *b->params, b->d_doms, b->d_items, b->nitems, b->d_need,
                                        b->d_next, b->d_done, b->d_status, b->spins, s);
}

int resident(const adzc_batch* b, int variant) {
  return b->prec == ADZC_FP64 ? adz::batch_resident_blocks<adz::kFp64>(variant)
                              : adz::batch_resident_blocks<adz::kMixed>(variant);
}

// the handles' positions now live in the domains' wpxyz (adzc_tricub may follow)
void record(adzc_batch* b) {
  for (int d = 0; d < b->ndom; d++)
    adz_internal_record_positions(b->handles[d], b->prec, (double*)b->doms[d].ta.wpxyz, b->doms[d].ta.zdt0,
                                  b->doms[d].ta.dt);
}

int capture(adzc_batch* b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return ADZC_ERR_CUDA;
  const cudaError_t e = enqueue(b, b->cap);
  cudaGraph_t g = nullptr;
  if (cudaStreamEndCapture(b->cap, &g) != cudaSuccess || e != cudaSuccess || !g) return ADZC_ERR_CUDA;
  b->graph = g;
  if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) return ADZC_ERR_CUDA;
  return ADZC_OK;
}

}  // namespace

extern "C" int adzc_batch_destroy(adzc_batch* b) {
  if (!b) return ADZC_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  for (int l = 0; l < adz::kBatchLanes; l++) {
    if (b->lane_s[l]) cudaStreamDestroy(b->lane_s[l]);
    if (b->join[l]) cudaEventDestroy(b->join[l]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b->params;
  cudaFree(b->d_doms);
  cudaFree(b->d_items);
  cudaFree(b->d_need);
  cudaFree(b->d_next);
  cudaFree(b->d_done);
  cudaFree(b->d_status);
  delete b;
  return ADZC_OK;
}

extern "C" int adzc_batch_create(int prec, int ndom, const adzc_domain* doms, adzc_batch** out) {
  if (!out || ndom < 1 || !doms || (prec != ADZC_FP64 && prec != ADZC_MIXED)) return adz_internal_fail(ADZC_ERR_ARG);
  if (ndom > ADZC_BATCH_MAX_DOMAINS) return adz_internal_fail(ADZC_ERR_SIZE);
  auto* b = new (std::nothrow) adzc_batch();
  if (!b) return adz_internal_fail(ADZC_ERR_ALLOC);
  b->prec = prec;
  b->ndom = ndom;
  b->doms.resize(ndom);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  b->bps = std::max(1, resident(b, 0));
  for (int p = 0; p < 3; p++) {
    const int r = b->prec == ADZC_FP64 ? adz::batch_phase_resident_blocks<adz::kFp64>(p)
                                       : adz::batch_phase_resident_blocks<adz::kMixed>(p);
    b->pgrid[p] = std::max(1, r) * b->sms;
  }
  for (int d = 0; d < ndom; d++) {
    const adzc_domain& in = doms[d];
    adz::BDom& D = b->doms[d];
    memset(&D, 0, sizeof(D));
    adzc_info I;
    adzc_grid G;
    int niter = 1, cold = 0;
    if (!in.h || !in.uu_ext || !in.vv_ext || !in.ww_ext || !in.ut0 || !in.vt0 || !in.zdt0 || !in.wpxyz ||
        adz_internal_view(in.h, &D.g, &I, &G, &niter, &cold) != ADZC_OK || cold || !adz_internal_warm(in.h)) {
      adzc_batch_destroy(b);
      return adz_internal_fail(ADZC_ERR_ARG);
    }
    void *uvw = nullptr, *wdep = nullptr;
    if (adz_internal_scratch(in.h, prec, &uvw, &wdep) != ADZC_OK) {
      adzc_batch_destroy(b);
      return adz_internal_fail(ADZC_ERR_ALLOC);
    }
    D.uu = in.uu_ext;
    D.vv = in.vv_ext;
    D.ww = in.ww_ext;
    D.ta.uvw_d = uvw;
    D.ta.ut0 = in.ut0;
    D.ta.vt0 = in.vt0;
    D.ta.zdt0 = in.zdt0;
    D.ta.wpxyz = in.wpxyz;
    D.ta.wdep = wdep;
    D.ta.niter = in.niter > 0 ? in.niter : niter;
    D.ta.cold = 0;
    D.ta.k00 = (D.g.k0 > 1) ? 1 : D.g.k0m;
    D.ta.dt = adz_internal_dt_split(G, in.dt);
    D.sa.wpxyz = in.wpxyz;
    D.sa.wdep = wdep;
    D.sa.zdt0 = in.zdt0;
    D.sa.dt = D.ta.dt;
    D.sa.k00 = std::max(I.k0t - 1, 1);
    if (G.bc_lam_flux != 0 && I.k0 > 1) D.sa.k00 = 1;
    adz_internal_set_inputs(in.h, &D.sa);
    if (D.sa.pert) {  // the batch kernels carry no perturbation: step such a domain on its own
      adzc_batch_destroy(b);
      return adz_internal_fail(ADZC_ERR_ARG);
    }
    const int r[4][5] = {{I.i0, I.in, I.j0, I.jn, I.k0},
                         {I.i0u, I.inu, I.j0, I.jn, I.k0},
                         {I.i0, I.in, I.j0v, I.jnv, I.k0},
                         {I.i0, I.in, I.j0, I.jn, I.k0t}};
    int f0 = 0;
    for (int set = 0; set < 4; set++) {
      const int nf = in.nfields[set];
      if (nf < 0) {
        adzc_batch_destroy(b);
        return adz_internal_fail(ADZC_ERR_ARG);
      }
      for (int q0 = 0; q0 < nf; q0 += adz::kMaxFields) {
        if (D.ngroups == adz::kMaxGroups) {
          adzc_batch_destroy(b);
          return adz_internal_fail(ADZC_ERR_SIZE);
        }
        const int gi = D.ngroups++;
        D.gset[gi] = set;
        D.grange[gi][0] = r[set][0];
        D.grange[gi][1] = r[set][1] - r[set][0] + 1;
        D.grange[gi][2] = r[set][2];
        D.grange[gi][3] = r[set][3] - r[set][2] + 1;
        D.grange[gi][4] = r[set][4];
        adz::FieldPtrs& fp = D.gfp[gi];
        fp.nf = std::min(adz::kMaxFields, nf - q0);
        for (int q = 0; q < fp.nf; q++) {
          const int f = f0 + q0 + q;
          if (!in.srcs || !in.dsts || !in.srcs[f] || !in.dsts[f]) {
            adzc_batch_destroy(b);
            return adz_internal_fail(ADZC_ERR_ARG);
          }
          fp.src[q] = in.srcs[f];
          fp.dst[q] = in.dsts[f];
          const int mv = in.mono ? in.mono[f] : 0;
          if (mv < 0 || mv > 2) {  // tricubic fields only
            adzc_batch_destroy(b);
            return adz_internal_fail(ADZC_ERR_ARG);
          }
          if (mv != 0) fp.mono_mask |= 1u << q;
          if (mv == 1) fp.clip_mask |= 1u << q;
        }
      }
      f0 += nf;
    }
    b->handles.push_back(in.h);
  }
  b->params = new (std::nothrow) adz::BatchParams();
  if (!b->params) {
    adzc_batch_destroy(b);
    return adz_internal_fail(ADZC_ERR_ALLOC);
  }
  for (int d = 0; d < ndom; d++) {
    adz::BDomC& C = b->params->d[d];
    C.g = b->doms[d].g;
    C.uu = b->doms[d].uu;
    C.vv = b->doms[d].vv;
    C.ww = b->doms[d].ww;
    C.ta = b->doms[d].ta;
    C.sa = b->doms[d].sa;
  }
  if (cudaMalloc(&b->d_doms, ndom * sizeof(adz::BDom)) != cudaSuccess ||
      cudaMalloc(&b->d_need, 2 * ndom * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&b->d_next, 4 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->d_done, 2 * ndom * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&b->d_status, sizeof(int)) != cudaSuccess ||
      cudaMemcpy(b->d_doms, b->doms.data(), ndom * sizeof(adz::BDom), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(b->d_status, 0, sizeof(int)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
    adzc_batch_destroy(b);
    return adz_internal_fail(ADZC_ERR_CUDA);
  }
  for (int l = 1; l < adz::kBatchLanes; l++) {
    if (cudaStreamCreateWithFlags(&b->lane_s[l], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join[l], cudaEventDisableTiming) != cudaSuccess) {
      adzc_batch_destroy(b);
      return adz_internal_fail(ADZC_ERR_CUDA);
    }
  }
  int st = build_items(b, b->rows);
  if (st == ADZC_OK) st = capture(b);
  if (st != ADZC_OK) {
    adzc_batch_destroy(b);
    return adz_internal_fail(st);
  }
  *out = b;
  return ADZC_OK;
}

extern "C" int adzc_batch_step(adzc_batch* b, void* stream) {
  AdzRange nvtx_range("ADZ_MAIN batch");
  if (!b || !b->exec) return adz_internal_fail(ADZC_ERR_ARG);
  if (cudaGraphLaunch(b->exec, (cudaStream_t)stream) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  record(b);
  return ADZC_OK;
}

extern "C" int adzc_batch_tune(adzc_batch* b, void* stream) {
  AdzRange nvtx_range("ADZ_MAIN batch tune");
  if (!b) return adz_internal_fail(ADZC_ERR_ARG);
  const cudaStream_t s = (cudaStream_t)stream;
  const int rows_c[] = {2, 8, 32};
  float best = 1e30f;
  for (int q = 0; q < 3; q++) b->tuned_ms[q] = -1.f;  // this tune's timings only
  int br = b->rows, bb = b->bps, bv = b->variant, bp = b->phased;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  int st = ADZC_OK;
  // variants 0..kBatchVariants-1: the one-launch kernel's register budgets;
  // kBatchVariants: the phased plan
  for (int v = 0; v <= adz::kBatchVariants && st == ADZC_OK; v++) {
    const bool ph = v == adz::kBatchVariants;
    const int res = ph ? b->bps : resident(b, v);  // persistent: every block resident
    if (res < 1) continue;
    for (int r : rows_c) {
      b->phased = ph ? 1 : 0;
      if (!ph) {
        b->variant = v;
        b->bps = res;
      }
      if (build_items(b, r) != ADZC_OK || enqueue(b, s) != cudaSuccess) {
        st = ADZC_ERR_CUDA;
        break;
      }
      cudaEventRecord(e0, s);
      for (int rep = 0; rep < 2; rep++) enqueue(b, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        st = ADZC_ERR_CUDA;
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      float& fam = b->tuned_ms[ph ? 1 : 0];
      if (fam < 0.f || ms / 2 < fam) fam = ms / 2;
      if (ms < best) {
        best = ms;
        br = r;
        bp = ph ? 1 : 0;
        if (!ph) {
          bb = res;
          bv = v;
        }
      }
    }
  }
  int blanes = b->lanes;
  for (int lanes : {1, adz::kBatchLanes}) {  // the per-domain launches (rows unused), in turn or concurrent
    if (st != ADZC_OK) break;
    b->phased = 2;
    b->lanes = lanes;
    float ms = 0.f;
    if (enqueue(b, s) != cudaSuccess || cudaEventRecord(e0, s) != cudaSuccess || enqueue(b, s) != cudaSuccess ||
        enqueue(b, s) != cudaSuccess || cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
      st = ADZC_ERR_CUDA;
    else if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
      if (b->tuned_ms[2] < 0.f || ms / 2 < b->tuned_ms[2]) b->tuned_ms[2] = ms / 2;
      if (ms < best) best = ms, bp = 2, blanes = lanes;
    }
  }
  b->lanes = bp == 2 ? blanes : 1;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->bps = bb;
  b->variant = bv;
  b->phased = bp;
  if (st == ADZC_OK) st = build_items(b, br);
  if (st == ADZC_OK) st = capture(b);
  record(b);
  return st == ADZC_OK ? ADZC_OK : adz_internal_fail(st);
}

extern "C" int adzc_batch_query(const adzc_batch* b, int* rows, int* blocks_per_sm, long long* nitems) {
  if (!b) return adz_internal_fail(ADZC_ERR_ARG);
  if (rows) *rows = b->rows;
  if (blocks_per_sm) *blocks_per_sm = b->phased == 2 ? 0 : b->phased ? b->pgrid[1] / b->sms : b->bps;
  if (nitems) *nitems = b->nitems;
  return ADZC_OK;
}

extern "C" int adzc_batch_select(adzc_batch* b, int rows, int plan) {
  if (!b || rows < 1 || plan < 0 || plan > ADZC_BATCH_DOMAINS_CONCURRENT) return adz_internal_fail(ADZC_ERR_ARG);
  if (plan < adz::kBatchVariants) {
    const int res = resident(b, plan);
    if (res < 1) return adz_internal_fail(ADZC_ERR_ARG);
    b->variant = plan;
    b->bps = res;
    b->phased = 0;
  } else {
    b->phased = plan == ADZC_BATCH_PHASED ? 1 : 2;
  }
  b->lanes = plan == ADZC_BATCH_DOMAINS_CONCURRENT ? adz::kBatchLanes : 1;
  int st = build_items(b, rows);
  if (st == ADZC_OK) st = capture(b);
  return st == ADZC_OK ? ADZC_OK : adz_internal_fail(st);
}

extern "C" int adzc_batch_inject(adzc_batch* b, int what, long long value) {
  if (!b || value < 0) return adz_internal_fail(ADZC_ERR_ARG);
  if (what == ADZC_INJECT_SPINS) {
    b->spins = value > 0 ? (unsigned long long)value : adz::kDepSpins;
  } else if (what == ADZC_INJECT_NEED) {
    if (value > 1000000) return adz_internal_fail(ADZC_ERR_ARG);
    b->inject_need = value;
  } else {
    return adz_internal_fail(ADZC_ERR_ARG);
  }
  int st = build_items(b, b->rows);
  if (st == ADZC_OK) st = capture(b);
  return st == ADZC_OK ? ADZC_OK : adz_internal_fail(st);
}

extern "C" int adzc_batch_tuned(const adzc_batch* b, float* ms) {
  if (!b || !ms) return adz_internal_fail(ADZC_ERR_ARG);
  for (int q = 0; q < 3; q++) ms[q] = b->tuned_ms[q];
  return ADZC_OK;
}

extern "C" int adzc_batch_plan(const adzc_batch* b, int* phased) {
  if (!b || !phased) return adz_internal_fail(ADZC_ERR_ARG);
  *phased = b->phased == 2 && b->lanes > 1 ? 3 : b->phased;
  return ADZC_OK;
}

extern "C" int adzc_batch_status(adzc_batch* b, int reset, void* stream) {
  if (!b) return adz_internal_fail(ADZC_ERR_ARG);
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return adz_internal_fail(ADZC_ERR_CUDA);
  int bits = 0;
  if (cudaMemcpy(&bits, b->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return adz_internal_fail(ADZC_ERR_CUDA);
  if (reset) cudaMemset(b->d_status, 0, sizeof(int));
  if (bits & adz::kErrTimeout) return ADZC_ERR_TIMEOUT;
  for (adzc_handle* h : b->handles) {
    const int st = adzc_status(h, reset, stream);
    if (st != ADZC_OK) return st;
  }
  return ADZC_OK;
}
