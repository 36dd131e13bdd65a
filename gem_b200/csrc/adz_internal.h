// Internal accessors between the host C-ABI translation units (not part of
// the public ABI).
#pragma once
#include <nvtx3/nvToolsExt.h>

#include <cstddef>
#include "../../include/adz_b200.h"
#include "adz_types.h"

// read-only view of what adzc_setup derived, plus the iteration state
int adz_internal_view(const adzc_handle* h, adz::DGrid* dg, adzc_info* info, adzc_grid* g, int* niter, int* cold);
// the bookkeeping adzc_traject does after its launches (Adz_niter := Adz_itraj)
void adz_internal_after_traject(adzc_handle* h);
// drop the handle's record of its last trajectory: calls that read it
// (adzc_tricub, adzc_bc_lam_flux) then refuse with ADZC_ERR_ARG
void adz_internal_forget_positions(adzc_handle* h);
// 1 when the handle has completed a trajectory and is past its cold start
int adz_internal_warm(const adzc_handle* h);
// dt split of adz_traject.F90:38-59
adz::DtSplit adz_internal_dt_split(const adzc_grid& g, double dt);
// after a trajectory computed outside adzc_traject: positions now live in wpxyz
void adz_internal_record_positions(adzc_handle* h, int prec, double* wpxyz, const void* zdt0, const adz::DtSplit& dt);
int adz_internal_fail(int status);
// the handle's departure-wind and departure-w scratch for a precision (allocated on first use)
int adz_internal_scratch(adzc_handle* h, int prec, void** uvw, void** wdep);
// a handle-owned device buffer of at least bytes for auxiliary passes (mass fixers)
int adz_internal_aux(adzc_handle* h, size_t bytes, void** p);
// the optional inputs of the position sets registered on the handle: the
// surface-layer winds (adzc_slt_winds) and the perturbation pattern
// (adzc_rhs_perturbation); NULL when not set
void adz_internal_set_inputs(const adzc_handle* h, adz::SetArgs* a);
// restore the iteration state (cold start pending, Adz_niter) from a restart
void adz_internal_set_iteration(adzc_handle* h, int cold, int niter);

// NVTX range over a C-ABI call (host enqueue time), named after the reference
// routine or gtmg timer it stands for (B/adz_tracers.F90:34-111,
// B/tstpdyn.F90:116); visible to nsys/ncu, a no-op without a tool attached
struct AdzRange {
  explicit AdzRange(const char* name) { nvtxRangePushA(name); }
  ~AdzRange() { nvtxRangePop(); }
  AdzRange(const AdzRange&) = delete;
  AdzRange& operator=(const AdzRange&) = delete;
};
