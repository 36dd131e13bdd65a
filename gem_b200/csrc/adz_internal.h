// Internal accessors between the host C-ABI translation units (not part of
// the public ABI).
#pragma once
#include "../../include/adz_b200.h"
#include "adz_types.h"

// read-only view of what adzc_setup derived, plus the iteration state
int adz_internal_view(const adzc_handle* h, adz::DGrid* dg, adzc_info* info, adzc_grid* g, int* niter, int* cold);
// the bookkeeping adzc_traject does after its launches (Adz_niter := Adz_itraj)
void adz_internal_after_traject(adzc_handle* h);
// dt split of adz_traject.F90:38-59
adz::DtSplit adz_internal_dt_split(const adzc_grid& g, double dt);
int adz_internal_fail(int status);
