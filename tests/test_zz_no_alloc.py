"""adzc_step_noalloc: the advection step for callers that cannot call
cudaMalloc while stepping (a host model whose device memory belongs to its own
pool or to a budget fixed at start-up, or one that must not let the step
synchronise the device).  Its scratch is a static device array shared by every
call, so these tests check it against the regular entry points (adzc_traject
followed by adzc_tricub) on two calls in a row: the second call must not be
disturbed by what the first left in the array.  Tolerance: bit-exact, as for
the regular path against the oracle (same kernels, same inputs).

This file sorts last so that a run stopping at the first failure has already
run every other test; it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a.view(np.int64)


def _setup(prec, shape=(48, 40, 20)):
    from gem_b200 import adz, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    cfg = synth.config_small(*shape)
    cfg.mono = True
    dt = torch.float64 if prec == adz.FP64 else torch.float32
    inp = synth.make_inputs(cfg, device="cuda", dtype=dt)
    return adz, cfg, inp


def _noalloc_call(adz, ad, prec, cfg, inp, px, wp, outs, tro):
    srcs = [inp["src_u"], inp["src_v"], inp["src_w"]] + list(inp["tracers"])
    dsts = [outs["u"], outs["v"], outs["w"]] + list(tro)
    nf = (C.c_int * 4)(0, 1, 1, 1 + len(tro))
    mono = (C.c_int * len(srcs))(*([0, 0, 0] + [1] * len(tro)))
    st = adz.lib().adzc_step_noalloc(
        ad.h, prec, C.c_double(cfg.dt), 0,
        *(inp[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")),
        None if px is None else px.data_ptr(), wp.data_ptr(), nf,
        C.cast(adz._ptr_array(srcs), C.c_void_p), C.cast(adz._ptr_array(dsts), C.c_void_p), mono,
        torch.cuda.current_stream().cuda_stream)
    assert st == 0, adz.lib().adzc_error_string(st)


@pytest.mark.parametrize("precname", ["ref32", "mixed", "fp64"])
def test_noalloc_step_matches_regular_path_twice(precname):
    from gem_b200 import adz as A
    prec = A.PREC_NAMES[precname]
    adz, cfg, inp = _setup(prec)
    dt = adz._field_dtype(prec)
    runs = {}
    for path in ("regular", "noalloc"):
        ad = adz.Adz.from_config(cfg)
        px, wp = ad.new_state(prec)
        ad.adz_inittraj(prec, px, wp)
        snaps = []
        for _ in range(2):  # cold step (6 iterations), then a warm one
            outs = {k: torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for k in ("u", "v", "w")}
            tro = [torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for _ in inp["tracers"]]
            if path == "regular":
                adz.step_fused(ad, prec, cfg.dt, inp, inp, inp["tracers"], px, wp, outs, tro, cfg.mono)
            else:
                _noalloc_call(adz, ad, prec, cfg, inp, px, wp, outs, tro)
            assert ad.status() == 0
            torch.cuda.synchronize()
            snaps.append([wp.cpu().numpy().copy()] + ([px.cpu().numpy().copy()] if px is not None else []) +
                         [o.cpu().numpy() for o in (outs["u"], outs["v"], outs["w"], *tro)])
        runs[path] = snaps
    for call in range(2):
        for a, b in zip(runs["regular"][call], runs["noalloc"][call]):
            assert np.array_equal(_bits(a), _bits(b)), f"call {call}"


def test_noalloc_rejects_tiles_above_capacity():
    from gem_b200 import adz, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    cfg = synth.config_large(1024, 1024, 80)
    ad = adz.Adz.from_config(cfg)  # tables only; nothing of the tile's size is allocated
    tiny = torch.zeros(16, device="cuda")
    wp = torch.zeros(16, dtype=torch.float64, device="cuda")
    nf = (C.c_int * 4)(0, 0, 0, 0)
    st = adz.lib().adzc_step_noalloc(ad.h, adz.MIXED, C.c_double(60.0), 0, *([tiny.data_ptr()] * 6), None,
                                     wp.data_ptr(), nf, None, None, None, torch.cuda.current_stream().cuda_stream)
    assert st == 9  # ADZC_ERR_SIZE, checked before any launch
    assert adz.lib().adzc_error_string(9) == b"size above capacity"


def test_noalloc_leaves_no_trajectory_on_the_handle():
    """The step's positions stay in the caller's wpxyz and its departure
    vertical wind in the shared array, so the calls that read the handle's
    last trajectory (adzc_tricub, adzc_bc_lam_flux) refuse after it instead of
    using an older step's positions; a non-finite dt is refused before any
    launch, as adzc_traject refuses it."""
    from gem_b200 import adz as A
    prec = A.MIXED
    adz, cfg, inp = _setup(prec)
    ad = adz.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    outs = {k: torch.zeros(ad.ext_shape, device="cuda") for k in ("u", "v", "w")}
    tro = [torch.zeros(ad.ext_shape, device="cuda") for _ in inp["tracers"]]
    # a regular trajectory first: without the reset the follow-on calls would use it
    ad.adz_traject(prec, cfg.dt, inp, px, wp)
    _noalloc_call(adz, ad, prec, cfg, inp, px, wp, outs, tro)
    assert ad.status() == 0
    with pytest.raises(A.AdzError) as e:
        ad.adz_tricub_hlt(prec, 3, [inp["src_w"]], [outs["w"]])
    assert e.value.status == 1  # ADZC_ERR_ARG
    fo = [torch.zeros(ad.ext_shape, device="cuda")]
    fi = [torch.zeros(ad.ext_shape, device="cuda")]
    with pytest.raises(A.AdzError) as e:
        ad.bc_lam_flux(prec, [inp["tracers"][0]], fo, fi)
    assert e.value.status == 1
    # the next regular trajectory restores them
    ad.adz_traject(prec, cfg.dt, inp, px, wp)
    ad.adz_tricub_hlt(prec, 3, [inp["src_w"]], [outs["w"]])
    assert ad.status() == 0
    nf = (C.c_int * 4)(0, 0, 0, 0)
    for bad in (float("nan"), float("inf")):
        st = adz.lib().adzc_step_noalloc(
            ad.h, prec, C.c_double(bad), 0,
            *(inp[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")),
            None, wp.data_ptr(), nf, None, None, None, torch.cuda.current_stream().cuda_stream)
        assert st == 1
