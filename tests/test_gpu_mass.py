"""Bermejo-Conde mass fixer (adzc_bermejo_conde) against the restatement
(oracle/adz_oracle_impl.h: orc_bermejo_conde) on the same inputs: tracers
after a real advection step with their post arrays (mono 2), synthetic air
masses and area mask.  Tolerances: masses and diagnostics 1e-12 relative
(FP64 sums in another order); fixed fields within 2 units in the last place
of the field type, plus the correction times the relative difference of the
two lambdas (a quotient of a cancelling difference of sums: up to ~1e-12);
the deficit carried to the next step within 1e-12 of the tracer mass.  The
fixed total must equal the total before advection to the field type's
rounding."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _case(prec_name, ntr=3, ni=56):
    from gem_b200 import adz as A, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    prec = A.PREC_NAMES[prec_name]
    dt = A._field_dtype(prec)
    cfg = synth.config_small(ni, 48, 20)
    cfg.ntracers, cfg.tracer_kind = ntr, "lognormal"
    inp = synth.make_inputs(cfg, device="cuda", dtype=dt)
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    ad.adz_traject(prec, cfg.dt, inp, px, wp)
    trs = inp["tracers"]
    z = lambda: torch.zeros(ad.ext_shape, dtype=dt, device="cuda")  # noqa: E731
    m = [z() for _ in trs]
    post = ([z() for _ in trs], [z() for _ in trs], [z() for _ in trs])
    ad.adz_tricub_hlt(prec, A.SET_T, trs, m, mono=[2] * len(trs), post=post)
    g = torch.Generator(device="cuda").manual_seed(5)
    shp = ad.ext_shape
    airm_p = (1.0 + 0.2 * torch.rand(shp, generator=g, device="cuda", dtype=torch.float64)).to(dt)
    airm_m = (airm_p.double() * (1.0 + 0.01 * torch.rand(shp, generator=g, device="cuda", dtype=torch.float64))).to(dt)
    mask = (cfg.dx ** 2 * (0.5 + torch.rand((cfg.nj, cfg.ni), generator=g, device="cuda", dtype=torch.float64)))
    torch.cuda.synchronize()
    return A, cfg, prec, ad, trs, m, post, airm_p, airm_m, mask


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a.view(np.int64)


def _np(t):
    return t.cpu().numpy()


def _close(a, b, before, ulps, dlam, dprop=0.0):
    """a, b agree to ulps units in the last place of the value, plus the
    correction m - before times the relative difference of the two lambdas
    (a quotient of two FP64 sums, summed in different orders), plus the value
    times the relative difference of the two proportional rescale factors
    (another quotient of sums, applied to the whole field when min_max)."""
    a, b = np.asarray(a), np.asarray(b)
    eps = np.finfo(a.dtype).eps
    tol = ulps * eps * np.maximum(np.abs(a), np.abs(b)) + (dlam + 4 * eps) * np.abs(b - before) + dprop * np.abs(b)
    return np.all(np.abs(a - b) <= tol + np.finfo(a.dtype).tiny)


# FP32 fields take four cells at a time where every row start is 16-byte
# aligned (ni = 56: extended rows of 64 cells); ni = 58 (rows of 66) takes the
# cell-by-cell kernels
# flux: LAM boundary fluxes fo, fi given (the flux pass), weight 3 with pkps
@pytest.mark.parametrize("prec_name,weight,p_exp,min_max,ni,flux", [("mixed", 1, 1.0, True, 56, False),
                                                                     ("ref32", 2, 2.0, True, 56, False),
                                                                     ("fp64", 1, 1.0, False, 56, False),
                                                                     ("mixed", 1, 1.0, False, 56, False),
                                                                     ("mixed", 1, 1.0, True, 58, False),
                                                                     ("ref32", 2, 2.0, True, 58, False),
                                                                     ("mixed", 3, 1.0, True, 56, True),
                                                                     ("ref32", 3, 1.5, True, 58, True),
                                                                     ("fp64", 3, 1.0, True, 56, True)])
def test_bermejo_conde_vs_oracle(prec_name, weight, p_exp, min_max, ni, flux):
    A, cfg, prec, ad, trs, m, post, airm_p, airm_m, mask = _case(prec_name, ni=ni)
    lin, mn, mx = post
    ntr = len(trs)
    # tracer 0 made smooth in its last step: high and low order equal -> no correction (almost_zero)
    m[0].copy_(lin[0])
    extra = [{} for _ in range(ntr)]
    if flux or weight == 3:
        g = torch.Generator(device="cuda").manual_seed(11)
        rnd = lambda a: (a * torch.rand(ad.ext_shape, generator=g, device="cuda", dtype=torch.float64)).to(m[0].dtype)  # noqa: E731
        for q in range(ntr):
            if flux:
                extra[q].update(fo=rnd(0.01), fi=rnd(0.01))
            if weight == 3:
                extra[q]["pkps"] = 0.5 + rnd(1.0)
    src = [dict(p=trs[q], m=m[q], lin=lin[q], min=mn[q], max=mx[q], weight=weight, p_exp=p_exp, **extra[q])
           for q in range(ntr)]
    before = [_np(t).copy() for t in m]
    deficit = torch.tensor([0.0, 1e-3, -2e-3][:ntr], dtype=torch.float64, device="cuda")
    d0 = _np(deficit).copy()
    diag = torch.zeros((ntr, 8), dtype=torch.float64, device="cuda")
    A.bermejo_conde(ad, prec, src, airm_p, airm_m, mask, deficit, min_max=min_max, diag=diag)
    torch.cuda.synchronize()
    st = O.Step(cfg, kind="oracle", prec="f32" if prec != A.FP64 else "f64")
    g_diag, g_def = _np(diag), _np(deficit)
    for q in range(ntr):
        ex = {k: _np(v) for k, v in extra[q].items()}
        o_m, o_def, o_diag = st.bermejo_conde(_np(trs[q]), before[q], _np(lin[q]), _np(mn[q]), _np(mx[q]),
                                              _np(airm_p), _np(airm_m), _np(mask), deficit=d0[q], weight=weight,
                                              p_exp=p_exp, min_max=min_max, **ex)
        scale = max(abs(o_diag[0]), abs(o_diag[1]))
        masses = [0, 1, 2, 3, 4, 6, 7]
        assert np.all(np.abs(g_diag[q][masses] - o_diag[masses]) <= 1e-12 * scale), (q, g_diag[q], o_diag)
        assert abs(g_diag[q][5] - o_diag[5]) <= 1e-10 * abs(o_diag[5]), (q, g_diag[q][5], o_diag[5])
        assert abs(g_def[q] - o_def) <= 1e-12 * scale
        gm = _np(m[q])
        bad = np.argmax(np.abs(gm - o_m))
        dlam = abs(g_diag[q][5] - o_diag[5]) / max(abs(o_diag[5]), 1e-300)
        # rescale factor mass_bc / mass_bc_r of each side (min_max only)
        dprop = 0.0
        if min_max and o_diag[6] != 0 and g_diag[q][6] != 0 and o_diag[7] != 0:
            dprop = 2 * abs((g_diag[q][7] / g_diag[q][6]) / (o_diag[7] / o_diag[6]) - 1.0)
        assert _close(gm, o_m, before[q], 2 if p_exp == 1.0 else 4, dlam, dprop), (
            q, np.unravel_index(bad, gm.shape), gm.flat[bad], o_m.flat[bad], before[q].flat[bad],
            int(np.sum(gm != o_m)))
    if flux:  # the mass balance then includes the boundary fluxes; the oracle comparison above covers it
        return
    # tracer 0: nothing to fix, epsilon carried unchanged
    assert np.array_equal(_np(m[0]), before[0]) and g_def[0] == d0[0]
    # the fixed tracers hold the mass they had before advection (minus the old epsilon)
    for q in range(1, ntr):
        assert abs(g_diag[q][7] - (g_diag[q][0] - d0[q])) <= 1e-6 * abs(g_diag[q][0])


def test_bermejo_conde_rejects_bad_arguments():
    A, cfg, prec, ad, trs, m, post, airm_p, airm_m, mask = _case("mixed", ntr=1)
    deficit = torch.zeros(1, dtype=torch.float64, device="cuda")
    bad = [dict(p=trs[0], m=m[0], lin=post[0][0], min=post[1][0], max=post[2][0], weight=4)]
    with pytest.raises(A.AdzError):
        A.bermejo_conde(ad, prec, bad, airm_p, airm_m, mask, deficit)
    bad = [dict(p=trs[0], m=m[0], lin=post[0][0], weight=1)]  # min/max needed when min_max
    with pytest.raises(A.AdzError):
        A.bermejo_conde(ad, prec, bad, airm_p, airm_m, mask, deficit, min_max=True)


@pytest.mark.parametrize("prec_name,gbpil,psadj", [("ref32", 0, False), ("fp64", 0, False), ("ref32", 4, False),
                                                   ("ref32", 0, True)])
def test_bc_lam_flux_vs_oracle(prec_name, gbpil, psadj):
    """LAM boundary fluxes (adz_BC_LAM_Aranami_hlt.F90) bit for bit against the
    restatement: the masked tracers interpolated at Adz_pb over range b, then
    zeroed; every element of fo and fi compared, including which ones are
    written (NaN elsewhere on both sides).  gbpil: a top pilot (k0t > 1), so
    FLUX_in is also zeroed above k0t.  psadj: no tracer, the masks themselves
    (the PSADJ branch)."""
    from gem_b200 import adz as A, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    prec = A.PREC_NAMES[prec_name]
    dt = A._field_dtype(prec)
    cfg = synth.config_small(48, 40, 20)
    cfg.ntracers, cfg.tracer_kind = 3, "lognormal"
    inp = synth.make_inputs(cfg, dtype=torch.float64)
    npd = np.float32 if dt == torch.float32 else np.float64
    keys = ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")
    np_in = {k: inp[k].numpy().astype(npd) for k in keys}
    trs = [t.numpy().astype(npd) for t in inp["tracers"]]
    st = O.Step(cfg, kind="ref" if (prec == A.REF32 and O.have_ref()) else "oracle",
                prec="f32" if prec == A.REF32 else "f64", lam_gbpil_t=gbpil)
    st.inittraj()
    st.traject(np_in)
    if psadj:
        trs = [None]
    o_fo, o_fi = st.bc_lam_flux(trs)
    ad = A.Adz.from_config(cfg, lam_gbpil_t=gbpil)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    ad.adz_traject(prec, cfg.dt, {k: torch.from_numpy(v).cuda() for k, v in np_in.items()}, px, wp)
    srcs = [None if t is None else torch.from_numpy(t).cuda() for t in trs]
    nan = lambda: torch.full(ad.ext_shape, float("nan"), dtype=dt, device="cuda")  # noqa: E731
    fo, fi = [nan() for _ in srcs], [nan() for _ in srcs]
    ad.bc_lam_flux(prec, srcs, fo, fi)
    torch.cuda.synchronize()
    assert ad.status() == 0
    for g, o in zip(fo + fi, o_fo + o_fi):
        g = g.cpu().numpy()
        assert np.array_equal(np.isnan(g), np.isnan(o))
        w = ~np.isnan(o)
        assert w.any()
        assert np.array_equal(_bits(g[w]), _bits(o[w]))
    # the fluxes are not trivially zero: both carry tracer outside the zeroed parts
    assert all(np.nanmax(np.abs(o)) > 0 for o in o_fo + o_fi)
