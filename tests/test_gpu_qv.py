"""BICUBH_QV (bicubic horizontal, quintic vertical) through adzc_tricub with
the ADZC_QV flag, against the restatement (oracle/adz_oracle_impl.h:
orc_tricub_qv), after a full trajectory on both sides.  Tolerances: REF32 and
FP64 bit-exact (same positions, same operation order, no contraction); MIXED
(FP32 weights and sums, positions from an FP32-sum trajectory) within 1e-5 of
the field range against the FP64 oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a.view(np.int64)


def _case(shape=(48, 40, 24), stretched=True):
    from gem_b200 import synth
    cfg = synth.config_small(*shape)
    if stretched:
        cfg.levels = synth.stretched_levels(shape[2], 50.0, 1500.0, 20e3)
    cfg.ntracers = 3
    cfg.tracer_kind = "lognormal"
    return cfg


def _run(prec_name, cfg, clip=True, pert=False):
    from gem_b200 import adz as A, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    prec = A.PREC_NAMES[prec_name]
    dt = A._field_dtype(prec)
    inp = synth.make_inputs(cfg, dtype=torch.float64)
    keys = ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")
    npd = np.float32 if dt == torch.float32 else np.float64
    np_in = {k: inp[k].numpy().astype(npd) for k in keys}
    trs = [t.numpy().astype(npd) for t in inp["tracers"]]
    # oracle
    st = O.Step(cfg, kind="oracle", prec="f32" if prec == A.REF32 else "f64")
    st.inittraj()
    mc = None
    if pert:  # ensemble perturbation pattern mcrhsint (nj, ni)
        mc = np.random.default_rng(17).uniform(-0.5, 0.5, (cfg.nj, cfg.ni)).astype(npd)
        st.set_rhs_perturbation(mc)
    st.traject({k: v.astype(st.dt) for k, v in np_in.items()})
    o_d, (o_l, o_mn, o_mx) = st.tricub_qv([t.astype(st.dt) for t in trs], clip=clip, post=True)
    # device
    dev = {k: torch.from_numpy(v).cuda() for k, v in np_in.items()}
    ad = A.Adz.from_config(cfg)
    if pert:
        ad.set_rhs_perturbation(torch.from_numpy(mc).cuda())
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    ad.adz_traject(prec, cfg.dt, dev, px, wp)
    srcs = [torch.from_numpy(t).cuda() for t in trs]
    nan = lambda: torch.full(ad.ext_shape, float("nan"), dtype=dt, device="cuda")  # noqa: E731
    dsts = [nan() for _ in srcs]
    post = ([nan() for _ in srcs], [nan() for _ in srcs], [nan() for _ in srcs])
    flag = A.QV | (1 if clip else 2)
    ad.adz_tricub_hlt(prec, A.SET_T, srcs, dsts, mono=[flag] * len(srcs), post=post)
    torch.cuda.synchronize()
    assert ad.status() == 0
    m = ad.range_mask(3).numpy()
    g = [[x.cpu().numpy() for x in arrs] for arrs in (dsts,) + post]
    o = [o_d, o_l, o_mn, o_mx]
    return A, ad, m, g, o


@pytest.mark.parametrize("prec_name,pert", [("ref32", False), ("fp64", False), ("ref32", True), ("fp64", True)])
def test_qv_bit_exact(prec_name, pert):
    """pert: with the ensemble perturbation mcrhsint set (adz_interp_hlt.F90:99-133)"""
    cfg = _case()
    A, ad, m, g, o = _run(prec_name, cfg, pert=pert)
    for gi, oi in zip(g, o):
        for a, b in zip(gi, oi):
            assert np.isnan(a[~m]).all()
            assert np.array_equal(_bits(a[m]), _bits(b[m].astype(a.dtype)))


def test_qv_mixed_tolerance():
    cfg = _case()
    A, ad, m, g, o = _run("mixed", cfg)
    for gi, oi in zip(g, o):
        for a, b in zip(gi, oi):
            ref = b[m]
            assert np.max(np.abs(a[m] - ref)) <= 1e-5 * (np.max(ref) - np.min(ref))


def test_qv_uniform_levels_and_bounds_only():
    cfg = _case((40, 36, 12), stretched=False)
    A, ad, m, g, o = _run("fp64", cfg, clip=False)
    for gi, oi in zip(g, o):
        for a, b in zip(gi, oi):
            assert np.array_equal(_bits(a[m]), _bits(b[m]))


def test_qv_rejected_outside_set_t():
    from gem_b200 import adz as A, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    cfg = _case((32, 32, 12))
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(A.MIXED)
    ad.adz_inittraj(A.MIXED, px, wp)
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32)
    ad.adz_traject(A.MIXED, cfg.dt, inp, px, wp)
    with pytest.raises(A.AdzError):
        ad.adz_tricub_hlt(A.MIXED, A.SET_U, [inp["src_u"]], [torch.zeros_like(inp["src_u"])], mono=[A.QV])
