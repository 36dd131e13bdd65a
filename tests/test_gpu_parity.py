"""GPU parity: the CUDA path, called through the C ABI, against the oracle.

* REF32 (the reference's own arithmetic) is bit-exact with the reference
  interpolator compiled unchanged (golden vectors, SELF_TEST known answers) and
  with the driver restatement: positions, cell indices and every field.
* FP64 is bit-exact with the FP64 oracle.
* MIXED (FP32 weights and sums) is within a stated relative tolerance of the
  FP64 oracle, with bit-exact cell indices for the same positions.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# MIXED tolerance: max |gpu - fp64 oracle| / max |fp64 oracle| per field
MIXED_REL_TOL = 1e-6


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a.view(np.int64)


@pytest.fixture(scope="module")
def A():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from gem_b200 import adz
    adz.lib()
    return adz


@pytest.fixture(scope="module")
def vec():
    return dict(np.load(os.path.join(GOLD, "tricublin_ref_vectors.npz")))


# ---------------------------------------------------------------- interpolators
def test_golden_vectors_device_ref32(A, vec):
    ni, nj = int(vec["ni"]), int(vec["nj"])
    zt = A.Ztab(vec["levels"], ni, nj, int(vec["offi"]), int(vec["offj"]))
    f = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in vec["fields"]]
    pos = torch.from_numpy(vec["pos"]).cuda()
    d = A.tricublin_m_n(zt, A.REF32, f, pos).cpu().numpy()
    assert np.array_equal(_bits(d), _bits(vec["zyx1"]))
    out = [o.cpu().numpy() for o in A.tricublin_mono_m_n(zt, A.REF32, f, pos)]
    for got, key in zip(out, ("mono_d", "mono_lin", "mono_min", "mono_max")):
        assert np.array_equal(_bits(got), _bits(vec[key])), key
    out = [o.cpu().numpy() for o in A.tricublin_mono_m_n(zt, A.REF32, f, pos, box=1)]
    assert np.array_equal(_bits(out[2]), _bits(vec["scalar_mono_min"]))
    assert np.array_equal(_bits(out[3]), _bits(vec["scalar_mono_max"]))
    f3 = torch.from_numpy(np.ascontiguousarray(vec["f3"])).cuda()
    d3 = A.tricublin_zyx3_n(zt, A.REF32, f3, pos).cpu().numpy()
    assert np.array_equal(_bits(d3), _bits(vec["zyx3"]))


def test_golden_vectors_level_a_host_pointers(A, vec):
    """The reference-named symbols with host pointers (drop-in for turbo_tricublin.o)."""
    import ctypes as C
    L = A.lib()
    ni, nj, nk = int(vec["ni"]), int(vec["nj"]), int(vec["nk"])
    lev = np.ascontiguousarray(vec["levels"])
    lv = L.Vsearch_setup_plus(lev.ctypes.data, nk, ni, nj, int(vec["offi"]), int(vec["offj"]))
    assert lv
    fields = [np.ascontiguousarray(x) for x in vec["fields"]]
    pos = np.ascontiguousarray(vec["pos"])
    n, m = pos.shape[0], len(fields)
    fs = (C.c_void_p * m)(*[x.ctypes.data for x in fields])
    d = np.empty((m, n), np.float32)
    L.Tricublin_zyx1_m_n(d.ctypes.data, C.cast(fs, C.c_void_p), pos.ctypes.data, lv, n, m)
    assert np.array_equal(_bits(d), _bits(vec["zyx1"]))
    dnm = np.empty((n, m), np.float32)
    L.Tricublin_zyx1_n_m(dnm.ctypes.data, C.cast(fs, C.c_void_p), pos.ctypes.data, lv, n, m)
    assert np.array_equal(_bits(dnm.T), _bits(vec["zyx1"]))
    d1 = np.empty(n, np.float32)
    L.Tricublin_zyx1_n(d1.ctypes.data, fields[1].ctypes.data, pos.ctypes.data, lv, n)
    assert np.array_equal(_bits(d1), _bits(vec["zyx1"][1]))
    rows = [np.empty(n, np.float32) for _ in range(m)]
    dp = (C.c_void_p * m)(*[r.ctypes.data for r in rows])
    L.Tricublin_zyx1_p(C.cast(dp, C.c_void_p), C.cast(fs, C.c_void_p), pos.ctypes.data, lv, n, m)
    assert all(np.array_equal(_bits(rows[q]), _bits(vec["zyx1"][q])) for q in range(m))
    outs = [np.empty((m, n), np.float32) for _ in range(4)]
    L.Tricublin_mono_zyx_m_n(*(o.ctypes.data for o in outs), C.cast(fs, C.c_void_p), pos.ctypes.data, lv, n, m)
    for got, key in zip(outs, ("mono_d", "mono_lin", "mono_min", "mono_max")):
        assert np.array_equal(_bits(got), _bits(vec[key])), key
    outs = [np.empty((n, m), np.float32) for _ in range(4)]
    L.Tricublin_mono_zyx_n_m(*(o.ctypes.data for o in outs), C.cast(fs, C.c_void_p), pos.ctypes.data, lv, n, m)
    assert np.array_equal(_bits(outs[0].T), _bits(vec["mono_d"]))
    o1 = [np.empty(n, np.float32) for _ in range(4)]
    L.Tricublin_mono_zyx_n(*(o.ctypes.data for o in o1), fields[2].ctypes.data, pos.ctypes.data, lv, n)
    assert np.array_equal(_bits(o1[3]), _bits(vec["mono_max"][2]))
    f3 = np.ascontiguousarray(vec["f3"])
    d3 = np.empty((n, 3), np.float32)
    L.Tricublin_zyx3_n(d3.ctypes.data, f3.ctypes.data, pos.ctypes.data, lv, n)
    assert np.array_equal(_bits(d3), _bits(vec["zyx3"]))
    # a non-finite position is refused on the host before anything is staged:
    # the output is left as it was and the thread's status is ADZC_ERR_ARG
    bad = pos.copy()
    bad[n // 2, 0] = np.nan
    d1[:] = 7.0
    L.Tricublin_zyx1_n(d1.ctypes.data, fields[1].ctypes.data, bad.ctypes.data, lv, n)
    assert L.adzc_last_error() == 1 and np.all(d1 == 7.0)
    L.Tricublin_zyx1_n(d1.ctypes.data, fields[1].ctypes.data, pos.ctypes.data, lv, n)
    assert np.array_equal(_bits(d1), _bits(vec["zyx1"][1]))


def test_level_a_concurrent_threads(A, vec):
    """Level A calls from several host threads at once (the reference calls
    its interpolators from every OpenMP thread) stay bit-exact in every
    layout."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor
    L = A.lib()
    ni, nj, nk = int(vec["ni"]), int(vec["nj"]), int(vec["nk"])
    lev = np.ascontiguousarray(vec["levels"])
    lv = L.Vsearch_setup_plus(lev.ctypes.data, nk, ni, nj, int(vec["offi"]), int(vec["offj"]))
    fields = [np.ascontiguousarray(x) for x in vec["fields"]]
    pos = np.ascontiguousarray(vec["pos"])
    n, m = pos.shape[0], len(fields)
    fs = (C.c_void_p * m)(*[x.ctypes.data for x in fields])

    def work(t):
        ok = True
        for rep in range(6):
            which = (t + rep) % 3
            if which == 0:
                outs = [np.empty((m, n), np.float32) for _ in range(4)]
                L.Tricublin_mono_zyx_m_n(*(o.ctypes.data for o in outs), C.cast(fs, C.c_void_p), pos.ctypes.data,
                                         lv, n, m)
                ok &= all(np.array_equal(_bits(g), _bits(vec[k]))
                          for g, k in zip(outs, ("mono_d", "mono_lin", "mono_min", "mono_max")))
            elif which == 1:
                outs = [np.empty((n, m), np.float32) for _ in range(4)]
                L.Tricublin_mono_zyx_n_m(*(o.ctypes.data for o in outs), C.cast(fs, C.c_void_p), pos.ctypes.data,
                                         lv, n, m)
                ok &= all(np.array_equal(_bits(g.T), _bits(vec[k]))
                          for g, k in zip(outs, ("mono_d", "mono_lin", "mono_min", "mono_max")))
            else:
                rows = [np.empty(n, np.float32) for _ in range(m)]
                dp = (C.c_void_p * m)(*[r.ctypes.data for r in rows])
                L.Tricublin_zyx1_p(C.cast(dp, C.c_void_p), C.cast(fs, C.c_void_p), pos.ctypes.data, lv, n, m)
                ok &= all(np.array_equal(_bits(rows[q]), _bits(vec["zyx1"][q])) for q in range(m))
            ok &= L.adzc_last_error() == 0
        return ok

    with ThreadPoolExecutor(max_workers=8) as ex:
        assert all(ex.map(work, range(24)))


def test_selftest_kat_through_cuda_library(A):
    subprocess.run(["make", "-s", "-C", O.HERE, "kat_selftest"], check=True)
    exe = os.path.join(O.HERE, "kat_selftest")
    out = subprocess.run([exe, A.LIB_PATH], capture_output=True, text=True, check=True).stdout.splitlines()
    gold = open(os.path.join(GOLD, "selftest_reference.txt")).read().splitlines()
    assert out == gold


def test_fp64_and_mixed_interpolators_vs_oracle(A, vec):
    ni, nj = int(vec["ni"]), int(vec["nj"])
    offi, offj = int(vec["offi"]), int(vec["offj"])
    zt = A.Ztab(vec["levels"], ni, nj, offi, offj)
    zo = O.Ztab(vec["levels"], ni, nj, offi, offj)
    f64 = [np.ascontiguousarray(x, dtype=np.float64) for x in vec["fields"]]
    rng = np.random.default_rng(5)
    pos = vec["pos"].astype(np.float64) + rng.uniform(-1e-3, 1e-3, vec["pos"].shape) * (vec["pos"] > 3)
    ref = O.zyx1_m_n(f64, pos, zo)
    fd = [torch.from_numpy(x).cuda() for x in f64]
    pd = torch.from_numpy(pos).cuda()
    got = A.tricublin_m_n(zt, A.FP64, fd, pd).cpu().numpy()
    assert np.array_equal(_bits(got), _bits(ref))
    gm = A.tricublin_mono_m_n(zt, A.FP64, fd, pd)
    rm = O.mono_m_n(f64, pos, zo)
    for a, b in zip(gm, rm):
        assert np.array_equal(_bits(a.cpu().numpy()), _bits(b))
    f3 = np.ascontiguousarray(vec["f3"], dtype=np.float64)
    assert np.array_equal(_bits(A.tricublin_zyx3_n(zt, A.FP64, torch.from_numpy(f3).cuda(), pd).cpu().numpy()),
                          _bits(O.zyx3_n(f3, pos, zo)))
    # MIXED: FP32 fields, FP64 positions, FP32 sums
    f32 = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in vec["fields"]]
    gmx = A.tricublin_m_n(zt, A.MIXED, f32, pd).cpu().numpy().astype(np.float64)
    for q in range(len(f64)):
        scale = np.max(np.abs(ref[q]))
        assert np.max(np.abs(gmx[q] - ref[q])) / scale < MIXED_REL_TOL
    mm = [o.cpu().numpy().astype(np.float64) for o in A.tricublin_mono_m_n(zt, A.MIXED, f32, pd)]
    for a, b in zip(mm, rm):
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < MIXED_REL_TOL
    assert np.array_equal(mm[2], rm[2]) and np.array_equal(mm[3], rm[3])  # min/max are exact values


def test_empty_and_invalid_calls(A, vec):
    ni, nj = int(vec["ni"]), int(vec["nj"])
    zt = A.Ztab(vec["levels"], ni, nj)
    f = [torch.zeros(ni * nj * int(vec["nk"]), device="cuda")]
    d = A.tricublin_m_n(zt, A.REF32, f, torch.zeros((0, 3), device="cuda"))
    assert d.shape == (1, 0)
    with pytest.raises(A.AdzError) as e:
        A.Ztab(vec["levels"][:3], ni, nj)
    assert e.value.status == 3  # ADZC_ERR_NK
    import ctypes as C
    assert A.lib().adzc_tricublin_m_n(zt.ptr, 7, None, None, None, 1, 1, None) == 1  # ADZC_ERR_ARG


# ---------------------------------------------------------------- full step
def _inputs(cfg, dtype):
    from gem_b200 import synth
    inp = synth.make_inputs(cfg, dtype=torch.float64)
    np_in = {k: (v.numpy() if torch.is_tensor(v) else [t.numpy() for t in v]) for k, v in inp.items()}
    dev = {k: (v.to(dtype).cuda() if torch.is_tensor(v) else [t.to(dtype).cuda() for t in v]) for k, v in inp.items()}
    return np_in, dev


def _gpu_step(A, cfg, prec, dev, steps=2):
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    dt = A._field_dtype(prec)
    outs = None
    for _ in range(steps):
        outs = {k: torch.full(ad.ext_shape, float("nan"), dtype=dt, device="cuda") for k in ("u", "v", "w")}
        tro = [torch.full(ad.ext_shape, float("nan"), dtype=dt, device="cuda") for _ in dev["tracers"]]
        A.step_fused(ad, prec, cfg.dt, dev, dev, dev["tracers"], px, wp, outs, tro, cfg.mono)
        outs["tracers"] = tro
    assert ad.status() == 0
    torch.cuda.synchronize()
    return ad, px, wp, outs


def _oracle_step(cfg, kind, prec, np_in, steps=2):
    st = O.Step(cfg, kind=kind, prec=prec)
    st.inittraj()
    out = None
    for _ in range(steps):
        out = st.step(np_in)
    return st, out


@pytest.mark.parametrize("shape", [(48, 40, 20), (128, 128, 40)])
def test_step_ref32_bit_exact(A, shape):
    from gem_b200 import synth
    cfg = synth.config_small(*shape)
    cfg.mono = True
    np_in, dev = _inputs(cfg, torch.float32)
    kind = "ref" if O.have_ref() else "oracle"
    st, o_out = _oracle_step(cfg, kind, "f32", np_in)
    ad, px, wp, g_out = _gpu_step(A, cfg, A.REF32, dev)
    assert np.array_equal(_bits(px.cpu().numpy()), _bits(st.pxyzm))
    assert np.array_equal(_bits(wp.cpu().numpy()), _bits(st.wpxyz))
    for k, s in (("u", 1), ("v", 2), ("w", 3)):
        m = ad.range_mask(s).numpy()
        assert np.array_equal(_bits(g_out[k].cpu().numpy()[m]), _bits(o_out[k][m])), k
    m = ad.range_mask(3).numpy()
    for a, b in zip(g_out["tracers"], o_out["tracers"]):
        assert np.array_equal(_bits(a.cpu().numpy()[m]), _bits(b[m]))


@pytest.mark.parametrize("branch", ["schm_advec2", "schm_advec3", "slt_winds", "lam_gbpil_t", "mcrhsint"])
def test_step_ref32_reference_branches(A, branch):
    """The less common switches of the path, REF32 bit-exact with the
    reference interpolator and the driver restatement:
    Schm_advec 2 and 3 (dt split with the off-centering weights,
    B/adz_traject.F90:38-59), Adz_slt_winds (surface-layer winds for the
    top-level pt positions, B/adz_interp_traj.F90:123-133) and
    Lam_gbpil_t > 0 (a top pilot: k0 > 1, B/adz_set.F90:94-114) and the
    ensemble perturbation mcrhsint of every interpolation
    (B/adz_interp_hlt.F90:99-133, momentum and tracers, before the clip)."""
    from gem_b200 import synth
    cfg = synth.config_small(40, 36, 24)
    cfg.mono = True
    kw = {"schm_advec2": dict(schm_advec=2), "schm_advec3": dict(schm_advec=3),
          "slt_winds": dict(slt_winds=True), "lam_gbpil_t": dict(lam_gbpil_t=4), "mcrhsint": {}}[branch]
    np_in, dev = _inputs(cfg, torch.float32)
    kind = "ref" if O.have_ref() else "oracle"
    st = O.Step(cfg, kind=kind, prec="f32", **kw)
    st.inittraj()
    ad = A.Adz.from_config(cfg, **kw)
    if branch == "slt_winds":
        ad.set_slt_winds(dev["uslt"], dev["vslt"])
    if branch == "mcrhsint":
        mc = np.random.default_rng(23).uniform(-0.5, 0.5, (cfg.nj, cfg.ni)).astype(np.float32)
        st.set_rhs_perturbation(mc)
        ad.set_rhs_perturbation(torch.from_numpy(mc).cuda())
    px, wp = ad.new_state(A.REF32)
    ad.adz_inittraj(A.REF32, px, wp)
    for _ in range(2):
        o_out = st.step(np_in)
        outs = {k: torch.full(ad.ext_shape, float("nan"), dtype=torch.float32, device="cuda") for k in ("u", "v", "w")}
        tro = [torch.full(ad.ext_shape, float("nan"), dtype=torch.float32, device="cuda") for _ in dev["tracers"]]
        A.step_fused(ad, A.REF32, cfg.dt, dev, dev, dev["tracers"], px, wp, outs, tro, cfg.mono)
    assert ad.status() == 0
    torch.cuda.synchronize()
    assert np.array_equal(_bits(px.cpu().numpy()), _bits(st.pxyzm))
    assert np.array_equal(_bits(wp.cpu().numpy()), _bits(st.wpxyz))
    for k, s in (("u", 1), ("v", 2), ("w", 3)):
        m = ad.range_mask(s).numpy()
        assert m.any()
        assert np.array_equal(_bits(outs[k].cpu().numpy()[m]), _bits(o_out[k][m])), k
    m = ad.range_mask(3).numpy()
    for a, b in zip(tro, o_out["tracers"]):
        assert np.array_equal(_bits(a.cpu().numpy()[m]), _bits(b[m]))
    if branch == "mcrhsint":  # the pattern changes the results
        ad.set_rhs_perturbation(None)
        plain = torch.zeros(ad.ext_shape, dtype=torch.float32, device="cuda")
        ad.adz_tricub_hlt(A.REF32, A.SET_U, [dev["src_u"]], [plain])
        torch.cuda.synchronize()
        m = ad.range_mask(1).numpy()
        assert not np.array_equal(_bits(plain.cpu().numpy()[m]), _bits(outs["u"].cpu().numpy()[m]))
    if branch == "slt_winds":  # the switch changes the top-level results
        ad2 = A.Adz.from_config(cfg)
        px2, wp2 = ad2.new_state(A.REF32)
        ad2.adz_inittraj(A.REF32, px2, wp2)
        o2 = [torch.zeros(ad.ext_shape, dtype=torch.float32, device="cuda") for _ in range(3)]
        for _ in range(2):
            A.step_fused(ad2, A.REF32, cfg.dt, dev, dev, [], px2, wp2, dict(zip("uvw", o2)), [], cfg.mono)
        torch.cuda.synchronize()
        top = np.zeros(ad.ext_shape, bool)
        top[-1] = True
        mw = ad.range_mask(3).numpy() & top
        assert not np.array_equal(_bits(o2[2].cpu().numpy()[mw]), _bits(outs["w"].cpu().numpy()[mw]))


@pytest.mark.parametrize("lam", [True, False])
def test_cfl_above_maxcfl_clips(A, lam):
    """Winds of about twice maxcfl grid lengths per step.  Departure points are
    clipped to the adz_set bounds: on a LAM-edge tile the BCS_BASE bounds, on
    an interior tile the halo (B/adz_set.F90:123-160, B/adz_traject.F90:94-98).
    No stencil leaves the extended array (status 0, nothing read out of
    bounds), and the REF32 step stays bit-exact with the reference."""
    from gem_b200 import synth
    cfg = synth.config_small(48, 40, 20)
    cfg.u0 = 2.0 * cfg.maxcfl * cfg.dx / cfg.dt
    cfg.phase = (0.5, 0.25)  # strongest eastward wind on the west edge: departures leave the tile
    cfg.mono = True
    np_in, dev = _inputs(cfg, torch.float32)
    kind = "ref" if O.have_ref() else "oracle"
    st = O.Step(cfg, kind=kind, prec="f32", lam=lam)
    st.inittraj()
    ad = A.Adz.from_config(cfg, lam=lam)
    px, wp = ad.new_state(A.REF32)
    ad.adz_inittraj(A.REF32, px, wp)
    for _ in range(2):
        o_out = st.step(np_in)
        outs = {k: torch.full(ad.ext_shape, float("nan"), dtype=torch.float32, device="cuda") for k in ("u", "v", "w")}
        tro = [torch.full(ad.ext_shape, float("nan"), dtype=torch.float32, device="cuda") for _ in dev["tracers"]]
        A.step_fused(ad, A.REF32, cfg.dt, dev, dev, dev["tracers"], px, wp, outs, tro, cfg.mono)
    assert ad.status() == 0
    torch.cuda.synchronize()
    pxc = px.cpu().numpy()
    lo, hi = np.float32(ad.info.iminposx), np.float32(ad.info.imaxposx)
    clipped = int(np.sum(pxc[..., 0] == lo) + np.sum(pxc[..., 0] == hi))
    assert clipped > 0  # the clip is exercised
    assert np.array_equal(_bits(pxc), _bits(st.pxyzm))
    assert np.array_equal(_bits(wp.cpu().numpy()), _bits(st.wpxyz))
    for k, s in (("u", 1), ("v", 2), ("w", 3)):
        m = ad.range_mask(s).numpy()
        assert np.array_equal(_bits(outs[k].cpu().numpy()[m]), _bits(o_out[k][m])), k
    m = ad.range_mask(3).numpy()
    for a, b in zip(tro, o_out["tracers"]):
        assert np.array_equal(_bits(a.cpu().numpy()[m]), _bits(b[m]))


@pytest.mark.parametrize("prec_name", ["ref32", "fp64"])
def test_step_bit_exact_full_size(A, prec_name):
    """The benchmark tile itself: 1024x1024x80 (84 M arrival points, ext
    arrays of 85 M cells), u, v, w + 4 tracers, a cold and a warm step, bit
    for bit on every point of every set: REF32 against the reference-linked
    oracle, FP64 against the FP64 oracle.  The oracle runs on all host cores."""
    from gem_b200 import synth
    prec = A.PREC_NAMES[prec_name]
    dt = A._field_dtype(prec)
    cfg = synth.config_large(1024, 1024, 80)
    cfg.mono = True
    dev = synth.make_inputs(cfg, device="cuda", dtype=dt)
    np_in = {k: (v.cpu().numpy() if torch.is_tensor(v) else [t.cpu().numpy() for t in v]) for k, v in dev.items()}
    if prec == A.REF32:
        st = O.Step(cfg, kind="ref" if O.have_ref() else "oracle", prec="f32", threads=os.cpu_count() or 1)
    else:
        st = O.Step(cfg, kind="oracle", prec="f64", threads=os.cpu_count() or 1)
    st.inittraj()
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    outs = {k: torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for k in ("u", "v", "w")}
    tro = [torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for _ in dev["tracers"]]
    for _ in range(2):
        o_out = st.step(np_in)
        A.step_fused(ad, prec, cfg.dt, dev, dev, dev["tracers"], px, wp, outs, tro, cfg.mono)
    assert ad.status() == 0
    torch.cuda.synchronize()
    if prec == A.REF32:
        assert np.array_equal(_bits(px.cpu().numpy()), _bits(st.pxyzm))
    assert np.array_equal(_bits(wp.cpu().numpy()), _bits(st.wpxyz))
    for k, s in (("u", 1), ("v", 2), ("w", 3)):
        m = ad.range_mask(s).numpy()
        assert np.array_equal(_bits(outs[k].cpu().numpy()[m]), _bits(o_out[k][m])), k
    m = ad.range_mask(3).numpy()
    for a, b in zip(tro, o_out["tracers"]):
        assert np.array_equal(_bits(a.cpu().numpy()[m]), _bits(b[m]))


def test_step_fp64_bit_exact_stretched_levels(A):
    from gem_b200 import synth
    cfg = synth.config_large(96, 80, 80)
    np_in, dev = _inputs(cfg, torch.float64)
    st, o_out = _oracle_step(cfg, "oracle", "f64", np_in)
    ad, px, wp, g_out = _gpu_step(A, cfg, A.FP64, dev)
    assert np.array_equal(_bits(wp.cpu().numpy()), _bits(st.wpxyz))
    for k, s in (("u", 1), ("v", 2), ("w", 3)):
        m = ad.range_mask(s).numpy()
        assert np.array_equal(_bits(g_out[k].cpu().numpy()[m]), _bits(o_out[k][m])), k
    m = ad.range_mask(3).numpy()
    for a, b in zip(g_out["tracers"], o_out["tracers"]):
        assert np.array_equal(_bits(a.cpu().numpy()[m]), _bits(b[m]))


def test_step_mixed_vs_fp64_oracle(A):
    """MIXED step against the FP64 oracle fed the same FP32 inputs."""
    from gem_b200 import synth
    cfg = synth.config_mixed(96, 80, 80)
    np_in, dev = _inputs(cfg, torch.float32)
    np64 = {k: (v.astype(np.float32).astype(np.float64) if not isinstance(v, list)
                else [t.astype(np.float32).astype(np.float64) for t in v]) for k, v in np_in.items()}
    st, o_out = _oracle_step(cfg, "oracle", "f64", np64)
    ad, px, wp, g_out = _gpu_step(A, cfg, A.MIXED, dev)
    w = wp.cpu().numpy()
    inner = (slice(None), slice(None), slice(2, -2), slice(2, -2))
    assert np.max(np.abs(w[inner] - st.wpxyz[inner])) < 1e-4  # positions, in grid cells
    for k, s in (("u", 1), ("v", 2), ("w", 3)):
        m = ad.range_mask(s).numpy()
        a, b = g_out[k].cpu().numpy()[m].astype(np.float64), o_out[k][m]
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-5, k
    m = ad.range_mask(3).numpy()
    for a, b in zip(g_out["tracers"], o_out["tracers"]):
        a, b = a.cpu().numpy()[m].astype(np.float64), b[m]
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-5


def test_mixed_interp_tolerance_same_positions(A):
    """MIXED interpolation error alone (identical FP64 positions): <= 1e-6."""
    from gem_b200 import synth
    cfg = synth.config_mixed(96, 80, 80)
    np_in, dev = _inputs(cfg, torch.float32)
    ad = A.Adz.from_config(cfg)
    I = ad.info
    rng = np.random.default_rng(11)
    n = 200000
    pos = np.stack([rng.uniform(I.iminposx, I.imaxposx, n), rng.uniform(I.iminposy, I.imaxposy, n),
                    rng.uniform(0.2, cfg.nk + 0.8, n)], 1)
    lev = cfg.levels.zt[1:cfg.nk + 1]
    zt = A.Ztab(lev, I.nit, I.njt, 1 - 1 + I.halox - 0, I.haloy)
    zo = O.Ztab(lev, I.nit, I.njt, I.halox, I.haloy)
    flds = [np_in["tracers"][q].astype(np.float32) for q in range(len(np_in["tracers"]))]
    ref = O.zyx1_m_n([f.astype(np.float64).ravel() for f in flds], pos, zo)
    got = A.tricublin_m_n(zt, A.MIXED, [torch.from_numpy(f.ravel()).cuda() for f in flds],
                          torch.from_numpy(pos).cuda()).cpu().numpy().astype(np.float64)
    for q in range(len(flds)):
        assert np.max(np.abs(got[q] - ref[q])) / np.max(np.abs(ref[q])) <= MIXED_REL_TOL
    off_g, zl_g = O.cells(pos, zo)
    off_r, zl_r = O.cells(pos.astype(np.float32), zo)
    assert np.array_equal(off_g, off_r) and np.array_equal(zl_g, zl_r)


def test_nonfinite_wind_sets_status(A):
    from gem_b200 import synth
    cfg = synth.config_small(40, 36, 16)
    np_in, dev = _inputs(cfg, torch.float32)
    dev["uu_ext"][5, 10:12, 10:12] = float("nan")
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(A.REF32)
    ad.adz_inittraj(A.REF32, px, wp)
    ad.adz_traject(A.REF32, cfg.dt, dev, px, wp)
    assert ad.status() in (4, 5)
    assert ad.status() == 0  # reset by the previous read


def test_step_mixed_wide_plane_unions(A):
    """Strong vertical wind noise scatters the departure levels of neighbouring
    points over many thin bottom layers (warps whose lanes span more than 8
    levels), including linear-z points at the bottom level, with mono bounds
    and clipping on every field.  One trajectory iteration on both sides keeps
    the comparison well conditioned (iterating a map whose vertical Lipschitz
    constant dt*dw/dz is far above 1 would amplify FP32/FP64 differences)."""
    from gem_b200 import synth
    cfg = synth.config_mixed(96, 80, 80)
    cfg.noise = 6.0
    np_in, dev = _inputs(cfg, torch.float32)
    np64 = {k: (v.astype(np.float32).astype(np.float64) if not isinstance(v, list)
                else [t.astype(np.float32).astype(np.float64) for t in v]) for k, v in np_in.items()}
    st = O.Step(cfg, kind="oracle", prec="f64")
    st.inittraj()
    st.traject(np64, niter=1)
    ref = st.tricub(3, [np64["src_w"]] + np64["tracers"], mono=True, clip=True)
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(A.MIXED)
    ad.adz_inittraj(A.MIXED, px, wp)
    ad.adz_traject(A.MIXED, cfg.dt, dev, px, wp, niter=1)
    srcs = [dev["src_w"]] + dev["tracers"]
    outs = [torch.full(ad.ext_shape, float("nan"), device="cuda") for _ in srcs]
    ad.adz_tricub_sets(A.MIXED, [0, 0, 0, len(srcs)], srcs, outs, [1] * len(srcs))
    assert ad.status() == 0
    # the oracle clips w as well here (mono on every field)
    m = ad.range_mask(3).numpy()
    # many warps span more than 8 levels in this case
    p = st.sets[3]
    iz = np.clip(np.trunc(p[:, 2].astype(np.float32)).astype(int), 1, cfg.nk - 1) - 1
    zl = (iz < 1) | (iz > cfg.nk - 3)
    zb = np.where(zl, iz, iz - 1)
    zh = np.where(zl, zb + 1, zb + 3)
    n = len(zb) // 32 * 32
    U = zh[:n].reshape(-1, 32).max(1) - zb[:n].reshape(-1, 32).min(1) + 1
    assert (U > 8).sum() > 100
    for a, b in zip(outs, ref):
        a, b = a.cpu().numpy()[m].astype(np.float64), b[m]
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-5
