"""Batched uneven domains (adzc_batch_*): one persistent launch steps every
domain exactly as the per-domain entry points do (adzc_traject, then
adzc_tricub_sets).  Tolerance: bit-exact; the batch runs the same per-point
device code on the same inputs, only the work is split and ordered
differently.  The domains are a scaled-down draw of the uneven-domain case
(sizes 40-96, 16-40 levels, 1-20 log-normal tracers, so one domain has two
field groups in its thermo set)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a.view(np.int64)


def _domains(prec, n=5, seed=77):
    from gem_b200 import adz, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    cfgs = synth.config_batch(n=n, seed=seed, size=(40, 96), levels=(16, 40), tracers=(1, 20))
    cfgs[0].ntracers = 20  # T set: w + 20 tracers -> two field groups
    dt = adz._field_dtype(prec)
    doms = []
    for cfg in cfgs:
        ad = adz.Adz.from_config(cfg)
        inp = synth.make_inputs(cfg, device="cuda", dtype=dt)
        _, wp = ad.new_state(prec)
        ad.adz_inittraj(prec, None, wp)
        ad.adz_traject(prec, cfg.dt, inp, None, wp)  # cold start, outside the batch
        doms.append((cfg, ad, inp, wp))
    assert ad.status() == 0
    return adz, doms


def _outs(ad, inp, dt):
    return [torch.full(ad.ext_shape, -7.0, dtype=dt, device="cuda") for _ in range(3 + len(inp["tracers"]))]


def _sources(inp):
    return [inp["src_u"], inp["src_v"], inp["src_w"]] + list(inp["tracers"])


def _regular_step(adz, prec, cfg, ad, inp, wp, outs):
    ntr = len(inp["tracers"])
    ad.adz_traject(prec, cfg.dt, inp, None, wp)
    ad.adz_tricub_sets(prec, [0, 1, 1, 1 + ntr], _sources(inp), outs, [0, 0, 0] + [1] * ntr)


def _batch(adz, prec, doms, wps, outs):
    spec = []
    for (cfg, ad, inp, _), wp, o in zip(doms, wps, outs):
        ntr = len(inp["tracers"])
        spec.append(dict(adz=ad, dt=cfg.dt, winds=inp, wpxyz=wp, nfields=[0, 1, 1, 1 + ntr],
                         srcs=_sources(inp), dsts=o, mono=[0, 0, 0] + [1] * ntr))
    return adz.Batch(prec, spec)


def _snap(wp, outs):
    torch.cuda.synchronize()
    return [wp.cpu().numpy().copy()] + [o.cpu().numpy().copy() for o in outs]


def _compare(a, b, what):
    for q, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(_bits(x), _bits(y)), f"{what}: array {q} differs"


@pytest.mark.parametrize("precname,plan", [("mixed", None), ("fp64", None), ("mixed", (8, 2)), ("mixed", (2, 3)),
                                           ("fp64", (32, 3)), ("mixed", (8, 4)), ("fp64", (8, 4)),
                                           ("mixed", (8, 5)), ("fp64", (8, 5))])
def test_batch_matches_per_domain_steps(precname, plan):
    """plan None: the default one-launch plan; (rows, 0..2): that register
    budget of the one-launch kernel; (rows, 3): the phased plan; (rows, 4):
    every domain's own launches in the graph; (rows, 5): the same on
    concurrent graph branches."""
    from gem_b200 import adz as A
    prec = A.PREC_NAMES[precname]
    adz, doms = _domains(prec)
    dt = adz._field_dtype(prec)
    wps_b = [wp.clone() for (_, _, _, wp) in doms]
    outs_b = [_outs(ad, inp, dt) for (_, ad, inp, _) in doms]
    batch = _batch(adz, prec, doms, wps_b, outs_b)
    if plan is not None:
        batch.select(*plan)
    q = batch.query()
    per_domain = plan is not None and plan[1] in (adz.Batch.DOMAINS, adz.Batch.DOMAINS_CONCURRENT)
    assert q["items"] > 0 and (q["blocks_per_sm"] == 0 if per_domain else q["blocks_per_sm"] >= 1)
    assert q["plan"].startswith("phased") == (plan is not None and plan[1] == adz.Batch.PHASED)
    assert q["plan"].startswith("per-domain") == per_domain
    assert q["plan"].endswith("concurrent branches") == (plan is not None and plan[1] == adz.Batch.DOMAINS_CONCURRENT)
    if plan is not None:
        assert q["rows_per_item"] == plan[0]
    for step in range(2):
        batch.step()
        assert batch.status() == 0
        snaps_b = [_snap(wp, o) for wp, o in zip(wps_b, outs_b)]
        for d, (cfg, ad, inp, wp) in enumerate(doms):
            o = _outs(ad, inp, dt)
            _regular_step(adz, prec, cfg, ad, inp, wp, o)
            assert ad.status() == 0
            _compare(_snap(wp, o), snaps_b[d], f"step {step} domain {d}")


def test_batch_tune_then_step():
    """The tuner's timed launches are real steps; afterwards the captured plan
    must still reproduce the per-domain step from the same positions, and
    adzc_tricub on a handle must see the positions the batch wrote."""
    from gem_b200 import adz as A
    prec = A.MIXED
    adz, doms = _domains(prec, n=4, seed=91)
    dt = adz._field_dtype(prec)
    wps_b = [wp.clone() for (_, _, _, wp) in doms]
    outs_b = [_outs(ad, inp, dt) for (_, ad, inp, _) in doms]
    batch = _batch(adz, prec, doms, wps_b, outs_b)
    batch.tune()
    assert batch.status() == 0
    q = batch.query()
    assert q["rows_per_item"] in (2, 8, 32)
    t = batch.tuned()  # every plan family was timed, and the kept plan is the fastest
    assert all(v is not None and v > 0 for v in t.values())
    kept = {"one launch": "one_launch", "phased (one launch per phase)": "phased"}.get(q["plan"], "per_domain")
    assert t[kept] == min(t.values())
    for (_, _, _, wp), wb in zip(doms, wps_b):
        wp.copy_(wb)
    batch.step()
    assert batch.status() == 0
    snaps_b = [_snap(wp, o) for wp, o in zip(wps_b, outs_b)]
    # the handles now point at the batch's positions
    cfg, ad, inp, _ = doms[1]
    extra = torch.full(ad.ext_shape, -7.0, dtype=dt, device="cuda")
    ad.adz_tricub_hlt(prec, A.SET_U, [inp["src_u"]], [extra])
    torch.cuda.synchronize()
    assert np.array_equal(_bits(extra.cpu().numpy()), _bits(snaps_b[1][1]))
    for d, (cfg, ad, inp, wp) in enumerate(doms):
        o = _outs(ad, inp, dt)
        _regular_step(adz, prec, cfg, ad, inp, wp, o)
        assert ad.status() == 0
        _compare(_snap(wp, o), snaps_b[d], f"tuned domain {d}")


def test_batch_rejects_bad_domains():
    from gem_b200 import adz as A
    adz, doms = _domains(A.MIXED, n=2, seed=5)
    dt = adz._field_dtype(A.MIXED)
    wps = [wp.clone() for (_, _, _, wp) in doms]
    outs = [_outs(ad, inp, dt) for (_, ad, inp, _) in doms]
    with pytest.raises(adz.AdzError):
        adz.Batch(A.REF32, [])  # no domains / REF32 not batched
    ok = _batch(adz, A.MIXED, doms, wps, outs)
    for rows, plan in ((0, 0), (8, -1), (8, 6)):
        with pytest.raises(adz.AdzError):
            ok.select(rows, plan)
    # a handle still in its cold start is refused
    cfg, _, inp, _ = doms[0]
    fresh = adz.Adz.from_config(cfg)
    ntr = len(inp["tracers"])
    with pytest.raises(adz.AdzError):
        adz.Batch(A.MIXED, [dict(adz=fresh, dt=cfg.dt, winds=inp, wpxyz=wps[0], nfields=[0, 1, 1, 1 + ntr],
                                 srcs=_sources(inp), dsts=outs[0], mono=[0, 0, 0] + [1] * ntr)])


def test_batch_wait_times_out_and_recovers():
    """Failure detection without a GPU fault: domain 0's trajectory items are
    made to wait for departure-wind items that do not exist (host-side
    injection) under a short wait bound.  The waits run out, the kernel skips
    those items and completes, the host reads ADZC_ERR_TIMEOUT, and the next
    step (fault cleared, same positions) is bit-exact with the per-domain
    entry points: the context stays usable."""
    import time
    from gem_b200 import adz as A
    prec = A.MIXED
    adz, doms = _domains(prec, n=2, seed=13)
    dt = adz._field_dtype(prec)
    wps_b = [wp.clone() for (_, _, _, wp) in doms]
    outs_b = [_outs(ad, inp, dt) for (_, ad, inp, _) in doms]
    batch = _batch(adz, prec, doms, wps_b, outs_b)
    batch.select(8, 0)  # the one-launch plan: the phased plan has no waits
    batch.inject(adz.Batch.INJECT_SPINS, 4096)
    batch.inject(adz.Batch.INJECT_NEED, 1)
    t0 = time.time()
    batch.step()
    assert batch.status() == 6  # ADZC_ERR_TIMEOUT
    assert time.time() - t0 < 60
    assert batch.status() == 0  # read and reset
    batch.inject(adz.Batch.INJECT_NEED, 0)
    batch.inject(adz.Batch.INJECT_SPINS, 0)
    for (_, _, _, wp), wb in zip(doms, wps_b):
        wb.copy_(wp)
    batch.step()
    assert batch.status() == 0
    snaps_b = [_snap(wp, o) for wp, o in zip(wps_b, outs_b)]
    for d, (cfg, ad, inp, wp) in enumerate(doms):
        o = _outs(ad, inp, dt)
        _regular_step(adz, prec, cfg, ad, inp, wp, o)
        assert ad.status() == 0
        _compare(_snap(wp, o), snaps_b[d], f"after recovery, domain {d}")
    with pytest.raises(adz.AdzError):
        batch.inject(9, 1)
