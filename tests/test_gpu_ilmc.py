"""ILMC (adzc_ilmc) against the sequential restatement (oracle/adz_oracle_impl.h:
orc_ilmc) on the same fields: bit-exact, FP32 and FP64, sparse and dense
violations (the dense case needs many rounds of the order-preserving parallel
schedule), sweeps 1 to 3, with and without the final clip."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _fields(st, dt, frac, seed):
    rng = np.random.default_rng(seed)
    sh = st.ext_shape
    mn = rng.random(sh).astype(dt)
    mx = (mn + 0.5 + rng.random(sh)).astype(dt)
    f = (mn + (mx - mn) * rng.random(sh)).astype(dt)
    air = (1.0 + 0.3 * rng.random(sh)).astype(dt)
    viol = rng.random(sh) < frac
    f = np.where(viol, np.where(rng.random(sh) < 0.5, mx + 0.3 * rng.random(sh), mn - 0.3 * rng.random(sh)),
                 f).astype(dt)
    return f, mn, mx, air


@pytest.mark.parametrize("prec_name,frac,sweeps,min_max", [("mixed", 0.01, 2, True), ("fp64", 0.01, 2, False),
                                                            ("ref32", 0.2, 2, True), ("mixed", 0.05, 1, False),
                                                            ("fp64", 0.05, 3, True), ("mixed", 0.2, 4, True)])
def test_ilmc_bit_exact(prec_name, frac, sweeps, min_max):
    from gem_b200 import adz as A, synth
    from oracle import oracle as O
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    prec = A.PREC_NAMES[prec_name]
    cfg = synth.config_small(40, 36, 16)
    st = O.Step(cfg, "oracle", "f64" if prec == A.FP64 else "f32")
    dt = np.float64 if prec == A.FP64 else np.float32
    trs = [_fields(st, dt, frac, seed) for seed in (3, 4)]
    air = trs[0][3]
    ad = A.Adz.from_config(cfg)
    fs = [torch.from_numpy(t[0].copy()).cuda() for t in trs]
    mns = [torch.from_numpy(t[1]).cuda() for t in trs]
    mxs = [torch.from_numpy(t[2]).cuda() for t in trs]
    rounds = A.ilmc(ad, prec, fs, mns, mxs, torch.from_numpy(air).cuda(), sweep_max=sweeps, min_max=min_max)
    torch.cuda.synchronize()
    assert rounds >= 1
    for t, g in zip(trs, fs):
        ref = st.ilmc(t[0], t[1], t[2], air, sweep_max=sweeps, min_max=min_max)
        got = g.cpu().numpy()
        diff = int(np.sum(got != ref))
        assert diff == 0, (diff, rounds)
        assert not np.array_equal(ref, t[0])  # the filter did something
