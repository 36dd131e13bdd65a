"""CFL diagnostic and restart state.  adzc_cfl against the restatement of
adz_courant (oracle/oracle.py: adz_cfl) on the same departure points:
bit-exact values and indices.  adzc_state_save/load: a step after restoring
the state into a fresh handle reproduces, bit for bit, the step of the handle
that kept running (REF32 with its FP32 positions, and MIXED)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _setup(prec_name, shape=(48, 40, 20)):
    from gem_b200 import adz as A, synth
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    prec = A.PREC_NAMES[prec_name]
    cfg = synth.config_small(*shape)
    cfg.mono = True
    inp = synth.make_inputs(cfg, device="cuda", dtype=A._field_dtype(prec))
    return A, prec, cfg, inp


def test_cfl_bit_exact():
    A, prec, cfg, inp = _setup("mixed")
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    ad.adz_traject(prec, cfg.dt, inp, px, wp)
    cfl, idx = ad.adz_cfl(wp)
    I = ad.info
    ref, ridx = O.adz_cfl(wp.cpu().numpy(), I.i0, I.in_, I.j0, I.jn, I.k0, cfg.nk)
    assert np.array_equal(cfl.view(np.int64), ref.view(np.int64)), (cfl, ref)
    assert np.array_equal(idx, ridx), (idx, ridx)
    # before any trajectory (departure = arrival): all zero, index 0 + offset
    _, wp0 = ad.new_state(prec)
    ad.adz_inittraj(prec, None, wp0)
    cfl0, idx0 = ad.adz_cfl(wp0)
    assert np.all(cfl0 == 0.0) and np.array_equal(idx0[:, 2], [0, 0, 0])


@pytest.mark.parametrize("prec_name", ["ref32", "mixed"])
def test_restart_state_round_trip(prec_name, tmp_path):
    A, prec, cfg, inp = _setup(prec_name)
    dt = A._field_dtype(prec)
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    nan = lambda: torch.full(ad.ext_shape, float("nan"), dtype=dt, device="cuda")  # noqa: E731

    def step(h, px_, wp_):
        outs = {k: nan() for k in ("u", "v", "w")}
        tro = [nan() for _ in inp["tracers"]]
        A.step_fused(h, prec, cfg.dt, inp, inp, inp["tracers"], px_, wp_, outs, tro, cfg.mono)
        torch.cuda.synchronize()
        return [wp_.cpu().numpy().copy()] + [o.cpu().numpy() for o in (outs["u"], outs["v"], outs["w"], *tro)]

    step(ad, px, wp)  # cold start (6 updates)
    path = str(tmp_path / "adz_state.bin")
    ad.state_save(prec, px, wp, path)
    ref = step(ad, px, wp)  # warm step of the running handle
    fresh = A.Adz.from_config(cfg)
    px2, wp2 = fresh.new_state(prec)
    fresh.state_load(prec, px2, wp2, path)
    got = step(fresh, px2, wp2)
    for a, b in zip(ref, got):
        assert np.array_equal(np.isnan(a), np.isnan(b))
        assert np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)])
    # a file of another precision or size is refused
    other = A.Adz.from_config(synth_small(cfg))
    pxo, wpo = other.new_state(prec)
    with pytest.raises(A.AdzError):
        other.state_load(prec, pxo, wpo, path)


def synth_small(cfg):
    from gem_b200 import synth
    return synth.config_small(cfg.ni + 8, cfg.nj, cfg.nk)
