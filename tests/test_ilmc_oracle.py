"""ILMC restatement (oracle/adz_oracle_impl.h: orc_ilmc), pinned without the
Fortran reference by the scheme's invariants on fields with seeded over- and
undershoots: the air-mass-weighted total over the domain is conserved while
no neighbour is clamped, every point ends inside its bounds after the final
clip, points already inside their bounds far from any violation are left
untouched, and nothing outside the filtered region changes."""
import numpy as np
import pytest


def _case(prec, frac=0.01, seed=3):
    from gem_b200 import synth
    from oracle import oracle as O
    cfg = synth.config_small(40, 36, 16)
    st = O.Step(cfg, "oracle", prec)
    rng = np.random.default_rng(seed)
    sh = st.ext_shape
    dt = np.float32 if prec == "f32" else np.float64
    mn = rng.random(sh).astype(dt)
    mx = (mn + 0.5 + rng.random(sh)).astype(dt)
    f = (mn + (mx - mn) * rng.random(sh)).astype(dt)
    air = (1.0 + 0.3 * rng.random(sh)).astype(dt)
    viol = rng.random(sh) < frac
    f = np.where(viol, np.where(rng.random(sh) < 0.5, mx + 0.3 * rng.random(sh), mn - 0.3 * rng.random(sh)),
                 f).astype(dt)
    return cfg, st, f, mn, mx, air


def _region(st, cfg):
    s, H = st.s, cfg.halo
    return (slice(s.k0t - 1, cfg.nk), slice(s.j0 - 1 + H, s.jn + H), slice(s.i0 - 1 + H, s.in_ + H))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_ilmc_invariants(prec):
    cfg, st, f, mn, mx, air = _case(prec)
    sl = _region(st, cfg)
    out = st.ilmc(f, mn, mx, air, sweep_max=2, min_max=False)
    mass0 = np.sum(f[sl].astype(np.float64) * air[sl])
    mass1 = np.sum(out[sl].astype(np.float64) * air[sl])
    tol = 1e-5 if prec == "f32" else 1e-12
    assert abs(mass1 - mass0) <= tol * mass0
    viol = (f[sl] > mx[sl]) | (f[sl] < mn[sl])
    assert ((out[sl] > mx[sl]) | (out[sl] < mn[sl])).sum() < viol.sum() / 4
    clipped = st.ilmc(f, mn, mx, air, sweep_max=2, min_max=True)
    assert np.all(clipped[sl] >= mn[sl]) and np.all(clipped[sl] <= mx[sl])
    # far from every violation nothing moves
    from scipy.ndimage import binary_dilation
    near = binary_dilation(viol, structure=np.ones((5, 5, 5), bool))
    assert np.array_equal(out[sl][~near], f[sl][~near])
    # outside the region nothing moves
    m = np.ones(f.shape, bool)
    m[sl] = False
    assert np.array_equal(out[m], f[m])
