"""Bermejo-Conde restatement (oracle/adz_oracle_impl.h: orc_bermejo_conde),
pinned without the Fortran reference: against an independent numpy
restatement of Bermejo_Conde.F90 (weights, lambda, clipped correction,
proportional rescale, epsilon) on an FP64 advection step of the oracle
itself, and against the scheme's invariant (the fixed total equals the
total before advection minus the carried epsilon)."""
import numpy as np
import pytest
import torch


def _case():
    from gem_b200 import synth
    from oracle import oracle as O
    cfg = synth.config_small(48, 40, 16)
    cfg.ntracers, cfg.tracer_kind = 2, "lognormal"
    inp = synth.make_inputs(cfg, "cpu", torch.float64)
    st = O.Step(cfg, "oracle", "f64")
    st.inittraj()
    st.traject({k: inp[k].numpy() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")})
    trs = [t.numpy() for t in inp["tracers"]]
    m, (lin, mn, mx) = st.tricub(3, trs, mono=True, clip=False, post=True)
    rng = np.random.default_rng(5)
    sh = st.ext_shape
    airm_p = 1.0 + 0.2 * rng.random(sh)
    airm_m = airm_p * (1 + 0.01 * rng.random(sh))
    mask = cfg.dx ** 2 * (0.5 + rng.random((cfg.nj, cfg.ni)))
    z = np.nan_to_num
    return cfg, st, trs, [z(x) for x in m], [z(x) for x in lin], [z(x) for x in mn], [z(x) for x in mx], \
        airm_p, airm_m, mask


def _numpy_bc(cfg, st, p, m, lin, mn, mx, airm_p, airm_m, mask, deficit, min_max):
    g, s, H = st.grid, st.s, cfg.halo
    i0, i1 = 1 + g.pil_w * g.west, cfg.ni - g.pil_e * g.east
    j0, j1 = 1 + g.pil_s * g.south, cfg.nj - g.pil_n * g.north
    sl = (slice(s.k0t - 1, cfg.nk), slice(j0 - 1 + H, j1 + H), slice(i0 - 1 + H, i1 + H))
    mk = mask[j0 - 1:j1, i0 - 1:i1][None]
    mass = lambda f, a: np.sum(f[sl] * a[sl] * mk)  # noqa: E731
    tot_p = mass(p, airm_p) - deficit
    de = mass(m, airm_m) - tot_p
    hml = m[sl] - lin[sl]
    sd = -1.0 if np.signbit(de) else 1.0
    w = np.where(np.where(np.signbit(hml), -1.0, 1.0) == sd, np.abs(hml) * sd, 0.0)
    wf = np.zeros_like(m)
    wf[sl] = w
    lam = de / mass(wf, airm_m)
    out = m.copy()
    corr = lam * w
    new = m[sl] - corr
    if min_max:
        new = np.where((corr > 0) & (new < mn[sl]), mn[sl], new)
        new = np.where((corr < 0) & (new > mx[sl]), mx[sl], new)
    out[sl] = new
    if min_max:
        out[sl] = tot_p / mass(out, airm_m) * out[sl]
    return out, mass(out, airm_m) - tot_p, tot_p


@pytest.mark.parametrize("min_max", [False, True])
def test_oracle_bc_matches_numpy_restatement(min_max):
    cfg, st, trs, m, lin, mn, mx, airm_p, airm_m, mask = _case()
    for q in range(len(trs)):
        out, d, diag = st.bermejo_conde(trs[q], m[q], lin[q], mn[q], mx[q], airm_p, airm_m, mask, deficit=1e-3,
                                        min_max=min_max)
        ref, d_ref, tot_p = _numpy_bc(cfg, st, trs[q], m[q], lin[q], mn[q], mx[q], airm_p, airm_m, mask, 1e-3,
                                      min_max)
        assert not np.shares_memory(out, m[q])
        assert np.max(np.abs(out - ref)) <= 1e-11 * np.max(np.abs(ref))
        assert abs(diag[7] - tot_p) <= 1e-12 * abs(tot_p)  # fixed total = total before advection - epsilon
        assert abs(d - d_ref) <= 1e-12 * abs(tot_p)
