"""The restated ZLF setups (orc_bc_lam_zlf, adz_BC_LAM_zlf_hlt.F90:18-319)
against an independent numpy statement of the regions each setup touches, and
the restated BICUBH_QV with Schm_autobar_L (bicubHQV_lin_mono.F90:95-96): a
field that varies in z only is interpolated linearly in z, so its value equals
the trilinear one."""
import numpy as np
import pytest

from oracle import oracle as O


def _regions(st, setup):
    """Boolean (nk, njt, nit) mask of the cells a setup writes."""
    s, g = st.s, st.s.g
    nk, ni, nj = g.nk, g.ni, g.nj
    k = np.arange(1, nk + 1)[:, None, None]
    j = np.arange(s.lminy, s.lminy + s.njt)[None, :, None]
    i = np.arange(s.lminx, s.lminx + s.nit)[None, None, :]
    inside = (i >= 1) & (i <= ni) & (j >= 1) & (j <= nj) & (k >= 1)
    w, e, so, no = g.west, g.east, g.south, g.north
    if setup == 1:
        ext = g.maxcfl + 1
        i0, i1 = 1 + g.pil_w - ext * w, ni - g.pil_e + ext * e
        j0, j1 = 1 + g.pil_s - ext * so, nj - g.pil_n + ext * no
        kcut = int(np.floor(s.k0t / 2.0 + 0.5))
    elif setup == 3:
        i0, i1, j0, j1, kcut = 1 + 4 * w, ni - 4 * e, 1 + 4 * so, nj - 4 * no, 1
    else:
        i0, i1, j0, j1, kcut = 1 + g.pil_w, ni - g.pil_e, 1 + g.pil_s, nj - g.pil_n, s.k0t
    out = (w & (i < i0)) | (e & (i > i1)) | (so & (j < j0)) | (no & (j > j1))
    box = (i >= i0) & (i <= i1) & (j >= j0) & (j <= j1) & (k <= kcut - 1)
    return inside & (out | (box if setup != 3 else False))


@pytest.mark.parametrize("gbpil,edges", [(0, (1, 1, 1, 1)), (5, (1, 1, 1, 1)), (2, (0, 1, 0, 1))])
def test_zlf_setups_against_region_masks(gbpil, edges):
    from gem_b200 import synth
    cfg = synth.config_small(40, 36, 16)
    st = O.Step(cfg, kind="oracle", prec="f64", lam_gbpil_t=gbpil, bc_lam_flux=2, edges=edges)
    rng = np.random.default_rng(1)
    for setup in (1, 2, 3, 4):
        f1 = rng.uniform(1, 2, st.ext_shape)
        f2 = rng.uniform(3, 4, st.ext_shape)
        a1, a2 = f1.copy(), f2.copy()
        st.bc_lam_zlf(setup, a1, a2 if setup in (2, 4) else None)
        m = _regions(st, setup)
        assert m.any()
        if setup in (1, 3):
            want1, want2 = np.where(m, 0.0, f1), f2
        elif setup == 2:
            want1, want2 = f1, np.where(m, f1, f2)
        else:
            want1, want2 = np.where(m, f2, f1), f2
        assert np.array_equal(a1, want1) and np.array_equal(a2, want2), setup


def test_qv_autobar_is_linear_in_z():
    from gem_b200 import synth
    cfg = synth.config_small(40, 36, 16)
    cfg.levels = synth.stretched_levels(16, 50.0, 1500.0, 20e3)
    inp = synth.make_inputs(cfg, dtype=__import__("torch").float64, with_fields=False)
    np_in = {k: v.numpy() for k, v in inp.items()}
    zt = cfg.levels.zt[1:cfg.nk + 1]
    fz = np.broadcast_to((np.sin(zt / 3000.0) + 2.0)[:, None, None], (cfg.nk, cfg.nj + 8, cfg.ni + 8)).copy()
    out = {}
    for autobar in (False, True):
        st = O.Step(cfg, kind="oracle", prec="f64", schm_autobar=autobar)
        st.inittraj()
        st.traject(np_in)
        d, (lin, mn, mx) = st.tricub_qv([fz], clip=False, post=True)
        m = ~np.isnan(d[0])
        out[autobar] = (d[0][m], lin[0][m], mn[0][m], mx[0][m])
    d, lin, mn, mx = out[True]
    inb = (d > mn) & (d < mx)  # lin is stored clipped to the box
    assert np.max(np.abs(d[inb] - lin[inb])) <= 1e-13 * np.max(np.abs(d))
    d0, lin0, _, _ = out[False]
    assert np.max(np.abs(d0 - lin0)) > 1e-6  # the quintic and cubic cases are really switched off
