"""BICUBH_QV restatement (oracle/adz_oracle_impl.h: qv_coef, qv_point,
orc_tricub_qv), pinned without the Fortran reference by what the scheme must
reproduce exactly: a field that is cubic in x and y plus quintic in height is
interpolated exactly where the quintic stencil applies (3 <= level <= nk-3),
a cubic in height exactly at the cubic levels, and the inner-box min/max and
trilinear value bracket the stencil values.  The FP32 (reference precision)
and FP64 restatements agree to FP32 rounding."""
import numpy as np
import pytest
import torch


def _setup(prec):
    from gem_b200 import synth
    from oracle import oracle as O
    cfg = synth.config_small(40, 36, 24)
    cfg.levels = synth.stretched_levels(24, 50.0, 1500.0, 20e3)
    dt = torch.float32 if prec == "f32" else torch.float64
    inp = synth.make_inputs(cfg, "cpu", dt)
    st = O.Step(cfg, kind="oracle", prec=prec)
    st.inittraj()
    st.traject({k: inp[k].numpy() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")})
    return cfg, st


def _field(cfg, zpow):
    H, nk = cfg.halo, cfg.nk
    zt = cfg.levels.zt
    i = np.arange(1 - H, cfg.ni + H + 1, dtype=np.float64)
    j = np.arange(1 - H, cfg.nj + H + 1, dtype=np.float64)
    Z = zt[1:nk + 1] / 1e4
    f = zpow(Z).reshape(-1, 1, 1) + (i.reshape(1, 1, -1) / 10.0) ** 3 + (j.reshape(1, -1, 1) / 10.0) ** 2
    return f


def _heights(cfg, pz):
    zt = cfg.levels.zt
    dz = np.diff(zt)  # delz_t(k) = zt(k+1) - zt(k), k = 0..nk
    nk = cfg.nk
    kk = pz.astype(np.float32).astype(np.int64)
    kk = np.where((kk >= 2) & (kk <= nk - 2), kk, np.clip(kk, 1, nk - 1))
    return zt[kk] + (pz - kk) * dz[kk], kk


def test_qv_reproduces_polynomials():
    cfg, st = _setup("f64")
    nk = cfg.nk
    r = st.ranges()["t"]
    p = st.sets[3]
    zt, kk = _heights(cfg, p[:, 2])
    for zpow, ok in ((lambda Z: Z ** 5 - 2 * Z ** 3 + 0.3, (kk >= 3) & (kk <= nk - 3)),
                     (lambda Z: Z ** 3 - Z + 0.1, (kk >= 2) & (kk <= nk - 2))):
        f = _field(cfg, zpow)
        d = st.tricub_qv([f])[0]
        i0, i1, j0, j1, k0 = r
        sub = d[k0 - 1:, j0 - 1 + cfg.halo:j1 + cfg.halo, i0 - 1 + cfg.halo:i1 + cfg.halo].reshape(-1)
        want = zpow(zt / 1e4) + (p[:, 0] / 10.0) ** 3 + (p[:, 1] / 10.0) ** 2
        assert ok.sum() > 1000
        err = np.abs(sub - want)[ok]
        assert err.max() <= 1e-9 * np.abs(want).max(), err.max()


def test_qv_box_and_precisions():
    cfg, st = _setup("f64")
    f = _field(cfg, lambda Z: np.sin(3 * Z)) + 0.1 * np.cos(np.arange(np.prod(_field(cfg, np.sin).shape))
                                                        ).reshape(_field(cfg, np.sin).shape)
    d, (lin, mn, mx) = st.tricub_qv([f], post=True)
    m = ~np.isnan(d[0])
    assert np.all(mn[0][m] <= lin[0][m]) and np.all(lin[0][m] <= mx[0][m])
    dc = st.tricub_qv([f], clip=True)[0]
    assert np.all(dc[m] >= mn[0][m]) and np.all(dc[m] <= mx[0][m])
    cfg32, st32 = _setup("f32")
    d32 = st32.tricub_qv([f.astype(np.float32)])[0]
    rel = np.abs(d32[m] - d[0][m]) / np.abs(d[0][m]).max()
    # positions differ by FP32 trajectory rounding, values by FP32 sums
    assert rel.max() < 1e-4 and np.median(rel) < 1e-6
