"""MIXED accuracy on the mixed-precision workload (u, v, w and 8 log-normal
tracers, sigma 1, monotone clipping on the tracers), against the FP64 oracle
fed the same FP32 source values at the same FP64 departure points.

Error of a field at arrival point i (x the MIXED value, r the oracle's):

    e_i = |x_i - r_i| / max(|r_i|, b_i)

where b_i is the largest |source value| of the point's monotone bound box
(the 16 nodes x 1..2, y 0..3, z 1..2 of its 4x4x4 stencil, the box whose
min/max the reference's AVX2 interpolator returns,
src/gemdyn/src/base/turbo_tricublin.c:883-980).  Where the interpolated value
is as large as its neighbours this is the plain relative error; where it
cancels towards zero (a sign change of w, a log-normal value far below its
neighbours) the error is measured against the neighbours' magnitude, the
scale the FP32 weights resolve.  The bar is max_i e_i <= 1e-6 per field.

Positions: the FP64 oracle trajectory's position sets (adz_interp_traj),
which the library's FP64 path reproduces bit for bit (checked here through
adzc_interp_traj).  The MIXED values come from the device interpolator with
explicit positions, which runs the same per-point arithmetic (coef_mixed,
interp1_mixed, interp_mono_mixed) as the step's set kernels.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# max over points of |mixed - fp64| / max(|fp64|, largest |source| of the bound box)
MIXED_LOCAL_TOL = 1e-6
# max |mixed - fp64| / max |fp64| over the field
MIXED_NORM_TOL = 1e-6


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int32) if a.dtype == np.float32 else a.view(np.int64)


@pytest.fixture(scope="module")
def case():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from gem_b200 import adz as A, synth
    cfg = synth.config_mixed(160, 144, 80)
    inp = synth.make_inputs(cfg, dtype=torch.float64)
    f32 = {k: (v.float() if torch.is_tensor(v) else [t.float() for t in v]) for k, v in inp.items()}
    np64 = {k: (v.double().numpy() if torch.is_tensor(v) else [t.double().numpy() for t in v])
            for k, v in f32.items()}
    st = O.Step(cfg, kind="oracle", prec="f64")
    st.inittraj()
    for _ in range(2):  # cold step, then a warm one
        st.traject(np64)
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(A.FP64)
    ad.adz_inittraj(A.FP64, px, wp)
    dev64 = {k: torch.from_numpy(v).cuda() for k, v in np64.items() if not isinstance(v, list)}
    for _ in range(2):
        ad.adz_traject(A.FP64, cfg.dt, dev64, px, wp)
    pos = {s: ad.adz_interp_traj(A.FP64, s) for s in range(4)}
    assert ad.status() == 0
    return A, cfg, f32, np64, st, ad, pos


def test_position_sets_match_the_oracle(case):
    """adzc_interp_traj: the FP64 path's position sets equal the oracle's
    adz_interp_traj outputs bit for bit."""
    A, cfg, f32, np64, st, ad, pos = case
    for s in range(4):
        assert np.array_equal(_bits(pos[s].cpu().numpy()), _bits(st.sets[s])), s


def _ztab(A, cfg, ad, set_id):
    lev = (cfg.levels.zt if set_id == 3 else cfg.levels.zm)[1:cfg.nk + 1]
    I = ad.info
    return A.Ztab(lev, I.nit, I.njt, 1 - ad.grid.i0g, 1 - ad.grid.j0g)


def _at111(ad, t):
    """1-D view of an ext tensor starting at element (1,1,1)."""
    I = ad.info
    return t.reshape(-1)[I.haloy * I.nit + I.halox:]


def _errors(x, r, b):
    d = np.abs(x - r)
    return {"local": float(np.max(d / np.maximum(np.abs(r), b))),
            "norm": float(d.max() / np.abs(r).max()),
            "pointwise_floor1e-3": float(np.max(d / np.maximum(np.abs(r), 1e-3 * np.abs(r).max())))}


@pytest.mark.parametrize("field", ["u", "v", "w"] + [f"tracer{q}" for q in range(1, 9)])
def test_mixed_interpolated_field_error(case, field):
    A, cfg, f32, np64, st, ad, pos = case
    if field.startswith("tracer"):
        q = int(field[6:]) - 1
        set_id, src32, src64, clip = 3, f32["tracers"][q], np64["tracers"][q], True
    else:
        set_id = {"u": 1, "v": 2, "w": 3}[field]
        src32, src64, clip = f32["src_" + field], np64["src_" + field], False
    out, (lin, mn, mx) = st.tricub(set_id, [src64], mono=True, clip=clip, post=True)
    m = ad.range_mask(set_id).numpy()
    r, rmn, rmx = out[0][m], mn[0][m], mx[0][m]
    zt = _ztab(A, cfg, ad, set_id)
    d, _, dmn, dmx = (o[0].cpu().numpy().astype(np.float64) for o in
                      A.tricublin_mono_m_n(zt, A.MIXED, [_at111(ad, src32.cuda())], pos[set_id]))
    # the bound box is made of source values: identical in both precisions
    assert np.array_equal(dmn, rmn) and np.array_equal(dmx, rmx)
    if clip:
        d = np.maximum(dmn, np.minimum(dmx, d))
    e = _errors(d, r, np.maximum(np.abs(rmn), np.abs(rmx)))
    assert e["local"] <= MIXED_LOCAL_TOL, e
    assert e["norm"] <= MIXED_NORM_TOL, e
