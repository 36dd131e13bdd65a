"""The oracle is pinned before anything is checked against it:

* the restated interpolator reproduces the reference's SELF_TEST known answers
  (src/gemdyn/src/base/turbo_tricublin.c:1314-1506) line for line;
* it reproduces the reference build's outputs on the committed golden vectors
  bit for bit (cubic, mono with the AVX2 2x4x2 bound box, 3-component);
* the driver restatement gives the same step whether it calls the restated
  interpolator or the reference's own (when the reference build is present).

Trajectory parity is pinned to the C restatement of the Fortran drivers, not to
a Fortran run (the Fortran cannot be built here).
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _bits(a):
    return np.ascontiguousarray(a).view(np.int32)


def test_selftest_kat_matches_reference_output():
    exe = os.path.join(os.path.dirname(O.HERE), "oracle", "kat_selftest")
    subprocess.run(["make", "-s", "-C", O.HERE, "kat_selftest"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines()
    gold = open(os.path.join(GOLD, "selftest_reference.txt")).read().splitlines()
    assert out == gold
    # the headline known answers
    assert "worst case error :  4.98177e-07, avg error : 6.866881e-08, exact :    36.43 percent" in out


@pytest.fixture(scope="module")
def vec():
    return dict(np.load(os.path.join(GOLD, "tricublin_ref_vectors.npz")))


def test_golden_vectors_bit_exact(vec):
    ni, nj, nk = int(vec["ni"]), int(vec["nj"]), int(vec["nk"])
    zt = O.Ztab(vec["levels"], ni, nj, int(vec["offi"]), int(vec["offj"]))
    fields = [np.ascontiguousarray(f) for f in vec["fields"]]
    pos = vec["pos"]
    assert np.array_equal(_bits(O.zyx1_m_n(fields, pos, zt)), _bits(vec["zyx1"]))
    d, lin, mi, ma = O.mono_m_n(fields, pos, zt, box=0)
    for got, key in ((d, "mono_d"), (lin, "mono_lin"), (mi, "mono_min"), (ma, "mono_max")):
        assert np.array_equal(_bits(got), _bits(vec[key])), key
    d3 = O.zyx3_n(np.ascontiguousarray(vec["f3"]), pos, zt)
    assert np.array_equal(_bits(d3), _bits(vec["zyx3"]))


def test_golden_scalar_box_option(vec):
    """The reference's scalar branch bounds the 2x2x2 inner box; the option
    reproduces it (its cubic and linear values equal the AVX2 ones)."""
    ni, nj = int(vec["ni"]), int(vec["nj"])
    zt = O.Ztab(vec["levels"], ni, nj, int(vec["offi"]), int(vec["offj"]))
    fields = [np.ascontiguousarray(f) for f in vec["fields"]]
    d, lin, mi, ma = O.mono_m_n(fields, vec["pos"], zt, box=1)
    assert np.array_equal(_bits(mi), _bits(vec["scalar_mono_min"]))
    assert np.array_equal(_bits(ma), _bits(vec["scalar_mono_max"]))
    assert np.array_equal(_bits(d), _bits(vec["mono_d"]))
    # the two bound boxes really differ on these inputs
    assert np.any(vec["scalar_mono_min"] != vec["mono_min"])


def test_f64_extension_agrees_with_f32_path(vec):
    ni, nj = int(vec["ni"]), int(vec["nj"])
    zt = O.Ztab(vec["levels"], ni, nj, int(vec["offi"]), int(vec["offj"]))
    f64 = [np.ascontiguousarray(f, dtype=np.float64) for f in vec["fields"]]
    pos64 = vec["pos"].astype(np.float64)
    d = O.zyx1_m_n(f64, pos64, zt)
    ref = vec["zyx1"].astype(np.float64)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(d - ref)) / scale < 1e-6


def test_cell_index_from_fp32_rounded_position():
    """An FP64 position within half an FP32 ulp below an integer selects the
    cell the FP32 position selects (turbo_tricublin.c:395-399)."""
    lev = np.linspace(10000.0, 500.0, 12)
    zt = O.Ztab(lev, 30, 30)
    p = np.array([[10.0 - 1e-9, 7.0 - 2e-8, 5.0 - 1e-9], [12.25, 9.5, 4.75]], np.float64)
    off64, zl64 = O.cells(p, zt)
    off32, zl32 = O.cells(p.astype(np.float32), zt)
    assert np.array_equal(off64, off32) and np.array_equal(zl64, zl32)
    assert np.floor(p[0, 0]) == 9.0  # floor would have picked the cell below


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_driver_with_reference_interpolator_is_bit_identical():
    from gem_b200 import synth
    cfg = synth.config_small(40, 36, 16)
    inp = synth.make_inputs(cfg, dtype=torch.float64)
    inp = {k: (v.numpy() if torch.is_tensor(v) else [t.numpy() for t in v]) for k, v in inp.items()}
    outs = []
    for kind in ("oracle", "ref"):
        st = O.Step(cfg, kind=kind, prec="f32")
        st.inittraj()
        o = st.step(inp)
        outs.append((st.pxyzm.copy(), st.wpxyz.copy(), o))
    (pa, wa, oa), (pb, wb, ob) = outs
    assert np.array_equal(_bits(pa), _bits(pb))
    assert np.array_equal(wa, wb)
    for k in ("u", "v", "w"):
        m = ~np.isnan(oa[k])
        assert np.array_equal(_bits(oa[k][m]), _bits(ob[k][m]))
    for x, y in zip(oa["tracers"], ob["tracers"]):
        m = ~np.isnan(x)
        assert np.array_equal(_bits(x[m]), _bits(y[m]))


def test_search_tables_and_ranges():
    from gem_b200 import synth
    cfg = synth.config_large(64, 64, 80)
    st = O.Step(cfg, kind="oracle", prec="f64")
    s = st.s
    assert s.sig == -1.0
    assert (s.halox, s.lminx, s.lmaxx) == (4, -3, 68)
    # LAM tile with an 8-point pilot zone: arrival ranges (adz_set.F90:94-114)
    assert (s.i0, s.in_, s.i0u, s.inu, s.i0b, s.inb) == (7, 57, 9, 55, 5, 60)
    assert abs(s.iminposx - (5 + 2e-5)) < 1e-12 and abs(s.imaxposx - (60 - 2e-5)) < 1e-12
    tab = np.ctypeslib.as_array(s.search_m, shape=(s.pnz_m,))
    assert tab[0] == 0 and tab[-1] <= cfg.nk + 1 and np.all(np.diff(tab) >= 0)


@pytest.mark.skipif(not O.have_ref(), reason="reference build absent")
def test_driver_reference_build_across_grids():
    """Successive steps on different grids with the reference interpolator
    match the restated one (each orc_set carries its own descriptors)."""
    from gem_b200 import synth
    for shape in ((40, 36, 12), (64, 48, 20), (40, 36, 12)):
        cfg = synth.config_small(*shape)
        inp = synth.make_inputs(cfg, dtype=torch.float64)
        inp = {k: (v.numpy() if torch.is_tensor(v) else [t.numpy() for t in v]) for k, v in inp.items()}
        res = []
        for kind in ("ref", "oracle"):
            st = O.Step(cfg, kind=kind, prec="f32")
            st.inittraj()
            st.step(inp)
            res.append(st.pxyzm.copy())
        assert np.array_equal(_bits(res[0]), _bits(res[1])), shape
