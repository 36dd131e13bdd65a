"""The C ABI library loads without a GPU and exports every function that
include/adz_b200.h declares; calls that need a device fail with a status, not
a crash."""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "adz_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "return", "sizeof")))


@pytest.fixture(scope="module")
def L():
    from gem_b200 import build
    build.build()
    from gem_b200 import adz
    return adz.lib()


def test_header_symbols_exported(L):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_reference_symbol_set_present(L):
    for n in ("Vsearch_setup", "Vsearch_setup_plus", "Tricublin_zyx1_n", "Tricublin_zyx1_n_m", "Tricublin_zyx1_m_n",
              "Tricublin_zyx1_p", "Tricublin_mono_zyx_n", "Tricublin_mono_zyx_n_m", "Tricublin_mono_zyx_m_n",
              "Tricublin_zyx3_n"):
        assert hasattr(L, n)


def test_errors_without_device(L):
    from gem_b200 import adz, synth
    if torch.cuda.is_available():
        pytest.skip("device present")
    with pytest.raises(adz.AdzError) as e:
        adz.Adz.from_config(synth.config_small(32, 32, 10))
    assert e.value.status in (8, 2)
    assert L.adzc_error_string(8) == b"no CUDA device"
    # argument checks come before any device work
    assert L.adzc_setup(None, None) == 1
    assert L.adzc_traject(None, 0, C.c_double(1.0), 1, *([None] * 9)) == 1
    assert L.adzc_tricub(None, 0, 0, 0, None, None, None, None, None, None, None) == 1
    # a tile whose extended volume needs offsets beyond 32 bits is refused
    g = adz.AdzcGrid()
    big = np.zeros(64)
    g.ni, g.nj, g.nk, g.maxcfl = 60000, 60000, 4, 3
    g.zm = g.zt = g.zx = g.cy = big.ctypes.data_as(C.POINTER(C.c_double))
    h = C.c_void_p()
    assert L.adzc_setup(C.byref(g), C.byref(h)) == 9
    lev = np.linspace(3000.0, 100.0, 3)
    out = C.c_void_p()
    assert L.adzc_ztab_create(lev.ctypes.data, 3, 10, 10, 0, 0, C.byref(out)) == 3  # nk < 4


def test_no_library_no_fallback(monkeypatch, tmp_path):
    """Without the built library every entry point raises: there is no CPU
    fallback behind the binding."""
    from gem_b200 import adz, synth
    monkeypatch.setattr(adz, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(adz, "_LIB", None)
    with pytest.raises(FileNotFoundError):
        adz.lib()
    with pytest.raises(FileNotFoundError):
        adz.Adz.from_config(synth.config_small(16, 16, 8))
