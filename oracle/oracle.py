"""ORACLE — test infrastructure only.

ctypes front end of the CPU restatement (``liboracle.so``) and of the
reference interpolator compiled unchanged (``_ref/libtricublin_ref.so``,
``_ref/libadz_ref.so``).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class OrcZtab(C.Structure):
    _fields_ = [("z", C.POINTER(C.c_double)), ("ocz", C.POINTER(C.c_double)),
                ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("nij", C.c_int),
                ("offi", C.c_int), ("offj", C.c_int)]


class OrcGrid(C.Structure):
    """Inputs of adz_set (src/gemdyn/src/base/adz_set.F90:16-538)."""
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("maxcfl", C.c_int),
                ("i0g", C.c_int), ("j0g", C.c_int),
                ("west", C.c_int), ("east", C.c_int), ("south", C.c_int), ("north", C.c_int),
                ("pil_w", C.c_int), ("pil_e", C.c_int), ("pil_s", C.c_int), ("pil_n", C.c_int),
                ("lam_gbpil_t", C.c_int), ("bc_lam_flux", C.c_int), ("schm_advec", C.c_int),
                ("itraj", C.c_int), ("slt_winds", C.c_int), ("schm_autobar", C.c_int),
                ("bA_m", C.c_double), ("bA", C.c_double), ("inv_rayt", C.c_double),
                ("inv_hx", C.c_double), ("inv_hy", C.c_double),
                ("cy", C.POINTER(C.c_double)), ("zm", C.POINTER(C.c_double)),
                ("zt", C.POINTER(C.c_double)), ("zx", C.POINTER(C.c_double)),
                ("zmin", C.c_double), ("zmax", C.c_double),
                ("wmstar_nk", C.c_double), ("idz_t_nkm1", C.c_double)]


class OrcSet(C.Structure):
    _fields_ = [("g", OrcGrid)] + [(n, C.c_int) for n in (
        "halox", "haloy", "lminx", "lmaxx", "lminy", "lmaxy", "nit", "njt", "nij",
        "i0", "in_", "j0", "jn", "i0u", "inu", "j0v", "jnv", "i0b", "inb", "j0b", "jnb",
        "k0", "k0t", "k0m", "niu", "njv")] + [
        ("iminposx", C.c_double), ("imaxposx", C.c_double), ("iminposy", C.c_double),
        ("imaxposy", C.c_double), ("sig", C.c_double), ("ovdzm", C.c_double), ("ovdzt", C.c_double),
        ("pnz_m", C.c_int), ("pnz_t", C.c_int),
        ("search_m", C.POINTER(C.c_int)), ("search_t", C.POINTER(C.c_int))] + [
        (n, C.POINTER(C.c_double)) for n in (
            "delz_m", "delz_t", "odelz_m", "odelz_t",
            "vw1m", "vw2m", "vw3m", "vw4m", "vw1t", "vw2t", "vw3t", "vw4t")] + [
        ("vw5", C.c_double), ("vw6", C.c_double), ("ww", C.c_double), ("wp", C.c_double),
        ("wm", C.c_double), ("cy", C.POINTER(C.c_double)),
        ("ztab_m", C.POINTER(OrcZtab)), ("ztab_t", C.POINTER(OrcZtab)),
        ("ref_m", C.c_void_p), ("ref_t", C.c_void_p), ("qv_t", C.c_void_p)]


def build(ref: bool | None = None) -> None:
    """Compile the restatement (and the reference objects when the reference
    tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    # the Makefile's REFDIR (overridable from the environment) names the reference source
    refsrc = subprocess.run(["make", "-s", "-C", HERE, "refsrc"], check=True, capture_output=True,
                            text=True).stdout.strip()
    if ref or (ref is None and os.path.exists(refsrc)):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def _ptrs(arrs, ctype):
    arr = (C.POINTER(ctype) * len(arrs))()
    for i, a in enumerate(arrs):
        arr[i] = a.ctypes.data_as(C.POINTER(ctype))
    return arr


class _Lib:
    def __init__(self, path: str):
        self.path = path
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_vsearch_setup_plus.restype = C.POINTER(OrcZtab)
        L.orc_vsearch_setup_plus.argtypes = [_f64p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_ztab_free.argtypes = [C.POINTER(OrcZtab)]
        vp = C.c_void_p
        for name in ("orc_zyx1_m_n_f32", "orc_zyx1_m_n_f64"):
            getattr(L, name).argtypes = [vp, vp, vp, C.POINTER(OrcZtab), C.c_int, C.c_int]
        L.orc_mono_m_n_f32.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(OrcZtab), C.c_int, C.c_int, C.c_int]
        L.orc_mono_m_n_f64.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(OrcZtab), C.c_int, C.c_int]
        for name in ("orc_zyx3_n_f32", "orc_zyx3_n_f64"):
            getattr(L, name).argtypes = [vp, vp, vp, C.POINTER(OrcZtab), C.c_int]
        for name in ("orc_cells_f32", "orc_cells_f64"):
            getattr(L, name).argtypes = [vp, vp, vp, C.POINTER(OrcZtab), C.c_int]
        L.orc_adz_set.argtypes = [C.POINTER(OrcGrid), C.POINTER(OrcSet)]
        L.orc_adz_free.argtypes = [C.POINTER(OrcSet)]
        L.orc_set_npoints.restype = C.c_long
        L.orc_set_npoints.argtypes = [C.POINTER(OrcSet), C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        for sfx in ("f32", "f64"):
            getattr(L, f"orc_prepare_winds_{sfx}").argtypes = [C.POINTER(OrcSet)] + [vp] * 10
            getattr(L, f"orc_inittraj_{sfx}").argtypes = [C.POINTER(OrcSet), vp, vp]
            getattr(L, f"orc_traject_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_double, C.c_int] + [vp] * 7
            getattr(L, f"orc_interp_traj_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_double] + [vp] * 10
            getattr(L, f"orc_tricub_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_int, vp, C.c_int, vp, vp,
                                                        C.c_int, C.c_int, vp, vp, vp]
            getattr(L, f"orc_tricub_qv_{sfx}").argtypes = [C.POINTER(OrcSet), vp, C.c_int, vp, vp, C.c_int,
                                                           vp, vp, vp]
            getattr(L, f"orc_bc_lam_flux_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_double, vp, vp, vp, vp, vp,
                                                             C.c_int, vp, vp, vp]
            getattr(L, f"orc_tricub_p_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_int, vp, C.c_int, vp, vp,
                                                          C.c_int, C.c_int, vp, vp, vp, vp, C.c_int]
            getattr(L, f"orc_tricub_qv_p_{sfx}").argtypes = [C.POINTER(OrcSet), vp, C.c_int, vp, vp, C.c_int,
                                                             vp, vp, vp, vp, C.c_int]
            getattr(L, f"orc_ilmc_{sfx}").argtypes = [C.POINTER(OrcSet), vp, vp, vp, vp, C.c_int, C.c_int]
            getattr(L, f"orc_pb_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_double, vp, vp, vp, vp, vp, vp]
            getattr(L, f"orc_bc_lam_zlf_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_int, vp, vp]
            getattr(L, f"orc_tricub_qv_set_p_{sfx}").argtypes = [C.POINTER(OrcSet), C.c_int, vp, C.c_int, vp, vp,
                                                                 C.c_int, vp, vp, vp, vp, C.c_int]
            getattr(L, f"orc_bermejo_conde_{sfx}").argtypes = [C.POINTER(OrcSet)] + [vp] * 8 + [
                C.c_int, C.c_double, C.c_int, vp, vp, vp, vp, vp]


_LIBS: dict[str, _Lib] = {}


def lib(kind: str = "oracle") -> _Lib:
    """kind: 'oracle' (restatement) or 'ref' (driver restatement linked with
    the reference's own interpolator)."""
    if kind not in _LIBS:
        path = os.path.join(HERE, "liboracle.so") if kind == "oracle" else os.path.join(REF_DIR, "libadz_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run oracle.build())")
        _LIBS[kind] = _Lib(path)
    return _LIBS[kind]


def have_ref() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libadz_ref.so")) and \
        os.path.exists(os.path.join(REF_DIR, "libtricublin_ref.so"))


# --------------------------------------------------------------------------
# interpolator-level API (reference call shapes, numpy in/out)
# --------------------------------------------------------------------------
class Ztab:
    """Level descriptor of the restatement (Vsearch_setup_plus)."""

    def __init__(self, levels, ni, nj, offi=0, offj=0, kind="oracle"):
        self.L = lib(kind)
        self.levels = np.ascontiguousarray(levels, dtype=np.float64)
        self.ptr = self.L.lib.orc_vsearch_setup_plus(self.levels, len(self.levels), ni, nj, offi, offj)
        self.ni, self.nj, self.nk = ni, nj, len(self.levels)

    def __del__(self):
        try:
            self.L.lib.orc_ztab_free(self.ptr)
        except Exception:
            pass


def zyx1_m_n(fields, pos, zt: Ztab):
    """Tricublin_zyx1_m_n; fields: list of flat arrays addressed at f(1,1,1)
    through ``base`` offsets handled by the caller (pass views)."""
    f64 = fields[0].dtype == np.float64
    n, m = pos.shape[0], len(fields)
    d = np.empty((m, n), dtype=fields[0].dtype)
    ct = C.c_double if f64 else C.c_float
    fs = _ptrs(fields, ct)
    fn = zt.L.lib.orc_zyx1_m_n_f64 if f64 else zt.L.lib.orc_zyx1_m_n_f32
    fn(d.ctypes.data, C.cast(fs, C.c_void_p), np.ascontiguousarray(pos).ctypes.data, zt.ptr, n, m)
    return d


def mono_m_n(fields, pos, zt: Ztab, box=0):
    f64 = fields[0].dtype == np.float64
    n, m = pos.shape[0], len(fields)
    out = [np.empty((m, n), dtype=fields[0].dtype) for _ in range(4)]
    ct = C.c_double if f64 else C.c_float
    fs = _ptrs(fields, ct)
    p = np.ascontiguousarray(pos)
    if f64:
        zt.L.lib.orc_mono_m_n_f64(*(o.ctypes.data for o in out), C.cast(fs, C.c_void_p), p.ctypes.data, zt.ptr, n, m)
    else:
        zt.L.lib.orc_mono_m_n_f32(*(o.ctypes.data for o in out), C.cast(fs, C.c_void_p), p.ctypes.data, zt.ptr, n, m,
                                  box)
    return out  # d, lin, min, max


def zyx3_n(f3, pos, zt: Ztab):
    f64 = f3.dtype == np.float64
    n = pos.shape[0]
    d = np.empty((n, 3), dtype=f3.dtype)
    fn = zt.L.lib.orc_zyx3_n_f64 if f64 else zt.L.lib.orc_zyx3_n_f32
    fn(d.ctypes.data, f3.ctypes.data, np.ascontiguousarray(pos).ctypes.data, zt.ptr, n)
    return d


def cells(pos, zt: Ztab):
    """(corner offset, zlinear) chosen for each position."""
    n = pos.shape[0]
    off = np.empty(n, np.int32)
    zl = np.empty(n, np.int32)
    fn = zt.L.lib.orc_cells_f64 if pos.dtype == np.float64 else zt.L.lib.orc_cells_f32
    fn(off.ctypes.data, zl.ctypes.data, np.ascontiguousarray(pos).ctypes.data, zt.ptr, n)
    return off, zl


# --------------------------------------------------------------------------
# the reference interpolator compiled unchanged (reference symbol names)
# --------------------------------------------------------------------------
class RefKernels:
    """Direct ctypes access to the reference's Tricublin_* (FP32 only)."""

    def __init__(self, scalar: bool = False):
        name = "libtricublin_ref_scalar.so" if scalar else "libtricublin_ref.so"
        self.lib = C.CDLL(os.path.join(REF_DIR, name))
        L = self.lib
        L.Vsearch_setup_plus.restype = C.c_void_p
        L.Vsearch_setup_plus.argtypes = [_f64p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        vp = C.c_void_p
        L.Tricublin_zyx1_n.argtypes = [vp, vp, vp, vp, C.c_int]
        L.Tricublin_zyx1_n_m.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int]
        L.Tricublin_zyx1_m_n.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int]
        L.Tricublin_zyx1_p.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int]
        L.Tricublin_mono_zyx_n.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int]
        L.Tricublin_mono_zyx_n_m.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int]
        L.Tricublin_mono_zyx_m_n.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int]
        L.Tricublin_zyx3_n.argtypes = [vp, vp, vp, vp, C.c_int]
        self._keep = []

    def setup(self, levels, ni, nj, offi=0, offj=0):
        lv = np.ascontiguousarray(levels, dtype=np.float64)
        self._keep.append(lv)
        return self.lib.Vsearch_setup_plus(lv, len(lv), ni, nj, offi, offj)

    def zyx1_m_n(self, fields, pos, zt):
        n, m = pos.shape[0], len(fields)
        d = np.empty((m, n), np.float32)
        fs = _ptrs(fields, C.c_float)
        self.lib.Tricublin_zyx1_m_n(d.ctypes.data, C.cast(fs, C.c_void_p), np.ascontiguousarray(pos).ctypes.data,
                                    zt, n, m)
        return d

    def mono_m_n(self, fields, pos, zt):
        n, m = pos.shape[0], len(fields)
        out = [np.empty((m, n), np.float32) for _ in range(4)]
        fs = _ptrs(fields, C.c_float)
        self.lib.Tricublin_mono_zyx_m_n(*(o.ctypes.data for o in out), C.cast(fs, C.c_void_p),
                                        np.ascontiguousarray(pos).ctypes.data, zt, n, m)
        return out

    def zyx3_n(self, f3, pos, zt):
        n = pos.shape[0]
        d = np.empty((n, 3), np.float32)
        self.lib.Tricublin_zyx3_n(d.ctypes.data, f3.ctypes.data, np.ascontiguousarray(pos).ctypes.data, zt, n)
        return d


# --------------------------------------------------------------------------
# driver restatement: one advection step (adz_main + adz_tracers subset)
# --------------------------------------------------------------------------
def make_grid(cfg, i0g=1, j0g=1, lam=True, slt_winds=False, schm_advec=1, lam_gbpil_t=0, bc_lam_flux=1,
              schm_autobar=False, edges=None):
    """orc_grid for a synth.Config tile: a LAM tile touching the edges
    flagged in edges = (west, east, south, north) (default: all four when
    lam), with pilot zones on those edges only."""
    from gem_b200 import synth
    ga = synth.grid_arrays(cfg)
    keep = {k: np.ascontiguousarray(ga[k], dtype=np.float64) for k in ("cy", "zm", "zt", "zx")}
    e = 1 if lam else 0
    w, ea, so, no = edges if edges is not None else (e, e, e, e)
    p = cfg.pil if lam else 0
    g = OrcGrid(ni=cfg.ni, nj=cfg.nj, nk=cfg.nk, maxcfl=cfg.maxcfl, i0g=i0g, j0g=j0g,
                west=w, east=ea, south=so, north=no, pil_w=p * w, pil_e=p * ea, pil_s=p * so, pil_n=p * no,
                lam_gbpil_t=lam_gbpil_t, bc_lam_flux=bc_lam_flux, schm_advec=schm_advec, itraj=cfg.niter,
                slt_winds=1 if slt_winds else 0, schm_autobar=1 if schm_autobar else 0, bA_m=0.6, bA=0.6, inv_rayt=ga["inv_rayt"],
                inv_hx=ga["inv_hx"], inv_hy=ga["inv_hy"],
                cy=keep["cy"].ctypes.data_as(C.POINTER(C.c_double)),
                zm=keep["zm"].ctypes.data_as(C.POINTER(C.c_double)),
                zt=keep["zt"].ctypes.data_as(C.POINTER(C.c_double)),
                zx=keep["zx"].ctypes.data_as(C.POINTER(C.c_double)),
                zmin=ga["zmin"], zmax=ga["zmax"], wmstar_nk=ga["wmstar_nk"], idz_t_nkm1=ga["idz_t_nkm1"])
    return g, keep


class Step:
    """adz_set + one advection step on the CPU (the reference's structure:
    prepareWinds, Adz_niter trajectory iterations, interp_traj, then
    adz_tricub_hlt per position set and the monotone clip).

    kind: 'oracle' (restated interpolator) or 'ref' (reference interpolator).
    prec: 'f32' (the reference's own precision) or 'f64' (FP64 extension).
    """

    def __init__(self, cfg, kind="oracle", prec="f32", threads=0, **gridkw):
        self.cfg, self.kind, self.prec = cfg, kind, prec
        self.L = lib(kind).lib
        self.L.orc_set_threads(threads)
        self.grid, self._keep = make_grid(cfg, **gridkw)
        self.s = OrcSet()
        self.L.orc_adz_set(C.byref(self.grid), C.byref(self.s))
        self.dt = np.float32 if prec == "f32" else np.float64
        s, c = self.s, cfg
        self.ext_shape = (c.nk, s.njt, s.nit)
        self.arr_shape = (c.nk, c.nj, c.ni)
        self.uvw_d = np.zeros(self.ext_shape + (3,), self.dt)
        self.uu_arr = np.zeros(self.arr_shape, self.dt)
        self.vv_arr = np.zeros(self.arr_shape, self.dt)
        self.ww_arr = np.zeros(self.arr_shape, self.dt)
        self.uvw_dep = np.zeros(self.arr_shape + (3,), self.dt)
        self.pxyzm = np.zeros(self.arr_shape + (3,), self.dt)
        self.wpxyz = np.zeros((3, c.nk, c.nj + 4, c.ni + 4), np.float64)
        self.sets = {q: np.zeros((self.L.orc_set_npoints(C.byref(s), q), 3), self.dt) for q in range(4)}
        self.cold = True

    def __del__(self):
        try:
            self.L.orc_adz_free(C.byref(self.s))
        except Exception:
            pass

    def ranges(self):
        s = self.s
        return dict(q=(s.i0, s.in_, s.j0, s.jn, s.k0), u=(s.i0u, s.inu, s.j0, s.jn, s.k0),
                    v=(s.i0, s.in_, s.j0v, s.jnv, s.k0), t=(s.i0, s.in_, s.j0, s.jn, s.k0t))

    def inittraj(self):
        fn = getattr(self.L, f"orc_inittraj_{self.prec}")
        fn(C.byref(self.s), self.pxyzm.ctypes.data, self.wpxyz.ctypes.data)
        self.cold = True

    def traject(self, inp, niter=None):
        """adz_prepareWinds + iterations + interp_traj. inp: dict of ext arrays."""
        P = self.prec
        a = {k: np.ascontiguousarray(inp[k], dtype=self.dt) for k in
             ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")}
        self._zdt0 = a["zdt0"]
        getattr(self.L, f"orc_prepare_winds_{P}")(
            C.byref(self.s), *(a[k].ctypes.data for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")),
            self.uvw_d.ctypes.data, self.uu_arr.ctypes.data, self.vv_arr.ctypes.data, self.ww_arr.ctypes.data)
        if niter is None:
            niter = max(6, self.cfg.niter) if self.cold else self.cfg.niter
        getattr(self.L, f"orc_traject_{P}")(
            C.byref(self.s), self.cfg.dt, niter, self.uvw_d.ctypes.data, self.uu_arr.ctypes.data,
            self.vv_arr.ctypes.data, self.ww_arr.ctypes.data, self.uvw_dep.ctypes.data,
            self.pxyzm.ctypes.data, self.wpxyz.ctypes.data)
        self.cold = False
        # Adz_uslt, Adz_vslt (nj, ni), used when the grid sets slt_winds
        slt = [np.ascontiguousarray(inp[k], dtype=self.dt) if inp.get(k) is not None else None
               for k in ("uslt", "vslt")]
        self._slt = slt
        getattr(self.L, f"orc_interp_traj_{P}")(
            C.byref(self.s), self.cfg.dt, self.wpxyz.ctypes.data, self.uvw_dep.ctypes.data,
            a["zdt0"].ctypes.data, self.pxyzm.ctypes.data, *(None if x is None else x.ctypes.data for x in slt),
            *(self.sets[q].ctypes.data for q in range(4)))

    def bc_lam_flux(self, srcs):
        """FLUX_out, FLUX_in of adz_BC_LAM_Aranami_hlt.F90 for the tracers srcs
        (ext arrays) at the last trajectory's Adz_pb; ext arrays, NaN where
        not written."""
        ct = C.c_float if self.prec == "f32" else C.c_double
        srcs = [None if x is None else np.ascontiguousarray(x, dtype=self.dt) for x in srcs]
        fo = [np.full(self.ext_shape, np.nan, self.dt) for _ in srcs]
        fi = [np.full(self.ext_shape, np.nan, self.dt) for _ in srcs]
        sp = (C.POINTER(ct) * len(srcs))(*[C.POINTER(ct)() if x is None else x.ctypes.data_as(C.POINTER(ct))
                                           for x in srcs])
        slt = getattr(self, "_slt", [None, None])
        getattr(self.L, f"orc_bc_lam_flux_{self.prec}")(
            C.byref(self.s), self.cfg.dt, self.wpxyz.ctypes.data, self.uvw_dep.ctypes.data, self._zdt0.ctypes.data,
            *(None if x is None else x.ctypes.data for x in slt), len(srcs), C.cast(sp, C.c_void_p),
            C.cast(_ptrs(fo, ct), C.c_void_p), C.cast(_ptrs(fi, ct), C.c_void_p))
        return fo, fi

    def pb(self):
        """Adz_pb: the t-set positions over range b (i0b:inb, j0b:jnb, 1:nk)
        of the last trajectory, (npoints, 3) with i fastest."""
        s = self.s
        n = (s.inb - s.i0b + 1) * (s.jnb - s.j0b + 1) * self.cfg.nk
        pb = np.zeros((n, 3), self.dt)
        slt = getattr(self, "_slt", [None, None])
        getattr(self.L, f"orc_pb_{self.prec}")(
            C.byref(s), self.cfg.dt, self.wpxyz.ctypes.data, self.uvw_dep.ctypes.data, self._zdt0.ctypes.data,
            *(None if x is None else x.ctypes.data for x in slt), pb.ctypes.data)
        return pb

    def tricub_b(self, srcs, mono=False, clip=False, post=False, qv=False):
        """adz_tricub_hlt at Adz_pb over range b, all levels (the ZLF call of
        adz_tracers.F90:91-93, 130-133); tricubic, or BICUBH_QV when qv."""
        m = len(srcs)
        srcs = [np.ascontiguousarray(x, dtype=self.dt) for x in srcs]
        dsts = [np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)]
        ct = C.c_float if self.prec == "f32" else C.c_double
        extra = [[np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)] for _ in range(3)]
        ptr = [C.cast(_ptrs(z, ct), C.c_void_p) for z in extra]
        pos = self.pb()
        pert, ld = self._pert_args()
        if qv:
            getattr(self.L, f"orc_tricub_qv_set_p_{self.prec}")(
                C.byref(self.s), 4, pos.ctypes.data, m, C.cast(_ptrs(srcs, ct), C.c_void_p),
                C.cast(_ptrs(dsts, ct), C.c_void_p), int(clip), *ptr, pert, ld)
        else:
            getattr(self.L, f"orc_tricub_p_{self.prec}")(
                C.byref(self.s), 4, pos.ctypes.data, m, C.cast(_ptrs(srcs, ct), C.c_void_p),
                C.cast(_ptrs(dsts, ct), C.c_void_p), int(mono), int(clip), *(ptr if mono else (None,) * 3), pert, ld)
        if post:
            return dsts, tuple(extra)
        return dsts

    def bc_lam_zlf(self, setup, f1, f2=None):
        """adz_BC_LAM_zlf_hlt setup 1-4 on ext arrays of the Step's precision,
        in place (f2 for setups 2 and 4)."""
        for a in (f1, f2):
            if a is not None:
                assert a.dtype == self.dt and a.flags.c_contiguous and a.shape == self.ext_shape
        getattr(self.L, f"orc_bc_lam_zlf_{self.prec}")(C.byref(self.s), int(setup), f1.ctypes.data,
                                                        None if f2 is None else f2.ctypes.data)

    def set_rhs_perturbation(self, mcrhsint=None):
        """mcrhsint (nj, ni) or None: the ensemble perturbation of every
        later interpolation (adz_interp_hlt.F90:99-133)."""
        self._pert = None if mcrhsint is None else np.ascontiguousarray(mcrhsint, dtype=self.dt)

    def _pert_args(self):
        p = getattr(self, "_pert", None)
        return (None, 0) if p is None else (p.ctypes.data, p.shape[1])

    def tricub(self, set_id, srcs, mono=False, clip=False, post=False):
        """adz_tricub_hlt on position set set_id (0=q,1=u,2=v,3=t); returns the
        destination arrays (ext layout, range written, NaN elsewhere) and, if
        post, (lin, min, max)."""
        m = len(srcs)
        srcs = [np.ascontiguousarray(x, dtype=self.dt) for x in srcs]
        dsts = [np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)]
        ct = C.c_float if self.prec == "f32" else C.c_double
        sp, dp = _ptrs(srcs, ct), _ptrs(dsts, ct)
        lin = mn = mx = None
        lp = mnp = mxp = None
        if mono and post:
            lin = [np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)]
            mn = [np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)]
            mx = [np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)]
            lp, mnp, mxp = (C.cast(_ptrs(z, ct), C.c_void_p) for z in (lin, mn, mx))
        pert, ld = self._pert_args()
        getattr(self.L, f"orc_tricub_p_{self.prec}")(
            C.byref(self.s), set_id, self.sets[set_id].ctypes.data, m, C.cast(sp, C.c_void_p),
            C.cast(dp, C.c_void_p), int(mono), int(clip), lp, mnp, mxp, pert, ld)
        if post:
            return dsts, (lin, mn, mx)
        return dsts

    def tricub_qv(self, srcs, clip=False, post=False):
        """adz_tricub_hlt with BICUBH_QV at position set t (bicubHQV_lin_mono.F90);
        returns the destinations (ext layout, range written, NaN elsewhere) and,
        if post, (lin, min, max)."""
        m = len(srcs)
        srcs = [np.ascontiguousarray(x, dtype=self.dt) for x in srcs]
        dsts = [np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)]
        ct = C.c_float if self.prec == "f32" else C.c_double
        extra = [[np.full(self.ext_shape, np.nan, self.dt) for _ in range(m)] for _ in range(3)]
        ptr = [C.cast(_ptrs(z, ct), C.c_void_p) for z in extra]
        pert, ld = self._pert_args()
        getattr(self.L, f"orc_tricub_qv_p_{self.prec}")(
            C.byref(self.s), self.sets[3].ctypes.data, m, C.cast(_ptrs(srcs, ct), C.c_void_p),
            C.cast(_ptrs(dsts, ct), C.c_void_p), int(clip), *ptr, pert, ld)
        if post:
            return dsts, tuple(extra)
        return dsts

    def bermejo_conde(self, p, m, lin, mn, mx, airm_p, airm_m, mask, deficit=0.0, weight=1, p_exp=1.0,
                      min_max=True, fo=None, fi=None, pkps=None):
        """Bermejo-Conde on one tracer (ext arrays of the Step's precision);
        returns (fixed m, new deficit, diag[8])."""
        A = lambda x: None if x is None else np.ascontiguousarray(x, dtype=self.dt)  # noqa: E731
        arrs = [A(x) for x in (p, m, lin, mn, mx, fo, fi, pkps)]
        arrs[1] = arrs[1].copy()  # fixed in place: never the caller's array
        am, bm = A(airm_p), A(airm_m)
        mk = np.ascontiguousarray(mask, dtype=np.float64)
        d = C.c_double(deficit)
        diag = np.zeros(8, np.float64)
        P = lambda x: None if x is None else x.ctypes.data  # noqa: E731
        getattr(self.L, f"orc_bermejo_conde_{self.prec}")(
            C.byref(self.s), *(P(x) for x in arrs), int(weight), float(p_exp), int(min_max), am.ctypes.data,
            bm.ctypes.data, mk.ctypes.data, C.byref(d), diag.ctypes.data)
        return arrs[1], d.value, diag

    def ilmc(self, f, mn, mx, air, sweep_max=2, min_max=True):
        """ILMC on one tracer (ext arrays of the Step's precision); returns the
        filtered copy."""
        A = lambda x: np.ascontiguousarray(x, dtype=self.dt)  # noqa: E731
        out = A(f).copy()
        a = [A(x) for x in (mn, mx, air)]
        getattr(self.L, f"orc_ilmc_{self.prec}")(C.byref(self.s), out.ctypes.data, *(x.ctypes.data for x in a),
                                                 int(sweep_max), int(min_max))
        return out

    def step(self, inp, niter=None):
        """Trajectory, then u@pmu, v@pmv, w@pt, tracers@pt (clip if cfg.mono)."""
        self.traject(inp, niter)
        out = {}
        out["u"] = self.tricub(1, [inp["src_u"]])[0]
        out["v"] = self.tricub(2, [inp["src_v"]])[0]
        out["w"] = self.tricub(3, [inp["src_w"]])[0]
        if inp.get("tracers"):
            out["tracers"] = self.tricub(3, inp["tracers"], mono=self.cfg.mono, clip=self.cfg.mono)
        return out


def adz_cfl(wpxyz, i0, in_, j0, jn, k0, nk, i0g=1, j0g=1):
    """adz_courant (src/gemdyn/src/base/adz_cfl.F90:63-189) on one domain:
    maximum horizontal, vertical and 3-D Courant numbers of the departure
    points, FP64 in the reference's order, first maximum in loop order
    (k, j, i); returns (cfl[3], idx[3, 3] global i, j, k)."""
    wp = np.asarray(wpxyz, np.float64)
    best = [(0.0, (0, 0, 0)) for _ in range(3)]
    kk = np.arange(k0, nk + 1)
    jj = np.arange(j0, jn + 1)
    ii = np.arange(i0, in_ + 1)
    sl = (slice(k0 - 1, nk), slice(j0 + 1, jn + 2), slice(i0 + 1, in_ + 2))
    x = np.abs(wp[0][sl] - float(i0g) + 1.0 - ii[None, None, :].astype(np.float64))
    y = np.abs(wp[1][sl] - float(j0g) + 1.0 - jj[None, :, None].astype(np.float64))
    z = np.abs(wp[2][sl] - kk[:, None, None].astype(np.float64))
    vals = [np.sqrt(x * x + y * y), z, np.sqrt(x * x + y * y + z * z)]
    cfl = np.zeros(3)
    idx = np.zeros((3, 3), np.int64)
    for q, v in enumerate(vals):
        flat = v.reshape(-1)
        n = int(np.argmax(flat))  # first of equal maxima in (k, j, i) order
        if flat[n] > 0.0:
            k, j, i = np.unravel_index(n, v.shape)
            cfl[q] = flat[n]
            idx[q] = (ii[i] + i0g - 1, jj[j] + j0g - 1, kk[k])
        else:
            idx[q] = (i0g - 1, j0g - 1, 0)
    return cfl, idx
