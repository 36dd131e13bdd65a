"""Python mirror of GEM's adz interface over the B200 C ABI (include/adz_b200.h).

The names follow the reference's Fortran drivers (src/gemdyn/src/base/):
``adz_set`` (adz_set.F90), ``adz_inittraj`` (adz_inittraj.F90),
``adz_traject`` (adz_traject.F90 + adz_prepareWinds.F90 + adz_interp_traj.F90),
``adz_tricub_hlt`` (adz_interp_hlt.F90), ``adz_main`` (adz_main.F90) and
``adz_tracers`` (adz_tracers.F90 with the clip of adz_post_tr.F90:81-94).

torch supplies device memory and the CUDA stream; all arithmetic runs in the
library's kernels.  There is no CPU path: without the built library or a CUDA
device every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libadz_b200.so")

REF32, FP64, MIXED = 0, 1, 2
SET_Q, SET_U, SET_V, SET_T, SET_B = 0, 1, 2, 3, 4
QV = 4  # mono flag bit: BICUBH_QV interpolation of that field (set T)
PREC_NAMES = {"ref32": REF32, "fp64": FP64, "mixed": MIXED}

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA runtime error", 3: "fewer than 4 levels",
          4: "stencil outside the extended array", 5: "non-finite wind or position",
          6: "bounded device wait expired", 7: "allocation failed", 8: "no CUDA device", 9: "size above capacity"}


class AdzError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: adz status {status} ({STATUS.get(status, '?')})")


class AdzcGrid(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "ni", "nj", "nk", "maxcfl", "i0g", "j0g", "west", "east", "south", "north",
        "pil_w", "pil_e", "pil_s", "pil_n", "lam_gbpil_t", "bc_lam_flux", "schm_advec", "itraj", "slt_winds",
        "schm_autobar")] + [
        ("bA_m", C.c_double), ("bA", C.c_double), ("inv_rayt", C.c_double), ("inv_hx", C.c_double),
        ("inv_hy", C.c_double), ("cy", C.POINTER(C.c_double)), ("zm", C.POINTER(C.c_double)),
        ("zt", C.POINTER(C.c_double)), ("zx", C.POINTER(C.c_double)), ("zmin", C.c_double), ("zmax", C.c_double),
        ("wmstar_nk", C.c_double), ("idz_t_nkm1", C.c_double)]


class AdzcInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "halox", "haloy", "nit", "njt", "i0", "in_", "j0", "jn", "i0u", "inu", "j0v", "jnv",
        "i0b", "inb", "j0b", "jnb", "k0", "k0t", "k0m")] + [
        ("npts", C.c_longlong * 4), ("iminposx", C.c_double), ("imaxposx", C.c_double),
        ("iminposy", C.c_double), ("imaxposy", C.c_double), ("pnz_m", C.c_int), ("pnz_t", C.c_int)]


class AdzcDomain(C.Structure):
    """adzc_domain: one domain of a batch (include/adz_b200.h)."""
    _fields_ = [("h", C.c_void_p), ("dt", C.c_double), ("niter", C.c_int),
                ("uu_ext", C.c_void_p), ("vv_ext", C.c_void_p), ("ww_ext", C.c_void_p),
                ("ut0", C.c_void_p), ("vt0", C.c_void_p), ("zdt0", C.c_void_p), ("wpxyz", C.c_void_p),
                ("nfields", C.c_int * 4), ("srcs", C.c_void_p), ("dsts", C.c_void_p), ("mono", C.c_void_p)]


class AdzcBcTracer(C.Structure):
    """adzc_bc_tracer: one tracer of a Bermejo-Conde call (include/adz_b200.h)."""
    _fields_ = [("p", C.c_void_p), ("m", C.c_void_p), ("lin", C.c_void_p), ("min", C.c_void_p),
                ("max", C.c_void_p), ("fo", C.c_void_p), ("fi", C.c_void_p), ("pkps", C.c_void_p),
                ("weight", C.c_int), ("p_exp", C.c_double)]


class PxPyPz(C.Structure):
    _fields_ = [("px", C.c_float), ("py", C.c_float), ("pz", C.c_float)]


_LIB = None


def lib() -> C.CDLL:
    """Load the CUDA library; raises when it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: build it with gem_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.adzc_setup.argtypes = [C.POINTER(AdzcGrid), C.POINTER(vp)]
        L.adzc_destroy.argtypes = [vp]
        L.adzc_query.argtypes = [vp, C.POINTER(AdzcInfo)]
        L.adzc_inittraj.argtypes = [vp, i, vp, vp, vp]
        L.adzc_traject.argtypes = [vp, i, d, i] + [vp] * 9
        L.adzc_tricub.argtypes = [vp, i, i, i, vp, vp, vp, vp, vp, vp, vp]
        L.adzc_status.argtypes = [vp, i, vp]
        L.adzc_ztab_create.argtypes = [vp, i, i, i, i, i, C.POINTER(vp)]
        L.adzc_ztab_destroy.argtypes = [vp]
        L.adzc_tricublin_m_n.argtypes = [vp, i, vp, vp, vp, i, i, vp]
        L.adzc_tricublin_mono_m_n.argtypes = [vp, i, vp, vp, vp, vp, vp, vp, i, i, i, vp]
        L.adzc_tricublin_zyx3_n.argtypes = [vp, i, vp, vp, vp, i, vp]
        L.adzc_tricub_sets.argtypes = [vp, i, vp, vp, vp, vp, vp]
        L.adzc_interp_traj.argtypes = [vp, i, i, vp, vp]
        L.adzc_bc_lam_zlf.argtypes = [vp, i, i, i, vp, vp, vp]
        L.adzc_traject_region.argtypes = [vp, i, d, i] + [vp] * 8 + [i, vp]
        L.adzc_tricub_sets_region.argtypes = [vp, i, vp, vp, vp, vp, i, vp]
        L.adzc_step_noalloc.argtypes = [vp, i, d, i] + [vp] * 8 + [vp, vp, vp, vp, vp]
        L.adzc_batch_create.argtypes = [i, i, vp, C.POINTER(vp)]
        L.adzc_batch_tune.argtypes = [vp, vp]
        L.adzc_batch_step.argtypes = [vp, vp]
        L.adzc_batch_query.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        L.adzc_batch_plan.argtypes = [vp, C.POINTER(C.c_int)]
        L.adzc_batch_tuned.argtypes = [vp, C.POINTER(C.c_float)]
        L.adzc_batch_select.argtypes = [vp, i, i]
        L.adzc_batch_inject.argtypes = [vp, i, C.c_longlong]
        L.adzc_batch_status.argtypes = [vp, i, vp]
        L.adzc_batch_destroy.argtypes = [vp]
        L.adzc_bermejo_conde.argtypes = [vp, i, i, vp, vp, vp, vp, i, vp, vp, vp]
        L.adzc_cfl.argtypes = [vp, vp, vp, vp, vp]
        L.adzc_ilmc.argtypes = [vp, i, i, vp, vp, vp, vp, i, i, C.POINTER(C.c_int), vp]
        L.adzc_state_save.argtypes = [vp, i, vp, vp, C.c_char_p]
        L.adzc_state_load.argtypes = [vp, i, vp, vp, C.c_char_p]
        L.adzc_slt_winds.argtypes = [vp, vp, vp]
        L.adzc_bc_lam_flux.argtypes = [vp, i, i, vp, vp, vp, vp]
        L.adzc_rhs_perturbation.argtypes = [vp, vp, i]
        L.adzc_halo_layout.argtypes = [vp, i, vp]
        L.adzc_halo_pack.argtypes = [vp, i, vp, vp, vp]
        L.adzc_halo_unpack.argtypes = [vp, i, vp, vp, vp]
        L.adzc_error_string.restype = C.c_char_p
        L.Vsearch_setup.restype = vp
        L.Vsearch_setup.argtypes = [vp, i, i, i]
        L.Vsearch_setup_plus.restype = vp
        L.Vsearch_setup_plus.argtypes = [vp, i, i, i, i, i]
        for name in ("Tricublin_zyx1_n", "Tricublin_zyx3_n"):
            getattr(L, name).argtypes = [vp, vp, vp, vp, i]
        for name in ("Tricublin_zyx1_n_m", "Tricublin_zyx1_m_n", "Tricublin_zyx1_p"):
            getattr(L, name).argtypes = [vp, vp, vp, vp, i, i]
        L.Tricublin_mono_zyx_n.argtypes = [vp, vp, vp, vp, vp, vp, vp, i]
        for name in ("Tricublin_mono_zyx_n_m", "Tricublin_mono_zyx_m_n"):
            getattr(L, name).argtypes = [vp, vp, vp, vp, vp, vp, vp, i, i]
        _LIB = L
    return _LIB


def _check(st: int, what: str):
    if st != 0:
        raise AdzError(st, what)


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr_array(tensors):
    arr = (C.c_void_p * len(tensors))()
    for q, t in enumerate(tensors):
        arr[q] = None if t is None else t.data_ptr()
    return arr


def _field_dtype(prec: int):
    return torch.float64 if prec == FP64 else torch.float32


def _pos_dtype(prec: int):
    return torch.float32 if prec == REF32 else torch.float64


# ---------------------------------------------------------------------------
# level descriptor + interpolators on device data (turbo_tricublin.c ABI)
# ---------------------------------------------------------------------------
class Ztab:
    """Vsearch_setup_plus on the device."""

    def __init__(self, levels, ni, nj, offi=0, offj=0):
        self.levels = np.ascontiguousarray(levels, dtype=np.float64)
        self.ptr = C.c_void_p()
        _check(lib().adzc_ztab_create(self.levels.ctypes.data, len(self.levels), ni, nj, offi, offj,
                                      C.byref(self.ptr)), "adzc_ztab_create")

    def __del__(self):
        try:
            lib().adzc_ztab_destroy(self.ptr)
        except Exception:
            pass


def tricublin_m_n(zt: Ztab, prec: int, fields, pos, stream=None):
    """Tricublin_zyx1_m_n on device tensors: returns d[m][n]."""
    n, m = pos.shape[0], len(fields)
    d = torch.empty((m, n), dtype=fields[0].dtype, device=pos.device)
    _check(lib().adzc_tricublin_m_n(zt.ptr, prec, d.data_ptr(), C.cast(_ptr_array(fields), C.c_void_p),
                                    pos.data_ptr(), n, m, _stream(stream)), "adzc_tricublin_m_n")
    return d


def tricublin_mono_m_n(zt: Ztab, prec: int, fields, pos, box=0, stream=None):
    n, m = pos.shape[0], len(fields)
    out = [torch.empty((m, n), dtype=fields[0].dtype, device=pos.device) for _ in range(4)]
    _check(lib().adzc_tricublin_mono_m_n(zt.ptr, prec, *(o.data_ptr() for o in out),
                                         C.cast(_ptr_array(fields), C.c_void_p), pos.data_ptr(), n, m, box,
                                         _stream(stream)), "adzc_tricublin_mono_m_n")
    return out


def tricublin_zyx3_n(zt: Ztab, prec: int, f3, pos, stream=None):
    n = pos.shape[0]
    d = torch.empty((n, 3), dtype=f3.dtype, device=pos.device)
    _check(lib().adzc_tricublin_zyx3_n(zt.ptr, prec, d.data_ptr(), f3.data_ptr(), pos.data_ptr(), n,
                                       _stream(stream)), "adzc_tricublin_zyx3_n")
    return d


# ---------------------------------------------------------------------------
# the adz step
# ---------------------------------------------------------------------------
class Adz:
    """adz_set for one tile, then the step entry points.

    Array layouts (torch shapes, C order = Fortran order reversed):
      ext fields (nk, njt, nit); wpxyz (3, nk, nj+4, ni+4) float64;
      pxyzm (nk, nj, ni, 3) float32 (REF32 warm start only).
    """

    def __init__(self, grid: AdzcGrid, keep=None, itraj: int | None = None):
        self._keep = keep
        self.grid = grid
        self.h = C.c_void_p()
        _check(lib().adzc_setup(C.byref(grid), C.byref(self.h)), "adzc_setup")
        self.info = AdzcInfo()
        _check(lib().adzc_query(self.h, C.byref(self.info)), "adzc_query")
        self.ni, self.nj, self.nk = grid.ni, grid.nj, grid.nk

    @classmethod
    def from_config(cls, cfg, lam=True, i0g=None, j0g=None, schm_advec=1, edges=None, slt_winds=False,
                    lam_gbpil_t=0, bc_lam_flux=1, schm_autobar=False):
        """adz_set for a synthetic LAM tile (gem_b200.synth.Config).  The
        tile starts at global (i0g, j0g) (default: the config's tile origin)
        and touches the LAM edges flagged in ``edges`` = (west, east, south,
        north) (default: all of them when ``lam``); pilot zones lie on those
        edges only.  bc_lam_flux: Adz_BC_LAM_flux (1 Aranami, 2 ZLF);
        schm_autobar: Schm_autobar_L."""
        from . import synth
        ga = synth.grid_arrays(cfg)
        keep = {k: np.ascontiguousarray(ga[k], dtype=np.float64) for k in ("cy", "zm", "zt", "zx")}
        e = 1 if lam else 0
        w, ea, so, no = edges if edges is not None else (e, e, e, e)
        p = cfg.pil if lam else 0
        i0g = cfg.gi0 if i0g is None else i0g
        j0g = cfg.gj0 if j0g is None else j0g
        P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        g = AdzcGrid(ni=cfg.ni, nj=cfg.nj, nk=cfg.nk, maxcfl=cfg.maxcfl, i0g=i0g, j0g=j0g,
                     west=w, east=ea, south=so, north=no, pil_w=p * w, pil_e=p * ea, pil_s=p * so, pil_n=p * no,
                     lam_gbpil_t=lam_gbpil_t, bc_lam_flux=bc_lam_flux, schm_advec=schm_advec, itraj=cfg.niter,
                     slt_winds=1 if slt_winds else 0, schm_autobar=1 if schm_autobar else 0,
                     bA_m=0.6, bA=0.6, inv_rayt=ga["inv_rayt"], inv_hx=ga["inv_hx"], inv_hy=ga["inv_hy"],
                     cy=P(keep["cy"]), zm=P(keep["zm"]), zt=P(keep["zt"]), zx=P(keep["zx"]),
                     zmin=ga["zmin"], zmax=ga["zmax"], wmstar_nk=ga["wmstar_nk"], idz_t_nkm1=ga["idz_t_nkm1"])
        return cls(g, keep)

    def __del__(self):
        try:
            lib().adzc_destroy(self.h)
        except Exception:
            pass

    # shapes ---------------------------------------------------------------
    @property
    def ext_shape(self):
        return (self.nk, self.info.njt, self.info.nit)

    def new_state(self, prec: int, device="cuda"):
        """Trajectory state arrays: (pxyzm or None, wpxyz)."""
        wp = torch.zeros((3, self.nk, self.nj + 4, self.ni + 4), dtype=torch.float64, device=device)
        px = torch.zeros((self.nk, self.nj, self.ni, 3), dtype=torch.float32, device=device) if prec == REF32 else None
        return px, wp

    def set_range(self, s: int):
        I = self.info
        return {SET_Q: (I.i0, I.in_, I.j0, I.jn, I.k0), SET_U: (I.i0u, I.inu, I.j0, I.jn, I.k0),
                SET_V: (I.i0, I.in_, I.j0v, I.jnv, I.k0), SET_T: (I.i0, I.in_, I.j0, I.jn, I.k0t),
                SET_B: (I.i0b, I.inb, I.j0b, I.jnb, 1)}[s]

    def range_mask(self, s: int, device="cpu"):
        """Boolean mask (ext layout) of the arrival points of set s."""
        i0, i1, j0, j1, k0 = self.set_range(s)
        I = self.info
        m = torch.zeros(self.ext_shape, dtype=torch.bool, device=device)
        m[k0 - 1:, j0 - 1 + I.haloy:j1 + I.haloy, i0 - 1 + I.halox:i1 + I.halox] = True
        return m

    # entry points ---------------------------------------------------------
    def adz_inittraj(self, prec: int, pxyzm, wpxyz, stream=None):
        _check(lib().adzc_inittraj(self.h, prec, None if pxyzm is None else pxyzm.data_ptr(), wpxyz.data_ptr(),
                                   _stream(stream)), "adzc_inittraj")

    def adz_traject(self, prec: int, dt: float, winds: dict, pxyzm, wpxyz, niter: int = 0, stream=None):
        """winds: uu_ext, vv_ext, ww_ext, ut0, vt0, zdt0 (ext layout, field dtype)."""
        self._zdt0 = winds["zdt0"]
        _check(lib().adzc_traject(self.h, prec, float(dt), int(niter),
                                  *(winds[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")),
                                  None if pxyzm is None else pxyzm.data_ptr(), wpxyz.data_ptr(), _stream(stream)),
               "adzc_traject")

    def adz_traject_region(self, prec: int, dt: float, winds: dict, pxyzm, wpxyz, region: int, niter: int = 0,
                           stream=None):
        """adzc_traject_region: 1 the interior of the tile, 2 the band around
        it (after the winds' halos arrived); 0 the whole tile."""
        self._zdt0 = winds["zdt0"]
        _check(lib().adzc_traject_region(self.h, prec, float(dt), int(niter),
                                         *(winds[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0",
                                                                         "zdt0")),
                                         None if pxyzm is None else pxyzm.data_ptr(), wpxyz.data_ptr(), int(region),
                                         _stream(stream)), "adzc_traject_region")

    def adz_tricub_sets_region(self, prec: int, nfields, srcs, dsts, mono, region: int, stream=None):
        """adzc_tricub_sets_region: the position sets' interior (1) or band (2)."""
        nf = (C.c_int * 4)(*nfields)
        mono_arr = (C.c_int * len(srcs))(*mono) if mono is not None else None
        _check(lib().adzc_tricub_sets_region(self.h, prec, nf, C.cast(_ptr_array(srcs), C.c_void_p),
                                             C.cast(_ptr_array(dsts), C.c_void_p), mono_arr, int(region),
                                             _stream(stream)), "adzc_tricub_sets_region")

    def set_slt_winds(self, uslt=None, vslt=None):
        """Adz_uslt, Adz_vslt (nj, ni) device tensors of the field type for
        the top-level pt positions when slt_winds is set; None to clear."""
        self._slt = (uslt, vslt)
        _check(lib().adzc_slt_winds(self.h, None if uslt is None else uslt.data_ptr(),
                                    None if vslt is None else vslt.data_ptr()), "adzc_slt_winds")

    def bc_lam_flux(self, prec: int, srcs, fo, fi, stream=None):
        """adz_BC_LAM_Aranami_hlt: FLUX_out / FLUX_in of the tracers srcs into
        fo, fi (ext tensors of the field type)."""
        _check(lib().adzc_bc_lam_flux(self.h, prec, len(srcs), C.cast(_ptr_array(srcs), C.c_void_p),
                                      C.cast(_ptr_array(fo), C.c_void_p), C.cast(_ptr_array(fi), C.c_void_p),
                                      _stream(stream)), "adzc_bc_lam_flux")

    def bc_lam_zlf(self, prec: int, setup: int, f1, f2=None, stream=None):
        """adz_BC_LAM_zlf_hlt setup 1-4 (Zerroukat-Shipway LAM treatment) on
        the ext tensors f1 (and f2 for setups 2 and 4), in place."""
        _check(lib().adzc_bc_lam_zlf(self.h, prec, int(setup), len(f1), C.cast(_ptr_array(f1), C.c_void_p),
                                     None if f2 is None else C.cast(_ptr_array(f2), C.c_void_p), _stream(stream)),
               "adzc_bc_lam_zlf")

    def set_rhs_perturbation(self, mcrhsint=None):
        """mcrhsint (nj, ni) device tensor of the field type: every later
        interpolation writes value + mcrhsint * |value - lin|; None clears."""
        self._pert = mcrhsint
        ld = 0 if mcrhsint is None else mcrhsint.stride(0)
        _check(lib().adzc_rhs_perturbation(self.h, None if mcrhsint is None else mcrhsint.data_ptr(), ld),
               "adzc_rhs_perturbation")

    def adz_tricub_hlt(self, prec: int, set_id: int, srcs, dsts, mono=None, post=None, stream=None):
        """Interpolate srcs at position set set_id into dsts (ext layout).
        mono: per-field 0 (none), 1 (bounds + clip), 2 (bounds only);
        post: optional (lin, min, max) lists of tensors for mono fields."""
        n = len(srcs)
        mono_arr = (C.c_int * n)(*mono) if mono is not None else None
        lin = mn = mx = None
        if post is not None:
            lin, mn, mx = (C.cast(_ptr_array(p), C.c_void_p) for p in post)
        _check(lib().adzc_tricub(self.h, prec, set_id, n, C.cast(_ptr_array(srcs), C.c_void_p),
                                 C.cast(_ptr_array(dsts), C.c_void_p), mono_arr, lin, mn, mx, _stream(stream)),
               "adzc_tricub")

    def adz_interp_traj(self, prec: int, set_id: int, stream=None):
        """Positions of set set_id of the last trajectory as adz_interp_traj
        stores them: an (n, 3) device tensor, float32 in REF32, float64
        otherwise, arrival points in (k, j, i) order with i fastest."""
        i0, i1, j0, j1, k0 = self.set_range(set_id)
        n = max(0, i1 - i0 + 1) * max(0, j1 - j0 + 1) * max(0, self.grid.nk - k0 + 1)
        pos = torch.empty((n, 3), dtype=torch.float32 if prec == REF32 else torch.float64, device="cuda")
        _check(lib().adzc_interp_traj(self.h, prec, set_id, pos.data_ptr(), _stream(stream)), "adzc_interp_traj")
        return pos

    def adz_tricub_sets(self, prec: int, nfields, srcs, dsts, mono=None, stream=None):
        """All position sets in one call: nfields = [nQ, nU, nV, nT]."""
        nf = (C.c_int * 4)(*nfields)
        mono_arr = (C.c_int * len(srcs))(*mono) if mono is not None else None
        _check(lib().adzc_tricub_sets(self.h, prec, nf, C.cast(_ptr_array(srcs), C.c_void_p),
                                      C.cast(_ptr_array(dsts), C.c_void_p), mono_arr, _stream(stream)),
               "adzc_tricub_sets")

    def adz_cfl(self, wpxyz, stream=None):
        """Maximum Courant numbers (horizontal, vertical, 3-D) and their global
        (i, j, k), as adz_cfl prints them."""
        cfl = torch.zeros(3, dtype=torch.float64, device=wpxyz.device)
        idx = torch.zeros(9, dtype=torch.int32, device=wpxyz.device)
        _check(lib().adzc_cfl(self.h, wpxyz.data_ptr(), cfl.data_ptr(), idx.data_ptr(), _stream(stream)), "adzc_cfl")
        return cfl.cpu().numpy(), idx.cpu().numpy().reshape(3, 3)

    def state_save(self, prec: int, pxyzm, wpxyz, path: str):
        _check(lib().adzc_state_save(self.h, prec, None if pxyzm is None else pxyzm.data_ptr(), wpxyz.data_ptr(),
                                     path.encode()), "adzc_state_save")

    def state_load(self, prec: int, pxyzm, wpxyz, path: str):
        _check(lib().adzc_state_load(self.h, prec, None if pxyzm is None else pxyzm.data_ptr(), wpxyz.data_ptr(),
                                     path.encode()), "adzc_state_load")

    def status(self, reset=True, stream=None) -> int:
        return lib().adzc_status(self.h, 1 if reset else 0, _stream(stream))

    def adz_main(self, prec, dt, winds, fields, pxyzm, wpxyz, outs, niter=0, stream=None):
        """Trajectory, then u@pmu, v@pmv, w@pt (adz_main.F90:32-60 with the
        synthetic momentum set u, v, w)."""
        self.adz_traject(prec, dt, winds, pxyzm, wpxyz, niter, stream)
        self.adz_tricub_hlt(prec, SET_U, [fields["src_u"]], [outs["u"]], stream=stream)
        self.adz_tricub_hlt(prec, SET_V, [fields["src_v"]], [outs["v"]], stream=stream)
        self.adz_tricub_hlt(prec, SET_T, [fields["src_w"]], [outs["w"]], stream=stream)

    def adz_tracers(self, prec, tracers, outs, mono: bool, stream=None):
        """All tracers of the t set in one fused launch, clipped when mono
        (adz_tracers.F90:74-99 + adz_post_tr.F90:81-94)."""
        if tracers:
            self.adz_tricub_hlt(prec, SET_T, tracers, outs, mono=[1 if mono else 0] * len(tracers), stream=stream)


def step_fused(adz: Adz, prec, dt, winds, fields, tracers, pxyzm, wpxyz, outs, tr_outs, mono, niter=0, stream=None):
    """One advection step: trajectory, then u@pmu, v@pmv and w + every tracer
    @pt through adzc_tricub_sets (one launch per position set)."""
    adz.adz_traject(prec, dt, winds, pxyzm, wpxyz, niter, stream)
    srcs = [fields["src_u"], fields["src_v"], fields["src_w"]] + list(tracers)
    dsts = [outs["u"], outs["v"], outs["w"]] + list(tr_outs)
    monos = [0, 0, 0] + [1 if mono else 0] * len(tracers)
    adz.adz_tricub_sets(prec, [0, 1, 1, 1 + len(tracers)], srcs, dsts, monos, stream)


class Batch:
    """Independent domains advanced by one persistent launch per step
    (adzc_batch_*).  ``domains``: dicts with adz (Adz, past its cold start),
    dt, winds (uu_ext, vv_ext, ww_ext, ut0, vt0, zdt0), wpxyz, nfields
    [nQ, nU, nV, nT], srcs, dsts (tensors in set order) and mono (per field)."""

    def __init__(self, prec: int, domains):
        self._keep = []
        arr = (AdzcDomain * len(domains))()
        for d, dom in enumerate(domains):
            w = dom["winds"]
            srcs, dsts = _ptr_array(dom["srcs"]), _ptr_array(dom["dsts"])
            mono = (C.c_int * len(dom["srcs"]))(*dom.get("mono", [0] * len(dom["srcs"])))
            self._keep += [dom["adz"], w, dom["wpxyz"], dom["srcs"], dom["dsts"], srcs, dsts, mono]
            a = arr[d]
            a.h, a.dt, a.niter = dom["adz"].h, float(dom["dt"]), int(dom.get("niter", 0))
            a.uu_ext, a.vv_ext, a.ww_ext = (w[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext"))
            a.ut0, a.vt0, a.zdt0 = (w[k].data_ptr() for k in ("ut0", "vt0", "zdt0"))
            a.wpxyz = dom["wpxyz"].data_ptr()
            for q in range(4):
                a.nfields[q] = int(dom["nfields"][q])
            a.srcs, a.dsts, a.mono = C.cast(srcs, C.c_void_p), C.cast(dsts, C.c_void_p), C.cast(mono, C.c_void_p)
        self.h = C.c_void_p()
        _check(lib().adzc_batch_create(prec, len(domains), C.cast(arr, C.c_void_p), C.byref(self.h)),
               "adzc_batch_create")

    def tune(self, stream=None):
        _check(lib().adzc_batch_tune(self.h, _stream(stream)), "adzc_batch_tune")

    def step(self, stream=None):
        _check(lib().adzc_batch_step(self.h, _stream(stream)), "adzc_batch_step")

    PHASED = 3  # plan of select(): one persistent launch per phase
    DOMAINS = 4  # plan of select(): every domain's own launches in turn
    DOMAINS_CONCURRENT = 5  # plan of select(): the same launches on 4 concurrent graph branches
    INJECT_SPINS, INJECT_NEED = 1, 2  # inject(): fault injection for failure-path tests

    def inject(self, what: int, value: int):
        """adzc_batch_inject: INJECT_SPINS sets the wait bound (0: default);
        INJECT_NEED makes domain 0's trajectory items wait for items that
        never come (0: clear)."""
        _check(lib().adzc_batch_inject(self.h, int(what), int(value)), "adzc_batch_inject")

    def tuned(self) -> dict:
        """The tuner's best ms per step of each plan family (None: not timed)."""
        ms = (C.c_float * 3)()
        _check(lib().adzc_batch_tuned(self.h, ms), "adzc_batch_tuned")
        return {k: (round(v, 3) if v >= 0 else None) for k, v in zip(("one_launch", "phased", "per_domain"), ms)}

    def select(self, rows: int, plan: int):
        """Pin a plan: rows per work item and 0..2 (register budget of the
        one-launch kernel), Batch.PHASED, Batch.DOMAINS or Batch.DOMAINS_CONCURRENT."""
        _check(lib().adzc_batch_select(self.h, int(rows), int(plan)), "adzc_batch_select")

    def query(self):
        r, b, n, p = C.c_int(), C.c_int(), C.c_longlong(), C.c_int()
        _check(lib().adzc_batch_query(self.h, C.byref(r), C.byref(b), C.byref(n)), "adzc_batch_query")
        _check(lib().adzc_batch_plan(self.h, C.byref(p)), "adzc_batch_plan")
        return {"rows_per_item": r.value, "blocks_per_sm": b.value, "items": n.value,
                "plan": {0: "one launch", 1: "phased (one launch per phase)",
                         2: "per-domain launches (3 per domain)",
                         3: "per-domain launches (3 per domain) on 4 concurrent branches"}[p.value]}

    def status(self, reset=True, stream=None) -> int:
        return lib().adzc_batch_status(self.h, 1 if reset else 0, _stream(stream))

    def __del__(self):
        try:
            lib().adzc_batch_destroy(self.h)
        except Exception:
            pass


def bermejo_conde(adz: Adz, prec: int, tracers, airm_p, airm_m, mask, deficit, min_max=True, diag=None,
                  stream=None):
    """Bermejo-Conde mass fixer (adzc_bermejo_conde) on a group of tracers.
    tracers: dicts with p, m (fixed in place), lin, min, max and optionally fo,
    fi, pkps, weight (1), p_exp (1.0); deficit: device float64 (ntr,)."""
    arr = (AdzcBcTracer * len(tracers))()
    ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    for q, t in enumerate(tracers):
        a = arr[q]
        a.p, a.m, a.lin = ptr(t["p"]), ptr(t["m"]), ptr(t["lin"])
        a.min, a.max = ptr(t.get("min")), ptr(t.get("max"))
        a.fo, a.fi, a.pkps = ptr(t.get("fo")), ptr(t.get("fi")), ptr(t.get("pkps"))
        a.weight, a.p_exp = int(t.get("weight", 1)), float(t.get("p_exp", 1.0))
    _check(lib().adzc_bermejo_conde(adz.h, prec, len(tracers), C.cast(arr, C.c_void_p), airm_p.data_ptr(),
                                    airm_m.data_ptr(), mask.data_ptr(), int(min_max), deficit.data_ptr(),
                                    None if diag is None else diag.data_ptr(), _stream(stream)),
           "adzc_bermejo_conde")


def ilmc(adz: Adz, prec: int, fields, mins, maxs, air, sweep_max=2, min_max=True, stream=None) -> int:
    """ILMC filter (adzc_ilmc) of tracers in place; returns the rounds used."""
    rounds = C.c_int(0)
    _check(lib().adzc_ilmc(adz.h, prec, len(fields), C.cast(_ptr_array(fields), C.c_void_p),
                           C.cast(_ptr_array(mins), C.c_void_p), C.cast(_ptr_array(maxs), C.c_void_p),
                           air.data_ptr(), int(sweep_max), int(min_max), C.byref(rounds), _stream(stream)), "adzc_ilmc")
    return rounds.value
