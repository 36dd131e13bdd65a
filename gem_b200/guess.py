"""Learned starting guess for the departure-point iteration, and the
iteration run to a convergence tolerance (adzc_traject_tol, adzc_guess_*,
adzc_mlp_* in include/adz_b200.h).

The reference runs a fixed number of fixed-point updates from the arrival
point on a cold start (adz_inittraj.F90, adz_traject.F90).  Here a network
guesses the departure displacement, and the plain update finishes from the
guess until no coordinate moves by more than ``TOL`` grid indices.  Points whose
guess does not converge within the update limit fall back to the plain start.

Convergence tolerance of this project: ``TOL = 1e-4`` grid indices (x, y and the
vertical level index), i.e. 0.25 m on a 2.5 km grid; the interpolation weights
then change by less than 1e-4 of their range.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import adz as A

NFEAT, HID, NOUT = 82, 128, 3
NPARAM = HID * NFEAT + HID + HID * HID + HID + NOUT * HID + NOUT
TOL = 1e-4
MAXIT = 30
SHAPES = {"W1": (HID, NFEAT), "b1": (HID,), "W2": (HID, HID), "b2": (HID,), "W3": (NOUT, HID), "b3": (NOUT,)}
ORDER = ("W1", "b1", "W2", "b2", "W3", "b3")
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(__file__), "data", "guess_mlp.npz")

_bound = False


def _lib():
    global _bound
    L = A.lib()
    if not _bound:
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.adzc_traject_tol.argtypes = [vp, i, d, d, i, i] + [vp] * 6 + [vp, vp, vp, vp]
        L.adzc_guess_create.argtypes = [vp, C.POINTER(vp)]
        L.adzc_guess_destroy.argtypes = [vp]
        L.adzc_guess_inject.argtypes = [vp, i, C.c_longlong]
        L.adzc_guess_npoints.argtypes = [vp]
        L.adzc_guess_npoints.restype = C.c_longlong
        L.adzc_guess_apply.argtypes = [vp, vp, d, vp, vp, vp, vp, vp, vp]
        L.adzc_guess_features.argtypes = [vp, d, vp, vp, vp, vp, C.c_longlong, vp, vp]
        L.adzc_guess_apply_coarse.argtypes = [vp, vp, d, vp, vp, vp, i, vp, vp]
        L.adzc_traject_guess.argtypes = [vp, vp, i, d, d, i] + [vp] * 6 + [vp, vp, vp, vp]
        L.adzc_mlp_create.argtypes = [vp, i, C.POINTER(vp)]
        L.adzc_mlp_destroy.argtypes = [vp]
        L.adzc_mlp_forward.argtypes = [vp, vp, i, vp, vp]
        L.adzc_mlp_grad.argtypes = [vp, vp, vp, i, vp]
        L.adzc_mlp_adam.argtypes = [vp, C.c_float, vp]
        L.adzc_mlp_read.argtypes = [vp, i, vp, vp]
        _bound = True
    return L


def flatten(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[k], np.float32).ravel() for k in ORDER]).astype(np.float32)


def unflatten(v) -> dict:
    v = np.asarray(v, np.float32)
    out, o = {}, 0
    for k in ORDER:
        n = int(np.prod(SHAPES[k]))
        out[k] = v[o:o + n].reshape(SHAPES[k]).copy()
        o += n
    return out


def init_params(seed: int = 0) -> dict:
    """Initial weights: normal with variance 2 / fan-in, output layer scaled
    by 0.1, zero biases."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, (n, k) in {"1": (HID, NFEAT), "2": (HID, HID), "3": (NOUT, HID)}.items():
        p["W" + name] = (rng.standard_normal((n, k)) * np.sqrt(2.0 / k)).astype(np.float32)
        p["b" + name] = np.zeros(n, np.float32)
    p["W3"] *= np.float32(0.1)
    return p


def load_weights(path: str = DEFAULT_WEIGHTS) -> dict:
    with np.load(path) as z:
        return {k: z[k].astype(np.float32) for k in ORDER}


def npoints(ad: A.Adz) -> int:
    return int(_lib().adzc_guess_npoints(ad.h))


def arrival_index(ad: A.Adz):
    """k00 and the (k, j, i) shape of the arrival points, in feature order."""
    n = npoints(ad)
    nk_pts = n // (ad.ni * ad.nj)
    return ad.nk - nk_pts + 1, (nk_pts, ad.nj, ad.ni)


class GuessNet:
    """BF16 tensor-core inference of the guess network (adzc_guess_*)."""

    def __init__(self, params: dict | None = None):
        p = load_weights() if params is None else params
        self._arrs = [np.ascontiguousarray(p[k], np.float32) for k in ORDER]
        ptrs = (C.c_void_p * 6)(*(a.ctypes.data for a in self._arrs))
        self.h = C.c_void_p()
        A._check(_lib().adzc_guess_create(C.cast(ptrs, C.c_void_p), C.byref(self.h)), "adzc_guess_create")

    INJECT_SPINS, INJECT_WITHHOLD = 1, 3  # inject(): fault injection for failure-path tests

    def inject(self, what: int, value: int):
        """adzc_guess_inject: INJECT_SPINS sets the bound of the kernel's
        waits in polls (0: default); INJECT_WITHHOLD 1 makes each CTA's first
        tile never signal its MMA, so the wait runs out (0 clears)."""
        A._check(_lib().adzc_guess_inject(self.h, int(what), int(value)), "adzc_guess_inject")

    def apply(self, ad: A.Adz, dt: float, winds: dict, wpxyz=None, disp=None, stream=None):
        """Start points into wpxyz and/or the displacement into disp (npoints x 3)."""
        A._check(_lib().adzc_guess_apply(ad.h, self.h, float(dt), *(winds[k].data_ptr() for k in
                                                                      ("uu_ext", "vv_ext", "ww_ext")),
                                         None if wpxyz is None else wpxyz.data_ptr(),
                                         None if disp is None else disp.data_ptr(), A._stream(stream)),
                 "adzc_guess_apply")

    def apply_coarse(self, ad: A.Adz, dt: float, winds: dict, wpxyz, stride: int, stream=None):
        """The network on every stride-th point in i and j only, start points
        of all points from the displacements interpolated bilinearly."""
        A._check(_lib().adzc_guess_apply_coarse(ad.h, self.h, float(dt),
                                                *(winds[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext")),
                                                int(stride), wpxyz.data_ptr(), A._stream(stream)),
                 "adzc_guess_apply_coarse")

    def __del__(self):
        try:
            _lib().adzc_guess_destroy(self.h)
        except Exception:
            pass


def features(ad: A.Adz, dt: float, winds: dict, idx=None, stream=None):
    """FP32 features (n x 82) of the arrival points idx (all when None)."""
    n = npoints(ad) if idx is None else int(idx.numel())
    out = torch.empty((n, NFEAT), dtype=torch.float32, device="cuda")
    A._check(_lib().adzc_guess_features(ad.h, float(dt), *(winds[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext")),
                                        None if idx is None else idx.data_ptr(), n, out.data_ptr(),
                                        A._stream(stream)), "adzc_guess_features")
    return out


def traject_tol(ad: A.Adz, prec: int, dt: float, winds: dict, wpxyz, tol=TOL, maxit=MAXIT, start=0, iters=None,
                stats=None, stream=None):
    """adzc_traject_tol: start 0 from the arrival point, 1 from wpxyz."""
    A._check(_lib().adzc_traject_tol(ad.h, prec, float(dt), float(tol), int(maxit), int(start),
                                     *(winds[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")),
                                     wpxyz.data_ptr(), None if iters is None else iters.data_ptr(),
                                     None if stats is None else stats.data_ptr(), A._stream(stream)),
             "adzc_traject_tol")


def traject_guess(ad: A.Adz, net: GuessNet, dt: float, winds: dict, wpxyz, stride=8, tol=TOL, maxit=MAXIT,
                  iters=None, stats=None, stream=None):
    """adzc_traject_guess (MIXED): the network on every stride-th point in i
    and j, then the tolerance iteration from the interpolated displacements."""
    A._check(_lib().adzc_traject_guess(ad.h, net.h, int(stride), float(dt), float(tol), int(maxit),
                                       *(winds[k].data_ptr() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0",
                                                                       "zdt0")),
                                       wpxyz.data_ptr(), None if iters is None else iters.data_ptr(),
                                       None if stats is None else stats.data_ptr(), A._stream(stream)),
             "adzc_traject_guess")


def displacement(ad: A.Adz, wpxyz, i0g=1, j0g=1):
    """Departure displacement (npoints x 3) of the positions in wpxyz, in
    feature order: (X - x, Y - y, k - z)."""
    k00, (nkp, nj, ni) = arrival_index(ad)
    wp = wpxyz[:, k00 - 1:, 2:nj + 2, 2:ni + 2]
    X = torch.arange(ni, device=wp.device, dtype=torch.float64) + i0g
    Y = torch.arange(nj, device=wp.device, dtype=torch.float64) + j0g
    Z = torch.arange(k00, k00 + nkp, device=wp.device, dtype=torch.float64)
    d = torch.stack([X.view(1, 1, -1) - wp[0], Y.view(1, -1, 1) - wp[1], Z.view(-1, 1, 1) - wp[2]], dim=-1)
    return d.reshape(-1, 3)


class Trainer:
    """FP32 training of the guess network on device data (adzc_mlp_*)."""

    def __init__(self, params: dict, max_batch: int):
        self._p = flatten(params)
        self.h = C.c_void_p()
        self.max_batch = max_batch
        A._check(_lib().adzc_mlp_create(self._p.ctypes.data, int(max_batch), C.byref(self.h)), "adzc_mlp_create")

    def grad(self, x, t, stream=None):
        A._check(_lib().adzc_mlp_grad(self.h, x.data_ptr(), t.data_ptr(), int(x.shape[0]), A._stream(stream)),
                 "adzc_mlp_grad")

    def adam(self, lr: float, stream=None):
        A._check(_lib().adzc_mlp_adam(self.h, C.c_float(lr), A._stream(stream)), "adzc_mlp_adam")

    def forward(self, x, stream=None):
        y = torch.empty((x.shape[0], NOUT), dtype=torch.float32, device=x.device)
        A._check(_lib().adzc_mlp_forward(self.h, x.data_ptr(), int(x.shape[0]), y.data_ptr(), A._stream(stream)),
                 "adzc_mlp_forward")
        return y

    def _read(self, what, n, stream=None):
        out = np.empty(n, np.float32)
        A._check(_lib().adzc_mlp_read(self.h, what, out.ctypes.data, A._stream(stream)), "adzc_mlp_read")
        return out

    def params(self) -> dict:
        return unflatten(self._read(0, NPARAM))

    def grads(self) -> dict:
        return unflatten(self._read(1, NPARAM))

    def loss(self) -> float:
        return float(self._read(2, 1)[0])

    def __del__(self):
        try:
            _lib().adzc_mlp_destroy(self.h)
        except Exception:
            pass
