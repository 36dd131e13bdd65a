"""Halo exchange between the tiles of a 2-D decomposition.

The path's rpn_comm_xch_halo calls (non-periodic limited-area domain):

- the departure winds before the step, width Adz_halox (dynstep.F90:52-53);
- the tracer sources, same width (adz_interp_hlt.F90:87-88);
- Adz_wpxyz between the trajectory and the position sets, width 2
  (adz_traject.F90:121-122).

rpn_comm itself (the rpncomm submodule, src/rpn-si/rpncomm, branch main) is
not vendored.  Its published behaviour is restated here: each tile's halo
strips are filled from the neighbours' interiors; halos on the domain edges
stay as they are.

The library packs a tile's strips for all eight neighbours into one buffer
and unpacks the received strips (adzc_halo_pack / adzc_halo_unpack, one
launch each).  The bytes move by torch.distributed point-to-point operations,
grouped into one batch per exchange (NCCL send/recv over NVLink on GPUs).
Corner strips come from the diagonal neighbours in the same batch.  Inside
the global domain this gives what rpn_comm's two passes (x, then y) give.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch
import torch.distributed as dist

from . import adz as A


class AdzcHalo(C.Structure):
    """adzc_halo (include/adz_b200.h)."""
    _fields_ = [("minx", C.c_int), ("maxx", C.c_int), ("miny", C.c_int), ("maxy", C.c_int), ("ni", C.c_int),
                ("nj", C.c_int), ("nplanes", C.c_longlong), ("hx", C.c_int), ("hy", C.c_int), ("elem", C.c_int),
                ("nbr", C.c_int * 9)]


def slot(dx: int, dy: int) -> int:
    """Neighbour slot of direction (dx, dy); 8 - slot is the opposite one."""
    return 3 * (dy + 1) + (dx + 1)


@dataclass(frozen=True)
class Tile:
    rank: int
    px: int
    py: int
    i0g: int   # global index of local (1, 1)
    j0g: int
    ni: int
    nj: int
    edges: tuple  # (west, east, south, north): 1 on the domain's edges


class Decomposition:
    """A gni x gnj domain cut into npx x npy tiles, rank = px + npx * py.
    Extents are split as evenly as possible, the first tiles taking the
    remainder."""

    def __init__(self, gni: int, gnj: int, npx: int, npy: int):
        if npx < 1 or npy < 1 or gni < npx or gnj < npy:
            raise ValueError("decomposition larger than the domain")
        self.gni, self.gnj, self.npx, self.npy = gni, gnj, npx, npy
        self.xs = self._split(gni, npx)
        self.ys = self._split(gnj, npy)

    @staticmethod
    def _split(n: int, p: int):
        base, extra = divmod(n, p)
        out, start = [], 1
        for q in range(p):
            size = base + (1 if q < extra else 0)
            out.append((start, size))
            start += size
        return out

    @property
    def size(self) -> int:
        return self.npx * self.npy

    def tile(self, rank: int) -> Tile:
        px, py = rank % self.npx, rank // self.npx
        (i0, ni), (j0, nj) = self.xs[px], self.ys[py]
        edges = (int(px == 0), int(px == self.npx - 1), int(py == 0), int(py == self.npy - 1))
        return Tile(rank, px, py, i0, j0, ni, nj, edges)

    def neighbour(self, rank: int, dx: int, dy: int):
        px, py = rank % self.npx + dx, rank // self.npx + dy
        if 0 <= px < self.npx and 0 <= py < self.npy:
            return px + self.npx * py
        return None

    def neighbours(self, rank: int) -> list:
        """Rank in each of the 9 slots (None: no neighbour; slot 4 is the tile)."""
        return [None if q == 4 else self.neighbour(rank, q % 3 - 1, q // 3 - 1) for q in range(9)]

    @staticmethod
    def grid_for(n: int) -> tuple:
        """The most nearly square npx x npy = n, npx >= npy."""
        npy = int(n ** 0.5)
        while n % npy:
            npy -= 1
        return n // npy, npy


class HaloExchange:
    """Exchange of one tile's arrays that share bounds, width and type.

    ``bounds`` = (minx, maxx, miny, maxy) of the arrays (Fortran, interior
    1..ni, 1..nj); ``nplanes`` the product of their trailing extents.  The
    arrays are torch tensors whose memory is that Fortran array.  The send
    and receive buffers are allocated once, on ``device``."""

    def __init__(self, decomp: Decomposition, rank: int, bounds, nplanes: int, hx: int, hy: int, dtype,
                 narrays: int, device="cuda", group=None):
        self.decomp, self.rank, self.group = decomp, rank, group
        self.tile = decomp.tile(rank)
        self.peers = decomp.neighbours(rank)
        self.narrays = narrays
        self.dtype = dtype
        elem = torch.empty((), dtype=dtype).element_size()
        minx, maxx, miny, maxy = bounds
        nbr = (C.c_int * 9)(*[0 if p is None else 1 for p in self.peers])
        self.desc = AdzcHalo(minx=minx, maxx=maxx, miny=miny, maxy=maxy, ni=self.tile.ni, nj=self.tile.nj,
                             nplanes=nplanes, hx=hx, hy=hy, elem=elem, nbr=nbr)
        self.array_numel = (maxx - minx + 1) * (maxy - miny + 1) * nplanes
        off = (C.c_longlong * 10)()
        A._check(A.lib().adzc_halo_layout(C.byref(self.desc), narrays, off), "adzc_halo_layout")
        self.offsets = [o // elem for o in off]
        total = self.offsets[9]
        self.send = torch.empty(total, dtype=dtype, device=device)
        self.recv = torch.empty(total, dtype=dtype, device=device)

    def segment(self, buf: torch.Tensor, q: int) -> torch.Tensor:
        return buf[self.offsets[q]:self.offsets[q + 1]]

    def _arrays(self, arrays):
        if len(arrays) != self.narrays:
            raise ValueError(f"{len(arrays)} arrays for an exchange of {self.narrays}")
        for a in arrays:
            if a.dtype != self.dtype or a.numel() != self.array_numel or not a.is_contiguous():
                raise ValueError("array does not match the exchange's bounds or type")
        return C.cast(A._ptr_array(arrays), C.c_void_p)

    def pack(self, arrays, stream=None):
        A._check(A.lib().adzc_halo_pack(C.byref(self.desc), self.narrays, self._arrays(arrays),
                                        self.send.data_ptr(), A._stream(stream)), "adzc_halo_pack")

    def unpack(self, arrays, stream=None):
        A._check(A.lib().adzc_halo_unpack(C.byref(self.desc), self.narrays, self._arrays(arrays),
                                          self.recv.data_ptr(), A._stream(stream)), "adzc_halo_unpack")

    def start(self):
        """Send segment q to the neighbour in slot q and receive segment q
        from it, for every neighbour, as one batch of point-to-point ops,
        without waiting: the requests to give to ``finish``.  Two tiles of a
        non-periodic grid are neighbours in one direction only, so every pair
        of ranks exchanges one message each way.  With NCCL the transfer runs
        on NCCL's stream, ordered after the work already on the current
        stream; work enqueued next on the current stream runs beside it."""
        ops = []
        for q, peer in enumerate(self.peers):
            if peer is None or self.offsets[q + 1] == self.offsets[q]:
                continue
            ops.append(dist.P2POp(dist.isend, self.segment(self.send, q), peer, self.group))
            ops.append(dist.P2POp(dist.irecv, self.segment(self.recv, q), peer, self.group))
        return dist.batch_isend_irecv(ops) if ops else []

    @staticmethod
    def finish(reqs):
        """Wait for a transfer started by ``start`` (with NCCL: the current
        stream waits for it; with gloo: the host does)."""
        for req in reqs:
            req.wait()

    def transfer(self):
        """``start`` then ``finish``."""
        self.finish(self.start())

    def exchange(self, arrays):
        """pack, transfer, unpack on the current stream (the one the
        point-to-point batch orders itself after): the halos of ``arrays``
        now hold the neighbours' interior values."""
        self.pack(arrays)
        self.transfer()
        self.unpack(arrays)


def ext_exchange(decomp: Decomposition, rank: int, ad: A.Adz, dtype, narrays: int, device="cuda", group=None):
    """Exchange of ext-layout arrays (1-H:ni+H, 1-H:nj+H, nk) of a tile's
    handle over the full halo H = Adz_halox (winds, sources)."""
    I = ad.info
    bounds = (1 - I.halox, ad.ni + I.halox, 1 - I.haloy, ad.nj + I.haloy)
    return HaloExchange(decomp, rank, bounds, ad.nk, I.halox, I.haloy, dtype, narrays, device, group)


def wpxyz_exchange(decomp: Decomposition, rank: int, ad: A.Adz, device="cuda", group=None):
    """Exchange of Adz_wpxyz (-1:ni+2, -1:nj+2, nk, 3), width 2."""
    bounds = (-1, ad.ni + 2, -1, ad.nj + 2)
    return HaloExchange(decomp, rank, bounds, 3 * ad.nk, 2, 2, torch.float64, 1, device, group)


WIND_KEYS = ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")


class TiledStep:
    """One advection step of a tile of a decomposed domain (adz_main with its
    halo exchanges):

    1. exchange the winds and the sources (width Adz_halox): departure winds
       as dynstep.F90:52-53, sources as adz_interp_hlt.F90:87-88, and the
       arrival winds, whose halo the host model fills with its own exchange
       before the step;
    2. adzc_traject;
    3. exchange Adz_wpxyz, width 2 (adz_traject.F90:121-122);
    4. adzc_tricub_sets: u@pmu, v@pmv, w and the tracers @pt.

    Packing, unpacking and the step run on the current CUDA stream; the
    transfers are torch.distributed point-to-point batches in the
    process group ``group``.

    With ``overlap`` (the default) each exchange runs beside the part of the
    step that needs none of its values (adzc_traject_region,
    adzc_tricub_sets_region): the winds' and sources' exchange beside the
    trajectory of the tile's interior, the exchange of wpxyz beside the
    interior's position sets; the band around the interior follows each
    exchange.  The results are those of the plain schedule bit for bit."""

    def __init__(self, decomp: Decomposition, rank: int, ad: A.Adz, prec: int, ntracers: int, device="cuda",
                 group=None):
        self.ad, self.prec = ad, prec
        self.ex = ext_exchange(decomp, rank, ad, A._field_dtype(prec), len(WIND_KEYS) + 3 + ntracers, device, group)
        self.exw = wpxyz_exchange(decomp, rank, ad, device, group)

    def __call__(self, dt, winds, fields, tracers, pxyzm, wpxyz, outs, tr_outs, mono, niter=0, overlap=True):
        srcs = [fields["src_u"], fields["src_v"], fields["src_w"]] + list(tracers)
        arrays = [winds[k] for k in WIND_KEYS] + srcs
        dsts = [outs["u"], outs["v"], outs["w"]] + list(tr_outs)
        monos = [0, 0, 0] + [1 if mono else 0] * len(tracers)
        nf = [0, 1, 1, 1 + len(tracers)]
        if not overlap:
            self.ex.exchange(arrays)
            self.ad.adz_traject(self.prec, dt, winds, pxyzm, wpxyz, niter)
            self.exw.exchange([wpxyz])
            self.ad.adz_tricub_sets(self.prec, nf, srcs, dsts, monos)
            return
        self.ex.pack(arrays)
        reqs = self.ex.start()
        self.ad.adz_traject_region(self.prec, dt, winds, pxyzm, wpxyz, 1, niter)
        self.ex.finish(reqs)
        self.ex.unpack(arrays)
        self.ad.adz_traject_region(self.prec, dt, winds, pxyzm, wpxyz, 2, niter)
        self.exw.pack([wpxyz])
        reqs = self.exw.start()
        self.ad.adz_tricub_sets_region(self.prec, nf, srcs, dsts, monos, 1)
        self.exw.finish(reqs)
        self.exw.unpack([wpxyz])
        self.ad.adz_tricub_sets_region(self.prec, nf, srcs, dsts, monos, 2)
