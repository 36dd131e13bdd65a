"""Halo exchange between tiles, host side (no GPU): the library's buffer
layout against the oracle (oracle/halo_oracle.py), argument checks, the
oracle's pack/route/unpack against its own statement of the exchange, and
gem_b200.halo's point-to-point transfer as gloo ranks on the CPU (2x2 tiles:
edge and corner neighbours; 3x1: a rank with two neighbours).  Packing on the
CPU ranks is the oracle's; the library's pack and unpack kernels are checked
on the GPU (tests/test_gpu_halo.py)."""
import ctypes as C
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import halo_oracle as HO


def _desc(ni, nj, bounds, nplanes, hx, hy, elem, nbr):
    from gem_b200 import halo
    return halo.AdzcHalo(minx=bounds[0], maxx=bounds[1], miny=bounds[2], maxy=bounds[3], ni=ni, nj=nj,
                         nplanes=nplanes, hx=hx, hy=hy, elem=elem, nbr=(C.c_int * 9)(*nbr))


@pytest.mark.parametrize("ni,nj,h,nplanes,narrays,elem,nbr", [
    (24, 20, 4, 10, 3, 4, [1] * 9),
    (17, 33, 2, 6, 1, 8, [0, 1, 0, 1, 0, 1, 0, 0, 0]),
    (5, 4, 4, 3, 13, 4, [0, 0, 0, 0, 0, 1, 0, 1, 1]),
    (9, 9, 1, 1, 64, 8, [1, 0, 1, 0, 0, 0, 1, 0, 1]),
])
def test_layout_matches_oracle(ni, nj, h, nplanes, narrays, elem, nbr):
    from gem_b200 import adz
    d = _desc(ni, nj, (1 - h, ni + h, 1 - h, nj + h), nplanes, h, h, elem, nbr)
    off = (C.c_longlong * 10)()
    assert adz.lib().adzc_halo_layout(C.byref(d), narrays, off) == 0
    nb = [0 if q == 4 else nbr[q] for q in range(9)]
    assert [o // elem for o in off] == HO.layout(ni, nj, h, h, nplanes, narrays, nb)


def test_layout_rejects_bad_descriptors():
    from gem_b200 import adz
    off = (C.c_longlong * 10)()
    ok = dict(ni=8, nj=8, bounds=(-3, 12, -3, 12), nplanes=2, hx=4, hy=4, elem=4, nbr=[1] * 9)
    assert adz.lib().adzc_halo_layout(C.byref(_desc(**ok)), 1, off) == 0
    bad = [dict(ok, hx=5), dict(ok, bounds=(-2, 12, -3, 12)), dict(ok, elem=2), dict(ok, nplanes=0),
           dict(ok, ni=3), dict(ok, bounds=(-3, 11, -3, 12))]
    for b in bad:
        assert adz.lib().adzc_halo_layout(C.byref(_desc(**b)), 1, off) == 1, b
    assert adz.lib().adzc_halo_layout(C.byref(_desc(**ok)), 0, off) == 1
    assert adz.lib().adzc_halo_layout(C.byref(_desc(**ok)), 65, off) == 1


def _tiles(decomp, h, nplanes, narrays, seed, dtype=np.float32):
    """Tile arrays cut from seeded global arrays (ext bounds 1-h:n+h), with
    the halo cells inside the domain poisoned with NaN."""
    rng = np.random.default_rng(seed)
    G = [rng.standard_normal((nplanes, decomp.gnj + 2 * h, decomp.gni + 2 * h)).astype(dtype)
         for _ in range(narrays)]
    out = []
    for r in range(decomp.size):
        t = decomp.tile(r)
        arrs = []
        for g in G:
            a = g[:, t.j0g - 1:t.j0g - 1 + t.nj + 2 * h, t.i0g - 1:t.i0g - 1 + t.ni + 2 * h].copy()
            for j in range(1 - h, t.nj + h + 1):
                for i in range(1 - h, t.ni + h + 1):
                    gi, gj = t.i0g - 1 + i, t.j0g - 1 + j
                    inside = 1 <= i <= t.ni and 1 <= j <= t.nj
                    if not inside and 1 <= gi <= decomp.gni and 1 <= gj <= decomp.gnj:
                        a[:, j + h - 1, i + h - 1] = np.nan
            arrs.append(a)
        out.append(arrs)
    return G, out


def _expected(decomp, tiles, h, k):
    bounds_of = lambda ni, nj: (1 - h, ni + h, 1 - h, nj + h)  # noqa: E731
    tl = [(decomp.tile(r).i0g, decomp.tile(r).j0g, decomp.tile(r).ni, decomp.tile(r).nj, tiles[r][k])
          for r in range(decomp.size)]
    return HO.expected(tl, bounds_of, decomp.gni, decomp.gnj, h, h)


@pytest.mark.parametrize("gni,gnj,npx,npy", [(23, 17, 3, 2), (12, 30, 1, 3), (16, 16, 2, 2)])
def test_oracle_route_equals_statement(gni, gnj, npx, npy):
    from gem_b200.halo import Decomposition
    D = Decomposition(gni, gnj, npx, npy)
    h, nplanes, narrays = 3, 4, 2
    G, tiles = _tiles(D, h, nplanes, narrays, seed=11)
    bufs = []
    for r in range(D.size):
        t = D.tile(r)
        nbr = [0 if p is None else 1 for p in D.neighbours(r)]
        bufs.append((HO.pack(tiles[r], (1 - h, t.ni + h, 1 - h, t.nj + h), t.ni, t.nj, h, h, nbr), nbr))
    for r in range(D.size):
        t = D.tile(r)
        nbr = bufs[r][1]
        off = HO.layout(t.ni, t.nj, h, h, nplanes, narrays, nbr)
        recv = np.empty(off[9], dtype=np.float32)
        for q, peer in enumerate(D.neighbours(r)):
            if peer is None:
                continue
            pt = D.tile(peer)
            poff = HO.layout(pt.ni, pt.nj, h, h, nplanes, narrays, bufs[peer][1])
            recv[off[q]:off[q + 1]] = bufs[peer][0][poff[8 - q]:poff[9 - q]]
        HO.unpack(tiles[r], recv, (1 - h, t.ni + h, 1 - h, t.nj + h), t.ni, t.nj, h, h, nbr)
    for k in range(narrays):
        exp = _expected(D, tiles, h, k)
        for r in range(D.size):
            np.testing.assert_array_equal(tiles[r][k], exp[r])
            t = D.tile(r)
            # interior-domain cells equal the global array's
            g = G[k][:, t.j0g - 1:t.j0g - 1 + t.nj + 2 * h, t.i0g - 1:t.i0g - 1 + t.ni + 2 * h]
            assert np.array_equal(tiles[r][k], g, equal_nan=True)


def test_decomposition_neighbours():
    from gem_b200.halo import Decomposition, slot
    D = Decomposition(100, 60, 4, 3)
    assert sum(D.tile(r).ni for r in range(4)) == 100
    assert [D.tile(r).i0g for r in range(4)] == [1, 26, 51, 76]
    for r in range(D.size):
        for q, p in enumerate(D.neighbours(r)):
            if p is not None:
                assert D.neighbours(p)[8 - q] == r
    assert D.tile(5).edges == (0, 0, 0, 0) and D.tile(0).edges == (1, 0, 1, 0)
    assert slot(-1, -1) == 0 and slot(1, 1) == 8 and slot(0, 1) == 7
    assert Decomposition.grid_for(8) == (4, 2) and Decomposition.grid_for(2) == (2, 1)


def _worker(rank, ws, port, npx, npy, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    import datetime
    import torch.distributed as dist
    from gem_b200 import halo
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    D = halo.Decomposition(21, 14, npx, npy)
    h, nplanes, narrays = 4, 3, 2
    _, tiles = _tiles(D, h, nplanes, narrays, seed=5)
    t = D.tile(rank)
    bounds = (1 - h, t.ni + h, 1 - h, t.nj + h)
    nbr = [0 if p is None else 1 for p in D.neighbours(rank)]

    class OracleExchange(halo.HaloExchange):  # the CPU ranks pack with the oracle
        def pack(self, arrays, stream=None):
            self.send.copy_(torch.from_numpy(HO.pack([a.numpy() for a in arrays], bounds, t.ni, t.nj, h, h, nbr)))

        def unpack(self, arrays, stream=None):
            HO.unpack([a.numpy() for a in arrays], self.recv.numpy(), bounds, t.ni, t.nj, h, h, nbr)

    ex = OracleExchange(D, rank, bounds, nplanes, h, h, torch.float32, narrays, device="cpu")
    mine = [torch.from_numpy(a) for a in tiles[rank]]
    ex.exchange(mine)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, [a.numpy() for a in mine]))


@pytest.mark.skipif(not torch.distributed.is_gloo_available(), reason="gloo backend missing")
@pytest.mark.parametrize("npx,npy", [(2, 2), (3, 1)])
def test_gloo_ranks_exchange(npx, npy):
    from gem_b200.halo import Decomposition
    ws = npx * npy
    port = 29600 + (os.getpid() % 1500) + 7 * npx
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, npx, npy, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    D = Decomposition(21, 14, npx, npy)
    _, tiles = _tiles(D, 4, 3, 2, seed=5)
    for k in range(2):
        exp = _expected(D, tiles, 4, k)
        for r in range(ws):
            np.testing.assert_array_equal(res[r][k], exp[r])


@pytest.mark.parametrize("ws", [1, 2, 4, 8])
def test_bench_tiles_form_one_domain(ws):
    import bench
    tiles = [bench.tile_config((64, 48, 10), r, ws, 2) for r in range(ws)]
    decomp = tiles[0][2]
    assert decomp.size == ws and decomp.gni == 64 * decomp.npx and decomp.gnj == 48 * decomp.npy
    seen = set()
    for r, (cfg, tile, _) in enumerate(tiles):
        assert (cfg.ni, cfg.nj, cfg.nk) == (64, 48, 10) and (tile.ni, tile.nj) == (64, 48)
        assert (cfg.gi0, cfg.gj0, cfg.gni, cfg.gnj) == (tile.i0g, tile.j0g, decomp.gni, decomp.gnj)
        seen.add((tile.i0g, tile.j0g))
    assert len(seen) == ws and len({c.seed for c, _, _ in tiles}) == ws
    if ws == 1:
        assert tiles[0][1].edges == (1, 1, 1, 1)


def _band_boxes(t, m, region):
    """Interior (region 1: at least m from every side with a neighbour) or
    the band around it (region 2), as (i0, i1, j0, j1) boxes of local
    indices, in the way adzc_traject_region cuts a tile."""
    w, e, s, n = [0 if edge else m for edge in t.edges]
    ni, nj = t.ni, t.nj
    if region == 1:
        return [(1 + w, ni - e, 1 + s, nj - n)] if ni - e >= 1 + w and nj - n >= 1 + s else []
    xw1, xe0 = min(w, ni), max(w + 1, ni - e + 1)
    ys1, yn0 = min(s, nj), max(s + 1, nj - n + 1)
    boxes = [(1, xw1, 1, nj), (xe0, ni, 1, nj), (xw1 + 1, xe0 - 1, 1, ys1), (xw1 + 1, xe0 - 1, yn0, nj)]
    return [b for b in boxes if b[1] >= b[0] and b[3] >= b[2]]


def _stencil_sum(a, h, boxes, out, r=2):
    """out(i, j) = sum of a over the (2r+1)^2 cells around (i, j), for the
    points of the boxes (a, out: (planes, nj + 2h, ni + 2h))."""
    for i0, i1, j0, j1 in boxes:
        for j in range(j0, j1 + 1):
            for i in range(i0, i1 + 1):
                out[:, j + h - 1, i + h - 1] = a[:, j + h - 1 - r:j + h + r, i + h - 1 - r:i + h + r].sum(axis=(1, 2))


def _overlap_worker(rank, ws, port, npx, npy, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank))
    import datetime
    import torch.distributed as dist
    from gem_b200 import halo
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    D = halo.Decomposition(21, 14, npx, npy)
    h, nplanes = 4, 3
    _, tiles = _tiles(D, h, nplanes, 1, seed=8)
    t = D.tile(rank)
    bounds = (1 - h, t.ni + h, 1 - h, t.nj + h)
    nbr = [0 if p is None else 1 for p in D.neighbours(rank)]

    class OracleExchange(halo.HaloExchange):
        def pack(self, arrays, stream=None):
            self.send.copy_(torch.from_numpy(HO.pack([a.numpy() for a in arrays], bounds, t.ni, t.nj, h, h, nbr)))

        def unpack(self, arrays, stream=None):
            HO.unpack([a.numpy() for a in arrays], self.recv.numpy(), bounds, t.ni, t.nj, h, h, nbr)

    ex = OracleExchange(D, rank, bounds, nplanes, h, h, torch.float32, 1, device="cpu")
    a = torch.from_numpy(tiles[rank][0])
    out = np.full_like(tiles[rank][0], np.nan)
    # the overlapped schedule: the interior while the halo is in flight (its
    # halo cells still NaN), the band once it has arrived
    ex.pack([a])
    reqs = ex.start()
    _stencil_sum(a.numpy(), h, _band_boxes(t, 2, 1), out)
    ex.finish(reqs)
    ex.unpack([a])
    _stencil_sum(a.numpy(), h, _band_boxes(t, 2, 2), out)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


@pytest.mark.skipif(not torch.distributed.is_gloo_available(), reason="gloo backend missing")
@pytest.mark.parametrize("npx,npy", [(2, 2), (3, 1)])
def test_gloo_ranks_overlap_interior_with_exchange(npx, npy):
    """The schedule of TiledStep(overlap=True) on CPU ranks: the transfer is
    started, the interior computed beside it, the transfer finished and
    unpacked, the band computed.  Every point equals the plain schedule's
    (exchange, then the whole tile), and the interior never read a halo cell
    (they were NaN until the unpack)."""
    from gem_b200.halo import Decomposition
    ws = npx * npy
    port = 31200 + (os.getpid() % 1500) + 7 * npx
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_overlap_worker, args=(r, ws, port, npx, npy, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    D = Decomposition(21, 14, npx, npy)
    _, tiles = _tiles(D, 4, 3, 1, seed=8)
    exp = _expected(D, tiles, 4, 0)
    for r in range(ws):
        t = D.tile(r)
        want = np.full_like(exp[r], np.nan)
        _stencil_sum(exp[r], 4, [(1, t.ni, 1, t.nj)], want)
        inner = (slice(None), slice(4, 4 + t.nj), slice(4, 4 + t.ni))
        assert not np.isnan(res[r][inner]).any()
        np.testing.assert_array_equal(res[r][inner], want[inner])
        # the band boxes and the interior cover the tile once
        cover = np.zeros((t.nj, t.ni), int)
        for reg in (1, 2):
            for i0, i1, j0, j1 in _band_boxes(t, 2, reg):
                cover[j0 - 1:j1, i0 - 1:i1] += 1
        assert (cover == 1).all()
