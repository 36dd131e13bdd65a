"""Halo exchange on the GPU (adzc_halo_pack / adzc_halo_unpack).

1. The library's send buffers and unpacked arrays equal the oracle's
   (oracle/halo_oracle.py) bit for bit: FP32 ext arrays of width 4 and the
   FP64 wpxyz layout of width 2, with every neighbour pattern of a 3x3
   decomposition.
2. A step on a decomposed domain equals the step on the undivided domain,
   bit for bit, on every tile's interior: positions (wpxyz) and every
   interpolated field.  Each tile starts from its window of the global
   inputs with the halo cells inside the domain set to NaN.  Exchanges
   refill them: winds and sources before the trajectory, wpxyz between the
   trajectory and the position sets.  Tiles are emulated on one GPU: every
   tile packs, the test copies segment 8 - q of the neighbour into segment q,
   every tile unpacks.  No kernel waits on another.  The undivided step is
   itself pinned to the adz oracle (tests/test_gpu_parity.py)."""
import numpy as np
import pytest
import torch

from oracle import halo_oracle as HO

pytestmark = pytest.mark.gpu


def _need_cuda():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")


@pytest.mark.parametrize("h,minx_off,dtype,narrays", [(4, 0, torch.float32, 5), (2, 0, torch.float64, 1),
                                                       (3, 2, torch.float32, 2)])
def test_pack_unpack_match_oracle(h, minx_off, dtype, narrays):
    _need_cuda()
    from gem_b200.halo import Decomposition, HaloExchange
    D = Decomposition(40, 29, 3, 3)
    g = torch.Generator(device="cuda").manual_seed(3)
    nplanes = 6
    for r in range(D.size):
        t = D.tile(r)
        # arrays may carry a wider halo than the one exchanged
        bounds = (1 - h - minx_off, t.ni + h + minx_off, 1 - h - minx_off, t.nj + h + minx_off)
        shape = (nplanes, bounds[3] - bounds[2] + 1, bounds[1] - bounds[0] + 1)
        arrs = [torch.randn(shape, generator=g, device="cuda", dtype=torch.float64).to(dtype) for _ in range(narrays)]
        ex = HaloExchange(D, r, bounds, nplanes, h, h, dtype, narrays)
        ex.pack(arrs)
        nbr = [0 if p is None else 1 for p in D.neighbours(r)]
        host = [a.cpu().numpy() for a in arrs]
        ref = HO.pack(host, bounds, t.ni, t.nj, h, h, nbr)
        torch.cuda.synchronize()
        assert np.array_equal(ex.send.cpu().numpy(), ref)
        ex.recv.copy_(torch.randn(ex.recv.shape, generator=g, device="cuda", dtype=torch.float64).to(dtype))
        ex.unpack(arrs)
        HO.unpack(host, ex.recv.cpu().numpy(), bounds, t.ni, t.nj, h, h, nbr)
        torch.cuda.synchronize()
        for a, b in zip(arrs, host):
            assert np.array_equal(a.cpu().numpy(), b)


def _route(exs, D, which_send="send", which_recv="recv"):
    for r, ex in enumerate(exs):
        for q, p in enumerate(D.neighbours(r)):
            if p is not None:
                ex.segment(getattr(ex, which_recv), q).copy_(exs[p].segment(getattr(exs[p], which_send), 8 - q))


def _poison_ext(a, t, gni, gnj, H):
    """NaN in the halo cells of a tile's ext array that lie inside the domain."""
    nk, nyt, nxt = a.shape
    i = torch.arange(1 - H, t.ni + H + 1, device=a.device)
    j = torch.arange(1 - H, t.nj + H + 1, device=a.device)
    gi, gj = i + t.i0g - 1, j + t.j0g - 1
    inside_dom = ((gj >= 1) & (gj <= gnj)).view(-1, 1) & ((gi >= 1) & (gi <= gni)).view(1, -1)
    interior = ((j >= 1) & (j <= t.nj)).view(-1, 1) & ((i >= 1) & (i <= t.ni)).view(1, -1)
    a[:, inside_dom & ~interior] = float("nan")


@pytest.mark.parametrize("prec_name,npx,npy,split", [("mixed", 2, 2, False), ("fp64", 3, 2, False),
                                                      ("ref32", 2, 2, False), ("mixed", 2, 2, True),
                                                      ("fp64", 3, 2, True), ("ref32", 2, 2, True)])
def test_decomposed_step_equals_single_tile(prec_name, npx, npy, split):
    """split: the schedule that overlaps the exchanges (adzc_traject_region,
    adzc_tricub_sets_region): each tile's interior runs while its halo cells
    are still NaN, the band after the exchange; bit-exact all the same."""
    _need_cuda()
    import copy
    from gem_b200 import adz as A, synth
    from gem_b200.halo import Decomposition, ext_exchange, wpxyz_exchange
    prec = A.PREC_NAMES[prec_name]
    dt_ = A._field_dtype(prec)
    cfg = synth.config_small(50, 40, 20)
    cfg.ntracers = 2
    H = cfg.halo
    inp = synth.make_inputs(cfg, device="cuda", dtype=dt_)
    names = ["uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0"]
    fields = [inp["src_u"], inp["src_v"], inp["src_w"]] + inp["tracers"]
    mono = [0, 0, 0] + [1] * len(inp["tracers"])
    nf = [0, 1, 1, 1 + len(inp["tracers"])]

    # undivided domain
    ad = A.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    ad.adz_traject(prec, cfg.dt, inp, px, wp)
    outs = [torch.zeros(ad.ext_shape, dtype=dt_, device="cuda") for _ in fields]
    ad.adz_tricub_sets(prec, nf, fields, outs, mono)
    assert ad.status() == 0

    # the same domain in npx x npy tiles
    D = Decomposition(cfg.ni, cfg.nj, npx, npy)
    tiles = []
    for r in range(D.size):
        t = D.tile(r)
        c = copy.copy(cfg)
        c.ni, c.nj, c.gi0, c.gj0, c.gni, c.gnj = t.ni, t.nj, t.i0g, t.j0g, cfg.ni, cfg.nj
        adt = A.Adz.from_config(c, edges=t.edges)
        win = lambda a: a[:, t.j0g - 1:t.j0g - 1 + t.nj + 2 * H, t.i0g - 1:t.i0g - 1 + t.ni + 2 * H].clone()  # noqa: E731,B023
        arrs = [win(inp[k]) for k in names] + [win(f) for f in fields]
        for a in arrs:
            _poison_ext(a, t, cfg.ni, cfg.nj, H)
        pxt, wpt = adt.new_state(prec)
        tiles.append(dict(t=t, ad=adt, arrs=arrs, px=pxt, wp=wpt,
                          ex=ext_exchange(D, r, adt, dt_, len(arrs)), exw=wpxyz_exchange(D, r, adt)))
    for T in tiles:
        T["ex"].pack(T["arrs"])
        T["winds"] = dict(zip(names, T["arrs"][:6]))
        T["ad"].adz_inittraj(prec, T["px"], T["wp"])
        if split:  # the interior's trajectory before any halo has arrived
            T["ad"].adz_traject_region(prec, cfg.dt, T["winds"], T["px"], T["wp"], 1)
    _route([T["ex"] for T in tiles], D)
    for T in tiles:
        T["ex"].unpack(T["arrs"])
        assert not any(torch.isnan(a).any() for a in T["arrs"])
        if split:
            T["ad"].adz_traject_region(prec, cfg.dt, T["winds"], T["px"], T["wp"], 2)
        else:
            T["ad"].adz_traject(prec, cfg.dt, T["winds"], T["px"], T["wp"])
        T["wp"][:, :, :2, :] = float("nan")
        T["wp"][:, :, -2:, :] = float("nan")
        T["wp"][:, :, :, :2] = float("nan")
        T["wp"][:, :, :, -2:] = float("nan")
        T["exw"].pack([T["wp"]])
        T["outs"] = [torch.zeros(T["ad"].ext_shape, dtype=dt_, device="cuda") for _ in fields]
        if split:  # the interior's position sets before wpxyz's halo has arrived
            T["ad"].adz_tricub_sets_region(prec, nf, T["arrs"][6:], T["outs"], mono, 1)
    _route([T["exw"] for T in tiles], D)
    for T in tiles:
        T["exw"].unpack([T["wp"]])
        if split:
            T["ad"].adz_tricub_sets_region(prec, nf, T["arrs"][6:], T["outs"], mono, 2)
        else:
            T["ad"].adz_tricub_sets(prec, nf, T["arrs"][6:], T["outs"], mono)
        assert T["ad"].status() == 0
    torch.cuda.synchronize()
    for T in tiles:
        t = T["t"]
        # wpxyz (-1:ni+2, -1:nj+2, nk, 3): local (1, 1) at [2, 2], global (i0g, j0g) at [i0g+1, j0g+1]
        assert torch.equal(T["wp"][:, :, 2:2 + t.nj, 2:2 + t.ni], wp[:, :, t.j0g + 1:t.j0g + 1 + t.nj,
                                                                       t.i0g + 1:t.i0g + 1 + t.ni]), t
        for q, (o_t, o_g) in enumerate(zip(T["outs"], outs)):
            gw = o_g[:, t.j0g - 1 + H:t.j0g - 1 + H + t.nj, t.i0g - 1 + H:t.i0g - 1 + H + t.ni]
            tw = o_t[:, H:H + t.nj, H:H + t.ni]
            assert torch.equal(tw, gw), (t, q, int((tw != gw).sum()))
