"""Seeded synthetic inputs for the semi-Lagrangian advection path.

They stand in for GEM's DCMIP-2012-style deformational transport cases
(src/gemdyn/src/canonical/dcmip_tracers11_transport.F90 is the reference's own
closest analogue; none of its items are reproduced).  A limited-area Cartesian
tile with GEM's height-coordinate staggering (src/gemdyn/src/base/set_zeta.F90:48-72,
fislh_hybrid.F90:147-210) carries an analytic 3-D deformational flow

    u =  U0 sin^2(pi x/Lx) sin(2 pi y/Ly) cos(pi t/T)
    v = -U0 sin^2(pi y/Ly) sin(2 pi x/Lx) cos(pi t/T)
    w =  W0 sin(pi z/H)    cos(2 pi x/Lx) cos(pi t/T)

plus seeded Gaussian noise, and tracers (cosine bells, uniform noise,
log-normal noise).  Everything is built with torch on any device; fields are
returned in the extended ("ext") Fortran layout (1-halo : n+halo, ..., 1:nk),
i.e. torch shape (nk, njt, nit), x fastest.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class Levels:
    """Ver_z_8 (m, t, x) for GEM's height coordinate (sig = -1)."""
    zm: np.ndarray  # (0:nk+1)
    zt: np.ndarray  # (0:nk+1)
    zx: np.ndarray  # (0:nk)
    ztop: float

    @property
    def nk(self) -> int:
        return len(self.zm) - 2

    @property
    def wmstar_nk(self) -> float:   # fislh_hybrid.F90:207-208
        nk = self.nk
        return (self.zx[nk] - self.zt[nk]) / (self.zx[nk] - self.zx[nk - 1])

    @property
    def idz_t_nkm1(self) -> float:  # fislh_hybrid.F90:186-187
        nk = self.nk
        return 1.0 / (self.zm[nk] - self.zm[nk - 1])


def levels_from_thickness(h_bottom_up: np.ndarray) -> Levels:
    """Momentum levels at layer mid-points (k=1 at the top), thermo levels
    between them, top and surface as in fislh_hybrid.F90:153-176."""
    nk = len(h_bottom_up)
    iface = np.concatenate([[0.0], np.cumsum(h_bottom_up)])
    mid = 0.5 * (iface[:-1] + iface[1:])          # bottom-up
    zm = np.empty(nk + 2)
    zm[1:nk + 1] = mid[::-1]
    zm[0] = 0.5 * (3.0 * zm[1] - zm[2])
    zm[nk + 1] = 0.0
    zt = np.empty(nk + 2)
    zt[0] = zm[0]
    for k in range(1, nk + 1):
        zt[k] = 0.5 * (zm[k] + zm[k + 1])
    zt[nk + 1] = 0.0
    zx = np.empty(nk + 1)
    zx[0] = zm[0]
    zx[1:nk] = zt[1:nk]
    zx[nk] = 0.0
    return Levels(zm, zt, zx, float(iface[-1]))


def uniform_levels(nk: int, top: float) -> Levels:
    return levels_from_thickness(np.full(nk, top / nk))


def stretched_levels(nk: int, dz_bottom: float, dz_cap: float, top: float) -> Levels:
    """Layer thickness grows geometrically from dz_bottom, capped at dz_cap,
    with the ratio chosen so the layers add up to ``top``."""
    def total(r):
        h = np.minimum(dz_bottom * r ** np.arange(nk), dz_cap)
        return h.sum()
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if total(mid) < top:
            lo = mid
        else:
            hi = mid
    r = 0.5 * (lo + hi)
    h = np.minimum(dz_bottom * r ** np.arange(nk), dz_cap)
    h *= top / h.sum()
    return levels_from_thickness(h)


@dataclass
class Config:
    """One synthetic advection case (a tile of a limited-area domain)."""
    name: str
    ni: int
    nj: int
    nk: int
    dx: float
    dt: float
    levels: Levels
    niter: int = 2
    maxcfl: int = 3
    pil: int = 8                 # LAM pilot zone width on every edge
    u0: float = 40.0
    w0: float = 0.5
    period: float = 12 * 3600.0
    noise: float = 0.5
    noise_w: float | None = None       # noise of the vertical winds (None: ``noise``)
    seed: int = 1234
    ntracers: int = 2
    tracer_kind: str = "bell+uniform"   # "bell+uniform" | "bells" | "lognormal"
    bell_radius: float = 500e3
    mono: bool = False
    phase: tuple = (0.0, 0.0)
    t_now: float = 0.0
    # tile of a larger domain: global index of local (1,1) and the global
    # extents (0: the tile is the whole domain); the flow and the tracers are
    # functions of the global position
    gi0: int = 1
    gj0: int = 1
    gni: int = 0
    gnj: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def domain(self) -> tuple:
        return (self.gni or self.ni, self.gnj or self.nj)

    @property
    def halo(self) -> int:
        return max(1, self.maxcfl) + 1

    @property
    def npoints(self) -> int:
        return self.ni * self.nj * self.nk


def config_small(ni=128, nj=128, nk=40, seed=1234) -> Config:
    """128x128x40, dx=10 km, 40 uniform levels over 0-20 km, dt=300 s,
    2 trajectory iterations, u,v,w + a cosine bell (R=500 km) + U[0,1) noise."""
    return Config("c0", ni, nj, nk, 10e3, 300.0, uniform_levels(nk, 20e3), seed=seed, ntracers=2,
                  tracer_kind="bell+uniform")


def config_large(ni=1024, nj=1024, nk=80, seed=4321, ntracers=4) -> Config:
    """1024x1024x80, dx=2.5 km, 80 levels stretched 20 m -> 1 km up to 25 km,
    dt=60 s, 2 iterations, u,v,w + cosine bells at seeded centres."""
    rng = np.random.default_rng(seed)
    ph = (float(rng.uniform(0, 1)), float(rng.uniform(0, 1)))
    return Config("c1", ni, nj, nk, 2.5e3, 60.0, stretched_levels(nk, 20.0, 1000.0, 25e3), seed=seed,
                  ntracers=ntracers, tracer_kind="bells", phase=ph, bell_radius=500e3)


def config_mixed(ni=1024, nj=1024, nk=80, seed=4321, ntracers=8) -> Config:
    """Same flow as config_large, u,v,w + 8 log-normal (sigma=1) tracers, mono on."""
    c = config_large(ni, nj, nk, seed, ntracers)
    c.name, c.tracer_kind, c.mono = "c2", "lognormal", True
    return c


def config_batch(n=16, seed=2024, size=(256, 1024), levels=(40, 80), tracers=(1, 20)) -> list:
    """Independent limited-area domains of uneven size for one batched step:
    ni, nj seeded integers in ``size``, nk in ``levels``, 1-20 log-normal
    FP32 tracers (mono on), each domain with its own deformational-flow phase,
    U0 in 20-60 m/s and dt in 60-300 s.  The grid length keeps the Courant
    number near 2 (dx = max(2.5 km, U0 dt / 2)); W0 keeps the vertical
    displacement per step at 30 m."""
    rng = np.random.default_rng(seed)
    out = []
    for d in range(n):
        ni = int(rng.integers(size[0], size[1] + 1))
        nj = int(rng.integers(size[0], size[1] + 1))
        nk = int(rng.integers(levels[0], levels[1] + 1))
        ntr = int(rng.integers(tracers[0], tracers[1] + 1))
        u0 = float(rng.uniform(20.0, 60.0))
        dt = float(rng.uniform(60.0, 300.0))
        ph = (float(rng.uniform(0, 1)), float(rng.uniform(0, 1)))
        dx = max(2.5e3, u0 * dt / 2.0)
        c = Config(f"batch{d}", ni, nj, nk, dx, dt, stretched_levels(nk, 20.0, 1000.0, 25e3), seed=seed + 97 * d,
                   ntracers=ntr, tracer_kind="lognormal", mono=True, phase=ph, u0=u0, w0=30.0 / dt,
                   bell_radius=0.2 * ni * dx)
        out.append(c)
    return out


def config_cold(ni=1024, nj=1024, nk=80, seed=4321) -> Config:
    """Cold start of the learned-guess workload: the flow of config_large with
    vertical-wind noise of 0.02 m/s.  With the 0.5 m/s of config_large on its
    20 m bottom layers the update of the departure level is not a contraction
    (dt/2 |dw/dz| > 1) at about 1 % of the points, so no starting point makes
    it converge there."""
    c = config_large(ni, nj, nk, seed, ntracers=0)
    c.name, c.noise_w = "c4", 0.02
    return c


def _coords(cfg: Config, device, dtype):
    H = cfg.halo
    nit, njt = cfg.ni + 2 * H, cfg.nj + 2 * H
    i = torch.arange(1 - H, cfg.ni + H + 1, device=device, dtype=dtype) + (cfg.gi0 - 1)
    j = torch.arange(1 - H, cfg.nj + H + 1, device=device, dtype=dtype) + (cfg.gj0 - 1)
    x = (i - 1) * cfg.dx
    y = (j - 1) * cfg.dx
    return x, y, nit, njt


def _flow(cfg: Config, x, y, z, t, comp):
    Lx, Ly = cfg.domain[0] * cfg.dx, cfg.domain[1] * cfg.dx
    ph = cfg.phase
    ct = math.cos(math.pi * t / cfg.period)
    X = x.view(1, 1, -1) / Lx + ph[0]
    Y = y.view(1, -1, 1) / Ly + ph[1]
    Z = z.view(-1, 1, 1)
    if comp == 0:
        return cfg.u0 * torch.sin(math.pi * X) ** 2 * torch.sin(2 * math.pi * Y) * ct
    if comp == 1:
        return -cfg.u0 * torch.sin(math.pi * Y) ** 2 * torch.sin(2 * math.pi * X) * ct
    H = cfg.levels.ztop
    return cfg.w0 * torch.sin(math.pi * Z / H) * torch.cos(2 * math.pi * X) * ct + 0.0 * Y


def make_inputs(cfg: Config, device="cpu", dtype=torch.float64, with_fields=True):
    """Winds and source fields of one advection step, ext layout (nk, njt, nit).

    Returns a dict: uu_ext, vv_ext, ww_ext (departure winds, time t),
    ut0, vt0 (arrival winds on C-grid u/v points, time t+dt), zdt0 (arrival
    vertical motion on thermo levels), src_u, src_v, src_w (momentum fields on
    u, v and thermo points) and tracers (list, thermo points)."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(cfg.seed)
    f64 = torch.float64
    x, y, nit, njt = _coords(cfg, dev, f64)
    nk = cfg.nk
    zm = torch.tensor(cfg.levels.zm[1:nk + 1], device=dev, dtype=f64)
    zt = torch.tensor(cfg.levels.zt[1:nk + 1], device=dev, dtype=f64)
    shp = (nk, njt, nit)

    def noise(sd=None):
        return torch.randn(shp, generator=g, device=dev, dtype=f64) * (cfg.noise if sd is None else sd)

    t0, t1 = cfg.t_now + cfg.dt, cfg.t_now
    out = {}
    out["uu_ext"] = (_flow(cfg, x, y, zm, t1, 0).expand(shp) + noise()).to(dtype).contiguous()
    out["vv_ext"] = (_flow(cfg, x, y, zm, t1, 1).expand(shp) + noise()).to(dtype).contiguous()
    out["ww_ext"] = (_flow(cfg, x, y, zt, t1, 2).expand(shp) + noise(cfg.noise_w)).to(dtype).contiguous()
    xu = x + 0.5 * cfg.dx
    yv = y + 0.5 * cfg.dx
    out["ut0"] = (_flow(cfg, xu, y, zm, t0, 0).expand(shp) + noise()).to(dtype).contiguous()
    out["vt0"] = (_flow(cfg, x, yv, zm, t0, 1).expand(shp) + noise()).to(dtype).contiguous()
    out["zdt0"] = (_flow(cfg, x, y, zt, t0, 2).expand(shp) + noise(cfg.noise_w)).to(dtype).contiguous()
    # surface-layer winds Adz_uslt, Adz_vslt (nj, ni): the lowest momentum
    # level's winds, weakened as near the ground
    i0 = j0 = cfg.halo
    out["uslt"] = (0.7 * out["uu_ext"][-1, j0:j0 + cfg.nj, i0:i0 + cfg.ni].to(torch.float64)).to(dtype).contiguous()
    out["vslt"] = (0.7 * out["vv_ext"][-1, j0:j0 + cfg.nj, i0:i0 + cfg.ni].to(torch.float64)).to(dtype).contiguous()
    if not with_fields:
        return out
    out["src_u"] = _flow(cfg, xu, y, zm, t1, 0).expand(shp).to(dtype).contiguous()
    out["src_v"] = _flow(cfg, x, yv, zm, t1, 1).expand(shp).to(dtype).contiguous()
    out["src_w"] = _flow(cfg, x, y, zt, t1, 2).expand(shp).to(dtype).contiguous()
    tr = []
    rng = np.random.default_rng(cfg.seed + 7)
    Lx, Ly = cfg.domain[0] * cfg.dx, cfg.domain[1] * cfg.dx
    H = cfg.levels.ztop
    for n in range(cfg.ntracers):
        kind = cfg.tracer_kind
        if kind == "bell+uniform":
            kind = "bell" if n % 2 == 0 else "uniform"
        elif kind == "bells":
            kind = "bell"
        if kind == "bell":
            cx = rng.uniform(0.25, 0.75) * Lx if n else 0.5 * Lx
            cyy = rng.uniform(0.25, 0.75) * Ly if n else 0.5 * Ly
            cz = rng.uniform(0.2, 0.6) * H
            r = torch.sqrt(((x.view(1, 1, -1) - cx) / cfg.bell_radius) ** 2 +
                           ((y.view(1, -1, 1) - cyy) / cfg.bell_radius) ** 2 +
                           ((zt.view(-1, 1, 1) - cz) / (0.25 * H)) ** 2)
            f = torch.where(r < 1.0, 0.5 * (1.0 + torch.cos(math.pi * r)), torch.zeros_like(r))
        elif kind == "uniform":
            f = torch.rand(shp, generator=g, device=dev, dtype=f64)
        elif kind == "lognormal":
            f = torch.exp(torch.randn(shp, generator=g, device=dev, dtype=f64))
        else:
            raise ValueError(kind)
        tr.append(f.expand(shp).to(dtype).contiguous())
    out["tracers"] = tr
    return out


def grid_arrays(cfg: Config):
    """Per-tile constants of adz_set for the Cartesian LAM tile: cy=1,
    inv_rayt=1, inv_hx=inv_hy=1/dx (so winds divided by dx give index/s)."""
    H = cfg.halo
    return dict(cy=np.ones(cfg.nj + 2 * H), zm=cfg.levels.zm.copy(), zt=cfg.levels.zt.copy(),
                zx=cfg.levels.zx.copy(), zmin=float(cfg.levels.zm[cfg.nk + 1]), zmax=float(cfg.levels.zm[0]),
                wmstar_nk=float(cfg.levels.wmstar_nk), idz_t_nkm1=float(cfg.levels.idz_t_nkm1),
                inv_hx=1.0 / cfg.dx, inv_hy=1.0 / cfg.dx, inv_rayt=1.0)
