"""Train the learned starting guess (gem_b200/guess.py) on the GPU.

Data: 64 seeded deformational flows (gem_b200.synth) on 256x256 tiles with
40, 60 or 80 stretched levels, U0 uniform in 10-70 m/s, dt in 60-300 s and a
grid length giving a Courant number U0 dt / dx between 0.3 and 2.5 (dx at
least 2.5 km), horizontal-wind noise 0.5 m/s and vertical-wind noise
0.02 m/s (the cold-start workload's, gem_b200.synth.config_cold).  For each flow the plain iteration runs from the arrival point
to 1e-6 grid indices (adzc_traject_tol, at most 60 updates); 312 500 converged
arrival points per flow are drawn at random, giving 2.0e7 (features, departure
displacement) pairs.  Two further flows are held out for validation.

Training: the FP32 kernels of adzc_mlp_* (mean squared error, Adam, batch
4096, learning rate 1e-3 decaying by a cosine to 1e-5 over the epochs).

    python -m gem_b200.guess_train --out gem_b200/data/guess_mlp.npz
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import adz as A
from . import guess, synth


def flow_config(seed: int, n: int = 256) -> synth.Config:
    rng = np.random.default_rng(seed)
    nk = int(rng.choice([40, 60, 80]))
    u0 = float(rng.uniform(10.0, 70.0))
    dt = float(rng.uniform(60.0, 300.0))
    courant = float(rng.uniform(0.3, 2.5))
    dx = max(2.5e3, u0 * dt / courant)
    ph = (float(rng.uniform(0, 1)), float(rng.uniform(0, 1)))
    return synth.Config(f"train{seed}", n, n, nk, dx, dt, synth.stretched_levels(nk, 20.0, 1000.0, 25e3),
                        seed=seed, ntracers=0, phase=ph, u0=u0, w0=0.5, noise_w=0.02)


def flow_samples(cfg: synth.Config, nsamp: int, gen: torch.Generator):
    """Features and converged displacements of nsamp random arrival points."""
    prec = A.MIXED
    ad = A.Adz.from_config(cfg)
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
    _, wp = ad.new_state(prec)
    iters = torch.zeros(ad.nk * ad.nj * ad.ni, dtype=torch.uint8, device="cuda")
    guess.traject_tol(ad, prec, cfg.dt, inp, wp, tol=1e-6, maxit=60, start=0, iters=iters)
    if ad.status() != 0:
        raise RuntimeError(f"trajectory status set for {cfg.name}")
    k00, _ = guess.arrival_index(ad)
    it = iters.view(ad.nk, ad.nj, ad.ni)[k00 - 1:].reshape(-1)
    good = torch.nonzero((it >= 1) & (it < 60)).view(-1)
    pick = good[torch.randint(0, good.numel(), (nsamp,), device="cuda", generator=gen)]
    x = guess.features(ad, cfg.dt, inp, idx=pick)
    y = guess.displacement(ad, wp)[pick].float()
    return x, y


def make_data(nflows: int, nsamp: int, seed0: int):
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed0)
    xs, ys = [], []
    for f in range(nflows):
        x, y = flow_samples(flow_config(seed0 + f), nsamp, gen)
        xs.append(x)
        ys.append(y)
    return torch.cat(xs), torch.cat(ys)


def train(x, y, xv, yv, epochs: int, batch: int, seed: int, lr0=1e-3, lr1=1e-5, log=None):
    p0 = guess.init_params(seed)
    tr = guess.Trainer(p0, max_batch=max(batch, 65536))
    n = x.shape[0]
    steps = epochs * (n // batch)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    step = 0
    t0 = time.time()
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        for b in range(n // batch):
            idx = perm[b * batch:(b + 1) * batch]
            tr.grad(x[idx].contiguous(), y[idx].contiguous())
            lr = lr1 + 0.5 * (lr0 - lr1) * (1.0 + math.cos(math.pi * step / max(1, steps)))
            tr.adam(lr)
            step += 1
        rmse = evaluate(tr, xv, yv)
        hist.append({"epoch": ep + 1, "val_rmse": rmse, "seconds": time.time() - t0})
        if log:
            log(hist[-1])
    return tr, hist


def evaluate(tr: guess.Trainer, x, y, chunk=65536) -> float:
    se, n = 0.0, 0
    for s in range(0, x.shape[0], chunk):
        yp = tr.forward(x[s:s + chunk].contiguous())
        se += float(((yp - y[s:s + chunk]) ** 2).sum().item())
        n += yp.shape[0]
    return math.sqrt(se / (3 * n))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=guess.DEFAULT_WEIGHTS)
    ap.add_argument("--flows", type=int, default=64)
    ap.add_argument("--samples", type=int, default=312_500)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=2025)
    ap.add_argument("--log", default=None)
    args = ap.parse_args()
    t0 = time.time()
    x, y = make_data(args.flows, args.samples, seed0=10_000)
    xv, yv = make_data(2, 100_000, seed0=90_000)
    t_data = time.time() - t0
    print(json.dumps({"samples": int(x.shape[0]), "data_seconds": t_data,
                      "target_rms": float(y.pow(2).mean().sqrt().item())}), flush=True)
    tr, hist = train(x, y, xv, yv, args.epochs, args.batch, args.seed, log=lambda h: print(json.dumps(h), flush=True))
    p = tr.params()
    meta = {"samples": int(x.shape[0]), "flows": args.flows, "epochs": args.epochs, "batch": args.batch,
            "val_rmse": hist[-1]["val_rmse"], "data_seconds": t_data, "train_seconds": hist[-1]["seconds"]}
    np.savez(args.out, **p, meta=json.dumps(meta))
    if args.log:
        with open(args.log, "w") as f:
            json.dump({"meta": meta, "history": hist}, f, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
