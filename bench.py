"""Benchmark of the semi-Lagrangian advection step on B200.

Workload (one "step"): one full GEM advection step of a 1024x1024x80 limited-area
tile (dx = 2.5 km, 80 levels stretched 20 m -> 1 km up to 25 km, dt = 60 s,
2 trajectory iterations): departure winds prepared, trajectories iterated,
then u@pmu, v@pmv, w + 4 cosine-bell tracers @pt interpolated (momentum plus 4
tracers).  Inputs are seeded synthetic fields of that shape (no dataset).

Metric: grid points advanced per second (ni*nj*nk per step / step time).
``value`` is the mixed-precision product path with inputs resident in HBM;
``fp64_value`` is the plain FP64 drop-in on the same GPU; ``e2e`` goes
through the same public API with inputs copied from pinned host memory and
results copied back every step.  Inputs (>10 GB) exceed the 126 MB L2, so no
flush is needed between steps.

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

HBM_FALLBACK_GBS = 6650.0
TENSOR_FALLBACK_TFLOPS = 1590.0
# DRAM bytes (read + write) per arrival point of each MIXED launch, measured
# by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on a 384x384x80 tile
# with u, v, w + 4 tracers; traffic grows in proportion to the points, so it
# scales to the benched tile
MEASURED_TRAFFIC_PER_POINT = {"traject": 73.59, "sets": 84.65}
# L1 data-pipe wavefronts (l1tex__data_pipe_lsu_wavefronts.sum) per grid point
# of each MIXED launch, same capture (384x384x80, u, v, w + 4 tracers); the
# pipe returns one wavefront per SM cycle, the bound both gather kernels reach
MEASURED_L1_WAVEFRONTS_PER_POINT = {"traject": 25.66, "sets": 30.24}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """nvidia-smi clock sampling during the timed region."""

    def __init__(self, index: int):
        self.index, self.samples, self.proc = index, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 8 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 8 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) > 8:
                for nm, v in zip(names, s[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_init():
    """One process per GPU under torchrun; NCCL on GPUs, gloo without."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)  # before the process group, so NCCL binds this rank's GPU
    if ws > 1 and not torch.distributed.is_initialized():
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def _dev():
    return "cuda" if torch.cuda.is_available() else "cpu"


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    t = torch.tensor([x], device=_dev(), dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def tile_seed(rank: int) -> int:
    """Each rank advances its own tile (weak scaling, no data-path collective)."""
    return 4321 + rank


# ---------------------------------------------------------------------------
def cpu_reference(size, steps, warmup, threads=0, ntracers=4, gen_device=None):
    """The reference's CPU path: its interpolator compiled unchanged plus the
    C restatement of the Fortran drivers (OpenMP over k-planes), FP32 fields,
    on a bounded sample of the workload.  Returns points/s and details."""
    from oracle import oracle as O
    from gem_b200 import synth
    kind = "ref" if O.have_ref() else "oracle"
    cfg = synth.config_large(*size, ntracers=ntracers)
    dev = gen_device or ("cuda" if torch.cuda.is_available() else "cpu")
    inp = synth.make_inputs(cfg, device=dev, dtype=torch.float32)
    np_in = {k: (v.cpu().numpy() if torch.is_tensor(v) else [t.cpu().numpy() for t in v]) for k, v in inp.items()}
    del inp
    ncores = threads or os.cpu_count()
    st = O.Step(cfg, kind=kind, prec="f32", threads=ncores)
    st.inittraj()
    st.traject(np_in)  # cold start (6 iterations) outside the timing
    times = []
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        st.step(np_in)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    med = statistics.median(times)
    cpu = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"value": cfg.npoints / med, "unit": "grid-points/s", "cores": ncores,
            "kind": "reference" if kind == "ref" else "port",
            "sample": f"{size[0]}x{size[1]}x{size[2]} tile, u,v,w+{ntracers} tracers, FP32 (reference precision), "
                      f"median of {steps} steps after {warmup} warm-up, {cpu}",
            "ms_per_step": med * 1e3}


# ---------------------------------------------------------------------------
def run_product(args):
    from gem_b200 import adz, synth
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    ni, nj, nk = args.size
    cfg, tile, decomp = tile_config(args.size, rank, ws, args.ntr)
    npts = cfg.npoints
    inp64 = synth.make_inputs(cfg, device="cuda", dtype=torch.float64)
    keys = ["uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0", "src_u", "src_v", "src_w"]

    def conv(d, dt):
        o = {k: d[k].to(dt) for k in keys}
        o["tracers"] = [t.to(dt) for t in d["tracers"]]
        return o

    ad = adz.Adz.from_config(cfg, edges=tile.edges)
    results = {}
    barrier(ws)  # first collective of the group, before any point-to-point batch

    def make_step(prec, data):
        px, wp = ad.new_state(prec)
        ad.adz_inittraj(prec, px, wp)
        dt = adz._field_dtype(prec)
        outs = {k: torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for k in ("u", "v", "w")}
        tro = [torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for _ in data["tracers"]]
        if ws > 1:  # a tile of one decomposed domain: halo exchanges inside the step
            from gem_b200.halo import TiledStep
            tiled = TiledStep(decomp, rank, ad, prec, len(data["tracers"]))

            def step():
                tiled(cfg.dt, data, data, data["tracers"], px, wp, outs, tro, cfg.mono)
        else:
            def step():
                adz.step_fused(ad, prec, cfg.dt, data, data, data["tracers"], px, wp, outs, tro, cfg.mono)
        step()  # cold start: 6 iterations, untimed
        return step, outs, tro, wp

    def timed(step, K, W, clocks=False):
        for _ in range(W):
            step()
        barrier(ws)
        clk = Clocks(local) if clocks else None
        if clk:
            clk.__enter__()
            time.sleep(0.3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(ws)
        e0.record()
        for _ in range(K):
            step()
        e1.record()
        barrier(ws)
        if clk:
            clk.__exit__()
        ms = e0.elapsed_time(e1) / K
        return max_over_ranks(ms, ws), (clk.summary() if clk else None)

    # plain FP64 drop-in
    ms64 = float("nan")
    if args.only is None:
        d64 = conv(inp64, torch.float64)
        step64, o64, t64, wp64 = make_step(adz.FP64, d64)
        ms64, _ = timed(step64, args.steps, args.warmup)
        # one more step from saved positions: the MIXED step below starts from the same ones
        ref64 = {"start": wp64.clone()}
        step64()
        ref64.update(fields=[o64["u"], o64["v"], o64["w"]] + t64, wp=wp64)
        del step64, d64
        torch.cuda.empty_cache()
    results["fp64"] = ms64
    # mixed precision (product)
    d32 = conv(inp64, torch.float32)
    del inp64
    torch.cuda.empty_cache()
    step32, outs32, tro32, wp32 = make_step(adz.MIXED, d32)
    ms32, clk = timed(step32, args.steps, args.warmup, clocks=True)
    if ad.status() != 0:
        raise RuntimeError("device status set during the timed steps")
    acc = None
    if args.only is None:
        wp32.copy_(ref64["start"])
        step32()
        acc = accuracy(ad, [outs32["u"], outs32["v"], outs32["w"]] + tro32, wp32, ref64)
        del ref64
        torch.cuda.empty_cache()
    # the reference's own arithmetic (REF32, bit-exact with the CPU reference) on the same inputs
    ms_ref32 = float("nan")
    if args.only is None:
        step_r, o_r, t_r, _ = make_step(adz.REF32, d32)
        ms_ref32, _ = timed(step_r, max(3, min(args.steps, 10)), args.warmup)
        if ad.status() != 0:
            raise RuntimeError("device status set during the REF32 steps")
        del step_r, o_r, t_r
        torch.cuda.empty_cache()

    # per-launch durations of one step (events between the API calls)
    s = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    px, wp = ad.new_state(adz.MIXED)
    ad.adz_inittraj(adz.MIXED, px, wp)
    ad.adz_traject(adz.MIXED, cfg.dt, d32, px, wp)
    torch.cuda.synchronize()
    per = {"traject": [], "sets": []}
    srcs = [d32["src_u"], d32["src_v"], d32["src_w"]] + d32["tracers"]
    dsts = [outs32["u"], outs32["v"], outs32["w"]] + tro32
    monos = [0, 0, 0] + [1 if cfg.mono else 0] * len(tro32)
    for _ in range(max(3, min(args.steps, 10))):
        ev[0].record(s)
        ad.adz_traject(adz.MIXED, cfg.dt, d32, px, wp)
        ev[1].record(s)
        ad.adz_tricub_sets(adz.MIXED, [0, 1, 1, 1 + len(tro32)], srcs, dsts, monos)
        ev[2].record(s)
        torch.cuda.synchronize()
        per["traject"].append(ev[0].elapsed_time(ev[1]))
        per["sets"].append(ev[1].elapsed_time(ev[2]))
    per = {k: statistics.median(v) for k, v in per.items()}
    I = ad.info
    n_t = int(I.npts[3])
    nf = 3 + len(tro32)
    # algorithmic bytes (each array read or written once):
    #   trajectory call, per grid point: departure winds 12 B + arrival winds
    #   12 B (FP32) + FP64 position in 24 B and out 24 B + departure w out 4 B
    #   sets launch, per arrival point: FP64 position 24 B + departure w and
    #   zdot 8 B + every field read and written 8 B
    bytes_launch = {"traject": npts * 76, "sets": n_t * (24 + 8 + nf * 8)}
    dom = max(per, key=per.get)
    hbm, hbm_kind = peaks()
    achieved = bytes_launch[dom] / (per[dom] * 1e-3) / 1e9
    traffic = MEASURED_TRAFFIC_PER_POINT[dom] * npts if args.ntr == 4 else None
    step_bytes = npts * (24 + 12 + 12 + 24 + (3 + args.ntr) * 8)

    # end to end: inputs from pinned host memory, results back, every step
    e2e = None
    if not args.no_e2e:
        host_in = {k: d32[k].cpu().pin_memory() for k in keys}
        host_tr = [t.cpu().pin_memory() for t in d32["tracers"]]
        host_out = [torch.empty(ad.ext_shape, dtype=torch.float32).pin_memory() for _ in range(3 + len(tro32))]
        h2d = sum(v.numel() * 4 for v in host_in.values()) + sum(t.numel() * 4 for t in host_tr)
        d2h = sum(t.numel() * 4 for t in host_out)

        def e2e_step():
            for k in keys:
                d32[k].copy_(host_in[k], non_blocking=True)
            for t, h in zip(d32["tracers"], host_tr):
                t.copy_(h, non_blocking=True)
            step32()
            for h, dsrc in zip(host_out, [outs32["u"], outs32["v"], outs32["w"]] + tro32):
                h.copy_(dsrc, non_blocking=True)
        K2 = max(3, min(args.steps, 5))
        ms_serial, _ = timed(e2e_step, K2, 3)
        ms_e2e = measure_e2e_pipelined(args, ws, rank, ad, cfg, decomp, d32, outs32, tro32, keys, host_in, host_tr,
                                       host_out)
        e2e = {"value": npts * ws / (ms_e2e * 1e-3), "unit": "grid-points/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e,
               "mode": "double-buffered: step n+1's inputs upload and step n-1's results download while step n "
                       "computes (copy streams + events); every step moves all its bytes inside the timed region",
               "serial": {"value": npts * ws / (ms_serial * 1e-3), "ms_per_step": ms_serial,
                          "mode": "upload, step, download one after another on one stream"}}

    batch = None
    if not args.no_batch:
        del d32, outs32, tro32, step32, px, wp, srcs, dsts
        torch.cuda.empty_cache()
        from gem_b200 import synth
        batch = measure_batch(args, timed, ws, synth.config_batch(n=args.batch_domains, seed=2024),
                              "uneven LAM domains (256-1024 squared, 40-80 levels, 1-20 tracers, mono)")
        batch["small_domains"] = measure_batch(
            args, timed, ws, synth.config_batch(n=40, seed=2025, size=(48, 160), levels=(20, 80), tracers=(1, 8)),
            "small LAM domains (48-160 squared, 20-80 levels, 1-8 tracers, mono)")

    tsum = None
    if not args.no_tracers:
        torch.cuda.empty_cache()
        tsum = measure_tracers(args, timed, ws, rank)

    psum = None
    if not args.no_post:
        torch.cuda.empty_cache()
        psum = measure_post(args, timed, ws, rank)

    gsum = None
    if not args.no_guess and os.path.exists(args.guess_weights):
        torch.cuda.empty_cache()
        gsum = measure_guess(args, timed, ws, rank)

    lvla = None
    if rank == 0 and ws == 1 and not args.no_level_a:
        torch.cuda.empty_cache()
        lvla = measure_level_a(args, with_cpu=not args.no_cpu)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        # the benchmarked tile, median of 5 steps after 1 warm-up, all host cores
        cpu = cpu_reference(args.cpu_size, 5, 1, ntracers=args.ntr)
        # the same path on one core, on a smaller sample (256x256x80)
        one = cpu_reference((256, 256, args.cpu_size[2]), 5, 1, threads=1, ntracers=args.ntr)
        cpu["single_core"] = {k: one[k] for k in ("value", "unit", "cores", "sample", "ms_per_step")}
    value = npts * ws / (ms32 * 1e-3)
    line = {
        "metric": "SL advection grid-points/s at 1024^2x80 (mixed-precision step; plain FP64 GPU drop-in alongside)",
        "value": value, "unit": "grid-points/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 sums / f64 positions", "data": "synthetic (seeded analytic deformational flow + noise)",
        "config": workload_config(args, ws, decomp),
        "fp64_value": npts * ws / (ms64 * 1e-3), "fp64_ms_per_step": ms64, "speedup_vs_fp64": ms64 / ms32,
        "ref32_value": npts * ws / (ms_ref32 * 1e-3), "ref32_ms_per_step": ms_ref32,
        "per_launch_ms": per,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": hbm_kind,
                     "l1": l1_roofline(args, per, npts, clk)},
        "step_roofline": {"algorithmic_bytes_per_point": step_bytes / npts,
                          "achieved_gbs": step_bytes / (ms32 * 1e-3) / 1e9,
                          "frac": step_bytes / (ms32 * 1e-3) / 1e9 / hbm},
        "accuracy": acc,
        "e2e": e2e, "gpu_launches": (LAUNCHES_PER_STEP + (HALO_LAUNCHES_PER_STEP if ws > 1 else 0)) * args.steps,
        "clocks": clk, "cpu_baseline": cpu,
        "tracers8": tsum, "post": psum, "batch": batch, "learned_guess": gsum, "level_a": lvla,
    }
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.destroy_process_group()


def l1_roofline(args, per, npts, clk):
    """The bound the gather kernels reach: the L1 data pipe, one wavefront per
    SM cycle.  Wavefronts per grid point from the ncu capture of the small
    case, times the points of the benched tile, over each launch's measured
    time, against the SM count times the SM clock sampled during the timed
    steps (the maximum clock when no sample)."""
    if args.ntr != 4:
        return None
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    peak = sms * mhz * 1e6
    out = {"metric": "l1tex__data_pipe_lsu_wavefronts", "unit": "wavefronts/s", "peak": peak,
           "peak_kind": f"1 wavefront per SM cycle, {sms} SMs at {mhz:g} MHz (sampled)", "kernels": {}}
    for k, ms in per.items():
        w = MEASURED_L1_WAVEFRONTS_PER_POINT[k] * npts
        out["kernels"][k] = {"wavefronts_per_point": MEASURED_L1_WAVEFRONTS_PER_POINT[k],
                             "achieved": w / (ms * 1e-3), "frac": w / (ms * 1e-3) / peak}
    # the trajectory call's time also holds its departure-wind launch
    # (k_prepare4, about 5 % of the call), so its fraction is a lower bound
    out["kernels"]["traject"]["time_includes"] = "departure-wind launch (k_prepare4)"
    dom = max(per, key=per.get)
    out["kernel"], out["achieved"], out["frac"] = dom, out["kernels"][dom]["achieved"], out["kernels"][dom]["frac"]
    return out


def level_a_inputs(size, ntr, seed=11):
    """Host arrays of the per-level Level A calls on the thermo set: w and the
    tracers on the extended tile (halo 4), FP32, and departure positions of
    every arrival point as fractional indices of the extended array, displaced
    up to 1.5 grid lengths horizontally and about 0.3 levels vertically."""
    ni, nj, nk = size
    h = 4
    nie, nje = ni + 2 * h, nj + 2 * h
    rng = np.random.default_rng(seed)
    fields = [rng.standard_normal(nie * nje * nk, dtype=np.float32) for _ in range(1 + ntr)]
    th = np.geomspace(20.0, 1000.0, nk)
    z = np.cumsum(th)[::-1].copy()
    levels = np.ascontiguousarray(z * (25000.0 / z[0]))
    ii, jj = np.meshgrid(np.arange(1, ni + 1, dtype=np.float32), np.arange(1, nj + 1, dtype=np.float32))
    planes = []
    for k in range(1, nk + 1):
        pos = np.empty((ni * nj, 3), np.float32)
        pos[:, 0] = np.clip(ii.ravel() + rng.uniform(-1.5, 1.5, ni * nj).astype(np.float32), 2.0 - h, nie - 2.0 - h - 1e-3)
        pos[:, 1] = np.clip(jj.ravel() + rng.uniform(-1.5, 1.5, ni * nj).astype(np.float32), 2.0 - h, nje - 2.0 - h - 1e-3)
        pos[:, 2] = np.clip(k + 0.3 * rng.standard_normal(ni * nj, dtype=np.float32), 1.0, float(nk))
        planes.append(pos)
    return {"fields": fields, "levels": levels, "planes": planes, "ext": (nie, nje, nk), "halo": h}


def time_level_a(lib, setup, inp, threads, reps=3):
    """Tricublin_mono_zyx_m_n once per level, as the reference's driver calls
    it (one slice of ni*nj points per OpenMP thread), from ``threads`` host
    threads; wall-clock seconds per pass over the tile (median), and the
    outputs of the first and the middle level."""
    import ctypes as C
    import threading
    from concurrent.futures import ThreadPoolExecutor
    nie, nje, nk = inp["ext"]
    h = inp["halo"]
    lv = setup(inp["levels"], nk, nie, nje, h, h)
    m = len(inp["fields"])
    fs = (C.c_void_p * m)(*[f.ctypes.data for f in inp["fields"]])
    n = inp["planes"][0].shape[0]
    local = threading.local()
    keep = {}
    status = getattr(lib, "adzc_last_error", None)  # per-thread status of the product library

    def call(k):
        if not hasattr(local, "out"):
            local.out = [np.empty((m, n), np.float32) for _ in range(4)]
        out = local.out
        lib.Tricublin_mono_zyx_m_n(*(o.ctypes.data for o in out), C.cast(fs, C.c_void_p),
                                   inp["planes"][k].ctypes.data, lv, n, m)
        if status is not None and status() != 0:
            raise RuntimeError(f"Level A call of level {k} failed with status {status()}")
        if k in (0, nk // 2):
            keep[k] = [o.copy() for o in out]

    times = []
    with ThreadPoolExecutor(max_workers=threads) as ex:
        for r in range(reps + 1):
            t0 = time.perf_counter()
            list(ex.map(call, range(nk)))
            if r > 0:
                times.append(time.perf_counter() - t0)
    return statistics.median(times), keep


def measure_level_a(args, with_cpu):
    """The reference-named interpolator symbols with host arrays (Level A, the
    link-level drop-in for the reference's interpolator) on the thermo set of
    the benched tile, against the reference's own interpolator on the host
    cores (the CPU leg, when the reference build is present)."""
    import ctypes as C
    from gem_b200 import adz
    ni, nj, nk = args.size
    inp = level_a_inputs(args.size, args.ntr)
    threads = min(16, os.cpu_count() or 1)
    L = adz.lib()
    n, m = ni * nj, 1 + args.ntr
    s_gpu, out_gpu = time_level_a(L, lambda lev, *a: L.Vsearch_setup_plus(lev.ctypes.data, *a), inp, threads)
    npts = n * nk
    res = {"workload": (f"thermo set of the {ni}x{nj}x{nk} tile: w + {args.ntr} tracers with bounds "
                        f"(Tricublin_mono_zyx_m_n), one call per level of {n} points from {threads} host threads, "
                        "host arrays in and out"),
           "threads": threads,
           "gpu": {"s_per_pass": s_gpu, "value": npts / s_gpu, "unit": "grid-points/s",
                   "d2h_bytes_per_pass": 4 * m * npts * 4}}
    if with_cpu:
        from oracle import oracle as O
        if O.have_ref():
            R = O.RefKernels()
            s_cpu, out_cpu = time_level_a(R.lib, lambda lev, *a: R.lib.Vsearch_setup_plus(lev, *a), inp, threads)
            same = all(np.array_equal(a.view(np.int32), b.view(np.int32))
                       for k in out_gpu for a, b in zip(out_gpu[k], out_cpu[k]))
            res["cpu_reference"] = {"s_per_pass": s_cpu, "value": npts / s_cpu, "unit": "grid-points/s",
                                    "cores": threads, "kind": "reference",
                                    "sample": "the same calls into the reference's interpolator compiled unchanged"}
            res["speedup_vs_cpu"] = s_cpu / s_gpu
            res["bit_identical_levels"] = same
    return res


def workload_config(args, ws, decomp=None):
    """The benched workload, shared by the product and the reference arm."""
    ni, nj, nk = args.size
    par = "1 tile"
    if ws > 1 and decomp is not None:
        par = (f"{decomp.npx}x{decomp.npy} tiles of one {decomp.gni}x{decomp.gnj} domain, one per GPU; "
               "halo exchange (NCCL send/recv) of winds and sources, then of wpxyz, every step")
    return {"workload": f"adz step {ni}x{nj}x{nk} LAM tile, u,v,w+{args.ntr} cosine-bell tracers, "
                        "2 trajectory iterations, dt=60 s, dx=2.5 km, 80 stretched levels",
            "points_per_step": ni * nj * nk, "l2": "inputs larger than L2 (no flush)", "parallelism": par}


# kernels of one MIXED step: departure winds, trajectory, and one
# interpolation launch per position set (u, v, then w + tracers at thermo points)
LAUNCHES_PER_STEP = 3  # k_prepare, k_traject, k_tricub_parts (every set's field groups)
HALO_LAUNCHES_PER_STEP = 4  # pack + unpack of the two exchanges (N > 1)


def accuracy(ad, fields32, wp32, ref64):
    """MIXED against the plain FP64 path (bit-exact with the FP64 oracle):
    one warm step of each from the same departure points (those the FP64
    path reached after its timed steps) on the same inputs.  One step, not
    the end of two separate runs: on this flow the fixed-point map of the
    trajectory amplifies position differences (vertical-wind noise of
    0.5 m/s over 60 s against 20 m levels), so separate runs drift apart by
    more than one step's rounding.  Per field: the largest
    error over the field's largest magnitude, the RMS error over the RMS
    value and the largest pointwise relative error (values below 1e-3 of the
    field's largest magnitude measured against that floor), over the set's
    arrival points; then the departure points' cell indices, (int)(float)
    of the position as the kernels form them, and the largest position
    difference in grid lengths."""
    names = ["u", "v", "w"] + [f"tracer{q + 1}" for q in range(len(fields32) - 3)]
    sets = [1, 2, 3] + [3] * (len(fields32) - 3)
    out = {"reference": "plain FP64 GPU path (bit-exact with the FP64 oracle), one step from the same positions",
           "fields": []}
    for name, st, a, b in zip(names, sets, fields32, ref64["fields"]):
        m = ad.range_mask(st, device="cuda")
        x, y = a[m].double(), b[m]
        d = (x - y).abs()
        scale = float(y.abs().max())
        rms = float(y.pow(2).mean().sqrt())
        out["fields"].append({
            "field": name, "max_err_over_max": float(d.max()) / scale,
            "rms_err_over_rms": float(d.pow(2).mean().sqrt()) / rms,
            "max_pointwise_rel": float((d / y.abs().clamp_min(1e-3 * scale)).max())})
        del m, x, y, d
    w32, w64 = wp32[:, :, 2:-2, 2:-2], ref64["wp"][:, :, 2:-2, 2:-2]
    c32 = w32.float().trunc()
    c64 = w64.float().trunc()
    out["cell_index_mismatches"] = int((c32 != c64).sum())
    out["positions"] = int(c32.numel())
    out["max_position_diff_grid"] = float((w32 - w64).abs().max())
    out["max_err_over_max_all_fields"] = max(f["max_err_over_max"] for f in out["fields"])
    return out


def measure_e2e_pipelined(args, ws, rank, ad, cfg, decomp, d32, outs32, tro32, keys, host_in, host_tr, host_out):
    """End to end through the public API with the copies overlapped: two
    device input sets and two output sets; step s computes on set s % 2
    while the copy streams upload step s+1's inputs from pinned host memory
    and download step s-1's results.  Every step's full inputs go up and
    its full results come down inside the timed region.  Returns ms per
    step (max over ranks), from CUDA events on the compute stream around
    the whole pipeline, fill and drain included."""
    from gem_b200 import adz
    prec = adz.MIXED
    D = [d32, {k: torch.empty_like(d32[k]) for k in keys}]
    D[1]["tracers"] = [torch.empty_like(t) for t in d32["tracers"]]
    OUT = [(outs32, tro32), ({k: torch.empty_like(v) for k, v in outs32.items()}, [torch.empty_like(t) for t in tro32])]
    HOUT = [host_out, [torch.empty(h.shape, dtype=h.dtype, pin_memory=True) for h in host_out]]
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    tiled = None
    if ws > 1:
        from gem_b200.halo import TiledStep
        tiled = TiledStep(decomp, rank, ad, prec, len(tro32))

    def run(b):
        data, (o, t) = D[b], OUT[b]
        if tiled is not None:
            tiled(cfg.dt, data, data, data["tracers"], px, wp, o, t, cfg.mono)
        else:
            adz.step_fused(ad, prec, cfg.dt, data, data, data["tracers"], px, wp, o, t, cfg.mono)
    run(0)  # cold start, untimed
    cin, cout = torch.cuda.Stream(), torch.cuda.Stream()

    def pipeline(nsteps):
        cur = torch.cuda.current_stream()
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_comp = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]
        used = [False, False]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(ws)
        e0.record(cur)
        cin.wait_event(e0)

        def h2d(b):
            with torch.cuda.stream(cin):
                if used[b]:
                    cin.wait_event(ev_comp[b])  # the step that read this set is done
                for k in keys:
                    D[b][k].copy_(host_in[k], non_blocking=True)
                for t, h in zip(D[b]["tracers"], host_tr):
                    t.copy_(h, non_blocking=True)
                ev_in[b].record(cin)
        h2d(0)
        for st in range(nsteps):
            b = st % 2
            if st + 1 < nsteps:
                h2d(1 - b)
            cur.wait_event(ev_in[b])
            if st >= 2:
                cur.wait_event(ev_out[b])  # this output set has been downloaded
            run(b)
            ev_comp[b].record(cur)
            used[b] = True
            with torch.cuda.stream(cout):
                cout.wait_event(ev_comp[b])
                for h, dsrc in zip(HOUT[b], [OUT[b][0]["u"], OUT[b][0]["v"], OUT[b][0]["w"]] + OUT[b][1]):
                    h.copy_(dsrc, non_blocking=True)
                ev_out[b].record(cout)
        for b in range(min(2, nsteps)):
            cur.wait_event(ev_out[b])
        e1.record(cur)
        barrier(ws)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / nsteps
    pipeline(3)  # warm-up
    ms = pipeline(max(5, min(args.steps, 20)))  # the device timing's K steps, fill and drain included
    if ad.status() != 0:
        raise RuntimeError("device status set during the end-to-end steps")
    del D, OUT, HOUT
    torch.cuda.empty_cache()
    return max_over_ranks(ms, ws)


def tile_config(size, rank, ws, ntr):
    """The bench tile of a rank: one ni x nj x nk tile of an (npx ni) x
    (npy nj) domain cut into npx x npy = ws tiles, the flow and tracers
    functions of the global position, the noise seeded per rank."""
    from gem_b200 import synth
    from gem_b200.halo import Decomposition
    ni, nj, nk = size
    npx, npy = Decomposition.grid_for(ws)
    decomp = Decomposition(ni * npx, nj * npy, npx, npy)
    tile = decomp.tile(rank)
    cfg = synth.config_large(ni, nj, nk, seed=tile_seed(rank), ntracers=ntr)
    cfg.gi0, cfg.gj0, cfg.gni, cfg.gnj = tile.i0g, tile.j0g, decomp.gni, decomp.gnj
    return cfg, tile, decomp


def measure_batch(args, timed, ws, cfgs, label):
    """Independent limited-area domains of uneven size (each with its own
    levels, log-normal tracers, flow phase, U0 and dt) in one persistent
    launch per step, replayed from a CUDA graph after the autotuner picked
    its tile height, register budget and resident blocks; beside it the same
    domains stepped one after another through the per-domain entry points."""
    from gem_b200 import adz, synth
    prec = adz.MIXED
    doms, spec = [], []
    for cfg in cfgs:
        ad = adz.Adz.from_config(cfg)
        inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32)
        _, wp = ad.new_state(prec)
        ad.adz_inittraj(prec, None, wp)
        ad.adz_traject(prec, cfg.dt, inp, None, wp)  # cold start, untimed
        ntr = len(inp["tracers"])
        srcs = [inp["src_u"], inp["src_v"], inp["src_w"]] + inp["tracers"]
        dsts = [torch.zeros(ad.ext_shape, dtype=torch.float32, device="cuda") for _ in srcs]
        mono = [0, 0, 0] + [1] * ntr
        doms.append((cfg, ad, inp, wp, srcs, dsts, mono))
        spec.append(dict(adz=ad, dt=cfg.dt, winds=inp, wpxyz=wp, nfields=[0, 1, 1, 1 + ntr], srcs=srcs,
                         dsts=dsts, mono=mono))
    npts = sum(c.npoints for c in cfgs)
    batch = adz.Batch(prec, spec)
    t0 = time.time()
    batch.tune()
    tune_s = time.time() - t0
    ms_b, clk = timed(batch.step, args.steps, args.warmup, clocks=True)
    if batch.status() != 0:
        raise RuntimeError("device status set during the batched steps")

    def sequential():
        for cfg, ad, inp, wp, srcs, dsts, mono in doms:
            ad.adz_traject(prec, cfg.dt, inp, None, wp)
            ad.adz_tricub_sets(prec, [0, 1, 1, len(srcs) - 2], srcs, dsts, mono)
    ms_s, _ = timed(sequential, args.steps, args.warmup)
    # per domain: winds, trajectory, and every set's field groups in one launch
    seq_launches = 3 * len(doms)
    plan = batch.query()
    nl = {"one launch": 1, "phased (one launch per phase)": 3}.get(plan["plan"], seq_launches)
    out = {"workload": f"{len(cfgs)} {label}",
           "points_per_step": npts, "value": npts * ws / (ms_b * 1e-3), "unit": "grid-points/s",
           "ms_per_step": ms_b, "launches_per_step": nl, "plan": plan, "tune_s": tune_s,
           "tuner_ms_per_plan": batch.tuned(),
           "sequential_ms_per_step": ms_s, "sequential_launches_per_step": seq_launches,
           "speedup_vs_sequential": ms_s / ms_b, "clocks": clk}
    del batch, doms, spec
    torch.cuda.empty_cache()
    return out


def measure_tracers(args, timed, ws, rank):
    """The mixed-precision workload: the 1024x1024x80 flow with u, v, w and 8
    log-normal (sigma 1) tracers, mono clipping on the tracers; MIXED and the
    FP64 drop-in, one step each as in the headline, then the accuracy of the
    MIXED interpolated fields against the FP64 path on the same FP32 source
    values (interp_accuracy)."""
    from gem_b200 import adz, synth
    ni, nj, nk = args.size
    cfg = synth.config_mixed(ni, nj, nk, seed=tile_seed(rank), ntracers=8)
    out = {"workload": f"adz step {ni}x{nj}x{nk}, u,v,w + 8 log-normal tracers, mono clipping",
           "points_per_step": cfg.npoints}
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float64)
    d32 = {k: (v.float() if torch.is_tensor(v) else [t.float() for t in v]) for k, v in inp.items()}
    del inp
    state = {}
    for name, prec in (("fp64", adz.FP64), ("mixed", adz.MIXED)):
        dt = adz._field_dtype(prec)
        # the FP64 path reads the same FP32 source values, promoted
        data = d32 if prec == adz.MIXED else {k: (v.double() if torch.is_tensor(v) else [t.double() for t in v])
                                               for k, v in d32.items()}
        ad = adz.Adz.from_config(cfg)
        px, wp = ad.new_state(prec)
        ad.adz_inittraj(prec, px, wp)
        outs = {k: torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for k in ("u", "v", "w")}
        tro = [torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for _ in data["tracers"]]

        # bound now: the accuracy passes call each precision's step after the loop
        def step(ad=ad, prec=prec, data=data, px=px, wp=wp, outs=outs, tro=tro):
            adz.step_fused(ad, prec, cfg.dt, data, data, data["tracers"], px, wp, outs, tro, cfg.mono)
        step()  # cold start, untimed
        ms, _ = timed(step, max(3, min(args.steps, 10)), args.warmup)
        if ad.status() != 0:
            raise RuntimeError("device status set during the multi-tracer steps")
        out[name + "_ms_per_step"] = ms
        out[name + "_value"] = cfg.npoints * ws / (ms * 1e-3)
        state[name] = (ad, prec, data, px, wp, outs, tro, step)
    out["speedup_vs_fp64"] = out["fp64_ms_per_step"] / out["mixed_ms_per_step"]
    hbm, _ = peaks()
    out["step_roofline"] = {"algorithmic_bytes_per_point": 160.0,
                            "achieved_gbs": 160.0 * cfg.npoints / (out["mixed_ms_per_step"] * 1e-3) / 1e9}
    out["step_roofline"]["frac"] = out["step_roofline"]["achieved_gbs"] / hbm
    if not args.no_accuracy:
        out["accuracy"] = interp_accuracy(cfg, state["fp64"], d32)
        out["accuracy_full_step"] = step_accuracy(state["fp64"], state["mixed"])
    del state, d32
    torch.cuda.empty_cache()
    return out


def _local_errors(x, r, mn, mx):
    """Error metrics of one field (device tensors of arrival points, FP64):
    local = max |x - r| / max(|r|, largest |source| of the point's monotone
    bound box); norm = max |x - r| / max |r|; rms = RMS error / RMS value;
    pointwise_floor_1e-3 = max |x - r| / max(|r|, 1e-3 max |r|)."""
    d = (x - r).abs()
    ra = r.abs()
    b = torch.maximum(mn.abs(), mx.abs())
    top = float(ra.max())
    return {"local": float((d / torch.maximum(ra, b)).max()), "norm": float(d.max()) / top,
            "rms": float(d.pow(2).mean().sqrt()) / float(r.pow(2).mean().sqrt()),
            "pointwise_floor_1e-3": float((d / ra.clamp_min(1e-3 * top)).max())}


def interp_accuracy(cfg, ref, d32):
    """MIXED interpolated fields against the plain FP64 path (bit-exact with
    the FP64 oracle) on the same FP32 source values at the same FP64
    departure points: the position sets of one more FP64 step
    (adzc_interp_traj), interpolated by the device interpolator with explicit
    positions in both precisions.  That interpolator runs the same per-point
    arithmetic as the step's set kernels.  Tracers are clipped to their bound
    box as in the step.  The bar is local <= 1e-6 (see _local_errors)."""
    from gem_b200 import adz
    ad, prec, data, px, wp, outs, tro, step = ref
    step()
    I = ad.info
    res = {"reference": "plain FP64 GPU path, same FP32 source values, same FP64 departure points "
                        "(position sets of one FP64 step)",
           "definition": "local: max |mixed - fp64| / max(|fp64|, largest |source| of the point's "
                         "monotone bound box); bar 1e-6",
           "fields": []}
    names = ["u", "v", "w"] + [f"tracer{q + 1}" for q in range(len(d32["tracers"]))]
    sets = [1, 2, 3] + [3] * len(d32["tracers"])
    srcs32 = [d32["src_u"], d32["src_v"], d32["src_w"]] + list(d32["tracers"])
    off = I.haloy * I.nit + I.halox
    for s_id in (1, 2, 3):
        pos = ad.adz_interp_traj(prec, s_id)
        lev = (cfg.levels.zt if s_id == 3 else cfg.levels.zm)[1:cfg.nk + 1]
        zt = adz.Ztab(lev, I.nit, I.njt, 1 - ad.grid.i0g, 1 - ad.grid.j0g)
        for name, st, src in zip(names, sets, srcs32):
            if st != s_id:
                continue
            f32 = src.reshape(-1)[off:]
            f64 = src.double().reshape(-1)[off:]
            r, _, rmn, rmx = (o[0] for o in adz.tricublin_mono_m_n(zt, adz.FP64, [f64], pos))
            x, _, xmn, xmx = (o[0].double() for o in adz.tricublin_mono_m_n(zt, adz.MIXED, [f32], pos))
            if name.startswith("tracer"):
                r = torch.maximum(rmn, torch.minimum(rmx, r))
                x = torch.maximum(xmn, torch.minimum(xmx, x))
            e = _local_errors(x, r, rmn, rmx)
            e["field"] = name
            e["clipped"] = name.startswith("tracer")
            res["fields"].append(e)
            del f64, r, rmn, rmx, x, xmn, xmx
        del pos, zt
        torch.cuda.empty_cache()
    res["max_local_all_fields"] = max(f["local"] for f in res["fields"])
    res["max_norm_all_fields"] = max(f["norm"] for f in res["fields"])
    return res


def step_accuracy(ref, mix):
    """Whole MIXED step (its own FP32-interpolated trajectory) against the
    FP64 step, both from the same start positions.  The departure points
    then differ by the trajectory's sensitivity to the winds' FP32
    interpolation, so this measures the step, not the interpolation alone."""
    ad64, p64, _, _, wp64, o64, t64, step64 = ref
    ad32, p32, _, _, wp32, o32, t32, step32 = mix
    start = wp64.clone()
    step64()
    wp32.copy_(start)
    step32()
    res = {"fields": []}
    names = ["u", "v", "w"] + [f"tracer{q + 1}" for q in range(len(t64))]
    sets = [1, 2, 3] + [3] * len(t64)
    for name, st, a, b in zip(names, sets, [o32["u"], o32["v"], o32["w"]] + t32, [o64["u"], o64["v"], o64["w"]] + t64):
        m = ad64.range_mask(st, device="cuda")
        x, y = a[m].double(), b[m]
        d = (x - y).abs()
        res["fields"].append({"field": name, "norm": float(d.max()) / float(y.abs().max()),
                              "rms": float(d.pow(2).mean().sqrt()) / float(y.pow(2).mean().sqrt())})
        del m, x, y, d
    w32, w64 = wp32[:, :, 2:-2, 2:-2], wp64[:, :, 2:-2, 2:-2]
    res["cell_index_mismatches"] = int((w32.float().trunc() != w64.float().trunc()).sum())
    res["positions"] = int(w32.numel())
    res["max_position_diff_grid"] = float((w32 - w64).abs().max())
    return res


def measure_post(args, timed, ws, rank):
    """The passes after the interpolation on the multi-tracer workload (8
    log-normal tracers, 1024x1024x80, MIXED): BICUBH_QV instead of the
    tricubic at the thermo set, the Bermejo-Conde mass fixer (clipped
    correction and proportional rescale), the ILMC filter (2 sweeps, then
    the clip), and the CFL diagnostic; each timed alone."""
    from gem_b200 import adz, synth
    prec = adz.MIXED
    ni, nj, nk = args.size
    cfg = synth.config_mixed(ni, nj, nk, seed=tile_seed(rank), ntracers=8)
    data = synth.make_inputs(cfg, device="cuda", dtype=torch.float32)
    ad = adz.Adz.from_config(cfg)
    px, wp = ad.new_state(prec)
    ad.adz_inittraj(prec, px, wp)
    ad.adz_traject(prec, cfg.dt, data, px, wp)
    trs = data["tracers"]
    z = lambda: torch.zeros(ad.ext_shape, dtype=torch.float32, device="cuda")  # noqa: E731
    m = [z() for _ in trs]
    lin, mn, mx = [z() for _ in trs], [z() for _ in trs], [z() for _ in trs]
    K, W = max(3, min(args.steps, 10)), args.warmup
    out = {"workload": f"{len(trs)} log-normal tracers at {ni}x{nj}x{nk}, MIXED", "ms": {}}

    def tricub():
        ad.adz_tricub_hlt(prec, adz.SET_T, trs, m, mono=[2] * len(trs), post=(lin, mn, mx))

    def qv():
        ad.adz_tricub_hlt(prec, adz.SET_T, trs, m, mono=[2 | adz.QV] * len(trs), post=(lin, mn, mx))
    out["ms"]["tricubic_t_set"] = timed(tricub, K, W)[0]
    out["ms"]["bicubh_qv_t_set"] = timed(qv, K, W)[0]
    g = torch.Generator(device="cuda").manual_seed(5)
    airm_p = 1.0 + 0.2 * torch.rand(ad.ext_shape, generator=g, device="cuda")
    airm_m = airm_p * (1.0 + 0.01 * torch.rand(ad.ext_shape, generator=g, device="cuda"))
    mask = torch.full((nj, ni), cfg.dx ** 2, dtype=torch.float64, device="cuda")
    deficit = torch.zeros(len(trs), dtype=torch.float64, device="cuda")
    tricub()
    base = [t.clone() for t in m]
    spec = [dict(p=trs[q], m=m[q], lin=lin[q], min=mn[q], max=mx[q]) for q in range(len(trs))]

    def restore():
        for t, b in zip(m, base):
            t.copy_(b)

    def bc():
        restore()
        adz.bermejo_conde(ad, prec, spec, airm_p, airm_m, mask, deficit)
    out["ms"]["bermejo_conde_incl_restore"] = timed(bc, K, W)[0]
    out["ms"]["restore_only"] = timed(restore, K, W)[0]
    viol = sum(int(((b < n_) | (b > x_)).sum()) for b, n_, x_ in zip(base, mn, mx))
    rounds = []

    def ilmc():
        restore()
        rounds.append(adz.ilmc(ad, prec, m, mn, mx, airm_m, sweep_max=2, min_max=True))
    out["ms"]["ilmc_incl_restore"] = timed(ilmc, K, W)[0]
    out["ilmc"] = {"violating_points": viol, "points": cfg.npoints * len(trs), "rounds": max(rounds)}
    out["ms"]["cfl"] = timed(lambda: ad.adz_cfl(wp), K, W)[0]
    if ad.status() != 0:
        raise RuntimeError("device status set during the post-processing measurement")
    del data, m, lin, mn, mx, base
    torch.cuda.empty_cache()
    return out


def measure_guess(args, timed, ws, rank):
    """The learned starting guess against the starts the reference has.

    Cold start of the 1024x1024x80 tile (no previous departure points): the
    reference's 6 fixed updates from the arrival point, the plain update run
    to the project tolerance from the arrival point, and the learned guess
    (BF16 tensor-core inference on every point, or on every stride-th point in
    i and j with bilinear interpolation between them) followed by the plain
    update to the same tolerance.  Also at dt = 150 s (Courant numbers near
    2.4), where the arrival point is a worse start.

    Warm step: the next step of the same flow (time t + dt, fresh wind noise)
    from the previous step's departure points, the reference's start after
    its first step (adz_traject.F90:69-70), against the learned guess.

    Reports updates per point, fallbacks, the guess error against the
    converged departure points (1e-6) and the time of each."""
    from gem_b200 import adz, guess, synth
    prec = adz.MIXED
    ni, nj, nk = args.size
    net = guess.GuessNet(guess.load_weights(args.guess_weights))
    K, W = max(3, min(args.steps, 10)), args.warmup
    strides = (1, 2, 4, 8, 16)

    def starts(cfg, inp, ad, prev=None):
        """Time and updates of every start on one workload; prev: the previous
        step's departure points (warm step)."""
        n = guess.npoints(ad)
        _, wp_ref = ad.new_state(prec)
        guess.traject_tol(ad, prec, cfg.dt, inp, wp_ref, tol=1e-6, maxit=60, start=0)
        d_ref = guess.displacement(ad, wp_ref)
        wps, fns = {}, {}
        stats = {}

        def tol_from(name, start, before=None):
            wps[name] = ad.new_state(prec)[1]
            stats[name] = torch.zeros(3, dtype=torch.int64, device="cuda")

            def fn():
                stats[name].zero_()
                if before is not None:
                    before(wps[name])
                guess.traject_tol(ad, prec, cfg.dt, inp, wps[name], start=start, stats=stats[name])
            fns[name] = fn

        tol_from("plain", 0)
        if prev is not None:
            tol_from("warm", 1, lambda wp: wp.copy_(prev))
        # every point: the start points stored, then the iteration from them
        tol_from("learned_s1", 1, lambda wp: net.apply(ad, cfg.dt, inp, wpxyz=wp))
        # coarse grids: one call, the displacements interpolated inside the iteration
        for s_ in strides[1:]:
            name = f"learned_s{s_}"
            wps[name] = ad.new_state(prec)[1]
            stats[name] = torch.zeros(3, dtype=torch.int64, device="cuda")

            def fn(name=name, s_=s_):
                stats[name].zero_()
                guess.traject_guess(ad, net, cfg.dt, inp, wps[name], stride=s_, stats=stats[name])
            fns[name] = fn
        if prev is None:
            def fixed():
                wps.setdefault("fixed", ad.new_state(prec)[1])
                ad.adz_inittraj(prec, None, wps["fixed"])
                ad.adz_traject(prec, cfg.dt, inp, None, wps["fixed"])
            fixed_name = "fixed6"
        else:
            def fixed():  # the reference's warm step: Adz_itraj = 2 updates from the previous departure points
                wps.setdefault("fixed", ad.new_state(prec)[1])
                wps["fixed"].copy_(prev)
                ad.adz_traject(prec, cfg.dt, inp, None, wps["fixed"], niter=2)
            fixed_name = "fixed2_from_previous"
        ms = {fixed_name: timed(fixed, K, W)[0]}
        for name, fn in fns.items():
            ms[name] = timed(fn, K, W)[0]
        for s_ in strides:  # the guess alone (inference + the departure-wind preparation)
            wp = ad.new_state(prec)[1]
            ms[f"inference_s{s_}"] = timed((lambda: net.apply(ad, cfg.dt, inp, wpxyz=wp)) if s_ == 1 else
                                           (lambda s_=s_: net.apply_coarse(ad, cfg.dt, inp, wp, s_)), K, W)[0]
        if ad.status() != 0:
            raise RuntimeError("device status set during the guess measurement")
        out = {"updates_per_point": {}, "fallback_rate": {}, "not_converged": {}, "guess_error_rms": {},
               "max_error_vs_converged": {}, "ms": ms}
        for name in fns:
            st = stats[name].cpu().tolist()
            out["updates_per_point"][name] = st[0] / n
            out["fallback_rate"][name] = st[1] / n
            out["not_converged"][name] = st[2]
            out["max_error_vs_converged"][name] = [float(v) for v in
                                                   (guess.displacement(ad, wps[name]) - d_ref).abs().max(0).values]
        # error of each start itself against the converged departure points
        for s_ in strides:
            wp = ad.new_state(prec)[1]
            if s_ == 1:
                net.apply(ad, cfg.dt, inp, wpxyz=wp)
            else:
                net.apply_coarse(ad, cfg.dt, inp, wp, s_)
            e = guess.displacement(ad, wp) - d_ref
            out["guess_error_rms"][f"learned_s{s_}"] = [float(v) for v in e.pow(2).mean(0).sqrt()]
        if prev is not None:
            e = guess.displacement(ad, prev) - d_ref
            out["guess_error_rms"]["warm"] = [float(v) for v in e.pow(2).mean(0).sqrt()]
        base = "warm" if prev is not None else "plain"
        best = min((k for k in ms if k.startswith("learned")), key=ms.get)
        out["best_learned"] = best
        out["speedup_best_learned_vs_" + base] = ms[base] / ms[best]
        out["updates_saved_per_point_vs_" + base] = (out["updates_per_point"][base] -
                                                     out["updates_per_point"][best])
        out["wp_ref"] = wp_ref
        return out

    res = {"tolerance": guess.TOL, "max_updates": guess.MAXIT, "unit": "grid indices (x, y, level)",
           "strides": list(strides)}
    # cold starts
    for label, dt in (("cold", None), ("cold_dt150", 150.0)):
        cfg = synth.config_cold(ni, nj, nk, seed=tile_seed(rank))
        if dt is not None:
            cfg.dt = dt
        inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
        ad = adz.Adz.from_config(cfg)
        r = starts(cfg, inp, ad)
        r.pop("wp_ref")
        r["workload"] = (f"cold start of the {ni}x{nj}x{nk} tile, {guess.npoints(ad)} arrival points, MIXED, "
                         f"dt={cfg.dt:g} s, vertical-wind noise 0.02 m/s")
        res[label] = r
        del inp, ad
        torch.cuda.empty_cache()
    # warm step: previous step at t, this step at t + dt with fresh wind noise
    cfg = synth.config_cold(ni, nj, nk, seed=tile_seed(rank))
    ad = adz.Adz.from_config(cfg)
    inp0 = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
    _, prev = ad.new_state(prec)
    guess.traject_tol(ad, prec, cfg.dt, inp0, prev, tol=1e-6, maxit=60, start=0)
    del inp0
    cfg.t_now, cfg.seed = cfg.dt, cfg.seed + 1
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
    r = starts(cfg, inp, ad, prev=prev)
    r.pop("wp_ref")
    r["workload"] = (f"warm step of the {ni}x{nj}x{nk} tile: winds at t + dt with fresh noise, started from the "
                     "previous step's departure points (converged to 1e-6)")
    res["warm"] = r
    # tensor-core roofline of the inference on every point (stride 1)
    _, hbm_kind = peaks()
    pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if hbm_kind == "measured" else {}
    peak_tf = float(pk.get("bf16_tflops", TENSOR_FALLBACK_TFLOPS))
    n = guess.npoints(ad)
    flops = n * 2.0 * 128 * (96 + 128 + 16)  # padded MMA work per arrival point
    tf = flops / (res["cold"]["ms"]["inference_s1"] * 1e-3) / 1e12
    res["inference_roofline"] = {"bound": "tensor", "achieved": tf, "peak": peak_tf, "unit": "TFLOP/s",
                                 "frac": tf / peak_tf, "flops_per_point": flops / n,
                                 "note": "stride 1; includes the departure-wind preparation launch"}
    res["speedup_learned_vs_plain"] = res["cold"]["speedup_best_learned_vs_plain"]
    del ad, inp, prev
    torch.cuda.empty_cache()
    res["composite_cold_step"] = measure_composite(args, timed, ws, rank, net)
    return res


def measure_composite(args, timed, ws, rank, net):
    """The whole first step of a run (no previous departure points), u, v, w
    and 4 cosine-bell tracers on the learned-guess flow: the plain FP64
    drop-in as the reference runs it (arrival-point start, max(6, itraj)
    fixed updates, then every set) against the mixed-precision step with the
    learned start on every 16th point and the iteration to the tolerance,
    then every set."""
    from gem_b200 import adz, guess, synth
    ni, nj, nk = args.size
    cfg = synth.config_cold(ni, nj, nk, seed=tile_seed(rank))
    cfg.ntracers, cfg.tracer_kind = 4, "bells"
    inp64 = synth.make_inputs(cfg, device="cuda", dtype=torch.float64)
    K, W = max(3, min(args.steps, 10)), args.warmup
    out = {"workload": f"first step of a run, {ni}x{nj}x{nk}, u,v,w + 4 cosine-bell tracers, dt={cfg.dt:g} s, "
                       "vertical-wind noise 0.02 m/s"}
    for name, prec in (("fp64_fixed6", adz.FP64), ("mixed_learned_s16", adz.MIXED)):
        dt = adz._field_dtype(prec)
        data = {k: (v.to(dt) if torch.is_tensor(v) else [t.to(dt) for t in v]) for k, v in inp64.items()}
        ad = adz.Adz.from_config(cfg)
        px, wp = ad.new_state(prec)
        outs = [torch.zeros(ad.ext_shape, dtype=dt, device="cuda") for _ in range(3 + len(data["tracers"]))]
        srcs = [data["src_u"], data["src_v"], data["src_w"]] + data["tracers"]
        mono = [0, 0, 0] + [0] * len(data["tracers"])
        nf = [0, 1, 1, 1 + len(data["tracers"])]

        def step(ad=ad, prec=prec, data=data, px=px, wp=wp, srcs=srcs, outs=outs, name=name):
            if name.startswith("fp64"):
                ad.adz_inittraj(prec, px, wp)
                ad.adz_traject(prec, cfg.dt, data, px, wp)
            else:
                guess.traject_guess(ad, net, cfg.dt, data, wp, stride=16)
            ad.adz_tricub_sets(prec, nf, srcs, outs, mono)
        ms, _ = timed(step, K, W)
        if ad.status() != 0:
            raise RuntimeError("device status set during the first-step measurement")
        out[name + "_ms"] = ms
        out[name + "_value"] = cfg.npoints * ws / (ms * 1e-3)
        del data, ad, outs, srcs, step
        torch.cuda.empty_cache()
    out["speedup"] = out["fp64_fixed6_ms"] / out["mixed_learned_s16_ms"]
    return out


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # inputs made on the host: nothing of this package runs on the GPU in this arm
    r = cpu_reference(args.cpu_size, args.steps, args.warmup, ntracers=args.ntr, gen_device="cpu")
    line = {"impl": "reference",
            "metric": "SL advection grid-points/s at 1024^2x80 (mixed-precision step; plain FP64 GPU drop-in alongside)",
            "value": r["value"], "unit": "grid-points/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 fields / f64 coefficients (reference precision)", "data": "synthetic",
            "config": workload_config(args, 1),
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": "grid-points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--size", type=lambda s: tuple(int(x) for x in s.split(",")), default=(1024, 1024, 80))
    ap.add_argument("--cpu-size", type=lambda s: tuple(int(x) for x in s.split(",")), default=None,
                    help="tile of the CPU reference (default: --size, the benchmarked tile)")
    ap.add_argument("--ntr", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched uneven-domain measurement")
    ap.add_argument("--batch-domains", type=int, default=16)
    ap.add_argument("--no-guess", action="store_true", help="skip the learned-guess cold-start measurement")
    ap.add_argument("--no-tracers", action="store_true", help="skip the 8-tracer mono measurement")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the accuracy passes of the 8-tracer leg")
    ap.add_argument("--no-post", action="store_true", help="skip the QV / mass-fixer / ILMC / CFL measurement")
    ap.add_argument("--no-level-a", action="store_true",
                    help="skip the reference-named interpolator calls on host arrays")
    ap.add_argument("--guess-weights", default=os.path.join(ROOT, "gem_b200", "data", "guess_mlp.npz"))
    ap.add_argument("--only", choices=["mixed"], default=None,
                    help="run the mixed-precision path alone (small profiling runs)")
    args = ap.parse_args()
    if args.cpu_size is None:
        args.cpu_size = args.size
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
