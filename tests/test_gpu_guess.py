"""Trajectory to a tolerance, the learned starting guess and its training
kernels, against oracle/guess_oracle.py and the fixed-count trajectory.

Tolerances:
  training kernels (FP32 SIMT): forward 1e-5, gradients 1e-4 of each
    tensor's largest entry (FP32 sums in another order), Adam 1e-6;
  features: 1e-6 relative (same double arithmetic, one FP32 rounding);
  BF16 tensor-core inference against the oracle's BF16 emulation: 0.02 + 1 %
    (hardware tanh approximation and BF16 rounding of the hidden layers),
    mean error below 0.003;
  trajectory with tol 0 and maxit 6 from the arrival point: bit-exact with the
    reference's cold start of 6 fixed updates.
"""
import numpy as np
import pytest
import torch

from oracle import guess_oracle as G

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")


def _params(seed):
    rng = np.random.default_rng(seed + 100)
    p = G.init_params(seed)
    for k in ("b1", "b2", "b3"):
        p[k] = (0.1 * rng.standard_normal(p[k].shape)).astype(np.float32)
    return p


def test_training_kernels_vs_oracle():
    _need_gpu()
    from gem_b200 import guess
    rng = np.random.default_rng(3)
    p = _params(7)
    B = 300
    x = rng.standard_normal((B, G.NFEAT)).astype(np.float32)
    t = rng.standard_normal((B, G.NOUT)).astype(np.float32)
    tr = guess.Trainer(p, max_batch=512)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = tr.forward(xd).cpu().numpy()
    y_ref, _ = G.forward(p, x)
    assert np.max(np.abs(y - y_ref)) <= 1e-5 * max(1.0, np.max(np.abs(y_ref)))
    tr.grad(xd, td)
    g = tr.grads()
    g_ref = G.backward(p, x, t)
    for k in guess.ORDER:
        scale = max(np.max(np.abs(g_ref[k])), 1e-6)
        assert np.max(np.abs(g[k] - g_ref[k])) <= 1e-4 * scale, k
    assert abs(tr.loss() - G.loss(p, x, t)) <= 1e-5 * G.loss(p, x, t)
    # Adam on the device's own gradients
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(v) for k, v in p.items()}
    q = {k: a.copy() for k, a in p.items()}
    for step in (1, 2):
        tr.adam(1e-3)
        G.adam_step(q, m, v, g, step, 1e-3)
    got = tr.params()
    for k in guess.ORDER:
        assert np.max(np.abs(got[k] - q[k])) <= 1e-6, k


def _case(prec, shape=(48, 40, 20)):
    from gem_b200 import adz, synth
    cfg = synth.config_small(*shape)
    dt = adz._field_dtype(prec)
    inp = synth.make_inputs(cfg, device="cuda", dtype=dt)
    ad = adz.Adz.from_config(cfg)
    return adz, cfg, inp, ad


@pytest.mark.parametrize("precname", ["mixed", "fp64"])
def test_tol_from_arrival_point_equals_fixed_cold_start(precname):
    _need_gpu()
    from gem_b200 import adz as A, guess
    prec = A.PREC_NAMES[precname]
    adz, cfg, inp, ad = _case(prec)
    dt = adz._field_dtype(prec)
    _, wp_a = ad.new_state(prec)
    ad.adz_inittraj(prec, None, wp_a)
    ad.adz_traject(prec, cfg.dt, inp, None, wp_a)  # 6 fixed updates from the arrival point
    ua = torch.full(ad.ext_shape, -7.0, dtype=dt, device="cuda")
    ad.adz_tricub_hlt(prec, A.SET_T, [inp["src_w"]], [ua])
    _, wp_b = ad.new_state(prec)
    ad.adz_inittraj(prec, None, wp_b)
    stats = torch.zeros(3, dtype=torch.int64, device="cuda")
    guess.traject_tol(ad, prec, cfg.dt, inp, wp_b, tol=0.0, maxit=6, start=0, stats=stats)
    ub = torch.full(ad.ext_shape, -7.0, dtype=dt, device="cuda")
    ad.adz_tricub_hlt(prec, A.SET_T, [inp["src_w"]], [ub])
    torch.cuda.synchronize()
    assert ad.status() == 0
    assert torch.equal(wp_a, wp_b)
    assert torch.equal(ua, ub)
    s = stats.cpu().numpy()
    assert s[1] == 0 and s[0] <= 6 * guess.npoints(ad)


def test_tol_converges_and_guess_paths():
    _need_gpu()
    from gem_b200 import adz as A, guess, synth
    prec = A.MIXED
    adz, cfg, inp, ad = _case(prec, (64, 56, 24))
    n = guess.npoints(ad)
    # converged reference: tight tolerance
    _, wp_ref = ad.new_state(prec)
    guess.traject_tol(ad, prec, cfg.dt, inp, wp_ref, tol=1e-9, maxit=60, start=0)
    # plain, project tolerance
    _, wp_p = ad.new_state(prec)
    it_p = torch.zeros(ad.nk * ad.nj * ad.ni, dtype=torch.uint8, device="cuda")
    st_p = torch.zeros(3, dtype=torch.int64, device="cuda")
    guess.traject_tol(ad, prec, cfg.dt, inp, wp_p, start=0, iters=it_p, stats=st_p)
    torch.cuda.synchronize()
    assert ad.status() == 0
    s = st_p.cpu().numpy()
    assert s[2] == 0 and s[1] == 0
    k00, _ = guess.arrival_index(ad)
    iters = it_p.view(ad.nk, ad.nj, ad.ni)[k00 - 1:].cpu().numpy().astype(np.int64)
    assert iters.sum() == s[0] and iters.min() >= 1
    d_ref = guess.displacement(ad, wp_ref)
    assert torch.max(torch.abs(guess.displacement(ad, wp_p) - d_ref)).item() <= 10 * guess.TOL
    # a guess from random weights: converges (with fallbacks where it must)
    net = guess.GuessNet(_params(9))
    _, wp_g = ad.new_state(prec)
    disp = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    net.apply(ad, cfg.dt, inp, wpxyz=wp_g, disp=disp)
    torch.cuda.synchronize()
    start = guess.displacement(ad, wp_g)
    dz_ok = (start[:, 2] - disp[:, 2].double()).abs() <= 1e-6  # vertical may be clipped
    assert torch.max(torch.abs(start[:, :2] - disp[:, :2].double())).item() <= 1e-5
    assert dz_ok.float().mean().item() > 0.5
    st_g = torch.zeros(3, dtype=torch.int64, device="cuda")
    guess.traject_tol(ad, prec, cfg.dt, inp, wp_g, start=1, stats=st_g)
    torch.cuda.synchronize()
    assert ad.status() == 0 and st_g[2].item() == 0
    assert torch.max(torch.abs(guess.displacement(ad, wp_g) - d_ref)).item() <= 10 * guess.TOL


def _odelz_m(levels):
    zm = np.asarray(levels.zm, np.float64)
    nk = len(zm) - 2
    return np.array([1.0 / (zm[k + 1] - zm[k]) for k in range(nk + 1)])


# 40x36x16: 180 full tiles, one or two per CTA (no stage reused); 67x53x29:
# about 800 tiles with a partial last one, so every CTA reuses its four stages
@pytest.mark.parametrize("size", [(40, 36, 16), (67, 53, 29)])
def test_features_and_bf16_inference_vs_oracle(size):
    _need_gpu()
    from gem_b200 import adz as A, guess, synth
    from oracle import oracle as O
    prec = A.MIXED
    adz, cfg, inp, ad = _case(prec, size)
    # oracle departure winds from the same FP32 inputs, in FP64
    st = O.Step(cfg, kind="oracle", prec="f64")
    st.inittraj()
    st.traject({k: inp[k].double().cpu().numpy() for k in ("uu_ext", "vv_ext", "ww_ext", "ut0", "vt0", "zdt0")})
    planes = np.moveaxis(st.uvw_d, -1, 0).astype(np.float32)
    ga = synth.grid_arrays(cfg)
    k00, _ = guess.arrival_index(ad)
    f_ref = G.features(planes, ad.info.nit, ad.info.njt, cfg.nk, ad.info.halox, cfg.ni, cfg.nj, k00, cfg.dt,
                       ga["inv_hx"], ga["inv_hy"], _odelz_m(cfg.levels))
    f_gpu = guess.features(ad, cfg.dt, inp).cpu().numpy()
    assert f_gpu.shape == f_ref.shape
    assert np.max(np.abs(f_gpu - f_ref) / (np.abs(f_ref) + 1e-3)) <= 1e-5
    idx = torch.tensor([0, 5, f_gpu.shape[0] - 1], dtype=torch.int64, device="cuda")
    assert np.array_equal(guess.features(ad, cfg.dt, inp, idx=idx).cpu().numpy(), f_gpu[[0, 5, -1]])
    # BF16 tensor-core inference
    p = _params(13)
    net = guess.GuessNet(p)
    disp = torch.zeros((f_gpu.shape[0], 3), dtype=torch.float32, device="cuda")
    net.apply(ad, cfg.dt, inp, disp=disp)
    torch.cuda.synchronize()
    assert ad.status() == 0
    y = disp.cpu().numpy()
    y_ref = G.forward_bf16(p, f_gpu)
    err = np.abs(y - y_ref)
    print("bf16 inference: max err", err.max(), "mean err", err.mean(), "max |y|", np.abs(y_ref).max())
    assert np.all(err <= 0.02 + 0.01 * np.abs(y_ref))
    assert err.mean() <= 0.003


def test_trained_network_saves_updates():
    """The committed network (gem_b200/data/guess_mlp.npz, trained by the
    project's kernels on the plain iteration's own trajectories) on a cold
    start of the learned-guess flow: fewer updates per point than the plain
    start from the arrival point, at most 1 % of points falling back, every
    point converged to the tolerance; on every point and on a coarse grid of
    every 4th point in i and j."""
    _need_gpu()
    from gem_b200 import adz as A, guess, synth
    prec = A.MIXED
    cfg = synth.config_cold(192, 160, 80, seed=77)
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
    ad = A.Adz.from_config(cfg)
    n = guess.npoints(ad)
    net = guess.GuessNet(guess.load_weights())
    _, wp_ref = ad.new_state(prec)
    guess.traject_tol(ad, prec, cfg.dt, inp, wp_ref, tol=1e-6, maxit=60, start=0)
    d_ref = guess.displacement(ad, wp_ref)
    upd = {}
    for name, stride in (("plain", 0), ("learned", 1), ("learned_coarse4", 4)):
        _, wp = ad.new_state(prec)
        if stride == 1:
            net.apply(ad, cfg.dt, inp, wpxyz=wp)
        elif stride > 1:
            net.apply_coarse(ad, cfg.dt, inp, wp, stride)
        if stride:
            err = (guess.displacement(ad, wp) - d_ref).pow(2).mean(0).sqrt()
            print(name, "guess RMS error (x, y, level)", err.tolist())
            assert torch.all(err < 0.05)  # the arrival point is ~1 grid length and ~1.5 levels away
        st = torch.zeros(3, dtype=torch.int64, device="cuda")
        guess.traject_tol(ad, prec, cfg.dt, inp, wp, start=1 if stride else 0, stats=st)
        torch.cuda.synchronize()
        s = st.cpu().tolist()
        assert ad.status() == 0 and s[2] == 0, (name, s)
        assert s[1] <= 0.01 * n, (name, s)
        upd[name] = s[0] / n
        assert torch.max(torch.abs(guess.displacement(ad, wp) - d_ref)).item() <= 10 * guess.TOL
    print("updates per point", upd)
    assert upd["learned"] < upd["plain"] - 0.5
    assert upd["learned_coarse4"] < upd["plain"] - 0.3


def test_coarse_guess_interpolates_the_node_displacements():
    """adzc_guess_apply_coarse: on the coarse nodes the start points equal
    those of the network on every point; in between they are the bilinear
    interpolation (in i, j) of the nodes' displacements."""
    _need_gpu()
    from gem_b200 import adz as A, guess, synth
    prec = A.MIXED
    cfg = synth.config_cold(45, 38, 16, seed=5)  # sizes not multiples of the stride
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
    ad = A.Adz.from_config(cfg)
    net = guess.GuessNet(guess.load_weights())
    n = guess.npoints(ad)
    disp = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    net.apply(ad, cfg.dt, inp, disp=disp)
    k00, (nkp, nj, ni) = guess.arrival_index(ad)
    d = disp.view(nkp, nj, ni, 3).double().cpu().numpy()
    for stride in (3, 4):
        _, wp = ad.new_state(prec)
        net.apply_coarse(ad, cfg.dt, inp, wp, stride)
        got = guess.displacement(ad, wp).view(nkp, nj, ni, 3).cpu().numpy()
        xs = np.minimum(1 + stride * np.arange((ni - 2 + stride) // stride + 1), ni) - 1
        ys = np.minimum(1 + stride * np.arange((nj - 2 + stride) // stride + 1), nj) - 1
        want = np.empty_like(d)
        for i in range(ni):
            m = min(i // stride, len(xs) - 2)
            wx = (i - xs[m]) / (xs[m + 1] - xs[m])
            for j in range(nj):
                q = min(j // stride, len(ys) - 2)
                wy = (j - ys[q]) / (ys[q + 1] - ys[q])
                c = lambda a, b: d[:, ys[b], xs[a]]  # noqa: E731
                lo = c(m, q) + wx * (c(m + 1, q) - c(m, q))
                hi = c(m, q + 1) + wx * (c(m + 1, q + 1) - c(m, q + 1))
                want[:, j, i] = lo + wy * (hi - lo)
        # the vertical start is clipped to the levels; compare where it is not
        ok = np.abs(got[..., 2] - want[..., 2]) <= 1e-5
        interior = (np.arange(nkp)[:, None, None] + k00 - want[..., 2] >= 1.0) & \
                   (np.arange(nkp)[:, None, None] + k00 - want[..., 2] <= ad.nk)
        assert np.all(ok | ~interior)
        assert np.max(np.abs(got[..., :2] - want[..., :2])) <= 1e-5
        # the nodes themselves: the network's own displacement
        node = np.zeros((nj, ni), bool)
        node[np.ix_(ys, xs)] = True
        assert np.max(np.abs(got[:, node, :2] - d[:, node, :2])) <= 1e-6


def test_fused_learned_trajectory_matches_the_two_calls():
    """adzc_traject_guess (network on the coarse grid, displacements
    interpolated inside the tolerance iteration) gives bit for bit the
    positions and counters of adzc_guess_apply_coarse followed by
    adzc_traject_tol from the stored start points."""
    _need_gpu()
    from gem_b200 import adz as A, guess, synth
    prec = A.MIXED
    cfg = synth.config_cold(70, 52, 24, seed=3)
    inp = synth.make_inputs(cfg, device="cuda", dtype=torch.float32, with_fields=False)
    ad = A.Adz.from_config(cfg)
    net = guess.GuessNet(guess.load_weights())
    for stride in (1, 4, 8):
        _, wp_a = ad.new_state(prec)
        st_a = torch.zeros(3, dtype=torch.int64, device="cuda")
        net.apply_coarse(ad, cfg.dt, inp, wp_a, stride)
        guess.traject_tol(ad, prec, cfg.dt, inp, wp_a, start=1, stats=st_a)
        _, wp_b = ad.new_state(prec)
        st_b = torch.zeros(3, dtype=torch.int64, device="cuda")
        guess.traject_guess(ad, net, cfg.dt, inp, wp_b, stride=stride, stats=st_b)
        torch.cuda.synchronize()
        assert ad.status() == 0
        assert torch.equal(st_a, st_b), stride
        assert torch.equal(wp_a.view(torch.int64), wp_b.view(torch.int64)), stride
        assert st_b[2].item() == 0


def test_inference_wait_times_out_and_recovers():
    """Failure detection without a GPU fault: each CTA's first tile is made to
    withhold its signal to the MMA thread (host-side injection) under a short
    wait bound.  The wait runs out, every role of the kernel stops, the host
    reads ADZC_ERR_TIMEOUT, and the next call (injection cleared) gives the
    same displacements as a network that never saw the fault: the context
    stays usable."""
    import time
    _need_gpu()
    from gem_b200 import adz as A, guess
    _, cfg, inp, ad = _case(A.MIXED, (67, 53, 29))
    n = guess.npoints(ad)
    ref = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    guess.GuessNet(_params(13)).apply(ad, cfg.dt, inp, disp=ref)
    torch.cuda.synchronize()
    assert ad.status() == 0
    net = guess.GuessNet(_params(13))
    net.inject(net.INJECT_SPINS, 1 << 14)
    net.inject(net.INJECT_WITHHOLD, 1)
    out = torch.zeros_like(ref)
    t0 = time.time()
    net.apply(ad, cfg.dt, inp, disp=out)
    torch.cuda.synchronize()
    assert time.time() - t0 < 60
    assert ad.status() == 6  # ADZC_ERR_TIMEOUT, read and reset
    assert ad.status() == 0
    net.inject(net.INJECT_WITHHOLD, 0)
    net.inject(net.INJECT_SPINS, 0)
    net.apply(ad, cfg.dt, inp, disp=out)
    torch.cuda.synchronize()
    assert ad.status() == 0
    assert torch.equal(out, ref)
    with pytest.raises(A.AdzError):
        net.inject(9, 1)
