"""The guess network's CPU restatement (oracle/guess_oracle.py), pinned
without a GPU: its backward pass against central finite differences of the
loss in float64, its GELU derivative likewise, Adam against the published
update written out by hand, and its BF16 rounding against known bit patterns.
These are the checks that make it usable as the oracle of the CUDA training
and inference kernels."""
import numpy as np

from oracle import guess_oracle as G


def _loss64(p, x, t):
    c = np.sqrt(2.0 / np.pi)

    def gelu(h):
        return 0.5 * h * (1.0 + np.tanh(c * (h + 0.044715 * h ** 3)))
    x = x.astype(np.float64)
    a1 = gelu(x @ p["W1"].T.astype(np.float64) + p["b1"])
    a2 = gelu(a1 @ p["W2"].T.astype(np.float64) + p["b2"])
    y = a2 @ p["W3"].T.astype(np.float64) + p["b3"]
    return np.mean(np.sum((y - t) ** 2, axis=1))


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = G.init_params(seed=11)
    for k in ("b1", "b2", "b3"):
        p[k] = (0.1 * rng.standard_normal(p[k].shape)).astype(np.float32)
    x = rng.standard_normal((40, G.NFEAT)).astype(np.float32)
    t = rng.standard_normal((40, G.NOUT)).astype(np.float32)
    g = G.backward(p, x, t)
    h = 1e-3
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        flat = p[name].reshape(-1)
        for q in rng.choice(flat.size, size=min(12, flat.size), replace=False):
            q64 = {k: v.astype(np.float64) for k, v in p.items()}
            base = q64[name].reshape(-1)[q]
            q64[name].reshape(-1)[q] = base + h
            lp = _loss64(q64, x, t)
            q64[name].reshape(-1)[q] = base - h
            lm = _loss64(q64, x, t)
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[q]
            assert abs(an - fd) <= 2e-3 * max(1.0, abs(fd)), (name, q, an, fd)


def test_gelu_grad_and_bf16():
    x = np.linspace(-6, 6, 241)
    h = 1e-5
    c = np.sqrt(2.0 / np.pi)
    f = lambda z: 0.5 * z * (1.0 + np.tanh(c * (z + 0.044715 * z ** 3)))  # noqa: E731
    fd = (f(x + h) - f(x - h)) / (2 * h)
    assert np.max(np.abs(G.gelu_grad(x) - fd)) < 1e-5
    vals = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-40, 65504.0], np.float32)
    want = np.array([1.0, 1.0, 1.0078125, -2.5, 0.0, 65536.0], np.float32)
    got = G.bf16(vals)
    assert np.array_equal(got[[0, 2, 3, 5]], want[[0, 2, 3, 5]])
    assert got[1] in (1.0, 1.0078125) and abs(got[4]) < 1e-38


def test_adam_step_by_hand():
    p = {"a": np.array([1.0, -2.0], np.float32)}
    m = {"a": np.zeros(2, np.float32)}
    v = {"a": np.zeros(2, np.float32)}
    g = {"a": np.array([0.5, -0.25], np.float32)}
    G.adam_step(p, m, v, g, 1, 0.01)
    # first step: m/c1 = g, v/c2 = g^2, update = lr * sign(g)
    assert np.allclose(p["a"], [0.99, -1.99], atol=1e-6)
