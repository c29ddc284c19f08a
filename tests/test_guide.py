"""CPU tests of the guide oracle: its analytic gradients agree with finite
differences (FP64), so it can judge the GPU's tensor-core backward."""
import numpy as np

from oracle import guide_ref as G


def _setup(n=6, seed=0):
    rng = np.random.default_rng(seed)
    Ws = [rng.uniform(-1, 1, (G.layer_out(l), G.layer_in(l))) * np.sqrt(6.0 / G.layer_in(l)) for l in range(G.LAYERS)]
    X = rng.normal(size=(n, G.IN))
    w = rng.normal(size=(n, 3))
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    weight = rng.uniform(0.5, 2.0, n)
    return Ws, X, w, weight


def test_output_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    raw = rng.normal(size=(5, G.OUT))
    raw[:, 3:40:5] = rng.uniform(-1, 3, (5, 8))  # log kappa inside the clamp
    w = rng.normal(size=(5, 3))
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    weight = rng.uniform(0.5, 2, 5)
    g = G.output_grad(raw, w, weight)
    eps = 1e-6
    for i in range(5):
        for k in range(40):
            rp, rm = raw.copy(), raw.copy()
            rp[i, k] += eps
            rm[i, k] -= eps
            fd = (G.loss(rp, w, weight) - G.loss(rm, w, weight)) / (2 * eps)
            assert abs(fd - g[i, k]) < 1e-5 * max(1.0, abs(fd)), (i, k, fd, g[i, k])


def test_weight_gradient_matches_finite_differences():
    Ws, X, w, weight = _setup()
    raw, acts = G.forward(X, Ws)
    dWs, dX = G.backward(acts, Ws, G.output_grad(raw, w, weight))
    rng = np.random.default_rng(2)
    eps = 1e-6
    for l in range(G.LAYERS):
        for _ in range(6):
            i, j = rng.integers(G.layer_out(l)), rng.integers(G.layer_in(l))
            Wp = [W.copy() for W in Ws]
            Wm = [W.copy() for W in Ws]
            Wp[l][i, j] += eps
            Wm[l][i, j] -= eps
            fd = (G.loss(G.forward(X, Wp)[0], w, weight) - G.loss(G.forward(X, Wm)[0], w, weight)) / (2 * eps)
            assert abs(fd - dWs[l][i, j]) < 1e-5 * max(1.0, abs(fd)), (l, i, j, fd, dWs[l][i, j])
    for _ in range(10):  # input gradient (feeds the hash-grid gradient)
        i, j = rng.integers(X.shape[0]), rng.integers(G.IN)
        Xp, Xm = X.copy(), X.copy()
        Xp[i, j] += eps
        Xm[i, j] -= eps
        fd = (G.loss(G.forward(Xp, Ws)[0], w, weight) - G.loss(G.forward(Xm, Ws)[0], w, weight)) / (2 * eps)
        assert abs(fd - dX[i, j]) < 1e-5 * max(1.0, abs(fd))


def test_mixture_density_integrates_to_one():
    rng = np.random.default_rng(3)
    raw = rng.normal(size=(1, G.OUT))
    raw[0, 3:40:5] = rng.uniform(0, 4, 8)
    n = 400000
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    est = 4 * np.pi * G.mixture_pdf(np.repeat(raw, n, 0), v).mean()
    assert abs(est - 1.0) < 0.02
