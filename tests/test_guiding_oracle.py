"""The guiding model's CPU restatement (oracle/guiding_ref.py): analytic gradients against finite
differences, and the vMF mixture is a normalised density.  CPU only."""
import numpy as np

from oracle import guiding_ref as G


def _model(rng):
    ws = [rng.normal(0, 0.3, (64, 48)), rng.normal(0, 0.2, (64, 64)), rng.normal(0, 0.2, (64, 64)),
          rng.normal(0, 0.2, (64, 64)), rng.normal(0, 0.3, (48, 64))]
    return ws


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n = 9
    ws = _model(rng)
    u = rng.normal(0, 1, (n, 48))
    u[:, 38:] = 0
    wd = rng.normal(size=(n, 3))
    wd /= np.linalg.norm(wd, axis=1, keepdims=True)
    cw = rng.uniform(0.1, 2, n)

    def loss(ws_, u_):
        y, _ = G.forward(ws_, u_, emulate_bf16=False)
        return G.loss_and_grad_y(y, wd, cw)[0]

    y, xs = G.forward(ws, u, emulate_bf16=False)
    _, gy = G.loss_and_grad_y(y, wd, cw)
    gws, gu = G.backward(ws, xs, gy, emulate_bf16=False)
    eps = 1e-6
    for li, (a, b) in [(0, (0, 0)), (0, (3, 5)), (1, (10, 20)), (2, (7, 7)), (3, (0, 9)), (4, (3, 5)), (4, (21, 40))]:
        w2 = [w.copy() for w in ws]
        w2[li][a, b] += eps
        w3 = [w.copy() for w in ws]
        w3[li][a, b] -= eps
        fd = (loss(w2, u) - loss(w3, u)) / (2 * eps)
        assert abs(fd - gws[li][a, b]) <= 1e-6 + 1e-4 * abs(fd), (li, a, b)
    for j in (0, 5, 31, 33, 37):
        u2, u3 = u.copy(), u.copy()
        u2[2, j] += eps
        u3[2, j] -= eps
        fd = (loss(ws, u2) - loss(ws, u3)) / (2 * eps)
        assert abs(fd - gu[2, j]) <= 1e-6 + 1e-4 * abs(fd)


def test_mixture_is_normalised():
    rng = np.random.default_rng(1)
    y = rng.normal(0, 1.5, (1, 48))
    d = rng.normal(size=(400000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    integral = (G.mixture_pdf(np.repeat(y, len(d), 0), d) * 4 * np.pi).mean()
    assert abs(integral - 1.0) < 0.01


def test_hash_grid_levels():
    res = [G.level_res(l) for l in range(G.L)]
    assert res[0] == 16 and res[-1] == 1024 and all(a < b for a, b in zip(res, res[1:]))
    dense = [(r + 1) ** 3 <= G.T for r in res]
    assert dense[0] and not dense[-1]
