"""The guiding model on the GPU against its CPU restatement (oracle/guiding_ref.py): forward pass
(bf16 tensor-core MLP), gradients of the loss (MLP weights and hash grid) on both training paths and
the Adam step."""
import numpy as np
import pytest

import swpathtracer_b200 as spt
from swpathtracer_b200 import abi
from oracle import guiding_ref as G

pytestmark = pytest.mark.gpu


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _mlp_list(flat):
    out, off = [], 0
    for o, i in abi.GUIDE_MLP_SHAPES:
        out.append(flat[off:off + o * i].reshape(o, i).astype(np.float64))
        off += o * i
    return out


def _guide(device, seed=3, train_path=abi.GUIDE_TRAIN_TCGEN05):
    g = spt.Guide(device, spt.guide_config(seed=seed, train_path=train_path))
    grid, mlp = g.get_params()
    rng = np.random.default_rng(seed)
    grid = rng.uniform(-0.5, 0.5, grid.shape).astype(np.float32)   # non-trivial features
    g.set_params(grid=grid)
    return g, grid, mlp


def _records(rng, n):
    r = np.zeros(n, abi.GUIDE_RECORD_DTYPE)
    r["pos"] = rng.uniform(0.02, 0.98, (n, 3))
    r["normal"] = _unit(rng, n)
    r["wo"] = _unit(rng, n)
    r["wi"] = _unit(rng, n)
    r["weight"] = rng.uniform(0.0, 2.0, n)
    return r


def _oracle_outputs(grid, mlp, pos, normal, wo):
    table = G.bf16(grid.reshape(G.L, G.T, G.F))
    feats, corners = G.encode(table, pos)
    u = G.inputs(feats, normal, wo)
    y, xs = G.forward(_mlp_list(mlp), u)
    return y, xs, corners


def test_forward_matches_oracle(device):
    g, grid, mlp = _guide(device)
    rng = np.random.default_rng(5)
    n = 999
    pos, normal, wo = rng.uniform(0, 1, (n, 3)), _unit(rng, n), _unit(rng, n)
    got = g.eval(pos, normal, wo)
    y, _, _ = _oracle_outputs(grid, mlp, pos, normal, wo)
    mu, kappa, w, _, _ = G.decode(y)
    cos = (got[:, :, 0:3] * mu).sum(2)
    assert np.quantile(cos, 0.01) > 0.995
    np.testing.assert_allclose(got[:, :, 4], w, rtol=0.05, atol=2e-3)
    np.testing.assert_allclose(np.log(got[:, :, 3]), np.log(kappa), atol=0.05)
    g.close()


@pytest.mark.parametrize("path,n", [(abi.GUIDE_TRAIN_TCGEN05, 4000), (abi.GUIDE_TRAIN_MMA_SYNC, 4000),
                                    (abi.GUIDE_TRAIN_TCGEN05, 1 << 18), (abi.GUIDE_TRAIN_TCGEN05, 77)])
def test_gradients_match_oracle(device, path, n):
    """Both training paths (tcgen05 tiles of 128 records with tensor-memory accumulators, and the
    warp-level mma.sync kernels), at the configured batch of 2^18 records, a ragged batch and one
    smaller than a tile."""
    g, grid, mlp = _guide(device, seed=4, train_path=path)
    rng = np.random.default_rng(6)
    recs = _records(rng, n)
    ggrid, gmlp, loss = g.gradients(recs)
    y, xs, corners = _oracle_outputs(grid, mlp, recs["pos"], recs["normal"], recs["wo"])
    cw = recs["weight"] / recs["weight"].mean()
    oloss, gy = G.loss_and_grad_y(y, recs["wi"].astype(np.float64), cw)
    gws, gu = G.backward(_mlp_list(mlp), xs, gy)
    assert abs(loss - oloss) < 1e-2 * abs(oloss) + 1e-3
    off = 0
    for (o, i), gw in zip(abi.GUIDE_MLP_SHAPES, gws):
        a = gmlp[off:off + o * i].reshape(o, i)
        off += o * i
        rel = np.linalg.norm(a - gw) / max(np.linalg.norm(gw), 1e-30)
        assert rel < 0.05, rel
    gt = G.grid_grad(corners, gu, (G.L, G.T, G.F)).reshape(-1)
    touched = gt != 0
    rel = np.linalg.norm(ggrid[touched] - gt[touched]) / np.linalg.norm(gt[touched])
    assert rel < 0.05, rel
    assert np.count_nonzero(ggrid[~touched]) == 0
    g.close()


def test_adam_step_matches_oracle(device):
    g, grid, mlp = _guide(device, seed=7)
    rng = np.random.default_rng(8)
    recs = _records(rng, 2048)
    _, gmlp, _ = g.gradients(recs)
    g.train(recs)
    _, mlp1 = g.get_params()
    exp, _, _ = G.adam(mlp.astype(np.float64), gmlp.astype(np.float64), 0.0, 0.0, 1)
    np.testing.assert_allclose(mlp1, exp, rtol=1e-4, atol=1e-6)
    g.close()


def test_grid_adam_is_lazy(device):
    """The hash grid's Adam step moves exactly the entries the batch touched, by the Adam update."""
    g, grid, mlp = _guide(device, seed=11)
    rng = np.random.default_rng(12)
    recs = _records(rng, 512)
    ggrid, _, _ = g.gradients(recs)
    g.train(recs)
    grid1, _ = g.get_params()
    exp, _, _ = G.adam_lazy(grid.astype(np.float64), ggrid.astype(np.float64), 0.0, 0.0, 1)
    touched = ggrid != 0
    assert 0 < touched.sum() < touched.size // 10
    np.testing.assert_array_equal(grid1[~touched], grid[~touched])
    np.testing.assert_allclose(grid1[touched], exp[touched], rtol=1e-4, atol=1e-6)
    g.close()


def test_training_learns_a_directional_distribution(device):
    """Records whose incident directions cluster around a position-dependent direction: the loss
    falls and the learned mixture puts far more density there than uniform (1/4pi)."""
    g = spt.Guide(device, spt.guide_config(seed=9))
    rng = np.random.default_rng(10)

    def batch(n):
        r = np.zeros(n, abi.GUIDE_RECORD_DTYPE)
        p = rng.uniform(0.05, 0.95, (n, 3))
        r["pos"] = p
        r["normal"] = np.array([0.0, 1.0, 0.0])
        r["wo"] = np.array([0.0, 1.0, 0.0])
        target = np.where(p[:, :1] < 0.5, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
        d = target + 0.15 * rng.normal(size=(n, 3))
        r["wi"] = d / np.linalg.norm(d, axis=1, keepdims=True)
        r["weight"] = 1.0
        return r

    losses = [g.train(batch(1 << 14)) for _ in range(60)]
    assert losses[-1] < losses[0] - 1.0
    test = batch(500)
    out = g.eval(test["pos"], test["normal"], test["wo"])
    target = np.where(test["pos"][:, :1] < 0.5, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    yy = np.zeros((500, 48))
    y5 = yy[:, :40].reshape(500, 8, 5)
    y5[:, :, 0:3] = out[:, :, 0:3]
    y5[:, :, 3] = np.log(out[:, :, 3])
    y5[:, :, 4] = np.log(np.maximum(out[:, :, 4], 1e-30))
    yy[:, :40] = y5.reshape(500, 40)
    q = G.mixture_pdf(yy, target)
    assert np.median(q) > 20 * (1 / (4 * np.pi))
    g.close()
