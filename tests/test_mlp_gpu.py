"""GPU: the learned initialiser's MLP (tensor-core forward/backward + Adam) against the oracle.

The oracle (oracle/mlp.py) rounds to BF16 at the same points as the kernels,
so the remaining differences are FP32-vs-FP64 accumulation and the occasional
BF16 rounding that flips because of it. Gates: output 2e-3 relative L2, loss
1e-3 relative, each weight/bias gradient 1e-2 relative L2, padding rows of W3
and b3 exactly zero. The first Adam step moves each weight by about lr*sign(g):
its sign must agree with the oracle's gradient wherever |g| is not negligible.
"""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import mlp as om

pytestmark = pytest.mark.gpu

D, H, O = 1024, 512, 156


def _batch(M, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(0, 1, (M, D)).astype(np.float32)
    T = rng.normal(0, 0.5, (M, O)).astype(np.float32)
    wout = rng.uniform(0.5, 1.5, O).astype(np.float32)
    return X, T, wout


@pytest.mark.parametrize("M", [300, 1024])
def test_mlp_forward_and_gradients_match_oracle(M):
    from complex_valued_quadratic_phase_gaussian_b200.mlp import TileMLP
    X, T, wout = _batch(M, M)
    w0 = om.init_weights(D, H, O, seed=3)
    w0 += om.valid_mask(D, H, O) * np.random.default_rng(4).normal(0, 0.01, w0.shape).astype(np.float32)
    net = TileMLP(M, weights=torch.from_numpy(w0))
    Y = net.forward(torch.from_numpy(X).cuda())
    loss, g = net.gradients(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda(), torch.from_numpy(wout).cuda())
    torch.cuda.synchronize()
    assert int(net.status.item()) == 0
    ref_loss, ref_Y, ref_g = om.forward_backward(w0, X, T, wout.astype(np.float64), D, H, O, rounding=True)
    assert rel_l2(Y.cpu().numpy(), ref_Y) < 2e-3
    assert abs(float(loss.item()) - ref_loss) < 1e-3 * abs(ref_loss)
    g = g.cpu().numpy()
    lay, _ = om.layout(D, H, O)
    for name, (o, shp) in lay.items():
        n = int(np.prod(shp))
        assert rel_l2(g[o:o + n], ref_g[o:o + n]) < 1e-2, (name, rel_l2(g[o:o + n], ref_g[o:o + n]))
    assert np.all(g[~om.valid_mask(D, H, O)] == 0)


def test_mlp_adam_step_and_training_reduces_loss():
    from complex_valued_quadratic_phase_gaussian_b200.mlp import TileMLP
    M, lr = 512, 1e-3
    X, T, wout = _batch(M, 7)
    w0 = om.init_weights(D, H, O, seed=5)
    net = TileMLP(M, lr=lr, weights=torch.from_numpy(w0))
    Xg, Tg, wg = (torch.from_numpy(a).cuda() for a in (X, T, wout))
    l0 = float(net.train_step(Xg, Tg, wg).item())
    w1 = net.weights.cpu().numpy()
    _, _, ref_g = om.forward_backward(w0, X, T, wout.astype(np.float64), D, H, O, rounding=True)
    step = w1 - w0
    valid = om.valid_mask(D, H, O)
    big = valid & (np.abs(ref_g) > 1e-3 * np.abs(ref_g).max())
    assert np.mean(np.sign(step[big]) == -np.sign(ref_g[big])) > 0.99
    assert np.abs(step[big]).max() <= lr * 1.001
    assert np.all(w1[~valid] == 0)
    assert int(net.step_count.item()) == 1
    for _ in range(60):
        loss = net.train_step(Xg, Tg, wg)
    torch.cuda.synchronize()
    assert int(net.status.item()) == 0
    assert float(loss.item()) < 0.7 * l0


def test_mlp_train_step_replays_from_a_cuda_graph():
    from complex_valued_quadratic_phase_gaussian_b200.mlp import TileMLP
    M = 256
    X, T, wout = _batch(M, 9)
    Xg, Tg, wg = (torch.from_numpy(a).cuda() for a in (X, T, wout))
    a = TileMLP(M, weights=torch.from_numpy(om.init_weights(D, H, O, seed=6)))
    b = TileMLP(M, weights=torch.from_numpy(om.init_weights(D, H, O, seed=6)))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b.train_step(Xg, Tg, wg)  # warm-up outside capture (kernel attributes, tensor maps)
    torch.cuda.current_stream().wait_stream(s)
    a.train_step(Xg, Tg, wg)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        b.train_step(Xg, Tg, wg)
    for _ in range(5):
        a.train_step(Xg, Tg, wg)
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(a.weights, b.weights)
    assert int(a.step_count.item()) == int(b.step_count.item()) == 6


def test_data_parallel_step_on_one_rank_equals_train_step():
    from complex_valued_quadratic_phase_gaussian_b200.mlp import TileMLP
    M = 384
    X, T, wout = _batch(M, 13)
    Xg, Tg, wg = (torch.from_numpy(a).cuda() for a in (X, T, wout))
    a = TileMLP(M, weights=torch.from_numpy(om.init_weights(D, H, O, seed=8)))
    b = TileMLP(M, weights=torch.from_numpy(om.init_weights(D, H, O, seed=8)))
    la = a.train_step(Xg, Tg, wg).clone()
    lb = b.data_parallel_step(Xg, Tg, wg)
    torch.cuda.synchronize()
    # same kernels; the row weighting (x rows / rows) of the all-reduce path rounds the gradient by an ulp
    assert rel_l2(b.weights.cpu().numpy(), a.weights.cpu().numpy()) < 1e-6
    assert rel_l2(b.adam.cpu().numpy(), a.adam.cpu().numpy()) < 1e-5
    assert int(b.step_count.item()) == 1
    assert abs(float(la.item()) - float(lb.item())) <= 1e-6 * abs(float(la.item()))
