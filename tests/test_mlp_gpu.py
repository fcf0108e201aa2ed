"""The learned-guess network's tensor-core kernels against the CPU oracle
(GPU tests): forward pass, gradients of one batch, one Adam step, and a
short training run that must lower the loss.

The device products (tcgen05.mma) are BF16 x BF16 with FP32 accumulation
and the oracle rounds to BF16 at the same points in float64, so the two
differ by FP32 accumulation order and by the rare value that lands on the
other side of a BF16 rounding boundary: relative error norms below 2e-3 per
parameter block (measured: at most 2.1e-4, on the 112-256-256-232 network),
and below 1e-4 for the forward output (measured: at most 3.5e-5)."""
import numpy as np
import pytest

from oracle import mlp_ref
from helpers import pfk

pytestmark = pytest.mark.gpu


def _net(dims, seed=0, max_batch=512):
    pfk()
    import importlib
    M = importlib.import_module("planck-refactored_b200.mlp")
    return M.MLP(dims, max_batch, seed=seed)


def _data(dims, n, seed):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, dims[0])).astype(np.float32)
    T = rng.normal(size=(n, dims[-1])).astype(np.float32)
    return X, T


@pytest.mark.parametrize("dims,n", [([112, 256, 256, 232], 300), ([16, 24, 8], 7), ([40, 64, 32, 48], 130)])
def test_forward_and_gradients_match_oracle(dims, n):
    torch = pytest.importorskip("torch")
    net = _net(dims, seed=1)
    X, T = _data(dims, n, 2)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    p = net.params()
    Y = net.forward(Xd).cpu().numpy()
    Yo = mlp_ref.forward(dims, p, X)[0]
    assert np.linalg.norm(Y - Yo) < 1e-4 * np.linalg.norm(Yo)
    g, loss = net.gradients(Xd, Td)
    go, losso = mlp_ref.gradients(dims, p, X, T)
    assert abs(loss - losso) < 1e-4 * losso
    o = 0
    for din, dout in zip(dims[:-1], dims[1:]):
        for size in (din * dout, dout):
            a, b = g[o:o + size], go[o:o + size]
            assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-12
            o += size
    net.close()


def test_adam_step_matches_oracle():
    torch = pytest.importorskip("torch")
    dims = [32, 64, 16]
    net = _net(dims, seed=3)
    X, T = _data(dims, 64, 4)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    p0 = net.params().astype(np.float64)
    g, _ = net.gradients(Xd, Td)           # the gradient the step will use
    net.train_step(Xd, Td, 1e-2)
    p1 = net.params()
    po, _, _ = mlp_ref.adam(p0, g.astype(np.float64), np.zeros_like(p0), np.zeros_like(p0), 1, 1e-2)
    assert np.abs(p1 - po).max() < 1e-5
    net.close()


def test_training_lowers_the_loss():
    torch = pytest.importorskip("torch")
    dims = [16, 64, 64, 8]
    rng = np.random.default_rng(5)
    X = rng.normal(size=(512, 16)).astype(np.float32)
    W = rng.normal(size=(16, 8)) / 4
    T = np.tanh(X @ W).astype(np.float32)            # a smooth target the network can fit
    net = _net(dims, seed=6)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    first = net.gradients(Xd, Td)[1]
    for _ in range(300):
        net.train_step(Xd, Td, 3e-3)
    last = net.gradients(Xd, Td)[1]
    assert last < 0.1 * first
    net.close()
