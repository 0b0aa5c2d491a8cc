"""The FP64 reference MLP (oracle/mlp.py) against central differences of its
own loss, and its BF16 rounding against torch's conversion."""
import numpy as np

from oracle import mlp


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    p = np.zeros(mlp.NPARAMS)
    for name in ("W1", "W2", "W3", "W4"):
        w = mlp.view(p, name)
        w[:] = rng.normal(0, 0.3, size=w.shape)
    for name in ("b1", "b2", "b3", "b4"):
        mlp.view(p, name)[:] = rng.normal(0, 0.1, size=mlp.view(p, name).shape)
    mlp.view(p, "W1")[:, mlp.IN:] = 0
    mlp.view(p, "W4")[mlp.OUT:] = 0
    mlp.view(p, "b4")[mlp.OUT:] = 0
    X = np.zeros((7, mlp.IN_PAD))
    X[:, :mlp.IN] = rng.normal(size=(7, mlp.IN))
    T = rng.normal(size=(7, 4))
    T[:, 3] = rng.uniform(0.5, 2.0, size=7)  # row weights
    loss, g = mlp.loss_and_grad(p, X, T)
    idx = np.concatenate([rng.choice(np.arange(off, off + int(np.prod(sh))), 12, replace=False)
                          for off, sh in mlp.LAYOUT.values()])
    for i in idx:
        if g[i] == 0 and ((i >= 37248 and (i - 37248) // 128 >= 3) or (i >= 39296 and i - 39296 >= 3) or
                          (i < 4096 and i % 32 >= 27)):
            continue  # padding
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.loss_and_grad(pp, X, T)[0] - mlp.loss_and_grad(pm, X, T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(1).normal(size=1000) * 10.0 ** np.random.default_rng(2).integers(-5, 5, 1000)
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(mlp.to_bf16(x), ref)
