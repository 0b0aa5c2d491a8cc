"""Host side of the learned warm start, on CPU: the parameter layout shared
by the engine, the trainer and the FP64 reference MLP; the initialisation
that leaves the inertial guess unchanged; the input standardisation; and the
folding of that standardisation into the first layer and of the output scale
into the last, checked through the FP64 reference forward pass."""
import numpy as np
import torch

from avbd_b200 import warmstart
from oracle import mlp


def _random_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(warmstart.NPARAMS)
    for name in ("W1", "W2", "W3", "W4", "b1", "b2", "b3", "b4"):
        v = warmstart.view(p, name)
        v[:] = rng.normal(0, 0.2, size=v.shape)
    warmstart.view(p, "W1")[:, warmstart.IN:] = 0
    warmstart.view(p, "W4")[warmstart.OUT:] = 0
    warmstart.view(p, "b4")[warmstart.OUT:] = 0
    return p


def test_layout_is_contiguous_and_shared_with_the_reference_mlp():
    assert warmstart.LAYOUT == mlp.LAYOUT
    end = 0
    for off, shape in sorted(warmstart.LAYOUT.values()):
        assert off == end
        end = off + int(np.prod(shape))
    assert end == warmstart.NPARAMS == mlp.NPARAMS


def test_untrained_network_leaves_the_guess_unchanged():
    p = warmstart.init_params(3)
    assert p.dtype == np.float32 and p.shape == (warmstart.NPARAMS,)
    # padding columns of the first layer stay zero, the output layer is zero
    assert (warmstart.view(p, "W1")[:, warmstart.IN:] == 0).all()
    assert (warmstart.view(p, "W4") == 0).all() and (warmstart.view(p, "b4") == 0).all()
    X = np.random.default_rng(0).normal(size=(64, warmstart.IN_PAD))
    y, _ = mlp.forward(p, X)
    assert (y == 0).all()
    assert np.array_equal(warmstart.init_params(3), p)


def test_standardise_keeps_the_padding_neutral():
    rng = np.random.default_rng(1)
    F = np.zeros((4096, warmstart.IN_PAD), dtype=np.float32)
    F[:, :warmstart.IN] = rng.normal(2.0, 3.0, size=(4096, warmstart.IN))
    F[:, 7] = 5.0  # a constant feature
    mean, std = warmstart.standardise(torch.from_numpy(F).to(torch.bfloat16))
    assert mean.shape == std.shape == (warmstart.IN_PAD,)
    assert (mean[warmstart.IN:] == 0).all() and (std[warmstart.IN:] == 1).all()
    assert std[7] == 1.0 and abs(mean[7] - 5.0) < 1e-6
    live = [j for j in range(warmstart.IN) if j != 7]
    assert np.allclose(mean[live], 2.0, atol=0.2) and np.allclose(std[live], 3.0, rtol=0.1)


def test_residual_weights_grow_with_the_block_stiffness():
    from avbd_b200.train_warmstart import residual_weights
    F = torch.zeros((3, warmstart.IN_PAD), dtype=torch.bfloat16)
    # features 18-20: log(1 + H_aa h^2 / m) = 0, log 2, log 101
    for r, lam in enumerate((0.0, 1.0, 100.0)):
        F[r, 18:21] = float(np.log1p(lam))
    w = residual_weights(F)
    assert abs(float(w.mean()) - 1.0) < 1e-6
    # (1 + mean_a H_aa h^2/m)^2 of the BF16-rounded features, normalised
    lam = np.expm1(F[:, 18:21].float().numpy().astype(np.float64)).mean(1)
    raw = (1.0 + lam) ** 2
    assert np.allclose(w.numpy(), raw / raw.mean(), rtol=1e-5)
    assert w[0] < w[1] < w[2]


def test_fold_gives_the_raw_feature_network():
    rng = np.random.default_rng(2)
    p = _random_params(4)
    mean = np.concatenate([rng.normal(size=warmstart.IN), np.zeros(warmstart.IN_PAD - warmstart.IN)])
    std = np.concatenate([rng.uniform(0.1, 10.0, size=warmstart.IN), np.ones(warmstart.IN_PAD - warmstart.IN)])
    out_std = np.concatenate([rng.uniform(0.01, 5.0, size=warmstart.OUT),
                              np.ones(warmstart.OUT_PAD - warmstart.OUT)])
    X = np.zeros((256, warmstart.IN_PAD))
    X[:, :warmstart.IN] = mean[:warmstart.IN] + std[:warmstart.IN] * rng.normal(size=(256, warmstart.IN))
    y_std, _ = mlp.forward(p, (X - mean) / std)
    y_raw, _ = mlp.forward(warmstart.fold(p, mean, std, out_std), X)
    want = y_std[:, :warmstart.OUT] * out_std[:warmstart.OUT]
    # the folded parameters are stored in FP32
    scale = np.abs(want).max()
    assert np.abs(y_raw[:, :warmstart.OUT] - want).max() <= 1e-5 * scale
    assert (y_raw[:, warmstart.OUT:] == 0).all()
