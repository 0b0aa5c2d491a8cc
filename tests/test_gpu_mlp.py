"""The learned warm start's tensor-core kernels: the BF16 GEMM against an
FP32 matmul of the same BF16 inputs, the fused MLP against the FP64 oracle
MLP with the engine's BF16 rounding points, the trainer's gradient against
the oracle's, and the warm-start hooks of a context."""
import numpy as np
import pytest

from oracle import mlp as omlp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def bf(x, dev="cuda"):
    return torch.tensor(np.asarray(x, dtype=np.float32), device=dev).to(torch.bfloat16).contiguous()


@pytest.mark.parametrize("M,N,K", [(128, 128, 16), (256, 16, 32), (384, 32, 128), (200, 128, 64),
                                   (128, 200, 48), (128, 128, 8192), (1000, 16, 16)])
def test_gemm_bf16_matches_fp32_matmul(M, N, K):
    from avbd_b200 import warmstart
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    C = warmstart.gemm_bf16(A, B)
    torch.cuda.synchronize()
    ref = A.double() @ B.double().T
    err = (C.double() - ref).abs().max().item()
    assert err <= 1e-5 * max(1.0, ref.abs().max().item()) * (K / 16) ** 0.5, err
    # accumulate into an existing C
    C2 = warmstart.gemm_bf16(A, B, C.clone(), accumulate=True)
    assert (C2.double() - 2 * ref).abs().max().item() <= 2e-5 * max(1.0, ref.abs().max().item()) * (K / 16) ** 0.5


def random_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    from avbd_b200 import warmstart
    p = warmstart.init_params(seed)
    w4 = warmstart.view(p, "W4")
    w4[:3] = rng.normal(0, 0.2, size=(3, 128))
    for name in ("b1", "b2", "b3"):
        warmstart.view(p, name)[:] = rng.normal(0, 0.1, size=128)
    warmstart.view(p, "b4")[:3] = rng.normal(0, 0.1, size=3)
    return p * np.float32(scale)


@pytest.mark.parametrize("n", [1, 128, 1000, 70000])
def test_fused_mlp_matches_fp64_reference(n):
    from avbd_b200 import warmstart
    p = random_params(n)
    rng = np.random.default_rng(n)
    X = np.zeros((n, 32), dtype=np.float32)
    X[:, :27] = rng.normal(size=(n, 27))
    m = warmstart.MLP(p)
    Y = m.forward(bf(X)).cpu().numpy()
    m.close()
    Yr, _ = omlp.forward(p, X, bf16=True)
    scale = np.abs(Yr[:, :3]).max()
    assert np.abs(Y[:, :3] - Yr[:, :3]).max() <= 2e-2 * scale
    assert np.abs(Y[:, 3:]).max() == 0.0  # padding outputs


def test_trainer_gradient_matches_fp64_reference():
    from avbd_b200 import warmstart
    p = random_params(3)
    rng = np.random.default_rng(4)
    B = 256
    X = np.zeros((B, 32), dtype=np.float32)
    X[:, :27] = rng.normal(size=(B, 27))
    T = rng.normal(size=(B, 4)).astype(np.float32)
    T[:, 3] = rng.uniform(0.5, 2.0, size=B)  # row weights of the loss
    tr = warmstart.Trainer(B, p)
    loss, g = tr.grad(bf(X), torch.tensor(T, device="cuda"))
    tr.close()
    lr_, gr = omlp.loss_and_grad(p, omlp.to_bf16(X), T, bf16=True)
    assert abs(loss - lr_) <= 1e-3 * lr_
    for name in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        a, b = warmstart.view(g, name).astype(np.float64), omlp.view(gr, name)
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 3e-2, (name, rel)
    assert np.abs(warmstart.view(g, "W1")[:, 27:]).max() == 0
    assert np.abs(warmstart.view(g, "W4")[3:]).max() == 0


def test_trainer_fits_a_smooth_map():
    """Adam on the tensor cores fits y = A tanh(x) + small noise."""
    from avbd_b200 import warmstart
    rng = np.random.default_rng(5)
    N = 16384
    X = np.zeros((N, 32), dtype=np.float32)
    X[:, :27] = rng.normal(size=(N, 27))
    Amat = rng.normal(size=(27, 3)) / 5
    T = np.ones((N, 4), dtype=np.float32)
    T[:, :3] = np.tanh(X[:, :27]) @ Amat
    Xd, Td = bf(X), torch.tensor(T, device="cuda")
    tr = warmstart.Trainer(2048, warmstart.init_params(0))
    first = None
    for ep in range(30):
        for b in range(N // 2048):
            loss = tr.step(Xd[b * 2048:(b + 1) * 2048], Td[b * 2048:(b + 1) * 2048], 2e-3)
            first = first if first is not None else loss
    tr.close()
    assert loss < 0.05 * first, (first, loss)


def test_warmstart_record_and_apply():
    from avbd_b200 import Context, scenes, warmstart
    sc = scenes.batched_cubes(num_scenes=3, seed=11, n_min=3, n_max=5)
    e = Context()
    sc.load(e, residual_tolerance=1e-4, max_iters=100, precision="mixed")
    e.finalize()
    e.step(5)
    F, T = warmstart.collect(e, steps=3, rows_per_step=10 ** 6)
    assert F.shape[1] == 32 and T.shape[1] == 4
    assert torch.isfinite(F.float()).all() and torch.isfinite(T).all()
    assert (T[:, 3] == 1).all()
    assert (F[:, 27:].float() == 0).all()
    # a zero output layer leaves the inertial guess unchanged: same trajectory as plain
    a = Context()
    sc.load(a, residual_tolerance=1e-4, max_iters=100, precision="mixed")
    a.finalize()
    b = Context()
    sc.load(b, residual_tolerance=1e-4, max_iters=100, precision="mixed")
    b.finalize()
    b.set_warmstart(2, warmstart.init_params(1))
    a.step(8)
    b.step(8)
    assert np.array_equal(a.positions(), b.positions())
    # a nonzero MLP moves the guess, and every scene still ends its step at
    # the tolerance or at the iteration cap, like plain AVBD
    b.set_warmstart(2, random_params(7, 0.01))
    for _ in range(3):
        cap0 = b.stats()["capped_scene_steps"]
        b.step(1)
        st = b.stats()
        assert np.isfinite(b.positions()).all()
        assert st["last_residual"] <= 1e-4 or st["capped_scene_steps"] > cap0
