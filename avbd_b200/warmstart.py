"""Learned warm start: a per-vertex MLP that corrects the inertial initial
guess of every step (x0 <- x0 + s * MLP(features), s = g h^2), then plain
AVBD iterations run to the same residual tolerance.

The reference has no learned component; this module drives the engine's
tensor-core MLP kernels (include/avbd.h, "learned warm start") through the
C-ABI with device buffers owned by PyTorch:

* `MLP` -- fused inference on feature rows (BF16 [n][32] -> FP32 [n][16]);
* `Trainer` -- forward/backward/Adam on mini-batches;
* `gemm_bf16` -- the tensor-core GEMM the trainer is built on;
* `collect` -- features and targets recorded from the plain solver;
* `train` -- the training loop with input standardisation folded into the
  first layer and the output scale folded into the last.

Parameters are one FP32 array in PyTorch Linear layout (`LAYOUT`).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _lib
from ._lib import check

IN, IN_PAD, HID, OUT, OUT_PAD, NPARAMS = (_lib.MLP_IN, _lib.MLP_IN_PAD, _lib.MLP_HIDDEN, _lib.MLP_OUT,
                                          _lib.MLP_OUT_PAD, _lib.MLP_NPARAMS)
# name -> (offset, shape) in the flat parameter array
LAYOUT = {"W1": (0, (HID, IN_PAD)), "b1": (4096, (HID,)), "W2": (4224, (HID, HID)), "b2": (20608, (HID,)),
          "W3": (20736, (HID, HID)), "b3": (37120, (HID,)), "W4": (37248, (OUT_PAD, HID)), "b4": (39296, (OUT_PAD,))}
# the applied correction is gated off where the block residual at the
# inertial guess is below GATE m g (L1 of features 12-14), as in the kernel
GATE = 1e-4
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_mlp.npz")
FEATURE_NAMES = (["x0-y"] * 3 + ["v h"] * 3 + ["prev correction"] * 3 + ["ring dv h"] * 3 + ["rhs h2/m"] * 3 +
                 ["newton step"] * 3 + ["log1p diag H h2/m"] * 3 + ["mu/lambda", "log10 m + 3", "tanh x0_y/10",
                                                                    "lambda_n h2/m", "tets/24", "tanh y_y"])


def view(params: np.ndarray, name: str) -> np.ndarray:
    off, shape = LAYOUT[name]
    return params[off:off + int(np.prod(shape))].reshape(shape)


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform fan-in initialisation of the SiLU layers (zero padding columns)
    and a zero output layer, so the untrained MLP leaves the inertial guess
    unchanged."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, dtype=np.float32)
    for name, fan_in in (("W1", IN), ("W2", HID), ("W3", HID)):
        w = view(p, name)
        bound = math.sqrt(6.0 / fan_in)
        w[:, :fan_in] = rng.uniform(-bound, bound, size=(w.shape[0], fan_in))
    return p


def fold(params: np.ndarray, mean: np.ndarray, std: np.ndarray, out_std: np.ndarray) -> np.ndarray:
    """Parameters of an MLP trained on standardised inputs (x - mean) / std
    and scaled targets t / out_std, rewritten to take raw features and give
    raw outputs: W1' = W1 / std, b1' = b1 - W1' mean, W4' = out_std W4,
    b4' = out_std b4."""
    p = params.astype(np.float64).copy()
    W1, b1 = view(p, "W1"), view(p, "b1")
    W1[:, :IN] /= std[None, :IN]
    b1 -= W1[:, :IN] @ mean[:IN]
    W4, b4 = view(p, "W4"), view(p, "b4")
    W4[:OUT] *= out_std[:OUT, None]
    b4[:OUT] *= out_std[:OUT]
    return p.astype(np.float32)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dev(t) -> int:
    """Device pointer of a contiguous CUDA tensor."""
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return t.data_ptr()


def gemm_bf16(A, B, C_out=None, accumulate=False, stream=None):
    """C = A B^T (+ C) on the tensor cores: A [M, K], B [N, K] BF16 CUDA
    tensors, C [M, N] FP32."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    if C_out is None:
        C_out = torch.empty((M, N), dtype=torch.float32, device=A.device)
    L = _lib.load()
    st = stream if stream is not None else torch.cuda.current_stream(A.device).cuda_stream
    check(L.avbd_gemm_bf16(_dev(A), A.stride(0), _dev(B), B.stride(0), _dev(C_out), C_out.stride(0), M, N, K,
                           1 if accumulate else 0, st))
    return C_out


class MLP:
    """Fused tensor-core inference of one parameter set."""

    def __init__(self, params: np.ndarray, device: int = 0):
        self.L = _lib.load()
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == NPARAMS
        h = C.c_void_p()
        check(self.L.avbd_mlp_create(C.byref(h), device, _fptr(p)))
        self.h = h

    def forward(self, features, stream=None):
        """features: BF16 CUDA tensor [n, 32] -> FP32 [n, 16]."""
        import torch
        n = features.shape[0]
        out = torch.empty((n, OUT_PAD), dtype=torch.float32, device=features.device)
        st = stream if stream is not None else torch.cuda.current_stream(features.device).cuda_stream
        check(self.L.avbd_mlp_forward(self.h, _dev(features), n, _dev(out), st))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.avbd_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Trainer:
    """Mini-batch Adam training on the tensor cores (MSE over the 3 outputs)."""

    def __init__(self, batch: int, params: np.ndarray, device: int = 0):
        self.L = _lib.load()
        self.batch = batch
        p = np.ascontiguousarray(params, dtype=np.float32)
        h = C.c_void_p()
        check(self.L.avbd_mlp_trainer_create(C.byref(h), device, batch, _fptr(p)))
        self.h = h

    def step(self, X, T, lr: float) -> float:
        loss = C.c_float(0)
        check(self.L.avbd_mlp_trainer_step(self.h, _dev(X), _dev(T), lr, C.byref(loss)))
        return loss.value

    def grad(self, X, T):
        loss = C.c_float(0)
        g = np.zeros(NPARAMS, dtype=np.float32)
        check(self.L.avbd_mlp_trainer_grad(self.h, _dev(X), _dev(T), C.byref(loss), _fptr(g)))
        return loss.value, g

    def params(self) -> np.ndarray:
        p = np.zeros(NPARAMS, dtype=np.float32)
        check(self.L.avbd_mlp_trainer_get_params(self.h, _fptr(p)))
        return p

    def close(self):
        if getattr(self, "h", None):
            self.L.avbd_mlp_trainer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def collect(ctx, steps: int, rows_per_step: int, seed: int = 0):
    """Runs `steps` plain steps of a finalized Context in record mode and
    keeps a random subset of `rows_per_step` solved-vertex rows per step.
    Returns (features BF16 [N, 32], targets FP32 [N, 4]) CUDA tensors."""
    import torch
    dev = torch.device("cuda", ctx.device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    ctx.set_warmstart(1)
    n = ctx.num_particles
    F = torch.empty((n, IN_PAD), dtype=torch.bfloat16, device=dev)
    T = torch.empty((n, 4), dtype=torch.float32, device=dev)
    fs, ts = [], []
    for _ in range(steps):
        ctx.step(1)
        ctx.warmstart_sample(F, T)
        # solved tet vertices whose block residual at the inertial guess is
        # above GATE m g: the rows the applied MLP acts on
        gate = F[:, 12:15].float().abs().sum(1) > GATE
        valid = torch.nonzero((T[:, 3] > 0) & gate).squeeze(1)
        if valid.numel() == 0:
            continue
        k = min(rows_per_step, valid.numel())
        pick = valid[torch.randperm(valid.numel(), generator=g, device=dev)[:k]]
        fs.append(F.index_select(0, pick))
        ts.append(T.index_select(0, pick))
    ctx.set_warmstart(0)
    return torch.cat(fs), torch.cat(ts)


def standardise(F):
    """Per-feature mean and std of raw feature rows (pads: mean 0, std 1)."""
    import torch
    x = F[:, :IN].float()
    mean = x.mean(0).double().cpu().numpy()
    std = x.std(0).double().cpu().numpy()
    std = np.where(std > 1e-6, std, 1.0)
    mean = np.concatenate([mean, np.zeros(IN_PAD - IN)])
    std = np.concatenate([std, np.ones(IN_PAD - IN)])
    return mean, std


def train(F, T, Fv=None, Tv=None, epochs: int = 20, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
          device: int = 0, log=print):
    """Trains on raw features F (BF16 [N, 32]) and targets T (FP32 [N, 4]);
    returns (folded parameters, report)."""
    import torch
    dev = F.device
    mean, std = standardise(F)
    out_std = T[:, :OUT].float().std(0).double().cpu().numpy()
    out_std = np.where(out_std > 1e-9, out_std, 1.0)
    mean_t = torch.tensor(mean, dtype=torch.float32, device=dev)
    std_t = torch.tensor(std, dtype=torch.float32, device=dev)
    Xs = ((F.float() - mean_t) / std_t).to(torch.bfloat16).contiguous()
    Ts = T.clone()
    Ts[:, :OUT] /= torch.tensor(out_std, dtype=torch.float32, device=dev)
    N = Xs.shape[0]
    nb = N // batch
    if nb == 0:
        raise ValueError(f"need at least {batch} samples, got {N}")
    tr = Trainer(batch, init_params(seed), device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    total = epochs * nb
    it = 0
    report = {"samples": N, "epochs": epochs, "batch": batch, "loss": []}
    for ep in range(epochs):
        perm = torch.randperm(N, generator=g, device=dev)
        ep_loss = 0.0
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch]
            xb = Xs.index_select(0, idx)
            tb = Ts.index_select(0, idx)
            cur = lr * 0.5 * (1 + math.cos(math.pi * it / total)) + 1e-5
            ep_loss += tr.step(xb, tb, cur)
            it += 1
        report["loss"].append(ep_loss / nb)
        log(f"epoch {ep + 1}/{epochs}: standardised loss {ep_loss / nb:.4f}")
    params = fold(tr.params(), mean, std, out_std)
    tr.close()
    report["mean"], report["std"], report["out_std"] = mean, std, out_std
    if Fv is not None:
        report.update(evaluate(params, Fv, Tv, device))
    return params, report


def evaluate(params, Fv, Tv, device: int = 0):
    """RMS distance to the converged plain solution of the MLP guess vs the
    inertial guess, in units of g h^2 (targets are (x_end - x0) / (g h^2))."""
    import torch
    m = MLP(params, device)
    pred = m.forward(Fv.contiguous())[:, :OUT]
    m.close()
    t = Tv[:, :OUT]
    rms_plain = float(torch.sqrt((t ** 2).sum(1).mean()))
    rms_mlp = float(torch.sqrt(((t - pred) ** 2).sum(1).mean()))
    # the same distances weighted by (1 + mean_a H_aa h^2 / m)^2: a proxy for
    # the residual each guess leaves (features 18-20 hold log(1 + H_aa h^2/m))
    w = (1.0 + torch.expm1(Fv[:, 18:21].float()).mean(1)) ** 2
    wr_plain = float(torch.sqrt((w * (t ** 2).sum(1)).mean()))
    wr_mlp = float(torch.sqrt((w * ((t - pred) ** 2).sum(1)).mean()))
    return {"val_rows": int(Fv.shape[0]), "rms_inertial_guess": rms_plain, "rms_mlp_guess": rms_mlp,
            "rms_ratio": rms_mlp / max(rms_plain, 1e-30), "rms_weighted_inertial_guess": wr_plain,
            "rms_weighted_mlp_guess": wr_mlp}


def load_params(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    with np.load(path) as d:
        return np.ascontiguousarray(d["params"], dtype=np.float32)


def guess_bound(scene, steps: int, warmup: int = 3, precision: str = "mixed", tol: float = 1e-4,
                max_iters: int = 100, device: int = 0, solution_max_iters: int = None):
    """What any displacement warm start can save, measured: every step runs
    twice from the same start state -- once with the inertial initial guess
    (plain AVBD, at most `solution_max_iters` iterations, default max_iters),
    once with the first run's end positions as the guess
    (avbd_set_initial_guess) and at most max_iters.  Where the first run
    converged, its end positions are the step's solution: the second run
    then measures a perfect predictor of the converged displacement.  Both
    iterate to the same residual tolerance.  Returns per-step arrays of
    per-scene iterations (first run, guessed run)."""
    from .api import Context
    a, b = Context(device=device), Context(device=device)
    for e, mi in ((a, solution_max_iters or max_iters), (b, max_iters)):
        scene.load(e, residual_tolerance=tol, max_iters=max_iters, precision=precision)
        e.finalize()
        e.step(warmup)
        if mi != max_iters:
            e.set_solver(scene.solver_iters, scene.iter_acceleration, tol, mi, precision)
    plain, perfect = [], []
    for _ in range(steps):
        x0, v0 = a.positions(), a.velocities()
        a.step(1)
        plain.append(a.scene_iterations())
        b.set_state(x0, v0)
        b.set_initial_guess(a.positions())
        b.step(1)
        perfect.append(b.scene_iterations())
    a.close()
    b.close()
    return np.array(plain), np.array(perfect)


if __name__ == "__main__":
    # python -m avbd_b200.warmstart [scenes] [steps] [warmup]: the perfect-guess
    # bound on the benchmark batch (seed 0, MIXED, R <= 1e-4, <= 100 iterations)
    import json
    import sys

    from . import scenes as _scenes
    S = int(sys.argv[1]) if len(sys.argv) > 1 else 1024
    K = int(sys.argv[2]) if len(sys.argv) > 2 else 10
    W = int(sys.argv[3]) if len(sys.argv) > 3 else 3
    SOL = int(sys.argv[4]) if len(sys.argv) > 4 else 100
    sc = _scenes.batched_cubes(num_scenes=S, seed=0)
    plain, perfect = guess_bound(sc, K, W, solution_max_iters=SOL)
    verts = np.array([(c + 1) ** 3 for c in sc.meta["cells"]], dtype=np.float64)
    capped_p, capped_g = (plain >= SOL).mean(), (perfect >= 100).mean()
    conv = plain < SOL  # scene-steps whose first run met the tolerance: the guess is their solution
    print(json.dumps({
        "converged_scene_steps": {"fraction": float(conv.mean()), "plain": float(plain[conv].mean()),
                                  "perfect_guess": float(perfect[conv].mean())},
        "capped_scene_steps": {"plain": float(plain[~conv].mean()) if (~conv).any() else None,
                               "perfect_guess": float(perfect[~conv].mean()) if (~conv).any() else None},
        "scenes": S, "steps": K, "warmup": W, "solution_max_iters": SOL,
        "iterations_per_scene_step": {"plain": float(plain.mean()), "perfect_guess": float(perfect.mean())},
        "vertex_weighted_iterations": {"plain": float((plain * verts).sum() / (verts.sum() * K)),
                                       "perfect_guess": float((perfect * verts).sum() / (verts.sum() * K))},
        "capped_fraction": {"plain": float(capped_p), "perfect_guess": float(capped_g)},
        "reduction": float(plain.mean() / max(perfect.mean(), 1e-9)),
    }))
