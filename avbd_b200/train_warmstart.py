"""Trains the learned warm start on trajectories of the plain GPU solver.

    python -m avbd_b200.train_warmstart [--scenes 256] [--steps 100]
        [--samples 2000000] [--epochs 20] [--weighted]
        [--out avbd_b200/data/warmstart_mlp.npz]

Training data: batched uneven NeoHookean cubes (n ~ U{4..24} cells per side,
E log-uniform 1e4..1e7, nu ~ U(0.3, 0.49), random rotation, ground contact)
generated from seed 1000003, a seed set disjoint from the benchmark's
(seed 0 + 7919 * rank); every step runs plain AVBD to R <= 1e-4 in the mixed
precision mode and contributes a random subset of its solved vertices
(features at the inertial guess, target = converged position - guess).
Validation: 64 scenes from seed 2000003, the same way.  The report gives the
MLP's distance to the converged solution against the inertial guess's and
the iterations-to-tolerance of plain vs learned on the validation scenes.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

TRAIN_SEED = 1000003
VAL_SEED = 2000003


def make_context(sc, device, tol, max_iters):
    from avbd_b200 import Context
    e = Context(device=device)
    sc.load(e, residual_tolerance=tol, max_iters=max_iters, precision="mixed")
    e.finalize()
    return e


def iterations_per_step(sc, params, steps, device, tol, max_iters):
    """Scene-iterations per scene-step over `steps` steps: plain, learned with
    the acceptance test (kappa 0.5, the engine's default) and learned
    applied to every vertex the residual gate admits (kappa 0)."""
    out = {}
    for name, p, kappa in (("plain", None, None), ("learned", params, "0.5"), ("learned_ungated", params, "0")):
        e = make_context(sc, device, tol, max_iters)
        if p is not None:
            os.environ["AVBD_WS_KAPPA"] = kappa
            e.set_warmstart(2, p)
            del os.environ["AVBD_WS_KAPPA"]
        e.step(steps)
        st = e.stats()
        out[name] = st["iterations"] / (steps * sc.num_scenes)
        e.close()
    return out


def residual_weights(F):
    """Row weights of the residual-weighted loss: a position error e (in
    units of g h^2) changes the block residual (in units of m g) by about
    (I + H h^2 / m) e, so rows are weighted by (1 + mean_a H_aa h^2 / m)^2
    (features 18-20 hold log(1 + H_aa h^2 / m)), normalised to mean 1."""
    import torch
    lam = torch.expm1(F[:, 18:21].float()).mean(1)
    w = (1.0 + lam) ** 2
    return w / w.mean()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--val-scenes", type=int, default=64)
    ap.add_argument("--val-samples", type=int, default=500_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--max-iters", type=int, default=100)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--weighted", action="store_true",
                    help="residual-weighted loss: rows weighted by (1 + H h^2/m)^2 (see residual_weights)")
    a = ap.parse_args(argv)

    import torch

    from avbd_b200 import scenes, warmstart
    torch.cuda.set_device(a.device)
    out = a.out or warmstart.DEFAULT_WEIGHTS
    t0 = time.time()
    sc = scenes.batched_cubes(num_scenes=a.scenes, seed=TRAIN_SEED)
    e = make_context(sc, a.device, a.tol, a.max_iters)
    F, T = warmstart.collect(e, a.steps, a.samples // a.steps, seed=1)
    e.close()
    sv = scenes.batched_cubes(num_scenes=a.val_scenes, seed=VAL_SEED)
    e = make_context(sv, a.device, a.tol, a.max_iters)
    Fv, Tv = warmstart.collect(e, a.steps, a.val_samples // a.steps, seed=2)
    e.close()
    t_data = time.time() - t0
    print(f"data: {F.shape[0]} training rows, {Fv.shape[0]} validation rows in {t_data:.1f} s", flush=True)
    if a.weighted:
        T[:, 3] = residual_weights(F)
        Tv[:, 3] = residual_weights(Fv)

    t1 = time.time()
    params, rep = warmstart.train(F, T, Fv, Tv, epochs=a.epochs, batch=a.batch, lr=a.lr, device=a.device)
    t_train = time.time() - t1
    print(f"trained in {t_train:.1f} s: validation RMS distance to the converged solution "
          f"{rep['rms_mlp_guess']:.4f} (MLP guess) vs {rep['rms_inertial_guess']:.4f} (inertial guess), "
          f"ratio {rep['rms_ratio']:.3f}", flush=True)
    its = iterations_per_step(sv, params, 30, a.device, a.tol, a.max_iters)
    print(f"validation scenes, 30 steps: {its['plain']:.2f} plain vs {its['learned']:.2f} learned "
          "iterations per scene-step", flush=True)

    report = {"train_seed": TRAIN_SEED, "val_seed": VAL_SEED, "train_scenes": a.scenes, "val_scenes": a.val_scenes,
              "steps": a.steps, "train_rows": int(F.shape[0]), "val_rows": int(Fv.shape[0]), "epochs": a.epochs,
              "batch": a.batch, "lr": a.lr, "loss_per_epoch": rep["loss"],
              "rms_inertial_guess": rep["rms_inertial_guess"], "rms_mlp_guess": rep["rms_mlp_guess"],
              "rms_ratio": rep["rms_ratio"], "iterations_per_scene_step": its, "data_s": round(t_data, 1),
              "train_s": round(t_train, 1), "residual_tolerance": a.tol, "max_iters": a.max_iters,
              "loss": "residual-weighted" if a.weighted else "unweighted",
              "rms_weighted_mlp_guess": rep.get("rms_weighted_mlp_guess"),
              "rms_weighted_inertial_guess": rep.get("rms_weighted_inertial_guess")}
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.savez(out, params=params, mean=rep["mean"], std=rep["std"], out_std=rep["out_std"],
             report=json.dumps(report))
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()
