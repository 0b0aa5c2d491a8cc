"""What the trained warm-start network gains over plain AVBD, on held-out
scenes.

The committed network (avbd_b200/data/warmstart_mlp.npz) was trained on
trajectories of the plain GPU solver over scenes of seed 1000003; the scenes
here are the first 16 of its validation seed 2000003 (the benchmark's batch
is seed 0), run in the mixed precision mode to R <= 1e-4 with at most 100
iterations, as the benchmark runs.

* The network's guess of each solved vertex's converged displacement is
  closer to the converged plain solution than the inertial guess: the RMS
  distance (in units of g h^2, over the vertices whose block residual at
  the inertial guess passes the engine's gate) is about half of the
  inertial guess's (0.48 on the 64 validation scenes after training;
  measured here on a B200: 1.27 against 2.51, ratio 0.50).
* That does not buy iterations to the tolerance: with the engine's
  acceptance test a correction is applied only where it is predicted to
  lower the block residual, and the learned run then takes the plain run's
  iterations (within one per scene-step); applied to every vertex the gate
  admits, the network's residual error costs iterations instead (measured
  over 30 steps: plain 77.08, learned 77.08, ungated 86.67 iterations per
  scene-step).  Every
  scene still ends each step at the tolerance or at the iteration cap.
"""
import numpy as np
import pytest

from avbd_b200 import Context, scenes, warmstart
from avbd_b200.train_warmstart import VAL_SEED, iterations_per_step

pytestmark = pytest.mark.gpu

SCENES = range(16)


@pytest.fixture(scope="module")
def held_out():
    return scenes.batched_cubes(num_scenes=64, seed=VAL_SEED, scene_ids=SCENES)


@pytest.fixture(scope="module")
def params():
    return warmstart.load_params()


def test_trained_guess_is_closer_to_the_converged_state(held_out, params):
    e = Context()
    held_out.load(e, residual_tolerance=1e-4, max_iters=100, precision="mixed")
    e.finalize()
    # the cubes start 0.3 m above the ground: in free flight the inertial
    # guess is exact and the gate admits no vertex, so sample after landing
    e.step(20)
    F, T = warmstart.collect(e, steps=10, rows_per_step=50_000, seed=3)
    e.close()
    rep = warmstart.evaluate(params, F, T)
    print("held-out guess distances:", rep)
    assert rep["val_rows"] >= 10_000, rep
    assert rep["rms_ratio"] < 0.8, rep


def test_trained_network_keeps_plain_iterations(held_out, params):
    its = iterations_per_step(held_out, params, 30, 0, 1e-4, 100)
    print("held-out iterations per scene-step:", its)
    assert its["learned"] <= its["plain"] + 1.0, its
    assert its["learned_ungated"] >= its["learned"] - 1.0, its
    # the learned context's steps end at the tolerance or at the cap
    e = Context()
    held_out.load(e, residual_tolerance=1e-4, max_iters=100, precision="mixed")
    e.finalize()
    e.set_warmstart(2, params)
    for _ in range(25):
        cap0 = e.stats()["capped_scene_steps"]
        e.step(1)
        st = e.stats()
        assert st["last_residual"] <= 1e-4 or st["capped_scene_steps"] > cap0
    assert np.isfinite(e.positions()).all()
    e.close()
