"""The caller-supplied initial guess (avbd_set_initial_guess) and the bound
it gives on any displacement warm start: a step started from its own
converged positions (a perfect predictor of the converged displacement)
still runs plain AVBD iterations to the same tolerance."""
import numpy as np
import pytest

from avbd_b200 import Context, scenes, warmstart

pytestmark = pytest.mark.gpu


def test_initial_guess_converges_to_the_same_step():
    sc = scenes.batched_cubes(num_scenes=6, seed=4, n_min=4, n_max=10)
    a, b = Context(), Context()
    for e in (a, b):
        sc.load(e, residual_tolerance=1e-4, max_iters=200, precision="mixed")
        e.finalize()
        e.step(3)
    x0, v0 = a.positions(), a.velocities()
    a.step(1)
    xa, ia = a.positions(), a.scene_iterations()
    b.set_state(x0, v0)
    b.set_initial_guess(xa)
    b.step(1)
    xb, ib = b.positions(), b.scene_iterations()
    # a scene that converged from the inertial guess converges from its own
    # end state in no more iterations, to the same state within the tolerance's scale
    conv = ia < 200
    assert conv.any()
    assert (ib[conv] <= ia[conv]).all(), (ia, ib)
    assert np.abs(xa - xb).max() / sc.bbox_diagonal() < 1e-3
    # the next step starts from the inertial guess again and converges as usual
    b.step(1)
    assert b.stats()["last_residual"] <= 1e-4 or b.stats()["capped_scene_steps"] > 0


def test_perfect_guess_bound_on_batch_sample():
    """On 16 scenes of the benchmark batch: the perfect-guess iterations are
    reported next to plain ones and never exceed them in total."""
    sc = scenes.batched_cubes(num_scenes=1024, seed=0, scene_ids=range(16))
    plain, perfect = warmstart.guess_bound(sc, steps=4, warmup=3)
    assert plain.shape == perfect.shape == (4, 16)
    assert perfect.sum() <= plain.sum()
    print("iterations per scene-step: plain %.1f, perfect guess %.1f" % (plain.mean(), perfect.mean()))
