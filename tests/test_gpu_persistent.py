"""Persistent sweep (the default; AVBD_PERSISTENT=0 in the environment at
context creation turns it off): each run-to-tolerance sweep is one
cooperative launch whose blocks draw a color's pieces from a shared ticket
counter and meet at a grid barrier before the next color, instead of one
launch per color.

Vertices of one color never read each other, and every vertex is solved by
the same per-vertex code with the same lane count, so the positions match
the per-color launches (up to the order of the FP64 atomic sums of the
per-scene residuals, which can only move a stop decision that sits on the
tolerance).  The barrier's waits are bounded: with a wait limit of 0 every
block but the last to arrive gives up, the step returns
AVBD_ERR_BARRIER_TIMEOUT, and the context steps normally afterwards.
"""
import numpy as np
import pytest

from avbd_b200 import Context, _lib, scenes
from avbd_b200._lib import AvbdError

pytestmark = pytest.mark.gpu

ERR_TIMEOUT = 6


def _ctx(monkeypatch, persistent: bool, sc, precision="mixed"):
    monkeypatch.setenv("AVBD_PERSISTENT", "1" if persistent else "0")
    monkeypatch.setenv("AVBD_LANES", "2")  # the persistent sweep runs 2 threads per vertex
    e = Context()
    sc.load(e, residual_tolerance=1e-4, max_iters=100, precision=precision)
    e.finalize()
    return e


@pytest.mark.parametrize("precision", ["mixed", "fp64", "fp32"])
def test_persistent_sweep_matches_per_color_launches(monkeypatch, precision):
    sc = scenes.batched_cubes(num_scenes=1024, seed=0, scene_ids=range(12))
    a = _ctx(monkeypatch, False, sc, precision)
    b = _ctx(monkeypatch, True, sc, precision)
    diag = sc.bbox_diagonal()
    for step in range(4):
        la, lb = a.stats()["kernel_launches"], b.stats()["kernel_launches"]
        a.step(1)
        b.step(1)
        ia, ib = a.scene_iterations(), b.scene_iterations()
        assert (ia == ib).all(), (step, ia, ib)
        err = np.abs(a.positions() - b.positions()).max() / diag
        assert err <= 1e-12, (step, err)
        # one sweep launch per iteration instead of one per color
        da, db = a.stats()["kernel_launches"] - la, b.stats()["kernel_launches"] - lb
        assert db < da, (da, db)
    a.close()
    b.close()


def test_persistent_sweep_barrier_timeout_is_reported(monkeypatch):
    sc = scenes.batched_cubes(num_scenes=1024, seed=0, scene_ids=range(12))
    e = _ctx(monkeypatch, True, sc)
    e.step(1)
    x0, v0 = e.positions(), e.velocities()
    L = _lib.load()
    try:
        assert L.avbd_debug_set_wait_limit(0, 0) == 0
        with pytest.raises(AvbdError) as ex:
            e.step(1)
            e.synchronize()
        assert ex.value.code == ERR_TIMEOUT
    finally:
        assert L.avbd_debug_set_wait_limit(0, _lib.DEFAULT_WAIT_POLLS) == 0
    # the context is still usable: from the saved positions and velocities it
    # steps again without error (the contact multipliers and stiffnesses the
    # abandoned step left differ, so the result is not compared)
    e.set_state(x0, v0)
    e.step(2)
    e.synchronize()
    assert np.isfinite(e.positions()).all()
    assert (e.scene_iterations() <= 100).all()
    e.close()
