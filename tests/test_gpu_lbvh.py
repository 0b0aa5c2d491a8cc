"""LBVH of the engine vs the oracle on identical FP64 inputs: Morton codes,
sorted order, tree topology, node bounds and candidate pairs are compared bit
for bit (LBVHBuilder / LBVHTraversal, collision/*)."""
import numpy as np
import pytest

from avbd_b200 import Context, scenes

pytestmark = pytest.mark.gpu


def _both(oracle_lib, sc, precision, X, V):
    e = Context()
    sc.load(e, precision=precision)
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    e.set_positions(0, X)
    e.set_velocities(0, V)
    o.set_positions_raw(0, X)
    o.set_velocities(0, V)
    e.collision_stage()
    o.collision_stage()
    return e.lbvh(), o.lbvh(sc.num_primitives)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [3, 8, 16])
def test_lbvh_bit_exact(oracle_lib, precision, n):
    sc = scenes.cube_drop(n=n, surface=True)
    rng = np.random.default_rng(n)
    o0 = oracle_lib.Oracle()
    sc.load(o0)
    X = o0.positions() + rng.uniform(-0.01, 0.01, size=(sc.num_particles, 3))
    V = rng.normal(0, 1.0, size=(sc.num_particles, 3))
    if precision == "fp32":  # the FP32 engine stores positions as floats
        X = X.astype(np.float32).astype(np.float64)
        V = V.astype(np.float32).astype(np.float64)
    ge, go = _both(oracle_lib, sc, precision, X, V)
    for k in ("morton", "sorted_order", "left", "right", "parent", "subtree_size"):
        assert (ge[k] == go[k]).all(), k
    assert ge["root"] == go["root"]
    assert (ge["bounds"] == go["bounds"]).all()
    assert ge["pairs"].shape == go["pairs"].shape
    assert (ge["pairs"] == go["pairs"]).all()
    assert len(ge["pairs"]) > 0


def test_lbvh_runs_every_step_and_counts_pairs(oracle_lib):
    sc = scenes.cube_drop(n=8, surface=True)
    e = Context()
    sc.load(e)
    e.finalize()
    e.step(3)
    st = e.stats()
    assert st["candidate_pairs"] > 0
