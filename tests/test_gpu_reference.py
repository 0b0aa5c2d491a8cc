"""The engine against the reference implementation itself.

tests/golden/reference_outputs.npz holds outputs of the reference's own
sources (compiled against the Eigen-API shim into oracle/_ref by
oracle/Makefile; tests/golden/make_reference_golden.py wrote the fixture).
Here the CUDA engine runs the same scenes through the C-ABI:

* colors, Morton codes, sorted order, LBVH topology, node bounds and
  candidate pairs of the step-1 collision stage are identical (FP64 inputs);
* positions stay within the stated fraction of the bounding-box diagonal of
  the reference's: 1e-9 for the FP64 engine, 1e-6 for MIXED (FP32 element
  records), 1e-5 for FP32 on the C1 cube (no contact);
* contact pools (slots, particles) are identical and their multipliers agree
  to 1e-6 relative.
"""
import hashlib
import os

import numpy as np
import pytest

from avbd_b200 import Context

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.npz")
LBVH_KEYS = ("morton", "sorted_order", "left", "right", "parent", "subtree_size")


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_reference_golden", os.path.join(os.path.dirname(GOLD), "make_reference_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.cases()


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def cases():
    return _cases()


def quat_err(a, b):
    s = np.sign(np.sum(a * b, axis=1, keepdims=True))
    s[s == 0] = 1
    return np.abs(a - s * b).max()


def _engine(sc, precision):
    e = Context()
    sc.load(e, precision=precision)
    e.finalize()
    return e


def _trajectory(name, precision, tol, gold, cases):
    sc, plan = cases[name]
    e = _engine(sc, precision)
    colors, nc = e.coloring()
    assert nc == int(gold[f"{name}/num_colors"][0])
    assert (colors == gold[f"{name}/colors"]).all(), "colors differ from the reference"
    diag = sc.bbox_diagonal()
    done = 0
    worst = 0.0
    for step in sorted(plan):
        e.step(step - done)
        done = step
        key = f"{name}/s{step}"
        X = e.positions()
        for what, sub in (("pos", X), ("pos16", X[::16]), ("pos8", X[::8])):
            if what in plan[step]:
                err = np.abs(sub - gold[f"{key}/{what}"]).max() / diag
                worst = max(worst, err)
                assert err <= tol, f"{key} ({precision}): positions {err:.2e} of the diagonal from the reference"
        if "rot" in plan[step]:
            err = quat_err(e.rotations(), gold[f"{key}/rot"])
            assert err <= 10 * tol, f"{key} ({precision}): rotations {err:.2e} from the reference"
        for pool, getter in (("trc", e.contact_pool), ("trd", e.rod_contact_pool)):
            if pool in plan[step] and precision == "fp64":
                p = getter()
                g_act = gold[f"{key}/{pool}_active"]
                n = len(p["active"])
                assert n == len(g_act) or (n == 0 and not g_act.any())
                assert (p["active"] == g_act[:n]).all(), f"{key}: live slots differ from the reference"
                live = p["active"]
                assert (p["particles"][live] == gold[f"{key}/{pool}_particles"][:n][live]).all()
                for f in ("k", "lam"):
                    a, b = p[f][live], gold[f"{key}/{pool}_{f}"][:n][live]
                    assert np.abs(a - b).max(initial=0) <= 1e-6 * max(1.0, np.abs(b).max(initial=0)), f
    e.close()
    return worst


@pytest.mark.parametrize("name", ["c1", "drop8", "rods", "sph", "rodcube", "c4_0", "c4_1", "c4_7", "c2"])
def test_fp64_engine_tracks_reference(gold, cases, name):
    _trajectory(name, "fp64", 1e-9, gold, cases)


@pytest.mark.parametrize("name", ["c1", "rods", "c4_0", "c4_1", "c4_7", "c2"])
def test_mixed_engine_tracks_reference(gold, cases, name):
    _trajectory(name, "mixed", 1e-6, gold, cases)


def test_fp32_engine_tracks_reference_c1(gold, cases):
    _trajectory("c1", "fp32", 1e-5, gold, cases)


@pytest.mark.parametrize("name,precision", [("drop8", "fp64"), ("c2", "fp64"), ("drop8", "mixed"),
                                            ("c2", "mixed")])
def test_lbvh_identical_to_reference(gold, cases, name, precision):
    """The collision stage of step 1 (the scene's initial positions and
    velocities): 384 and 12,288 surface triangles; the larger takes the
    reference's parallel refit path."""
    sc, plan = cases[name]
    e = _engine(sc, precision)
    e.collision_stage()
    t = e.lbvh()
    key = f"{name}/s1"
    for k in LBVH_KEYS:
        assert (t[k] == gold[f"{key}/{k}"]).all(), f"{key}: {k} differs from the reference"
    assert t["root"] == int(gold[f"{key}/root"][0])
    if f"{key}/bounds" in gold.files:
        assert (t["bounds"] == gold[f"{key}/bounds"]).all()
    else:
        digest = np.frombuffer(hashlib.sha256(t["bounds"].tobytes()).digest(), np.uint8)
        assert (digest == gold[f"{key}/bounds_sha256"]).all(), f"{key}: node bounds differ"
    assert np.array_equal(t["pairs"], gold[f"{key}/pairs"]), f"{key}: candidate pairs differ"
    e.close()
