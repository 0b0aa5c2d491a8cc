"""Parity of the dynamic triangle-rigid contacts with the FP64 oracle: the
merge of the narrow phase's detections into the contact pool
(CollisionDetector::_handleDetectedCollisions, collision/CollisionDetector.cpp:
265-482), the incremental recoloring (ColorList.hpp:381-522), the contact
energies in the vertex blocks (TriangleRigidCollisionEnergySolver.hpp:14-118,
CollisionConstraintEnergySolver.hpp:60-285) and the conflict buffering
(VBDSolver.hpp:82-87,108-119,474-509).

Scene: four rigid spheres dropped on a soft 4^3-cell tet cube with a fixed
base.  In FP64 the pool (slots, particles), the colors and the conflicts are
compared exactly every step, positions within 1e-8 of the bounding-box
diagonal; with no recoloring rounds the conflict path runs every step."""
import numpy as np
import pytest

from avbd_b200 import Context, scenes

pytestmark = pytest.mark.gpu

N_CUBE = 125


def pair(oracle_lib, precision="fp64", rounds=None, tol=0.0, max_iters=0):
    sc = scenes.spheres_on_cube(n=4, num_spheres=4, seed=0)
    e = Context()
    sc.load(e, precision=precision, residual_tolerance=tol, max_iters=max_iters)
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o, residual_tolerance=tol, max_iters=max_iters)
    o.finalize()
    if rounds is not None:
        e.set_recolor_rounds(rounds)
        o.set_recolor_rounds(rounds)
    return sc, e, o


def quat_err(a, b):
    s = np.sign(np.sum(a * b, axis=1, keepdims=True))
    s[s == 0] = 1
    return np.abs(a - s * b).max()


@pytest.mark.parametrize("rounds", [None, 0])
def test_contacts_track_oracle_fp64(oracle_lib, rounds):
    sc, e, o = pair(oracle_lib, "fp64", rounds)
    d = sc.bbox_diagonal()
    conflicts = 0
    for step in range(60):
        e.step(1)
        o.step(1)
        ie, io = e.dynamic_info(), o.dynamic_info()
        assert ie == io, (step, ie, io)
        conflicts += ie["conflicted"]
        ce, nce = e.coloring()
        co, nco = o.coloring()
        assert nce == nco and (ce == co).all(), step
        ex = np.abs(e.positions() - o.positions()).max() / d
        assert ex < 1e-8, (step, ex)
    assert quat_err(e.rotations(), o.rotations()) < 1e-7
    pe, po = e.contact_pool(), o.contact_pool()
    assert (pe["active"] == po["active"]).all()
    act = po["active"]
    assert act.any()
    assert (pe["particles"][act] == po["particles"][act]).all()
    for key in ("n", "t", "b", "barys", "cp_local"):
        np.testing.assert_allclose(pe[key][act], po[key][act], rtol=0, atol=1e-7, err_msg=key)
    np.testing.assert_allclose(pe["k"][act], po["k"][act], rtol=1e-6)
    lam_scale = np.abs(po["lam"][act][:, :3]).max() + 1e-12
    assert np.abs(pe["lam"][act][:, :3] - po["lam"][act][:, :3]).max() <= 1e-6 * lam_scale
    assert (pe["flags"][act] == po["flags"][act]).all()
    if rounds == 0:
        assert conflicts > 0


def test_contact_blocks_and_residual_match_oracle(oracle_lib):
    """avbd_debug_block of a sphere and of triangle vertices in contact, and
    the residual, after 12 steps of both."""
    sc, e, o = pair(oracle_lib, "fp64")
    e.step(12)
    o.step(12)
    pool = o.contact_pool()
    act = np.nonzero(pool["active"])[0]
    assert len(act)
    parts = sorted({int(v) for s in act for v in pool["particles"][s]})
    for p in parts[:6] + parts[-2:]:
        Ge, He = e.debug_block(p)
        Go, Ho = o.debug_block(p)
        scale_h = np.abs(Ho).max()
        scale_g = max(np.abs(Go).max(), scale_h * 1e-3)
        assert np.abs(Ge - Go).max() <= 1e-6 * scale_g, (p, Ge, Go)
        assert np.abs(He - Ho).max() <= 1e-6 * scale_h, (p, He, Ho)
    re, ro = e.residual(), o.residual()
    assert abs(re - ro) <= 1e-6 * ro, (re, ro)


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_contacts_lower_precision_track_oracle(oracle_lib, precision):
    """MIXED and FP32 runs against the FP64 oracle over 60 steps.  A
    detection within rounding of the collision margin, or a friction
    stick/slip switch, moves with any rounding of the state, so the bar is
    the oracle's own sensitivity: a second oracle started from the positions
    rounded to FP32.  The engine stays within 3x that drift plus 1e-5 of the
    diagonal (MIXED) or 1e-4 (FP32, whose own arithmetic moves the iterates
    more than a rounding of the inputs: 2e-5 after 20 steps) at every
    checkpoint, forms contacts, and its live-contact count stays within 2 of
    the oracle's."""
    sc, e, o = pair(oracle_lib, precision)
    o32 = oracle_lib.Oracle()
    sc.load(o32)
    o32.finalize()
    o32.set_positions_raw(0, o32.positions().astype(np.float32).astype(np.float64))
    diag = sc.bbox_diagonal()
    live = 0
    seen = []
    for _ in range(6):
        e.step(10)
        o.step(10)
        o32.step(10)
        X = o.positions()
        err = np.abs(e.positions() - X).max() / diag
        sens = np.abs(o32.positions() - X).max() / diag
        seen.append((round(err, 7), round(sens, 7)))
        assert err <= (1e-4 if precision == "fp32" else 1e-5) + 3 * sens, (precision, seen)
        live = max(live, e.dynamic_info()["live"])
        assert abs(e.dynamic_info()["live"] - o.dynamic_info()["live"]) <= 2
    assert live > 0
    print(precision, "error vs oracle sensitivity per 10 steps:", seen)


def test_contacts_run_to_tolerance(oracle_lib):
    """Per-scene run-to-tolerance with contacts: iteration counts and states
    follow the oracle."""
    sc, e, o = pair(oracle_lib, "fp64", tol=1e-3, max_iters=200)
    for step in range(20):
        i0e, i0o = e.stats()["iterations"], o.iterations
        e.step(1)
        o.step(1)
        # each step's iterations within 2 of the oracle's
        de, do = e.stats()["iterations"] - i0e, o.iterations - i0o
        assert abs(de - do) <= 2, (step, de, do)
    assert np.abs(e.positions() - o.positions()).max() / sc.bbox_diagonal() < 1e-6
