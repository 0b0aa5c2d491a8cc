"""Parity of the triangle-rod contacts with the FP64 oracle: the
closest-point narrow phase (CollisionDetector::_triangleRod,
collision/CollisionDetector.cpp:601-666), the triangle-rod pool next to the
triangle-rigid one, the 3-DOF and 6-DOF contact blocks
(TriangleRodCollisionEnergySolver.hpp:14-149) and the recoloring with
five-particle contacts.

Scene: three 8-segment Cosserat rods (radius 1 cm) dropped flat on a 4^3-cell
tet cube with a fixed base.  FP64: pool slots, particles, flags, colors and
conflict counts exact every step, positions within 1e-8 of the bounding-box
diagonal; with one recoloring round the conflict path runs on rod nodes."""
import numpy as np
import pytest

from avbd_b200 import Context, scenes

pytestmark = pytest.mark.gpu

N_CUBE = 125


def pair(oracle_lib, precision="fp64", rounds=None):
    sc = scenes.rods_on_cube()
    e = Context()
    sc.load(e, precision=precision)
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    if rounds is not None:
        e.set_recolor_rounds(rounds)
        o.set_recolor_rounds(rounds)
    return sc, e, o


def quat_err(a, b):
    s = np.sign(np.sum(a * b, axis=1, keepdims=True))
    s[s == 0] = 1
    return np.abs(a - s * b).max()


@pytest.mark.parametrize("rounds", [None, 1])
def test_rod_contacts_track_oracle_fp64(oracle_lib, rounds):
    sc, e, o = pair(oracle_lib, "fp64", rounds)
    d = sc.bbox_diagonal()
    conflicts = live = 0
    for step in range(60):
        e.step(1)
        o.step(1)
        ie, io = e.dynamic_info(), o.dynamic_info()
        assert ie == io, (step, ie, io)
        conflicts += ie["conflicted"]
        live = max(live, ie["rod_live"])
        ce, nce = e.coloring()
        co, nco = o.coloring()
        assert nce == nco and (ce == co).all(), step
        ex = np.abs(e.positions() - o.positions()).max() / d
        assert ex < 1e-8, (step, ex)
    assert live > 0
    assert quat_err(e.rotations()[N_CUBE:], o.rotations()[N_CUBE:]) < 1e-7
    pe, po = e.rod_contact_pool(), o.rod_contact_pool()
    assert (pe["active"] == po["active"]).all()
    act = po["active"]
    if act.any():
        assert (pe["particles"][act] == po["particles"][act]).all()
        for key in ("n", "t", "b", "barys", "cp_local", "s"):
            np.testing.assert_allclose(pe[key][act], po[key][act], rtol=0, atol=1e-7, err_msg=key)
        np.testing.assert_allclose(pe["k"][act], po["k"][act], rtol=1e-6)
        assert (pe["flags"][act] == po["flags"][act]).all()
    if rounds == 1:
        assert conflicts > 0


def test_rod_detections_match_oracle_from_the_same_state(oracle_lib):
    """The engine's state is copied into the oracle before each detection:
    keys, triangles and rod nodes exact, s / barycentrics / normal exact to
    1e-12, the rod-frame point to 1e-9 (it uses the interpolated rotation:
    device vs host sin/cos)."""
    sc, e, o = pair(oracle_lib, "fp64")
    found = 0
    for step in range(30):
        e.step(1)
        o.set_positions_raw(0, e.positions())
        o.set_velocities(0, e.velocities())
        o.set_rotations_raw(N_CUBE, e.rotations()[N_CUBE:])
        o.set_angular_velocities(N_CUBE, e.angular_velocities()[N_CUBE:])
        e.collision_stage()
        o.collision_stage()
        ce, co = e.rod_contacts(), o.rod_contacts()
        assert (ce["key"] == co["key"]).all(), step
        assert (ce["tri"] == co["tri"]).all() and (ce["rod"] == co["rod"]).all()
        for k in ("normal", "barys", "s"):
            assert np.abs(ce[k] - co[k]).max(initial=0) <= 1e-12, (step, k)
        assert np.abs(ce["cp_local"] - co["cp_local"]).max(initial=0) <= 1e-9
        found += len(co["key"])
    assert found > 0


def test_rod_contact_blocks_match_oracle(oracle_lib):
    """avbd_debug_block of rod nodes and triangle vertices in contact after 8
    steps of both."""
    sc, e, o = pair(oracle_lib, "fp64")
    e.step(8)
    o.step(8)
    pool = o.rod_contact_pool()
    act = np.nonzero(pool["active"])[0]
    assert len(act)
    parts = sorted({int(v) for s in act for v in pool["particles"][s]})
    rods = [p for p in parts if p >= N_CUBE]
    tris = [p for p in parts if p < N_CUBE]
    for p in tris[:4] + rods[:6]:
        Ge, He = e.debug_block(p)
        Go, Ho = o.debug_block(p)
        scale_h = np.abs(Ho).max()
        scale_g = max(np.abs(Go).max(), scale_h * 1e-3)
        assert np.abs(Ge - Go).max() <= 1e-6 * scale_g, (p, Ge, Go)
        assert np.abs(He - Ho).max() <= 1e-6 * scale_h, (p, He, Ho)
    re, ro = e.residual(), o.residual()
    assert abs(re - ro) <= 1e-6 * ro, (re, ro)


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_rod_contacts_lower_precision(oracle_lib, precision):
    """MIXED and FP32 rod contacts against the FP64 oracle over 60 steps,
    with the live-contact count within 2 of the oracle's (FP32: while its
    trajectory tracks the oracle's, up to step 20; once it has moved away
    an FP32 run measured 18 live contacts against the oracle's 12).  MIXED is held to
    1e-5 of the diagonal plus 3x the oracle's own drift when its positions
    are rounded to FP32 (measured 2e-7 after 60 steps).  FP32 is held to
    1e-4 plus that drift up to step 20 (measured 4e-6 after 10 steps, 1.6e-5
    after 20); once the rods hit the cube (steps 25-30) FP32 arithmetic in
    the contact and rod blocks moves the trajectory: 1.1e-3 after 30 steps,
    2.6e-3 after 40, 2.1e-2 after 50, 2.3e-2 after 60, the same to 3 digits
    with every 6x6 block re-solved in FP64 (AVBD_KAPPA_MAX=0), so the FP32
    LDL^T is not the cause.  From step 30 on FP32 is held to 5e-2."""
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
        step = 10 * len(seen)
        bar = 1e-5 if precision == "mixed" else (1e-4 if step <= 20 else 5e-2)
        assert err <= bar + 3 * sens, (precision, seen)
        live = max(live, e.dynamic_info()["rod_live"])
        if precision == "mixed" or step <= 20:
            assert abs(e.dynamic_info()["rod_live"] - o.dynamic_info()["rod_live"]) <= 2
    assert live > 0
    print(precision, "error vs oracle sensitivity per 10 steps:", seen)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_recorded_iteration_matches_launch_by_launch(monkeypatch, precision):
    """A fixed-iteration step with dynamic contacts records one iteration
    after its host contact management and replays it; with AVBD_GRAPH=0 the
    same kernels are launched one by one.  Both take the same steps: pools,
    colors and positions identical over 40 steps (with one recoloring round,
    so the conflict commits are in the recorded iteration too)."""
    sc = scenes.rods_on_cube()
    runs = []
    for graph in ("1", "0"):
        monkeypatch.setenv("AVBD_GRAPH", graph)
        e = Context()
        sc.load(e, precision=precision)
        e.finalize()
        e.set_recolor_rounds(1)
        runs.append(e)
    a, b = runs
    for step in range(40):
        a.step(1)
        b.step(1)
        assert a.dynamic_info() == b.dynamic_info(), step
        assert (a.coloring()[0] == b.coloring()[0]).all(), step
        assert np.array_equal(a.positions(), b.positions()), step
    assert np.array_equal(a.rotations(), b.rotations())
    assert a.dynamic_info()["rod_live"] > 0
    a.close()
    b.close()


def test_recoloring_barrier_timeout_is_reported():
    """The recoloring's rounds run as one cooperative launch whose phases
    meet at bounded grid barriers.  With a wait limit of 0 every block but
    the last to arrive gives up: the step returns AVBD_ERR_BARRIER_TIMEOUT
    before any list it would have built is used, and with the limit restored
    the context steps again."""
    from avbd_b200 import _lib
    from avbd_b200._lib import AvbdError
    sc = scenes.rods_on_cube()
    e = Context()
    sc.load(e, precision="fp32")
    e.finalize()
    e.step(2)
    L = _lib.load()
    try:
        assert L.avbd_debug_set_wait_limit(0, 0) == 0
        with pytest.raises(AvbdError) as ex:
            e.step(1)
            e.synchronize()
        assert ex.value.code == 6  # AVBD_ERR_BARRIER_TIMEOUT
    finally:
        assert L.avbd_debug_set_wait_limit(0, _lib.DEFAULT_WAIT_POLLS) == 0
    e.step(3)
    e.synchronize()
    assert np.isfinite(e.positions()).all()
    e.close()
