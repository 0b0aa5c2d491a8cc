"""Narrow phase on the GPU vs the FP64 oracle: two spheres hit the top of a
coarse tet cube at 2-4 m/s (one step moves them 3-7 cm); their contact
energies throw one far off and let the other through to the ground.  Such
impacts amplify rounding differences between two solvers, so the engine's
state (positions, velocities, rotations, angular velocities) is copied into
the oracle before every detection.  From the same state the LBVH with sphere
primitives (rotated-box bounds, CollisionPrimitivePool.hpp:199-231) is
bit-exact, and the triangle-sphere detections
(CollisionDetector::_triangleSDF_CCD) match: same keys, triangles and spheres,
vectors to 1e-12 while the spheres do not spin and to 1e-9 once they roll
(device and host sin/cos may differ in the last bit)."""
import numpy as np
import pytest

from avbd_b200 import Context, scenes

pytestmark = pytest.mark.gpu


def scene(n=4, seed=3):
    """Two spheres over opposite corners of the cube's top face, moving apart
    (sphere-sphere candidates stop the reference)."""
    sc = scenes.cube_drop(n=n, iters=10, height=0.05, surface=True)
    rng = np.random.default_rng(seed)
    first = sc.num_particles
    for k, (gx, gz) in enumerate([(0.25, 0.25), (0.75, 0.75)]):
        r = rng.uniform(0.06, 0.1)
        p = (gx + rng.uniform(-0.05, 0.05), 1.05 + r + rng.uniform(0.0, 0.1), gz + rng.uniform(-0.05, 0.05))
        b = scenes.add_sphere(sc, r, 500.0, p)
        out = np.array([gx - 0.5, 0.0, gz - 0.5]) * 2.0
        v = np.array([[out[0], rng.uniform(-4, -2), out[2]]])
        sc.record("set_velocities", b, v, v)
        sc.record("add_spheres", [b], [r], [10 + k])
        sc.num_primitives += 1
    sc.meta["spheres"] = list(range(first, sc.num_particles))
    sc.meta["bbox_diagonal"] = 2.0
    return sc


def compare(ce, co, tol):
    assert (ce["key"] == co["key"]).all()
    assert (ce["tri"] == co["tri"]).all() and (ce["rigid"] == co["rigid"]).all()
    for k in ("normal", "barys", "cp_local"):
        assert np.abs(ce[k] - co[k]).max(initial=0) <= tol, k


def test_narrow_phase_matches_oracle(oracle_lib):
    sc = scene()
    e = Context()
    sc.load(e, precision="fp64")
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    found, spinning = 0, False
    sph = sc.meta["spheres"]
    for step in range(40):
        e.step(1)
        o.set_positions_raw(0, e.positions())
        o.set_velocities(0, e.velocities())
        o.set_rotations_raw(sph[0], e.rotations()[sph[0]:])
        o.set_angular_velocities(sph[0], e.angular_velocities()[sph[0]:])
        e.collision_stage()
        o.collision_stage()
        w = o.angular_velocities()[sc.meta["spheres"]]
        spinning = spinning or np.abs(w).max() > 0
        ce, co = e.contacts(), o.contacts()
        compare(ce, co, 1e-9 if spinning else 1e-12)
        found += len(co["key"])
        ge, go = e.lbvh(), o.lbvh(sc.num_primitives)
        if not spinning:
            for k in ("morton", "sorted_order", "left", "right", "parent"):
                assert (ge[k] == go[k]).all(), (step, k)
            assert (ge["pairs"] == go["pairs"]).all()
    assert found > 0  # the spheres crossed the cube's top surface


def test_sphere_pairs_other_than_triangle_are_rejected(oracle_lib):
    """Sphere-sphere candidates throw in the reference (CollisionDetector.cpp:678-687):
    the engine reports AVBD_ERR_UNSUPPORTED_PAIR at the next synchronising call."""
    from avbd_b200._lib import AvbdError
    sc = scenes.Scene(name="two_spheres", dt=1 / 60)
    for k, x in enumerate((0.0, 0.15)):
        b = scenes.add_sphere(sc, 0.1, 500.0, (x, 0.5, 0.0))
        sc.record("add_spheres", [b], [0.1], [k])
        sc.num_primitives += 1
    e = Context()
    sc.load(e, precision="fp64")
    e.finalize()
    with pytest.raises(AvbdError) as ex:
        e.collision_stage()
        e.synchronize()
        e.contacts()
    assert ex.value.code == 4
