"""Parity of the 6-DOF (oriented particle) path with the FP64 oracle: Cosserat
rods (CosseratRodEnergySolver.hpp:20-159), rigid-body ground contact
(RigidBodyGroundCollisionEnergySolver.hpp:14-183), one-sided fixed joints
(HardConstraintEnergySolver.hpp + OneSidedFixedJointEnergySolver.hpp) and the
6x6 block solve with q <- q (+) dtheta (VBDSolver.hpp:450-486).

Scene: helical rods of 1 cm segments hanging from joints, spheres dropped on
the ground beside them.  Positions are compared relative to the bounding-box
diagonal, quaternions up to sign by their component difference.
"""
import numpy as np
import pytest

from avbd_b200 import Context, scenes

pytestmark = pytest.mark.gpu


def rod_scene(rods=4, segments=20, spheres=4, seed=1, iters=20):
    return scenes.rods_and_spheres(num_rods=rods, segments=segments, num_spheres=spheres, seed=seed, iters=iters,
                                   length=segments * 0.01)


def pair(sc, oracle_lib, precision):
    e = Context()
    sc.load(e, precision=precision)
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o)
    o.finalize()
    return e, o


def quat_err(a, b):
    s = np.sign(np.sum(a * b, axis=1, keepdims=True))
    s[s == 0] = 1
    return np.abs(a - s * b).max()


def test_rod_scene_coloring_bit_exact(oracle_lib):
    sc = rod_scene(rods=9, segments=30, spheres=8)
    e, o = pair(sc, oracle_lib, "fp64")
    ce, nce = e.coloring()
    co, nco = o.coloring()
    assert nce == nco
    assert (ce == co).all()


@pytest.mark.parametrize("precision,tol_x,tol_q", [("fp64", 1e-9, 1e-8), ("mixed", 1e-9, 1e-8),
                                                  ("fp32", 1e-4, 3e-3)])
def test_rods_joints_rigid_ground_track_oracle(oracle_lib, precision, tol_x, tol_q):
    """Mixed mode keeps the rod, contact and joint records in FP64 (only tet
    records are FP32), so it meets the FP64 bound.  FP32 solves the 6x6
    blocks by a Jacobi-scaled FP32 LDL^T.  FP32 floor: positions near
    1 m carry ~1.2e-7 m of rounding, a strain error of ~1e-5 on 1 cm segments;
    with EA ~ 785 N that is a shear force noise of ~m g per node, which on the
    soft bending stiffness (EI/L ~ 0.49 N m) turns nodes by ~1e-4 rad,
    accumulated along the rod: quaternion components drift by ~1e-3 over 60
    steps while the FP64 oracle's own sensitivity to FP32-rounded initial
    state is ~3e-5."""
    sc = rod_scene()
    e, o = pair(sc, oracle_lib, precision)
    x0 = o.positions()
    for _ in range(6):
        e.step(10)
        o.step(10)
        ex = np.abs(e.positions() - o.positions()).max() / sc.bbox_diagonal()
        eq = quat_err(e.rotations(), o.rotations())
        assert ex < tol_x, ex
        assert eq < tol_q, eq
    assert np.abs(np.linalg.norm(e.rotations(), axis=1) - 1).max() < 1e-6
    assert np.abs(o.positions() - x0).max() > 1e-2  # rods sag, spheres fall
    if precision == "fp32":
        # the 6x6 blocks are solved by the scaled FP32 LDL^T; FP64 only above
        # the condition threshold, which the Jacobi-scaled rod blocks (~2) stay far below
        node_solves = 60 * sc.solver_iters * sc.num_particles
        assert e.stats()["fp64_fallbacks"] <= 0.01 * node_solves, e.stats()["fp64_fallbacks"]
    d = sc.bbox_diagonal()
    np.testing.assert_allclose(e.velocities(), o.velocities(), atol=tol_x * d * 60 * 10)
    np.testing.assert_allclose(e.angular_velocities(), o.angular_velocities(), atol=max(tol_q * 60 * 10, 1e-6))


def test_spheres_rest_on_ground(oracle_lib):
    """Spheres dropped on the rigid-body ground come to rest at y = radius."""
    sc = rod_scene(rods=1, segments=10, spheres=6)
    e, o = pair(sc, oracle_lib, "fp64")
    e.step(120)
    o.step(120)
    n_rod = 11
    ye = e.positions()[n_rod:, 1]
    yo = o.positions()[n_rod:, 1]
    assert np.abs(ye - yo).max() < 1e-9
    # lowest point of each sphere within 1 mm of the ground plane
    radii = np.array([args[2][0] for method, args, _ in sc.calls if method == "add_rigid_body_ground_collision"][1:])
    assert np.abs(ye - radii).max() < 1e-3


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_rod_block_gradient_hessian(oracle_lib, precision):
    """avbd_debug_block on 6-DOF nodes (rod interior, joint base, rigid
    ground, sphere) vs the oracle's accumulate, at a state reached by
    stepping and then copied into the oracle."""
    sc = rod_scene(rods=2, segments=20, spheres=2)
    e, o = pair(sc, oracle_lib, "fp64")
    e.step(20)
    o.step(20)
    o.set_positions_raw(0, e.positions())
    o.set_rotations_raw(0, e.rotations())
    if precision == "fp32":
        e2 = Context()
        sc.load(e2, precision="fp32")
        e2.finalize()
        e2.set_positions(0, e.positions().astype(np.float32).astype(np.float64))
        e = e2
        o2 = oracle_lib.Oracle()
        sc.load(o2)
        o2.finalize()
        o2.set_positions_raw(0, e.positions())
        o = o2
    rtol = 1e-7 if precision == "fp64" else 2e-4
    nodes = [0, 1, 10, 20, 21, 30, 41, 42]
    for p in nodes:
        Ge, He = e.debug_block(p)
        Go, Ho = o.debug_block(p)
        assert Ge.shape == (6,) and He.shape == (6, 6)
        scale_h = np.abs(Ho).max()
        scale_g = max(np.abs(Go).max(), scale_h * 1e-3)
        assert np.abs(Ge - Go).max() <= rtol * scale_g + 1e-12, (p, Ge, Go)
        assert np.abs(He - Ho).max() <= rtol * scale_h, (p, He, Ho)


def test_rod_residual_matches_oracle(oracle_lib):
    sc = rod_scene()
    e, o = pair(sc, oracle_lib, "fp64")
    e.step(5)
    o.step(5)
    re, ro = e.residual(), o.residual()
    assert abs(re - ro) <= 1e-6 * ro, (re, ro)


def test_rod_run_to_tolerance(oracle_lib):
    """Gauss-Seidel converges slowly on stiff rods (R ~ 0.2 after 100
    iterations), so the target is R <= 0.3 here."""
    sc = rod_scene(rods=2, segments=20, spheres=2)
    e = Context()
    sc.load(e, precision="fp64", residual_tolerance=0.3, max_iters=400)
    e.finalize()
    o = oracle_lib.Oracle()
    sc.load(o, residual_tolerance=0.3, max_iters=400)
    o.finalize()
    for _ in range(5):
        e.step(1)
        o.step(1)
    st = e.stats()
    assert 5 < o.iterations < 5 * 400
    assert abs(st["iterations"] - o.iterations) <= 2 * 5, (st["iterations"], o.iterations)
    assert np.abs(e.positions() - o.positions()).max() / sc.bbox_diagonal() < 1e-6
