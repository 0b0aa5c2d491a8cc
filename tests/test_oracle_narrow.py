"""The oracle's triangle-sphere narrow phase (a restatement of
CollisionDetector::_triangleSDF_CCD, collision/CollisionDetector.cpp:689-876)
on cases with known answers: the contact under a falling sphere, no contact
when the sphere stays away, the contact frame of a rotated sphere, and the
DetectedCollision key layout."""
import numpy as np
import pytest

from oracle.oracle import Oracle


def setup(center, radius, vel, rot=(1, 0, 0, 0), omega=(0, 0, 0), dt=0.01, margin=1e-3, tri=None):
    o = Oracle()
    o.set_params(dt, 0.0, margin)
    o.set_solver(1, 0.5)
    T = np.array(tri if tri is not None else [[0, 0, 0], [1, 0, 0], [0, 0, 1.0]])
    o.add_particles(T, np.ones(3))
    o.set_fixed([0, 1, 2], [1, 1, 1])
    o.add_oriented_particles(np.array([center], dtype=float), np.array([rot], dtype=float), [1.0], np.ones((1, 3)))
    o.set_velocities(3, np.array([vel], dtype=float))
    o.add_triangles(np.array([[0, 1, 2]]), 0)
    o.add_spheres([3], [radius], [1])
    o.finalize()
    if any(omega):
        o.set_angular_velocity(3, omega) if hasattr(o, "set_angular_velocity") else pytest.skip("no angular velocity setter")
    o.collision_stage()
    return o.contacts()


def test_falling_sphere_contact_under_its_centre():
    c = setup([0.25, 0.3, 0.25], 0.2, [0, -20, 0])
    assert len(c["key"]) == 1
    assert c["tri"].tolist() == [[0, 1, 2]] and c["rigid"].tolist() == [3]
    # contact point: the centre's projection on the triangle, barycentrics (0.5, 0.25, 0.25),
    # to the search's 1e-3 bracket
    assert np.allclose(c["barys"][0], [0.5, 0.25, 0.25], atol=2e-3)
    assert np.allclose(c["normal"][0], [0, -1, 0], atol=5e-3)       # sphere frame -> triangle
    assert np.allclose(c["cp_local"][0], [0, -0.2, 0], atol=1e-3)   # on the sphere's surface
    assert c["key"][0] == (2 << 59) | (0 << 33) | (1 << 7)        # TriangleRigid, primitives 0 and 1


def test_sphere_moving_away_has_no_contact():
    assert len(setup([0.25, 0.3, 0.25], 0.2, [0, 5, 0])["key"]) == 0


def test_approaching_sphere_within_margin():
    c = setup([0.3, 0.2005, 0.3], 0.2, [0, -0.1, 0], margin=1e-3)
    assert len(c["key"]) == 1
    assert np.allclose(c["barys"][0], [0.4, 0.3, 0.3], atol=2e-3)


def test_static_sphere_inside_margin_is_not_a_candidate():
    """The swept boxes carry no margin (CollisionPrimitivePool.hpp:160-236): a
    motionless sphere 0.5 mm above a motionless triangle never reaches the
    narrow phase, whatever the collision margin."""
    assert len(setup([0.3, 0.2005, 0.3], 0.2, [0, 0, 0], margin=1e-3)["key"]) == 0


def test_rotated_sphere_contact_frame():
    """A sphere turned 90 degrees about z: the contact point in its body frame
    is the world contact direction rotated back, the normal stays in the world."""
    s = np.sqrt(0.5)
    c = setup([0.25, 0.3, 0.25], 0.2, [0, -20, 0], rot=(s, 0, 0, s))
    assert len(c["key"]) == 1
    assert np.allclose(c["normal"][0], [0, -1, 0], atol=5e-3)
    assert np.allclose(c["cp_local"][0], [-0.2, 0, 0], atol=1e-3)   # R_z(-90) (0, -0.2, 0)
