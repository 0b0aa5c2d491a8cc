"""Scene builders reproduce the workload sizes and the set-up math of the
reference's TetMeshObject::setup (simobject/TetMeshObject.cpp:21-113)."""
import numpy as np

from avbd_b200 import scenes


class Recorder:
    def __init__(self):
        self.calls = {}

    def __getattr__(self, name):
        def f(*a, **k):
            self.calls.setdefault(name, []).append(a)
        return f


def test_cube_fixed_bottom_sizes():
    sc = scenes.cube_fixed_bottom(8)
    assert sc.num_particles == 729 and sc.num_tets == 3072
    r = Recorder()
    sc.load(r)
    (X, m), = r.calls["add_particles"]
    assert np.isclose(m.sum(), 1000.0)  # 1 m^3 at 1000 kg/m^3
    (slots, fl), = r.calls["set_fixed"]
    assert len(slots) == 81 and np.allclose(X[slots, 1], 0.0)


def test_cube_drop_sizes():
    sc = scenes.cube_drop(32)
    assert sc.num_particles == 35937 and sc.num_tets == 196608 and sc.num_primitives == 12288
    r = Recorder()
    sc.load(r)
    (X, m), = r.calls["add_particles"]
    assert X[:, 1].min() > 0.5 - 0.2 / 32 - 1e-12
    (p, ks, mus, muk), = r.calls["add_ground_collision"]
    assert np.allclose(ks, m / sc.dt ** 2) and np.allclose(mus, 0.4) and np.allclose(muk, 0.2)


def test_tet_volumes_and_Q():
    sc = scenes.cube_drop(4, seed=2)
    r = Recorder()
    sc.load(r)
    (X, m), = r.calls["add_particles"]
    (idx, lam, mu, kd, Q, V), = r.calls["add_neo_hookean"]
    assert np.isclose(V.sum(), 1.0, rtol=0.05)  # perturbed 1 m cube
    T = X[idx]
    Xm = np.stack([T[:, 0] - T[:, 3], T[:, 1] - T[:, 3], T[:, 2] - T[:, 3]], axis=2)
    assert np.allclose(np.einsum("nij,njk->nik", Xm, Q.reshape(-1, 3, 3)), np.eye(3), atol=1e-9)
    E, nu = 1e6, 0.49
    assert np.allclose(mu, E / (2 * (1 + nu))) and np.allclose(lam, E * nu / ((1 + nu) * (1 - 2 * nu)))


def test_batched_scene_count():
    sc = scenes.batched_cubes(num_scenes=5, seed=0, n_min=2, n_max=4)
    r = Recorder()
    sc.load(r)
    assert len(r.calls["begin_scene"]) == 4
    assert len(r.calls["add_particles"]) == 5


def test_benchmark_batch_sizes_and_ranges():
    """The 1024-cube batch of seed 0: 4,921,807 vertices and 25,132,554 tets,
    n in 4..24 cells per side, E in [1e4, 1e7], nu in [0.3, 0.49]."""
    P = [scenes.batched_cube_params(0, s) for s in range(1024)]
    n = np.array([p[0] for p in P])
    E = np.array([p[1] for p in P])
    nu = np.array([p[2] for p in P])
    assert int(((n + 1) ** 3).sum()) == 4_921_807 and int((6 * n ** 3).sum()) == 25_132_554
    assert n.min() == 4 and n.max() == 24
    assert 1e4 <= E.min() and E.max() <= 1e7 and 0.3 <= nu.min() and nu.max() <= 0.49
    for P0 in P[:4]:
        R = P0[3]
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-12) and np.isclose(np.linalg.det(R), 1.0)


def test_batch_subset_reproduces_its_scenes():
    """A subset of the batch (the CPU baselines' samples, the parity tests'
    scenes) holds exactly the cubes the full batch has at those ids."""
    def particles(ids):
        r = Recorder()
        scenes.batched_cubes(num_scenes=1024, seed=0, scene_ids=ids).load(r)
        return r.calls["add_particles"]
    a = particles([2, 5, 9])
    b = particles([9])
    c = particles([5])
    assert np.array_equal(a[2][0], b[0][0]) and np.array_equal(a[2][1], b[0][1])
    assert np.array_equal(a[1][0], c[0][0])


def test_rods_and_spheres_setup():
    """Rod::Rod set-up (simobject/Rod.cpp:10-68): lumped masses and inertias,
    Cosserat stiffness, frames advanced by Exp_s3(kappa ds)."""
    sc = scenes.rods_and_spheres()
    assert sc.num_particles == 256 * 101 + 64 and sc.num_primitives == 256 * 100
    sc = scenes.rods_and_spheres(num_rods=2, segments=10, num_spheres=3, length=0.1)
    r = Recorder()
    sc.load(r)
    (X, Q, m, I), = r.calls["add_oriented_particles"][:1]
    ds, area, Ix = 0.01, np.pi * 0.005 ** 2, np.pi * 0.005 ** 4 / 4
    me = ds * area * 1000.0
    assert np.isclose(m[0], me / 2) and np.isclose(m[1], me) and np.isclose(m.sum(), 10 * me)
    assert np.allclose(I[1], 1000.0 * ds * np.array([Ix, Ix, 2 * Ix]))
    assert np.allclose(np.linalg.norm(Q, axis=1), 1)
    assert np.allclose(np.linalg.norm(np.diff(X, axis=0), axis=1), ds)
    (idx, K, L, kap), = r.calls["add_cosserat_rod"][:1]
    G = 1e7 / (2 * 1.25)
    assert np.allclose(K[0], [G * area, G * area, 1e7 * area, 1e7 * Ix, 1e7 * Ix, G * 2 * Ix])
    # helix: every segment turns by the same angle |kappa| ds
    rel = [scenes.quat_mul(Q[i] * [1, -1, -1, -1], Q[i + 1]) for i in range(10)]
    ang = [2 * np.arctan2(np.linalg.norm(q[1:]), q[0]) for q in rel]
    assert np.allclose(ang, np.linalg.norm(kap[0]) * ds)
    # spheres: m = 4/3 pi r^3 rho, I = 2/5 m r^2, on or above the ground
    sph = r.calls["add_oriented_particles"][2:]
    assert len(sph) == 3
    for (Xs, Qs, ms, Is) in sph:
        assert np.isclose(Is[0][0], 0.4 * ms[0] * (ms[0] / (4 / 3 * np.pi * 1000.0)) ** (2 / 3))
    joints = r.calls["add_one_sided_fixed_joint"]
    assert len(joints) == 2 and np.allclose(joints[0][3][0], X[0])
