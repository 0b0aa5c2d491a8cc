"""Procedural scene builders for the engine's workloads.

A Scene records the set-up calls a host application makes against a
SimulationContext (particles, energies, collision primitives, parameters) and
replays them into any object exposing the same method names -- the engine's
avbd_b200.Context or the FP64 oracle used by the tests.

The per-object set-up math restates the reference's scene objects, which
build their particles and energies with plain FP64 arithmetic:
  * TetMeshObject::setup (simobject/TetMeshObject.cpp:21-113): Lame
    parameters mu = E/(2(1+nu)), lambda = E nu/((1+nu)(1-2nu)); per tet
    X = [v1-v4, v2-v4, v3-v4], Q = X^-1, V = |det X|/6; lumped mass V rho/4;
  * per-vertex ground contact (simulation/Simulation.hpp:117-126):
    k_start = m/dt^2, mu_s = 0.4, mu_k = 0.2;
  * Rod::Rod (simobject/Rod.cpp:10-68) and RigidSphere (simobject/rigid/
    RigidSphere.cpp:8-22) for the oriented particles.
Meshes are generated here (a hex grid split into 6 tets per cell) instead of
being read from gmsh files.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np


@dataclass
class Scene:
    name: str
    dt: float
    g_accel: float = 9.81
    collision_margin: float = 1e-3
    solver_iters: int = 10
    iter_acceleration: float = 0.5
    calls: list = field(default_factory=list)
    num_particles: int = 0
    num_tets: int = 0
    num_primitives: int = 0
    num_scenes: int = 1
    meta: dict = field(default_factory=dict)

    def record(self, method: str, *args, **kwargs):
        self.calls.append((method, args, kwargs))

    def load(self, target: Any, residual_tolerance: float = 0.0, max_iters: int = 0, precision=None):
        target.set_params(self.dt, self.g_accel, self.collision_margin)
        target.set_solver(self.solver_iters, self.iter_acceleration, residual_tolerance, max_iters, precision)
        for method, args, kwargs in self.calls:
            getattr(target, method)(*args, **kwargs)
        return target

    def bbox_diagonal(self) -> float:
        return float(self.meta.get("bbox_diagonal", 1.0))


def lame(E: float, nu: float):
    """TetMeshObject::setup (simobject/TetMeshObject.cpp:44-45)."""
    mu = E / (2 * (1 + nu))
    lam = (E * nu) / ((1 + nu) * (1 - 2 * nu))
    return lam, mu


def hex_grid_tets(n: int):
    """Vertex grid (n+1)^3 (x fastest) and 6 tets per cell (Kuhn split along the
    (0,0,0)-(1,1,1) cell diagonal, the same diagonal in every cell)."""
    m = n + 1

    def vid(i, j, k):
        return i + m * (j + m * k)

    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    corner = lambda a, b, c: vid(ii + a, jj + b, kk + c)
    e = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    tets = []
    for perm in [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]:
        p1 = e[perm[0]]
        p2 = tuple(e[perm[0]][t] + e[perm[1]][t] for t in range(3))
        tets.append(np.stack([corner(0, 0, 0), corner(*p1), corner(*p2), corner(1, 1, 1)], axis=1))
    # cell-major order: all 6 tets of a cell are consecutive
    T = np.stack(tets, axis=1).reshape(-1, 4)
    return T.astype(np.uint32)


def surface_triangles(tets: np.ndarray) -> np.ndarray:
    """Boundary faces of a tet mesh (faces used by exactly one tet)."""
    f = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    key = np.sort(f, axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    once = cnt[inv.ravel()] == 1
    return f[once].astype(np.uint32)


def tet_setup(X: np.ndarray, tets: np.ndarray, E, nu, density):
    """Q, rest volume and lumped masses of TetMeshObject::setup
    (simobject/TetMeshObject.cpp:62-97)."""
    v1, v2, v3, v4 = (X[tets[:, k]] for k in range(4))
    a, b, c = v1 - v4, v2 - v4, v3 - v4  # columns of X
    # X^-1 rows are the cross products of the columns over det X
    r0, r1, r2 = np.cross(b, c), np.cross(c, a), np.cross(a, b)
    det = np.einsum("ij,ij->i", a, r0)
    Q = np.stack([r0, r1, r2], axis=1) / det[:, None, None]
    V = np.abs(det / 6.0)
    lam, mu = lame(E, nu)
    masses = np.bincount(tets.ravel(), weights=np.repeat(0.25 * V * density, 4), minlength=len(X))
    return Q, V, lam, mu, masses


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def add_tet_cube(sc: Scene, n: int, size: float = 1.0, origin=(0.0, 0.0, 0.0), E=1e5, nu=0.45,
                 density=1000.0, kd=0.0, perturb=0.0, rng=None, rotation=None,
                 fix_bottom=False, ground=False, surface=False, object_id=0, velocity=None, bottom_at=None):
    """Adds one cube of n^3 hex cells (6 tets each) to the scene."""
    m = n + 1
    h = size / n
    g = np.arange(m) * h
    gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
    # vertex id = i + m*(j + m*k): x fastest
    X = np.stack([gx.transpose(2, 1, 0).ravel(), gy.transpose(2, 1, 0).ravel(), gz.transpose(2, 1, 0).ravel()], axis=1)
    jidx = (np.arange(m ** 3) // m) % m
    if perturb > 0:
        rng = rng if rng is not None else np.random.default_rng(0)
        X = X + rng.uniform(-perturb * h, perturb * h, size=X.shape)
    if rotation is not None:
        c = np.full(3, size / 2)
        X = (X - c) @ np.asarray(rotation).T + c
    X = X + np.asarray(origin, dtype=np.float64)
    if bottom_at is not None:
        X[:, 1] += bottom_at - X[:, 1].min()
    tets = hex_grid_tets(n)
    Q, V, lam, mu, masses = tet_setup(X, tets, E, nu, density)
    base = sc.num_particles
    sc.record("add_particles", X, masses)
    if velocity is not None:
        vel = np.tile(np.asarray(velocity, dtype=np.float64), (len(X), 1))
        sc.record("set_velocities", base, vel, vel)
    gt = tets.astype(np.int64) + base
    nt = len(tets)
    sc.record("add_neo_hookean", gt, np.full(nt, lam), np.full(nt, mu), np.full(nt, kd), Q.reshape(-1, 9), V)
    if fix_bottom:
        slots = np.nonzero(jidx == 0)[0] + base
        sc.record("set_fixed", slots, np.ones(len(slots), dtype=np.uint8))
    if ground:
        ks = masses / (sc.dt * sc.dt)
        sc.record("add_ground_collision", np.arange(len(X)) + base, ks, np.full(len(X), 0.4), np.full(len(X), 0.2))
    if surface:
        tri = surface_triangles(tets).astype(np.int64) + base
        sc.record("add_triangles", tri, object_id)
        sc.num_primitives += len(tri)
    sc.num_particles += len(X)
    sc.num_tets += nt
    lo, hi = X.min(0), X.max(0)
    sc.meta.setdefault("boxes", []).append((lo, hi))
    allb = sc.meta["boxes"]
    glo = np.min([b[0] for b in allb], axis=0)
    ghi = np.max([b[1] for b in allb], axis=0)
    sc.meta["bbox_diagonal"] = float(np.linalg.norm(ghi - glo))
    return base


def cube_fixed_bottom(n: int = 8, steps_dt: float = 1.0 / 60.0, iters: int = 10, rho: float = 0.5) -> Scene:
    """Single NeoHookean cube, bottom face fixed, no collision:
    1 m cube of n^3 cells, rho 1000 kg/m^3, E 1e5 Pa, nu 0.45, g 9.81, dt 1/60,
    10 iterations per step (n = 8: 729 vertices, 3072 tets)."""
    sc = Scene(name=f"cube{n}_fixed", dt=steps_dt, solver_iters=iters, iter_acceleration=rho)
    add_tet_cube(sc, n, E=1e5, nu=0.45, density=1000.0, fix_bottom=True)
    return sc


def cube_drop(n: int = 32, seed: int = 0, iters: int = 20, rho: float = 0.5, dt: float = 1.0 / 60.0,
              height: float = 0.5, surface: bool = True) -> Scene:
    """Cube dropped onto the ground plane with self-collision candidates:
    1 m cube of n^3 cells (n = 32: 35,937 vertices, 196,608 tets, 12,288
    surface triangles), E 1e6, nu 0.49, rho 1000, every vertex perturbed by
    seeded uniform noise of +-0.2 cell, bottom face at y = height, per-vertex
    ground contact, 20 iterations per step."""
    sc = Scene(name=f"cube{n}_drop", dt=dt, solver_iters=iters, iter_acceleration=rho)
    rng = np.random.default_rng(seed)
    add_tet_cube(sc, n, origin=(0.0, height, 0.0), E=1e6, nu=0.49, density=1000.0, perturb=0.2, rng=rng,
                 ground=True, surface=surface)
    return sc


def quat_mul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 + y1 * w2 + z1 * x2 - x1 * z2, w1 * z2 + z1 * w2 + x1 * y2 - y1 * x2])


def quat_rotate(q, v):
    u = np.asarray(q[1:])
    t = 2 * np.cross(u, v)
    return np.asarray(v) + q[0] * t + np.cross(u, t)


def quat_exp(v):
    """Math::Exp_s3 (common/Math.hpp:197-222)."""
    v = np.asarray(v, dtype=np.float64)
    th = np.linalg.norm(v)
    if th < 1e-6:
        q = np.array([1.0, 0.5 * v[0], 0.5 * v[1], 0.5 * v[2]])
        return q / np.linalg.norm(q)
    s = np.sin(0.5 * th) / th
    return np.array([np.cos(0.5 * th), s * v[0], s * v[1], s * v[2]])


def quat_from_xyz_euler(deg):
    """Math::QuaternionFromXYZEulerAngles (common/Math.hpp:298-318): qz qy qx."""
    x, y, z = np.radians(deg)
    qx = np.array([np.cos(x / 2), np.sin(x / 2), 0, 0])
    qy = np.array([np.cos(y / 2), 0, np.sin(y / 2), 0])
    qz = np.array([np.cos(z / 2), 0, 0, np.sin(z / 2)])
    return quat_mul(quat_mul(qz, qy), qx)


def add_rod(sc: Scene, elements: int, length: float, radius: float, E: float, nu: float, density: float,
            position, euler_deg, curvature, base_joint=True, base_fixed=False, ground=True, collide=True,
            object_id=0):
    """Rod::Rod (simobject/Rod.cpp:10-68): nodes integrated along the local z
    axis with frames advanced by Exp_s3(curvature ds); lumped translational and
    rotational mass; Cosserat stiffness (GA, GA, EA, EIx, EIy, GIz).  The base
    is held by a one-sided fixed joint at its initial pose (the commented
    alternative of Rod.cpp:79-91) instead of being fixed."""
    G = E / (2 * (1 + nu))
    nn = elements + 1
    ds = length / (nn - 1)
    dR = np.asarray(curvature, dtype=np.float64) * ds
    pos = np.asarray(position, dtype=np.float64).copy()
    rot = quat_from_xyz_euler(euler_deg)
    P, Qs = [], []
    for _ in range(nn):
        P.append(pos.copy())
        Qs.append(rot.copy())
        pos = pos + quat_rotate(rot, np.array([0.0, 0.0, ds]))
        rot = quat_mul(rot, quat_exp(dR))
    area = np.pi * radius ** 2
    Ix = np.pi * radius ** 4 / 4.0
    m_e = ds * area * density
    I_e = density * ds * np.array([Ix, Ix, 2 * Ix])
    masses = np.zeros(nn)
    inert = np.zeros((nn, 3))
    for e in range(elements):
        masses[e] += 0.5 * m_e
        masses[e + 1] += 0.5 * m_e
        inert[e] += 0.5 * I_e
        inert[e + 1] += 0.5 * I_e
    base = sc.num_particles
    sc.record("add_oriented_particles", np.array(P), np.array(Qs), masses, inert)
    idx = np.stack([np.arange(elements), np.arange(1, elements + 1)], axis=1) + base
    K = np.array([G * area, G * area, E * area, E * Ix, E * Ix, G * 2 * Ix])
    sc.record("add_cosserat_rod", idx, np.tile(K, (elements, 1)), np.full(elements, ds),
              np.tile(np.asarray(curvature, dtype=np.float64), (elements, 1)))
    if base_joint:
        sc.record("add_one_sided_fixed_joint", [base], np.zeros((1, 3)), np.array([[1.0, 0, 0, 0]]),
                  np.array([P[0]]), np.array([Qs[0]]))
    if base_fixed:
        sc.record("set_fixed", [base], [1])
    if ground:
        ks = masses / sc.dt ** 2
        sc.record("add_rigid_body_ground_collision", np.arange(nn) + base, np.full(nn, 1, dtype=np.uint8),
                  np.full(nn, radius), np.tile([0.0, -radius, 0.0], (nn, 1)), ks, np.full(nn, 0.5),
                  np.full(nn, 0.2))
    if collide:
        sc.record("add_rod_segments", idx, radius, object_id)
        sc.num_primitives += elements
    sc.num_particles += nn
    return base


def add_sphere(sc: Scene, radius: float, density: float, position, ground=True):
    """RigidSphere (simobject/rigid/RigidSphere.cpp:8-22): mass 4/3 pi r^3 rho,
    inertia 2/5 m r^2; rigid-body ground contact (Simulation.hpp:108-115)."""
    m = 4 * np.pi / 3 * radius ** 3 * density
    I = 0.4 * m * radius ** 2
    base = sc.num_particles
    sc.record("add_oriented_particles", np.array([position], dtype=np.float64), np.array([[1.0, 0, 0, 0]]), [m],
              np.array([[I, I, I]]))
    if ground:
        sc.record("add_rigid_body_ground_collision", [base], np.array([2], dtype=np.uint8), [radius],
                  np.array([[0.0, -radius, 0.0]]), [m / sc.dt ** 2], [0.5], [0.2])
    sc.num_particles += 1
    return base


def spheres_on_cube(n: int = 4, num_spheres: int = 4, seed: int = 0, iters: int = 20, rho: float = 0.5,
                    dt: float = 1.0 / 60.0, size: float = 1.0, E: float = 1e5, nu: float = 0.4,
                    radius=(0.08, 0.15), drop: float = 0.02, speed: float = 1.0, sphere_density: float = 500.0,
                    fix_bottom: bool = True) -> Scene:
    """Rigid spheres dropped on a soft tet cube: a cube of n^3 cells (E, nu,
    rho 1000) with its bottom face fixed (or resting on the ground when
    fix_bottom is False) and its surface triangles as collision primitives;
    spheres of seeded radius ~ U(radius) spread over the top face, `drop`
    above it and falling at `speed`, each a collision sphere of its own object
    with rigid-body ground contact.  Their contacts with the cube's surface are
    the triangle-rigid contact energies of the collision stage."""
    rng = np.random.default_rng(seed)
    sc = Scene(name=f"cube{n}_spheres{num_spheres}", dt=dt, solver_iters=iters, iter_acceleration=rho)
    add_tet_cube(sc, n, size=size, E=E, nu=nu, density=1000.0, fix_bottom=fix_bottom, ground=not fix_bottom,
                 surface=True, object_id=0)
    side = int(np.ceil(np.sqrt(num_spheres)))
    for s in range(num_spheres):
        r = rng.uniform(*radius)
        cx = (s % side + 0.5) / side * size + rng.uniform(-0.05, 0.05) * size / side
        cz = (s // side + 0.5) / side * size + rng.uniform(-0.05, 0.05) * size / side
        base = add_sphere(sc, r, sphere_density, (cx, size + r + drop, cz))
        vel = np.array([[0.0, -speed, 0.0]])
        sc.record("set_velocities", base, vel, vel)
        sc.record("add_spheres", [base], [r], [1 + s])
        sc.num_primitives += 1
    return sc


def rods_on_cube(n: int = 4, num_rods: int = 3, segments: int = 8, seed: int = 0, iters: int = 20,
                 rho: float = 0.5, dt: float = 1.0 / 60.0, size: float = 1.0, E_cube: float = 1e6,
                 nu_cube: float = 0.4, rod_length: float = 0.5, rod_radius: float = 0.01, drop: float = 0.002,
                 speed: float = 0.2) -> Scene:
    """Cosserat rods dropped flat on a soft tet cube: a cube of n^3 cells
    (bottom face fixed, surface triangles as collision primitives) and
    `num_rods` straight rods of `segments` elements (radius 1 cm, E 1e7, nu
    0.25, rho 1000) lying along x at seeded z over the top face, `drop` above
    it and falling at `speed`, each its own object with rigid-body ground
    contact.  Their segments' contacts with the cube's surface are the
    triangle-rod contact energies of the collision stage."""
    rng = np.random.default_rng(seed)
    sc = Scene(name=f"cube{n}_rods{num_rods}x{segments}", dt=dt, solver_iters=iters, iter_acceleration=rho)
    add_tet_cube(sc, n, size=size, E=E_cube, nu=nu_cube, density=1000.0, fix_bottom=True, surface=True,
                 object_id=0)
    for r in range(num_rods):
        z = (r + 0.5) / num_rods * size + rng.uniform(-0.05, 0.05) * size / num_rods
        x0 = 0.5 * (size - rod_length) + rng.uniform(-0.05, 0.05)
        base = add_rod(sc, segments, rod_length, rod_radius, 1e7, 0.25, 1000.0,
                       (x0, size + rod_radius + drop, z), (0.0, 90.0, 0.0), (0.0, 0.0, 0.0), base_joint=False,
                       ground=True, collide=True, object_id=1 + r)
        vel = np.tile([0.0, -speed, 0.0], (segments + 1, 1))
        sc.record("set_velocities", base, vel, vel)
    return sc


def rods_and_spheres(num_rods: int = 256, segments: int = 100, num_spheres: int = 64, seed: int = 0,
                     iters: int = 20, rho: float = 0.5, dt: float = 1.0 / 60.0, length: float = 1.0,
                     helix_radius: float = 0.02, spacing: float = 0.1) -> Scene:
    """Cosserat rods and rigid spheres: rods of `segments` elements (radius
    5 mm, E 1e7, G 4e6 so nu = 0.25, rho 1000), length 1 m, shaped as seeded
    helices (radius 2 cm, pitch ~ U(2, 10) cm) through a constant precurvature
    (kappa, 0, tau), hanging from one-sided fixed joints at their bases on a
    grid 1.2 m above the ground; spheres of radius ~ U(1, 5) cm dropped onto
    the ground beside them.  Rod nodes and spheres have rigid-body ground
    contact; rod segments are collision primitives."""
    rng = np.random.default_rng(seed)
    sc = Scene(name=f"rods{num_rods}x{segments}_spheres{num_spheres}", dt=dt, solver_iters=iters,
               iter_acceleration=rho)
    side = int(np.ceil(np.sqrt(num_rods)))
    E, nu = 1e7, 0.25
    for r in range(num_rods):
        pitch = rng.uniform(0.02, 0.10)
        b = pitch / (2 * np.pi)
        a = helix_radius
        kappa, tau = a / (a * a + b * b), b / (a * a + b * b)
        ox, oz = (r % side) * spacing, (r // side) * spacing
        add_rod(sc, segments, length, 0.005, E, nu, 1000.0, (ox, 1.2, oz), (90.0, 0.0, 0.0), (kappa, 0.0, tau),
                object_id=r)
    for s in range(num_spheres):
        rad = rng.uniform(0.01, 0.05)
        x = rng.uniform(0, side * spacing)
        z = side * spacing + 0.2 + rng.uniform(0, 1.0)
        add_sphere(sc, rad, 1000.0, (x, rad + rng.uniform(0.05, 0.5), z))
    sc.meta["bbox_diagonal"] = float(np.linalg.norm([side * spacing, 1.2, side * spacing + 1.2]))
    return sc


def batched_cube_params(seed: int, s: int, n_min: int = 4, n_max: int = 24):
    """Parameters of scene s of a batch: drawn from a generator seeded by
    (seed, s), so any subset of a batch is reproduced exactly."""
    rng = np.random.default_rng([seed, s])
    n = int(rng.integers(n_min, n_max + 1))
    E = float(10 ** rng.uniform(4, 7))
    nu = float(rng.uniform(0.3, 0.49))
    R = random_rotation(rng)
    return n, E, nu, R


def batched_cubes(num_scenes: int = 1024, seed: int = 0, n_min: int = 4, n_max: int = 24, iters: int = 15,
                  rho: float = 0.5, dt: float = 1.0 / 60.0, spacing: float = 2.0, scene_ids=None) -> Scene:
    """Many independent cubes of uneven size advanced together: cell counts
    n ~ U{n_min..n_max} per side (6 n^3 tets), E log-uniform in [1e4, 1e7],
    nu ~ U(0.3, 0.49), random initial rotation, per-vertex ground contact,
    15 iterations per step.  Each cube is its own scene (own coloring).
    scene_ids selects a subset of the batch (same cubes, same placement)."""
    ids = list(range(num_scenes)) if scene_ids is None else list(scene_ids)
    sc = Scene(name=f"batch{num_scenes}", dt=dt, solver_iters=iters, iter_acceleration=rho)
    side = int(np.ceil(np.sqrt(num_scenes)))
    cells = []
    for k, s in enumerate(ids):
        if k > 0:
            sc.record("begin_scene")
        n, E, nu, R = batched_cube_params(seed, s, n_min, n_max)
        cells.append(n)
        ox, oz = (s % side) * spacing, (s // side) * spacing
        add_tet_cube(sc, n, size=1.0, origin=(ox, 0.0, oz), E=E, nu=nu, density=1000.0, rotation=R, ground=True,
                     bottom_at=0.3)
    sc.num_scenes = len(ids)
    sc.meta["cells"] = cells
    return sc
