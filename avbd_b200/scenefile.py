"""Headless scenes from the reference's YAML scene files.

    python -m avbd_b200.scenefile scene.yaml [--steps N] [--frames DIR] [--every K]

`load_yaml` reads the subset of the scene schema that the per-step solve
uses and builds a `scenes.Scene` whose replay is the reference's set-up
(simulation/Simulation.cpp:48-90, simulation/Simulation.hpp:54-137):

* simulation keys (config/SimulationConfig.hpp:40-56, defaults :133-149):
  time-step (1e-3), g-accel (9.81), collision-margin (1e-3), solver-iters (1),
  iter-acceleration (0.5); rendering, logging and threading keys are ignored;
* objects, in file order, each getting the next object id
  (simobject/ObjectBase.hpp:17-33):
  - TetMeshObject (config/TetMeshObjectConfig.hpp, simobject/TetMeshObject.cpp:21-113):
    filename (MSH 4.1 ASCII, relative to the YAML file), position-by-com
    (true: centred on the volume centre of mass of its surface,
    common/mesh/ParticleMesh.cpp:129-160), scaling, rotation (XYZ Euler
    degrees, Math.hpp:248-270), position, velocity, E (1e6), nu (0.4),
    density (1000), damping-coeff (0); per tet Q = X^-1 of the columns
    (v1-v4, v2-v4, v3-v4), V = |det X| / 6, mass V rho / 4 to each vertex;
    surface triangles join the collision pool;
  - Rod (config/RodConfig.hpp, simobject/Rod.cpp:10-68): elements (20), length
    (1), diameter (0.1), density (1000), E (3e6), nu (0.45), curvature,
    base-fixed (true), tip-fixed (false), position, rotation, velocity;
  - RigidSphere (config/RigidSphereConfig.hpp, simobject/rigid/RigidSphere.cpp:8-22,
    RigidObjectBase.cpp:10-20): radius (0.5), density (1000), fixed (false),
    position, rotation (its velocity is not used by the reference);
* ground contact for every object, whatever `ground-plane` says
  (Simulation.hpp:108-137): tet vertices k_start = m/h^2, mu 0.4 / 0.2; rod
  nodes and spheres rigid-body ground with mu 0.5 / 0.2.

Sphere collision primitives are left out unless `sphere_primitives=True`:
with them, spheres near rods or near each other give sphere-rod and
sphere-sphere candidate pairs, on which the reference throws
(collision/CollisionDetector.cpp:180-213,678-687) and the engine returns
AVBD_ERR_UNSUPPORTED_PAIR; triangle-sphere pairs become contact energies.
"""
from __future__ import annotations

import argparse
import math
import os

import numpy as np

from . import meshio, scenes

SIM_DEFAULTS = {"time-step": 1e-3, "g-accel": 9.81, "collision-margin": 1e-3, "solver-iters": 1,
                "iter-acceleration": 0.5}


def rot_xyz(deg):
    """Math::RotMatFromXYZEulerAngles: Rz(z) Ry(y) Rx(x), degrees."""
    x, y, z = np.radians(np.asarray(deg, dtype=np.float64))
    Rx = np.array([[1, 0, 0], [0, math.cos(x), -math.sin(x)], [0, math.sin(x), math.cos(x)]])
    Ry = np.array([[math.cos(y), 0, math.sin(y)], [0, 1, 0], [-math.sin(y), 0, math.cos(y)]])
    Rz = np.array([[math.cos(z), -math.sin(z), 0], [math.sin(z), math.cos(z), 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def surface_mass_center(X, faces):
    """ParticleMesh::massCenter: volume-weighted centroid of the tetrahedra
    (origin, f0, f1, f2) over the surface triangles."""
    a, b, c = X[faces[:, 0]], X[faces[:, 1]], X[faces[:, 2]]
    vol = np.einsum("ij,ij->i", a, np.cross(b, c)) / 6.0
    cm = (a + b + c) * 0.25
    return (cm * vol[:, None]).sum(0) / vol.sum()


def _vec(node, key, default):
    return np.asarray(node.get(key, default), dtype=np.float64)


def add_tet_mesh_object(sc, node, base_dir, object_id):
    path = node.get("filename", "")
    if not os.path.isabs(path):
        path = os.path.join(base_dir, path)
    X, tets, faces = meshio.read_msh(path)
    X = X.copy()
    if node.get("position-by-com", True):
        if len(faces) == 0:
            raise ValueError(f"{path}: position-by-com needs surface triangles")
        X -= surface_mass_center(X, faces)
    X *= _vec(node, "scaling", [1, 1, 1])[None, :]
    X = X @ rot_xyz(_vec(node, "rotation", [0, 0, 0])).T
    X += _vec(node, "position", [0, 0, 0])[None, :]
    E, nu, rho = float(node.get("E", 1e6)), float(node.get("nu", 0.4)), float(node.get("density", 1000))
    kd = float(node.get("damping-coeff", 0.0))
    lam, mu = scenes.lame(E, nu)
    P = X[tets]
    Xm = np.stack([P[:, 0] - P[:, 3], P[:, 1] - P[:, 3], P[:, 2] - P[:, 3]], axis=2)
    Q = np.linalg.inv(Xm)
    V = np.abs(np.linalg.det(Xm)) / 6.0
    masses = np.zeros(len(X))
    np.add.at(masses, tets.reshape(-1), np.repeat(0.25 * V * rho, 4))
    base = sc.num_particles
    sc.record("add_particles", X, masses)
    vel = np.tile(_vec(node, "velocity", [0, 0, 0]), (len(X), 1))
    if np.any(vel):
        sc.record("set_velocities", base, vel, vel)
    nt = len(tets)
    sc.record("add_neo_hookean", tets + base, np.full(nt, lam), np.full(nt, mu), np.full(nt, kd), Q.reshape(-1, 9), V)
    if len(faces):
        sc.record("add_triangles", faces + base, object_id)
        sc.num_primitives += len(faces)
    sc.record("add_ground_collision", np.arange(len(X)) + base, masses / sc.dt ** 2, np.full(len(X), 0.4),
              np.full(len(X), 0.2))
    sc.num_particles += len(X)
    sc.num_tets += nt
    return X, faces


def add_rod_object(sc, node, object_id):
    E, nu = float(node.get("E", 3e6)), float(node.get("nu", 0.45))
    el = int(node.get("elements", 20))
    base = scenes.add_rod(sc, el, float(node.get("length", 1.0)), float(node.get("diameter", 0.1)) / 2, E, nu,
                          float(node.get("density", 1000)), _vec(node, "position", [0, 0, 0]),
                          _vec(node, "rotation", [0, 0, 0]), _vec(node, "curvature", [0, 0, 0]),
                          base_joint=False, base_fixed=bool(node.get("base-fixed", True)), ground=True, collide=True,
                          object_id=object_id)
    if node.get("tip-fixed", False):
        sc.record("set_fixed", [base + el], [1])
    vel = _vec(node, "velocity", [0, 0, 0])
    if np.any(vel):
        sc.record("set_velocities", base, np.tile(vel, (el + 1, 1)), np.tile(vel, (el + 1, 1)))
    return base


def add_sphere_object(sc, node, object_id, sphere_primitives):
    r = float(node.get("radius", 0.5))
    rho = float(node.get("density", 1000))
    m = 4 * math.pi / 3 * r ** 3 * rho
    I = 0.4 * m * r ** 2
    base = sc.num_particles
    q = scenes.quat_from_xyz_euler(_vec(node, "rotation", [0, 0, 0]))
    sc.record("add_oriented_particles", _vec(node, "position", [0, 0, 0])[None, :], q[None, :], [m],
              np.array([[I, I, I]]))
    if node.get("fixed", False):
        sc.record("set_fixed", [base], [1])
    sc.record("add_rigid_body_ground_collision", [base], np.array([2], dtype=np.uint8), [r],
              np.array([[0.0, -r, 0.0]]), [m / sc.dt ** 2], [0.5], [0.2])
    if sphere_primitives:
        sc.record("add_spheres", [base], [r], [object_id])
        sc.num_primitives += 1
    sc.num_particles += 1
    return base


def load_yaml(path: str, sphere_primitives: bool = False) -> scenes.Scene:
    import yaml
    with open(path) as f:
        cfg = yaml.safe_load(f) or {}
    get = lambda k: float(cfg.get(k, SIM_DEFAULTS[k]))
    sc = scenes.Scene(name=str(cfg.get("name", os.path.basename(path))), dt=get("time-step"),
                      g_accel=get("g-accel"), collision_margin=get("collision-margin"),
                      solver_iters=int(cfg.get("solver-iters", SIM_DEFAULTS["solver-iters"])),
                      iter_acceleration=get("iter-acceleration"))
    base_dir = os.path.dirname(os.path.abspath(path))
    surfaces, rods = [], []
    lo, hi = np.full(3, np.inf), np.full(3, -np.inf)
    for object_id, node in enumerate(cfg.get("objects") or []):
        kind = node.get("type")
        if kind == "TetMeshObject":
            base = sc.num_particles
            X, faces = add_tet_mesh_object(sc, node, base_dir, object_id)
            surfaces.append(faces + base)
            lo, hi = np.minimum(lo, X.min(0)), np.maximum(hi, X.max(0))
        elif kind == "Rod":
            base = add_rod_object(sc, node, object_id)
            rods.append(list(range(base, base + int(node.get("elements", 20)) + 1)))
        elif kind == "RigidSphere":
            add_sphere_object(sc, node, object_id, sphere_primitives)
        else:
            raise ValueError(f"object type {kind!r} is not supported")
    sc.meta["surfaces"] = np.concatenate(surfaces) if surfaces else np.zeros((0, 3), dtype=np.int64)
    sc.meta["rods"] = rods
    if np.all(np.isfinite(lo)):
        sc.meta["bbox_diagonal"] = float(np.linalg.norm(hi - lo))
    return sc


def dump_frame(sc: scenes.Scene, positions, path: str):
    """Surface triangles and rod polylines of the current positions (OBJ, or
    PLY triangles when the path ends in .ply)."""
    if path.endswith(".ply"):
        meshio.write_ply(path, positions, sc.meta["surfaces"])
    else:
        meshio.write_obj(path, positions, sc.meta["surfaces"], sc.meta["rods"])


def run(path: str, steps: int, frames: str | None = None, every: int = 1, precision: str = "fp64",
        device: int = 0, fmt: str = "obj"):
    """Loads a scene file into the engine and steps it, writing a frame every
    `every` steps when `frames` is a directory."""
    from . import Context
    sc = load_yaml(path)
    ctx = Context(device=device)
    sc.load(ctx, precision=precision)
    ctx.finalize()
    if frames:
        os.makedirs(frames, exist_ok=True)
    for s in range(steps):
        ctx.step(1)
        if frames and (s + 1) % every == 0:
            dump_frame(sc, ctx.positions(), os.path.join(frames, f"frame_{s + 1:05d}.{fmt}"))
    return ctx, sc


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("scene")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--frames", default=None)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--format", default="obj", choices=["obj", "ply"])
    ap.add_argument("--precision", default="fp64", choices=["fp32", "mixed", "fp64"])
    a = ap.parse_args(argv)
    ctx, sc = run(a.scene, a.steps, a.frames, a.every, a.precision, fmt=a.format)
    x = ctx.positions()
    print(f"{sc.name}: {sc.num_particles} particles, {sc.num_tets} tets, {a.steps} steps; "
          f"min y {x[:, 1].min():.4f}, max |x| {np.abs(x).max():.4f}")


if __name__ == "__main__":
    main()
