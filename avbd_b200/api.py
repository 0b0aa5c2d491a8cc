"""Python facade of the engine over its C-ABI.

Two layers:
  * Context -- bulk, array-oriented calls (one C call per batch of particles or
    energies), used by the scene builders, tests and bench;
  * SimulationContext / EnergyRegistry / VBDSolver / SimulationExecutor --
    the reference's step-API names and argument meanings
    (simulation/SimulationContext.hpp:18-60, energy/EnergyRegistry.hpp:17-173,
    simulation/VBDSolver.hpp:37-103, simulation/SimulationExecutor.hpp:65-115),
    so code written against the reference's objects ports line by line.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import AvbdError, Params, SolverParams, Stats, check

_dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
_up = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint))
_u8p = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint8))


def _d(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def _u(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class Context:
    """One engine context (a SimulationContext plus its executor) on one GPU."""

    def __init__(self, device: int = 0, particles_capacity: int = 1 << 26, oriented_capacity: int = 1 << 24,
                 energies_capacity: int = 1 << 28, primitives_capacity: int = 1 << 24, sdf_capacity: int = 1 << 20):
        self.L = _lib.load()
        h = C.c_void_p()
        check(self.L.avbd_create(C.byref(h), device, particles_capacity, oriented_capacity, energies_capacity,
                                 primitives_capacity, sdf_capacity))
        self.h = h
        self.device = device
        self._params = Params(1e-3, 60.0, 9.81, 33.0, 1e-3)
        self._solver = SolverParams(1, 0.5, 0.0, 0, _lib.PRECISION_FP32)

    def close(self):
        if getattr(self, "h", None):
            self.L.avbd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters
    def set_params(self, dt, g_accel=9.81, collision_margin=1e-3):
        self._params = Params(dt, 60.0, g_accel, 33.0, collision_margin)
        check(self.L.avbd_set_params(self.h, C.byref(self._params)))

    def set_solver(self, solver_iters, iter_acceleration, residual_tolerance=0.0, max_iters=0, precision=None):
        codes = {"fp32": 0, "fp64": 1, "mixed": 2, 0: 0, 1: 1, 2: 2}
        prec = self._solver.precision if precision is None else codes[precision]
        self._solver = SolverParams(int(solver_iters), float(iter_acceleration), float(residual_tolerance),
                                    int(max_iters), prec)
        check(self.L.avbd_set_solver(self.h, C.byref(self._solver)))

    def set_precision(self, precision):
        self.set_solver(self._solver.solver_iters, self._solver.iter_acceleration, self._solver.residual_tolerance,
                        self._solver.max_iters, precision)

    def set_stream(self, stream_ptr: int | None):
        check(self.L.avbd_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def begin_scene(self):
        out = C.c_uint(0)
        check(self.L.avbd_begin_scene(self.h, C.byref(out)))
        return out.value

    # ---- particles
    def add_particles(self, positions, masses):
        x, m = _d(positions, (-1, 3)), _d(masses)
        first = C.c_uint(0)
        check(self.L.avbd_particles_add(self.h, len(m), _dp(x), _dp(m), C.byref(first)))
        return first.value

    def add_oriented_particles(self, positions, rotations, masses, inertias):
        x, q, m, I = _d(positions, (-1, 3)), _d(rotations, (-1, 4)), _d(masses), _d(inertias, (-1, 3))
        first = C.c_uint(0)
        check(self.L.avbd_particles_add_oriented(self.h, len(m), _dp(x), _dp(q), _dp(m), _dp(I), C.byref(first)))
        return first.value

    def set_fixed(self, slots, fixed):
        s, f = _u(slots), np.ascontiguousarray(fixed, dtype=np.uint8)
        check(self.L.avbd_particles_set_fixed(self.h, len(s), _up(s), _u8p(f)))

    def set_velocities(self, first, velocities, previous_velocities=None):
        v = _d(velocities, (-1, 3))
        vp = _d(previous_velocities, (-1, 3)) if previous_velocities is not None else v
        check(self.L.avbd_set_velocities(self.h, first, len(v), _dp(v), _dp(vp)))

    def set_positions(self, first, positions):
        x = _d(positions, (-1, 3))
        check(self.L.avbd_set_positions(self.h, first, len(x), _dp(x)))

    def set_state(self, positions=None, velocities=None):
        x = _d(positions, (-1, 3)) if positions is not None else None
        v = _d(velocities, (-1, 3)) if velocities is not None else None
        check(self.L.avbd_set_state(self.h, _dp(x) if x is not None else None, _dp(v) if v is not None else None))

    @property
    def num_particles(self):
        n = C.c_uint(0)
        check(self.L.avbd_num_particles(self.h, C.byref(n)))
        return n.value

    # ---- energies
    def add_neo_hookean(self, indices, lam, mu, kd, Q, V):
        idx = _u(indices).reshape(-1, 4)
        n = len(idx)
        first = C.c_uint(0)
        check(self.L.avbd_neo_hookean_add(self.h, n, _up(idx), _dp(_d(lam)), _dp(_d(mu)), _dp(_d(kd)),
                                          _dp(_d(Q, (-1, 9))), _dp(_d(V)), C.byref(first)))
        return first.value

    def add_cosserat_rod(self, indices, stiffness, rest_length, precurvature):
        idx = _u(indices).reshape(-1, 2)
        first = C.c_uint(0)
        check(self.L.avbd_cosserat_rod_add(self.h, len(idx), _up(idx), _dp(_d(stiffness, (-1, 6))),
                                           _dp(_d(rest_length)), _dp(_d(precurvature, (-1, 3))), C.byref(first)))
        return first.value

    def add_ground_collision(self, particle_index, k_start, mu_s, mu_k):
        p = _u(particle_index)
        first = C.c_uint(0)
        check(self.L.avbd_ground_collision_add(self.h, len(p), _up(p), _dp(_d(k_start)), _dp(_d(mu_s)),
                                               _dp(_d(mu_k)), C.byref(first)))
        return first.value

    def add_rigid_body_ground_collision(self, particle_index, shape_type, shape_radius, cp_rb_local, k_start,
                                        mu_s, mu_k):
        p = _u(particle_index)
        st = np.ascontiguousarray(shape_type, dtype=np.uint8)
        first = C.c_uint(0)
        check(self.L.avbd_rigid_body_ground_collision_add(self.h, len(p), _up(p), _u8p(st), _dp(_d(shape_radius)),
                                                          _dp(_d(cp_rb_local, (-1, 3))), _dp(_d(k_start)),
                                                          _dp(_d(mu_s)), _dp(_d(mu_k)), C.byref(first)))
        return first.value

    def add_one_sided_fixed_joint(self, particle_index, position_offset, rotation_offset, ref_position,
                                  ref_rotation):
        p = _u(particle_index)
        first = C.c_uint(0)
        check(self.L.avbd_one_sided_fixed_joint_add(self.h, len(p), _up(p), _dp(_d(position_offset, (-1, 3))),
                                                    _dp(_d(rotation_offset, (-1, 4))), _dp(_d(ref_position, (-1, 3))),
                                                    _dp(_d(ref_rotation, (-1, 4))), C.byref(first)))
        return first.value

    def add_triangles(self, indices, object_id=0):
        idx = _u(indices).reshape(-1, 3)
        first = C.c_uint(0)
        check(self.L.avbd_collision_add_triangles(self.h, len(idx), _up(idx), object_id, C.byref(first)))
        return first.value

    def add_rod_segments(self, indices, radius, object_id=0):
        idx = _u(indices).reshape(-1, 2)
        first = C.c_uint(0)
        check(self.L.avbd_collision_add_rod_segments(self.h, len(idx), _up(idx), float(radius), object_id,
                                                     C.byref(first)))
        return first.value

    def add_spheres(self, particle_index, radius, object_id):
        p = _u(particle_index)
        first = C.c_uint(0)
        check(self.L.avbd_collision_add_spheres(self.h, len(p), _up(p), _dp(_d(radius)), _up(_u(object_id)),
                                                C.byref(first)))
        return first.value

    # ---- set-up / stepping
    def finalize(self):
        check(self.L.avbd_finalize(self.h))

    def step(self, n=1):
        check(self.L.avbd_step(self.h, n))

    def synchronize(self):
        check(self.L.avbd_synchronize(self.h))

    def collision_stage(self):
        check(self.L.avbd_collision_stage(self.h))

    # ---- queries
    def positions(self, out=None):
        n = self.num_particles
        out = np.empty((n, 3)) if out is None else out
        check(self.L.avbd_get_positions(self.h, 0, n, _dp(out)))
        return out

    def velocities(self, out=None):
        n = self.num_particles
        out = np.empty((n, 3)) if out is None else out
        check(self.L.avbd_get_velocities(self.h, 0, n, _dp(out)))
        return out

    def rotations(self, out=None):
        """Unit quaternions (w, x, y, z); identity for positional particles."""
        n = self.num_particles
        out = np.empty((n, 4)) if out is None else out
        check(self.L.avbd_get_rotations(self.h, 0, n, _dp(out)))
        return out

    def angular_velocities(self, out=None):
        n = self.num_particles
        out = np.empty((n, 3)) if out is None else out
        check(self.L.avbd_get_angular_velocities(self.h, 0, n, _dp(out)))
        return out

    def coloring(self):
        out = np.zeros(self.num_particles, dtype=np.uint32)
        nc = C.c_uint(0)
        check(self.L.avbd_get_coloring(self.h, _up(out), C.byref(nc)))
        return out, nc.value

    def lbvh(self):
        n = C.c_uint(0)
        check(self.L.avbd_get_lbvh(self.h, C.byref(n), None, None, None, None, None, None, None, None))
        n = n.value
        nn = max(2 * n - 1, 0)
        out = dict(morton=np.zeros(n, dtype=np.uint64), sorted_order=np.zeros(n, dtype=np.uint32),
                   left=np.zeros(nn, dtype=np.uint32), right=np.zeros(nn, dtype=np.uint32),
                   parent=np.zeros(nn, dtype=np.uint32), subtree_size=np.zeros(nn, dtype=np.uint32),
                   bounds=np.zeros((nn, 6)))
        root = C.c_uint(0)
        cnt = C.c_uint(0)
        check(self.L.avbd_get_lbvh(self.h, C.byref(cnt), out["morton"].ctypes.data_as(C.POINTER(C.c_uint64)),
                                   _up(out["sorted_order"]), _up(out["left"]), _up(out["right"]), _up(out["parent"]),
                                   _up(out["subtree_size"]), _dp(out["bounds"]), C.byref(root)))
        out["root"] = root.value
        out["pairs"] = self.candidate_pairs()
        return out

    def candidate_pairs(self):
        cnt = C.c_uint(0)
        check(self.L.avbd_get_candidate_pairs(self.h, 0, None, C.byref(cnt)))
        out = np.zeros((cnt.value, 2), dtype=np.uint32)
        if cnt.value:
            check(self.L.avbd_get_candidate_pairs(self.h, cnt.value, _up(out), C.byref(cnt)))
        return out

    def contacts(self):
        """Triangle-sphere contacts of the last collision stage, ascending key:
        dict of key [k], tri [k, 3], rigid [k], normal / barys / cp_local [k, 3]."""
        cnt = C.c_uint(0)
        check(self.L.avbd_get_contacts(self.h, 0, None, None, None, C.byref(cnt)))
        n = cnt.value
        keys = np.zeros(n, dtype=np.uint64)
        idx = np.zeros((n, 4), dtype=np.uint32)
        vec = np.zeros((n, 9))
        if n:
            check(self.L.avbd_get_contacts(self.h, n, keys.ctypes.data_as(C.POINTER(C.c_uint64)), _up(idx),
                                           _dp(vec), C.byref(cnt)))
        return {"key": keys, "tri": idx[:, :3], "rigid": idx[:, 3], "normal": vec[:, 0:3], "barys": vec[:, 3:6],
                "cp_local": vec[:, 6:9]}

    def dynamic_info(self):
        """Contact pool and recoloring state of the last step: live contacts,
        pool size, colors, conflicted particles, particles still dirty,
        dynamic adjacency entries."""
        out = np.zeros(8, dtype=np.uint32)
        check(self.L.avbd_dynamic_info(self.h, _up(out)))
        return dict(zip(["live", "pool_size", "colors", "conflicted", "dirty", "entries", "rod_live", "rod_pool_size"],
                        (int(v) for v in out)))

    def contact_pool(self):
        """Triangle-rigid contact pool by slot (layout of avbd_get_contact_pool)."""
        size = C.c_uint(0)
        check(self.L.avbd_get_contact_pool(self.h, 0, None, None, None, C.byref(size)))
        n = size.value
        p4 = np.zeros((n, 4), dtype=np.uint32)
        act = np.zeros(n, dtype=np.uint8)
        d = np.zeros((n, 24))
        if n:
            check(self.L.avbd_get_contact_pool(self.h, n, _up(p4), _u8p(act), _dp(d), C.byref(size)))
        return {"particles": p4, "active": act.astype(bool), "n": d[:, 0:3], "t": d[:, 3:6], "b": d[:, 6:9],
                "barys": d[:, 9:12], "cp_local": d[:, 12:15], "k": d[:, 15:19], "lam": d[:, 19:23],
                "flags": d[:, 23].astype(np.uint8)}

    def rod_contact_pool(self):
        """Triangle-rod contact pool by slot (layout of avbd_get_rod_contact_pool)."""
        size = C.c_uint(0)
        check(self.L.avbd_get_rod_contact_pool(self.h, 0, None, None, None, C.byref(size)))
        n = size.value
        p5 = np.zeros((n, 5), dtype=np.uint32)
        act = np.zeros(n, dtype=np.uint8)
        d = np.zeros((n, 25))
        if n:
            check(self.L.avbd_get_rod_contact_pool(self.h, n, _up(p5), _u8p(act), _dp(d), C.byref(size)))
        return {"particles": p5, "active": act.astype(bool), "n": d[:, 0:3], "t": d[:, 3:6], "b": d[:, 6:9],
                "barys": d[:, 9:12], "cp_local": d[:, 12:15], "s": d[:, 15], "k": d[:, 16:20], "lam": d[:, 20:24],
                "flags": d[:, 24].astype(np.uint8)}

    def rod_contacts(self):
        """Triangle-rod contacts of the last collision stage, ascending key:
        key [k], tri [k, 3], rod [k, 2], normal / barys / cp_local [k, 3], s [k]."""
        cnt = C.c_uint(0)
        check(self.L.avbd_get_rod_contacts(self.h, 0, None, None, None, C.byref(cnt)))
        n = cnt.value
        keys = np.zeros(n, dtype=np.uint64)
        idx = np.zeros((n, 5), dtype=np.uint32)
        vec = np.zeros((n, 10))
        if n:
            check(self.L.avbd_get_rod_contacts(self.h, n, keys.ctypes.data_as(C.POINTER(C.c_uint64)), _up(idx),
                                               _dp(vec), C.byref(cnt)))
        return {"key": keys, "tri": idx[:, :3], "rod": idx[:, 3:5], "normal": vec[:, 0:3], "barys": vec[:, 3:6],
                "cp_local": vec[:, 6:9], "s": vec[:, 9]}

    def scene_iterations(self):
        """Iterations each scene ran in the last run-to-tolerance step."""
        st = self.stats()
        out = np.zeros(st["num_scenes"], dtype=np.uint32)
        check(self.L.avbd_get_scene_iterations(self.h, _up(out)))
        return out

    def set_pair_capacity(self, capacity):
        check(self.L.avbd_debug_set_pair_capacity(self.h, int(capacity)))

    def set_recolor_rounds(self, rounds):
        check(self.L.avbd_debug_set_recolor_rounds(self.h, rounds))

    def debug_block(self, p):
        G, H, dof = np.zeros(6), np.zeros(36), C.c_int(0)
        check(self.L.avbd_debug_block(self.h, p, _dp(G), _dp(H), C.byref(dof)))
        d = dof.value
        return G[:d].copy(), H[: d * d].reshape(d, d).copy()

    def residual(self):
        r = C.c_double(0)
        check(self.L.avbd_residual(self.h, C.byref(r)))
        return r.value

    def set_warmstart(self, mode, params=None):
        """Learned warm start: 0 off (inertial guess), 1 record features and
        targets every step, 2 apply the MLP `params` (FP32 flat array)."""
        p = None
        if params is not None:
            params = np.ascontiguousarray(params, dtype=np.float32)
            p = params.ctypes.data_as(C.POINTER(C.c_float))
        check(self.L.avbd_set_warmstart(self.h, int(mode), p))

    def warmstart_sample(self, features=None, targets=None):
        """Copies the last recorded step's feature rows (BF16 CUDA tensor
        [n, 32]) and target rows (FP32 CUDA tensor [n, 4]; column 3 is 1 on
        solved tet vertices) in internal vertex order; returns n."""
        rows = C.c_uint(0)
        f = features.data_ptr() if features is not None else None
        t = targets.data_ptr() if targets is not None else None
        check(self.L.avbd_warmstart_sample(self.h, f, t, C.byref(rows)))
        return rows.value

    def profile_solve(self, iterations=2):
        """Kernel time (ms) and algorithmic bytes of the per-color solve launches
        of `iterations` further iterations (advances the state)."""
        ms, b, nl = C.c_double(0), C.c_double(0), C.c_uint(0)
        check(self.L.avbd_profile_solve(self.h, iterations, C.byref(ms), C.byref(b), C.byref(nl)))
        return ms.value, b.value, nl.value

    def set_initial_guess(self, positions):
        """The next step's initial guess for every solved positional particle
        (particles x 3), used once in place of the inertial initialisation."""
        if positions is None:
            check(self.L.avbd_set_initial_guess(self.h, None))
            return
        x = _d(positions, (-1, 3))
        check(self.L.avbd_set_initial_guess(self.h, _dp(x)))

    def profile_step(self):
        """One run-to-tolerance step with the timed step's launches: kernel
        time (ms) and algorithmic bytes of its vertex-solve launches, the
        launch count and the iterations (advances the state)."""
        ms, b, nl, it = C.c_double(0), C.c_double(0), C.c_uint(0), C.c_uint(0)
        check(self.L.avbd_profile_step(self.h, C.byref(ms), C.byref(b), C.byref(nl), C.byref(it)))
        return ms.value, b.value, nl.value, it.value

    def stats(self):
        s = Stats()
        check(self.L.avbd_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}


# ------------------------------------------------------------------------
# Reference-named objects (the step API of smtobin/avbd)

class SimulationParams:
    """Sim::SimulationParams (simulation/SimulationParams.hpp:9-16)."""

    def __init__(self, dt=1e-3, end_time=60.0, g_accel=9.81, viewer_refresh_time_ms=33.0, collision_margin=1e-3):
        self.dt, self.end_time, self.g_accel = dt, end_time, g_accel
        self.viewer_refresh_time_ms, self.collision_margin = viewer_refresh_time_ms, collision_margin


class ParticlePool:
    """ParticlePool (common/ParticlePool.hpp:76-285): addParticle / addOrientedParticle / fixed."""

    def __init__(self, ctx: Context):
        self._c = ctx

    def addParticle(self, position, mass):
        return self._c.add_particles(np.asarray(position, dtype=np.float64)[None], [mass])

    def addOrientedParticle(self, position, rotation, mass, rotational_inertia):
        return self._c.add_oriented_particles(np.asarray(position, float)[None], np.asarray(rotation, float)[None],
                                              [mass], np.asarray(rotational_inertia, float)[None])

    def setFixed(self, p_idx, fixed=True):
        self._c.set_fixed([p_idx], [1 if fixed else 0])

    @property
    def positions(self):
        return self._c.positions()

    @property
    def velocities(self):
        return self._c.velocities()


class _Pool:
    def __init__(self, ctx: Context):
        self._c = ctx


class NeoHookeanEnergyPool(_Pool):
    """NeoHookeanEnergyPool::addEnergy (energy/elastic/NeoHookeanEnergyPool.hpp:40-67)."""

    def addEnergy(self, indices, lambda_, mu, kd, Q, rest_volume):
        return self._c.add_neo_hookean(np.asarray(indices)[None], [lambda_], [mu], [kd],
                                       np.asarray(Q, float).reshape(1, 9), [rest_volume])


class CosseratRodEnergyPool(_Pool):
    """CosseratRodEnergyPool::addEnergy (energy/elastic/CosseratRodEnergyPool.hpp:36-51)."""

    def addEnergy(self, indices, stiffness, rest_length, precurvature):
        return self._c.add_cosserat_rod(np.asarray(indices)[None], np.asarray(stiffness, float)[None], [rest_length],
                                        np.asarray(precurvature, float)[None])


class GroundCollisionEnergyPool(_Pool):
    """GroundCollisionEnergyPool::addEnergy (energy/collision/GroundCollisionEnergyPool.hpp:32-43)."""

    def addEnergy(self, particle_index, k_start, mu_s, mu_k):
        return self._c.add_ground_collision([particle_index], [k_start], [mu_s], [mu_k])


class RigidBodyGroundCollisionEnergyPool(_Pool):
    """RigidBodyGroundCollisionEnergyPool::addEnergy (energy/collision/RigidBodyGroundCollisionEnergyPool.hpp:36-58)."""

    def addEnergy(self, particle_index, shape_type, shape_radius, cp_rb_local, k_start, mu_s, mu_k):
        return self._c.add_rigid_body_ground_collision([particle_index], [shape_type], [shape_radius],
                                                       np.asarray(cp_rb_local, float)[None], [k_start], [mu_s], [mu_k])


class OneSidedFixedJointEnergyPool(_Pool):
    """OneSidedFixedJointEnergyPool::addEnergy (energy/joint/OneSidedFixedJointEnergyPool.hpp:36-55)."""

    def addEnergy(self, particle_index, pos_offset, rot_offset, ref_position, ref_rotation):
        return self._c.add_one_sided_fixed_joint([particle_index], np.asarray(pos_offset, float)[None],
                                                 np.asarray(rot_offset, float)[None],
                                                 np.asarray(ref_position, float)[None],
                                                 np.asarray(ref_rotation, float)[None])


class EnergyRegistry:
    """Energy::EnergyRegistry (energy/EnergyRegistry.hpp:17-37): one pool per energy type."""

    def __init__(self, ctx: Context):
        self.neo_hookean = NeoHookeanEnergyPool(ctx)
        self.cosserat_rod = CosseratRodEnergyPool(ctx)
        self.ground_collision = GroundCollisionEnergyPool(ctx)
        self.rigid_body_ground_collision = RigidBodyGroundCollisionEnergyPool(ctx)
        self.one_sided_fixed_joint = OneSidedFixedJointEnergyPool(ctx)


class SimulationContext:
    """Sim::SimulationContext(particles, oriented, energies, prims, sdf)
    (simulation/SimulationContext.hpp:46-59)."""

    def __init__(self, particles_capacity=10000, oriented_particles_capacity=1000, energies_capacity=100000,
                 collision_primitive_capacity=20000, collision_sdf_capacity=1000, device=0):
        self.engine = Context(device, particles_capacity, oriented_particles_capacity, energies_capacity,
                              collision_primitive_capacity, collision_sdf_capacity)
        self.particles = ParticlePool(self.engine)
        self.energies = EnergyRegistry(self.engine)
        self.params = SimulationParams()


class VBDSolver:
    """Sim::VBDSolver(ctx, solver_iters, iter_acceleration) (simulation/VBDSolver.hpp:37-42).
    solve() advances one step on the device (VBDSolver::solve_Parallel)."""

    def __init__(self, ctx: SimulationContext, solver_iters: int, iter_acceleration: float):
        self.ctx, self.solver_iters, self.iter_acceleration = ctx, solver_iters, iter_acceleration
        self._ready = False

    def _setup(self):
        p = self.ctx.params
        e = self.ctx.engine
        e.set_params(p.dt, p.g_accel, p.collision_margin)
        e.set_solver(self.solver_iters, self.iter_acceleration)
        e.finalize()
        self._ready = True

    def solve(self):
        if not self._ready:
            self._setup()
        self.ctx.engine.step(1)


class SimulationExecutor:
    """Sim::SimulationExecutor(ctx, solver_iters, iter_acceleration, num_threads)
    (simulation/SimulationExecutor.hpp:65-115).  num_threads is accepted for
    signature compatibility; the work runs on the context's GPU stream."""

    def __init__(self, ctx: SimulationContext, solver_iters: int, iter_acceleration: float, num_threads: int = 0):
        self._solver = VBDSolver(ctx, solver_iters, iter_acceleration)

    def timeStep(self):
        self._solver.solve()
