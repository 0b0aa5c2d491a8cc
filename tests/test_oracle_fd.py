"""Finite-difference pins of the FP64 oracle on the inputs of the reference's
own accumulate tests.

The reference tests print FD comparisons without asserting
(test/test_neohookean_accumulate.cpp:88-154, test/test_cosserat_accumulate.cpp:25-70,
test/test_one_sided_fixed_joint_accumulate.cpp:25-70, FD scheme in
test/finite_difference.hpp:6-50).  Here the same inputs and the same schemes
are asserted.  For a single NeoHookean vertex the block Hessian is exact (det F
is linear in each vertex, the deviatoric and damping terms are quadratic and
quartic with exact second derivatives), so gradient and Hessian are both
checked; the Cosserat and joint Hessians are Gauss-Newton, so those are checked
where Gauss-Newton is exact (zero residual).
"""
import numpy as np
import pytest

from conftest import golden


def _nh_oracle(oracle_lib, fx):
    o = oracle_lib.Oracle()
    o.set_params(fx["dt"])
    V = np.array(fx["vertices"], dtype=np.float64)
    o.add_particles(V, np.ones(4))
    X = np.stack([V[0] - V[3], V[1] - V[3], V[2] - V[3]], axis=1)
    Q = np.linalg.inv(X)
    o.add_neo_hookean([[0, 1, 2, 3]], [fx["lambda"]], [fx["mu"]], [fx["kd"]], Q.reshape(1, 9), [fx["rest_volume"]])
    o.after_time_step()  # E_prev at the rest state (NeoHookeanEnergySolver::updateAfterTimeStep)
    Vp = V + np.array(fx["perturbations"])
    o.set_positions_raw(0, Vp)
    return o, Vp


@pytest.mark.parametrize("local", [0, 1, 2, 3])
def test_neohookean_gradient_and_hessian_fd(oracle_lib, local):
    fx = golden("neohookean_element0.json")
    o, Vp = _nh_oracle(oracle_lib, fx)
    G, H = o.element_accumulate(oracle_lib.NEO_HOOKEAN, 0, local)
    E0 = o.energy(oracle_lib.NEO_HOOKEAN, 0)
    # central differences (more accurate than the reference's forward scheme)
    d = 1e-5
    Gfd = np.zeros(3)
    Hfd = np.zeros((3, 3))
    for k in range(3):
        for sgn in (+1, -1):
            P = Vp.copy()
            P[local, k] += sgn * d
            o.set_positions_raw(0, P)
            Gs, _ = o.element_accumulate(oracle_lib.NEO_HOOKEAN, 0, local)
            Es = o.energy(oracle_lib.NEO_HOOKEAN, 0)
            Gfd[k] += sgn * Es / (2 * d)
            Hfd[:, k] += sgn * Gs / (2 * d)
    o.set_positions_raw(0, Vp)
    assert np.isfinite(E0)
    np.testing.assert_allclose(G, Gfd, rtol=1e-6, atol=1e-6 * np.abs(G).max())
    np.testing.assert_allclose(H, Hfd, rtol=1e-5, atol=1e-6 * np.abs(H).max())
    np.testing.assert_allclose(H, H.T, rtol=1e-12, atol=1e-12 * np.abs(H).max())


def test_neohookean_forward_fd_matches_reference_scheme(oracle_lib):
    """The reference's own one-sided scheme with delta = 1e-6."""
    fx = golden("neohookean_element0.json")
    o, Vp = _nh_oracle(oracle_lib, fx)
    for local in range(4):
        G, _ = o.element_accumulate(oracle_lib.NEO_HOOKEAN, 0, local)
        E0 = o.energy(oracle_lib.NEO_HOOKEAN, 0)
        Gfd = np.zeros(3)
        for k in range(3):
            P = Vp.copy()
            P[local, k] += 1e-6
            o.set_positions_raw(0, P)
            Gfd[k] = (o.energy(oracle_lib.NEO_HOOKEAN, 0) - E0) / 1e-6
            o.set_positions_raw(0, Vp)
        np.testing.assert_allclose(G, Gfd, rtol=1e-4, atol=1e-4 * np.abs(G).max())


def _oriented_fd(o, oracle_lib, slot_particle, etype, slot, eps=1e-6):
    """Gradient_FD / Hessian_FD of test/finite_difference.hpp on the perturbation
    [dp, dtheta] applied as p += dp, q = q * Exp_s3(dtheta)."""
    p0 = o.positions()[slot_particle].copy()
    q0 = o.rotations()[slot_particle].copy()

    def F(dx):
        o.set_positions_raw(slot_particle, (p0 + dx[:3])[None])
        o.set_rotations_raw(slot_particle, oracle_lib.plus_s3(q0, dx[3:])[None])
        e = o.energy(etype, slot)
        o.set_positions_raw(slot_particle, p0[None])
        o.set_rotations_raw(slot_particle, q0[None])
        return e

    G = np.zeros(6)
    for i in range(6):
        e = np.zeros(6)
        e[i] = eps
        G[i] = (F(e) - F(-e)) / (2 * eps)
    H = np.zeros((6, 6))
    h = 1e-4
    for i in range(6):
        for j in range(6):
            ei = np.zeros(6); ei[i] = h
            ej = np.zeros(6); ej[j] = h
            H[i, j] = (F(ei + ej) - F(ei - ej) - F(-ei + ej) + F(-ei - ej)) / (4 * h * h)
    return G, H


def _cosserat_oracle(oracle_lib, fx, p2=None, q2=None):
    o = oracle_lib.Oracle()
    o.set_params(fx["dt"])
    q1 = oracle_lib.quat_from_xyz_euler(fx["euler1_deg"])
    q2 = oracle_lib.quat_from_xyz_euler(fx["euler2_deg"]) if q2 is None else q2
    p2 = np.array(fx["p2"], dtype=float) if p2 is None else p2
    o.add_oriented_particles(np.array([fx["p1"], p2], dtype=float), np.stack([q1, q2]), [fx["mass"]] * 2,
                             np.array([fx["inertia"]] * 2, dtype=float))
    o.add_cosserat_rod([[0, 1]], np.array([fx["stiffness"]]), [fx["rest_length"]], np.array([fx["precurvature"]]))
    return o


@pytest.mark.parametrize("local", [0, 1])
def test_cosserat_gradient_fd(oracle_lib, local):
    fx = golden("cosserat_pair.json")
    o = _cosserat_oracle(oracle_lib, fx)
    G, H = o.element_accumulate(oracle_lib.COSSERAT_ROD, 0, local)
    Gfd, _ = _oriented_fd(o, oracle_lib, local, oracle_lib.COSSERAT_ROD, 0)
    np.testing.assert_allclose(G, Gfd, rtol=1e-6, atol=1e-7 * max(1.0, np.abs(G).max()))
    np.testing.assert_allclose(H, H.T, atol=1e-12)
    assert np.linalg.eigvalsh(H).min() > -1e-10  # Gauss-Newton: positive semi-definite


@pytest.mark.parametrize("local", [0, 1])
def test_cosserat_hessian_fd_near_rest(oracle_lib, local):
    """Near zero strain the Gauss-Newton Hessian equals the exact one."""
    fx = golden("cosserat_pair.json")
    q1 = oracle_lib.quat_from_xyz_euler(fx["euler1_deg"])
    L = fx["rest_length"]
    p2 = np.array([0.0, 0.0, L]) + 1e-7
    o = _cosserat_oracle(oracle_lib, fx, p2=p2, q2=q1)
    _, H = o.element_accumulate(oracle_lib.COSSERAT_ROD, 0, local)
    _, Hfd = _oriented_fd(o, oracle_lib, local, oracle_lib.COSSERAT_ROD, 0)
    np.testing.assert_allclose(H, Hfd, rtol=2e-3, atol=2e-3 * np.abs(H).max())


def test_joint_gradient_fd(oracle_lib):
    fx = golden("joint.json")
    o = oracle_lib.Oracle()
    o.set_params(fx["dt"])
    o.add_oriented_particles(np.array([fx["p"]], dtype=float), np.array([[1.0, 0, 0, 0]]), [fx["mass"]],
                             np.array([fx["inertia"]], dtype=float))
    o.add_one_sided_fixed_joint([0], np.array([fx["position_offset"]]),
                                oracle_lib.quat_from_xyz_euler(fx["rotation_offset_euler_deg"])[None],
                                np.array([fx["ref_position"]]),
                                oracle_lib.quat_from_xyz_euler(fx["ref_rotation_euler_deg"])[None])
    G, H = o.element_accumulate(oracle_lib.JOINT, 0, 0)
    Gfd, _ = _oriented_fd(o, oracle_lib, 0, oracle_lib.JOINT, 0)
    np.testing.assert_allclose(G, Gfd, rtol=1e-6, atol=1e-6 * np.abs(G).max())
    np.testing.assert_allclose(H, H.T, atol=1e-9 * np.abs(H).max())
