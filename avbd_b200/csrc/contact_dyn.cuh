// contact_dyn.cuh -- device side of the triangle-rigid contact energies
// (dynamic energies of the collision stage).
//
// Reference behaviour followed:
//   TriangleRigidCollisionConstraintSolver   energy/collision/TriangleRigidCollisionEnergySolver.hpp:14-118
//   CollisionConstraintEnergySolver          energy/collision/CollisionConstraintEnergySolver.hpp:60-285
//     (updateAfterIteration :60-134, updateAfterTimeStep :141-167, accumulate<DOF> :179-285)
//
// A contact joins three triangle vertices (3-DOF) and one rigid body (6-DOF):
// C = (n, t, b) . (cp_rb - cp_tri) with cp_tri = sum_i bary_i x_i and
// cp_rb = p + R(q) cp_local.  A triangle vertex's gradients are -bary (n, t, b)
// and it has no constraint Hessian.  The rigid body's normal gradient is
// (n, -(R S)^T n) with S = skew(cp_local); its tangent and binormal gradients
// are zero (the reference overwrites them) while the rotational Hessian blocks
// sym(R^T skew(d) R S) of d = n, t, b all enter, scaled by the unclamped
// multipliers.
#pragma once

#include "engine.h"
#include "s3math.cuh"

namespace avbd {

template <typename R>
AVBD_D void trc_eval(const DevState<R>& s, unsigned k, R& Cn, R& Ct, R& Cb) {
    const uint4 id = s.trc_p[k];
    const typename Vec4Of<R>::T br = s.trc_bar[k];
    const V3<R> cp_tri = br.x * xyz(s.x[id.x]) + br.y * xyz(s.x[id.y]) + br.z * xyz(s.x[id.z]);
    const V3<R> cp_rb = xyz(s.x[id.w]) + qrot(q_of(s.q[s.rot[id.w]]), xyz(s.trc_cpl[k]));
    const V3<R> d = cp_rb - cp_tri;
    Cn = dot3(xyz(s.trc_n[k]), d);
    Ct = dot3(xyz(s.trc_t[k]), d);
    Cb = dot3(xyz(s.trc_b[k]), d);
}

// Multipliers of CollisionConstraintEnergySolver::accumulate: the clamped
// normal multiplier, the friction multipliers clamped to the Coulomb cone,
// and the unclamped ones that scale the constraint Hessians.
template <typename R>
struct TrcMult {
    R lnp, lt, lb;      // gradient weights
    R sn, st, sb;       // constraint-Hessian weights
    R kn, kt, kb;       // stiffnesses (Gauss-Newton terms)
};

template <typename R>
AVBD_D TrcMult<R> trc_multipliers(const DevState<R>& s, unsigned k, R Cn, R Ct, R Cb) {
    const typename Vec4Of<R>::T kk = s.trc_k[k], lam = s.trc_lam[k];
    const bool use_static = s.trc_flag[k] & CF_USE_STATIC;
    const R mu = use_static ? s.trc_bar[k].w : s.trc_cpl[k].w;
    TrcMult<R> m;
    const R cc = Cn - R(AVBD_ALPHA) * lam.w;
    m.sn = kk.x * cc + lam.x;
    m.st = kk.y * Ct + lam.y;
    m.sb = kk.z * Cb + lam.z;
    m.lnp = m.sn > R(0) ? m.sn : R(0);
    m.lt = m.st;
    m.lb = m.sb;
    const R mag = sqrt(m.lt * m.lt + m.lb * m.lb);
    const R mx = mu * m.lnp;
    if (mag > mx) {
        m.lt = m.lt / (mag + R(1e-8)) * mx;
        m.lb = m.lb / (mag + R(1e-8)) * mx;
    }
    m.kn = kk.x;
    m.kt = kk.y;
    m.kb = kk.z;
    return m;
}

// The 3x3 block of triangle vertex `local` (0..2) of contact k: gradient in
// P, Hessian in HT (the Block3 of the tet solve).
template <typename P, typename HT, typename Block>
AVBD_D void trc_accumulate3(const DevState<P>& s, unsigned k, unsigned local, Block& B) {
    P Cn, Ct, Cb;
    trc_eval<P>(s, k, Cn, Ct, Cb);
    const TrcMult<P> m = trc_multipliers<P>(s, k, Cn, Ct, Cb);
    const typename Vec4Of<P>::T br = s.trc_bar[k];
    const P bary = local == 0 ? br.x : (local == 1 ? br.y : br.z);
    const V3<P> n = xyz(s.trc_n[k]), t = xyz(s.trc_t[k]), b = xyz(s.trc_b[k]);
    const V3<P> gn = (-bary) * n, gt = (-bary) * t, gb = (-bary) * b;
    B.g0 += m.lnp * gn.x + m.lt * gt.x + m.lb * gb.x;
    B.g1 += m.lnp * gn.y + m.lt * gt.y + m.lb * gb.y;
    B.g2 += m.lnp * gn.z + m.lt * gt.z + m.lb * gb.z;
    B.h00 += (HT)(m.kn * gn.x * gn.x + m.kt * gt.x * gt.x + m.kb * gb.x * gb.x);
    B.h11 += (HT)(m.kn * gn.y * gn.y + m.kt * gt.y * gt.y + m.kb * gb.y * gb.y);
    B.h22 += (HT)(m.kn * gn.z * gn.z + m.kt * gt.z * gt.z + m.kb * gb.z * gb.z);
    B.h01 += (HT)(m.kn * gn.x * gn.y + m.kt * gt.x * gt.y + m.kb * gb.x * gb.y);
    B.h02 += (HT)(m.kn * gn.x * gn.z + m.kt * gt.x * gt.z + m.kb * gb.x * gb.z);
    B.h12 += (HT)(m.kn * gn.y * gn.z + m.kt * gt.y * gt.z + m.kb * gb.y * gb.z);
}

// sym(R^T skew(d) R S), the rotational Hessian block of direction d
template <typename R>
AVBD_D M3<R> trc_rot_hess(const M3<R>& Rm, const M3<R>& S, V3<R> d) {
    const M3<R> H = mmul(mmul(mmul(mT(Rm), skew(d)), Rm), S);
    M3<R> o;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) o.a[i][j] = R(0.5) * (H.a[i][j] + H.a[j][i]);
    return o;
}

// The 6x6 block of the rigid body of contact k (g: 6, h: 6x6 in R).
template <typename R, typename Block>
AVBD_D void trc_accumulate6(const DevState<R>& s, unsigned k, Block& B) {
    R Cn, Ct, Cb;
    trc_eval<R>(s, k, Cn, Ct, Cb);
    const TrcMult<R> m = trc_multipliers<R>(s, k, Cn, Ct, Cb);
    const uint4 id = s.trc_p[k];
    const M3<R> Rm = qmat(q_of(s.q[s.rot[id.w]]));
    const M3<R> S = skew(xyz(s.trc_cpl[k]));
    const M3<R> RS = mmul(Rm, S);
    const V3<R> n = xyz(s.trc_n[k]);
    R gn[6] = {n.x, n.y, n.z, R(0), R(0), R(0)};
#pragma unroll
    for (int j = 0; j < 3; j++) gn[3 + j] = -(n.x * RS.a[0][j] + n.y * RS.a[1][j] + n.z * RS.a[2][j]);
    const M3<R> Hn = trc_rot_hess<R>(Rm, S, n);
    const M3<R> Ht = trc_rot_hess<R>(Rm, S, xyz(s.trc_t[k]));
    const M3<R> Hb = trc_rot_hess<R>(Rm, S, xyz(s.trc_b[k]));
#pragma unroll
    for (int i = 0; i < 6; i++) {
        B.g[i] += m.lnp * gn[i];
#pragma unroll
        for (int j = 0; j < 6; j++) B.h[i][j] += m.kn * gn[i] * gn[j];
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) B.h[3 + i][3 + j] += m.sn * Hn.a[i][j] + m.st * Ht.a[i][j] + m.sb * Hb.a[i][j];
}

// CollisionConstraintEnergySolver::updateAfterIteration for contact k
template <typename R>
AVBD_D void trc_after_iter(DevState<R>& s, unsigned k) {
    R Cn, Ct, Cb;
    trc_eval<R>(s, k, Cn, Ct, Cb);
    typename Vec4Of<R>::T kk = s.trc_k[k], lam = s.trc_lam[k];
    uint8_t f = s.trc_flag[k];
    const R mu_s = s.trc_bar[k].w, mu_k = s.trc_cpl[k].w;
    const R cc = Cn - R(AVBD_ALPHA) * lam.w;
    const R ln = kk.x * cc + lam.x;
    const R lt = kk.y * Ct + lam.y;
    const R lb = kk.z * Cb + lam.z;
    if (ln > R(0)) kk.x += R(AVBD_BETA) * fabs(cc);
    lam.x = ln > R(0) ? ln : R(0);
    const R mag = sqrt(lt * lt + lb * lb);
    const bool use_static = f & CF_USE_STATIC;
    R mx = (use_static ? mu_s : mu_k) * lam.x;
    if (mag < mx) {
        kk.y += R(AVBD_BETA) * fabs(Ct);
        kk.z += R(AVBD_BETA) * fabs(Cb);
        lam.y = lt;
        lam.z = lb;
        f |= CF_UNCLAMPED;
    } else {
        if (use_static) {
            f &= ~CF_USE_STATIC;
            mx = mu_k * ln;
        }
        lam.y = lt / (mag + R(1e-8)) * mx;
        lam.z = lb / (mag + R(1e-8)) * mx;
        f &= ~CF_UNCLAMPED;
    }
    s.trc_k[k] = kk;
    s.trc_lam[k] = lam;
    s.trc_flag[k] = f;
}

// CollisionConstraintEnergySolver::updateAfterTimeStep for contact k (at the
// positions of the step start)
template <typename R>
AVBD_D void trc_after_step(DevState<R>& s, unsigned k) {
    typename Vec4Of<R>::T kk = s.trc_k[k], lam = s.trc_lam[k];
    uint8_t f = s.trc_flag[k];
    if (lam.x > R(0)) {
        R Cn, Ct, Cb;
        trc_eval<R>(s, k, Cn, Ct, Cb);
        lam.w = Cn;
    }
    if ((f & CF_UNCLAMPED) && !(f & CF_USE_STATIC)) f |= CF_USE_STATIC;
    lam.x *= R(AVBD_ALPHA * AVBD_GAMMA);
    lam.y *= R(AVBD_GAMMA);
    lam.z *= R(AVBD_GAMMA);
    R g;
    g = R(AVBD_GAMMA) * kk.x; kk.x = (g < kk.w) ? kk.w : g;
    g = R(AVBD_GAMMA) * kk.y; kk.y = (g < kk.w) ? kk.w : g;
    g = R(AVBD_GAMMA) * kk.z; kk.z = (g < kk.w) ? kk.w : g;
    s.trc_k[k] = kk;
    s.trc_lam[k] = lam;
    s.trc_flag[k] = f;
}

}  // namespace avbd
