// contact_dyn.cuh -- device side of the dynamic contact energies of the
// collision stage: triangle-rigid (pool 0) and triangle-rod (pool 1).
//
// Reference behaviour followed:
//   TriangleRigidCollisionConstraintSolver   energy/collision/TriangleRigidCollisionEnergySolver.hpp:14-118
//   TriangleRodCollisionConstraintSolver     energy/collision/TriangleRodCollisionEnergySolver.hpp:14-149
//   CollisionConstraintEnergySolver          energy/collision/CollisionConstraintEnergySolver.hpp:60-285
//     (updateAfterIteration :60-134, updateAfterTimeStep :141-167, accumulate<DOF> :179-285)
//
// Both contacts are C = (n, t, b) . (cp_body - cp_tri) with cp_tri =
// sum_i bary_i x_i.  Triangle-rigid: cp_body = p + R(q) cp_local.
// Triangle-rod: cp_body = p_mid + R(q_mid) cp_local with p_mid = (1-s) p1 +
// s p2 and q_mid = q1 (+) s (q2 (-) q1).  A triangle vertex's gradients are
// -bary (n, t, b) and it has no constraint Hessian.  For an oriented particle
// only the normal has a gradient (the reference overwrites the tangent and
// binormal ones with zero).  Rigid body: (n, -(R S)^T n) with S =
// skew(cp_local), plus the rotational Hessian blocks sym(R^T skew(d) R S) of
// d = n, t, b scaled by the unclamped multipliers.  Rod node 3 / 4: ((1-s) n
// / s n, -n^T (-R S) dR_s/dR) with dR_s/dR = Exp(s dq)^T - s J_r(s dq)
// J_r^-1(dq)^T for node 3 and s J_r(s dq) J_r^-1(dq) for node 4, and no
// constraint Hessian (Gauss-Newton).
#pragma once

#include "engine.h"
#include "s3math.cuh"

namespace avbd {

// the body-side contact point of contact k of pool `pool`
template <typename R>
AVBD_D V3<R> dyn_body_point(const DevState<R>& s, int pool, unsigned k) {
    const ContactPoolDev<R>& P = s.cp[pool];
    const uint4 id = P.p[k];
    const V3<R> cpl = xyz(P.cpl[k]);
    if (pool == POOL_TRI_RIGID) return xyz(s.x[id.w]) + qrot(q_of(s.q[s.rot[id.w]]), cpl);
    const unsigned b = P.p5[k];
    const R sp = P.n[k].w;
    const Q4<R> q1 = q_of(s.q[s.rot[id.w]]), q2 = q_of(s.q[s.rot[b]]);
    const Q4<R> qm = plus_s3(q1, sp * minus_s3(q2, q1));
    const V3<R> pm = (R(1) - sp) * xyz(s.x[id.w]) + sp * xyz(s.x[b]);
    return pm + qrot(qm, cpl);
}

template <typename R>
AVBD_D void dyn_eval(const DevState<R>& s, int pool, unsigned k, R& Cn, R& Ct, R& Cb) {
    const ContactPoolDev<R>& P = s.cp[pool];
    const uint4 id = P.p[k];
    const typename Vec4Of<R>::T br = P.bar[k];
    const V3<R> cp_tri = br.x * xyz(s.x[id.x]) + br.y * xyz(s.x[id.y]) + br.z * xyz(s.x[id.z]);
    const V3<R> d = dyn_body_point<R>(s, pool, k) - cp_tri;
    Cn = dot3(xyz(P.n[k]), d);
    Ct = dot3(xyz(P.t[k]), d);
    Cb = dot3(xyz(P.b[k]), d);
}

// Multipliers of CollisionConstraintEnergySolver::accumulate: the clamped
// normal multiplier, the friction multipliers clamped to the Coulomb cone,
// and the unclamped ones that scale the constraint Hessians.
template <typename R>
struct ContactMult {
    R lnp, lt, lb;      // gradient weights
    R sn, st, sb;       // constraint-Hessian weights
    R kn, kt, kb;       // stiffnesses (Gauss-Newton terms)
};

template <typename R>
AVBD_D ContactMult<R> dyn_multipliers(const ContactPoolDev<R>& P, unsigned k, R Cn, R Ct, R Cb) {
    const typename Vec4Of<R>::T kk = P.k[k], lam = P.lam[k];
    const bool use_static = P.flag[k] & CF_USE_STATIC;
    const R mu = use_static ? P.bar[k].w : P.cpl[k].w;
    ContactMult<R> m;
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
AVBD_D void dyn_accumulate3(const DevState<P>& s, int pool, unsigned k, unsigned local, Block& B) {
    P Cn, Ct, Cb;
    dyn_eval<P>(s, pool, k, Cn, Ct, Cb);
    const ContactPoolDev<P>& Q = s.cp[pool];
    const ContactMult<P> m = dyn_multipliers<P>(Q, k, Cn, Ct, Cb);
    const typename Vec4Of<P>::T br = Q.bar[k];
    const P bary = local == 0 ? br.x : (local == 1 ? br.y : br.z);
    const V3<P> n = xyz(Q.n[k]), t = xyz(Q.t[k]), b = xyz(Q.b[k]);
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
AVBD_D M3<R> dyn_rot_hess(const M3<R>& Rm, const M3<R>& S, V3<R> d) {
    const M3<R> H = mmul(mmul(mmul(mT(Rm), skew(d)), Rm), S);
    M3<R> o;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) o.a[i][j] = R(0.5) * (H.a[i][j] + H.a[j][i]);
    return o;
}

// The 6x6 block of the oriented particle `local` of contact k (g: 6, h: 6x6
// in R): the rigid body (pool 0, local 3) or a rod node (pool 1, local 3/4).
template <typename R, typename Block>
AVBD_D void dyn_accumulate6(const DevState<R>& s, int pool, unsigned k, unsigned local, Block& B) {
    R Cn, Ct, Cb;
    dyn_eval<R>(s, pool, k, Cn, Ct, Cb);
    const ContactPoolDev<R>& P = s.cp[pool];
    const ContactMult<R> m = dyn_multipliers<R>(P, k, Cn, Ct, Cb);
    const uint4 id = P.p[k];
    const V3<R> n = xyz(P.n[k]);
    const M3<R> S = skew(xyz(P.cpl[k]));
    R gn[6];
    if (pool == POOL_TRI_RIGID) {
        const M3<R> Rm = qmat(q_of(s.q[s.rot[id.w]]));
        const M3<R> RS = mmul(Rm, S);
        gn[0] = n.x; gn[1] = n.y; gn[2] = n.z;
#pragma unroll
        for (int j = 0; j < 3; j++) gn[3 + j] = -(n.x * RS.a[0][j] + n.y * RS.a[1][j] + n.z * RS.a[2][j]);
        const M3<R> Hn = dyn_rot_hess<R>(Rm, S, n);
        const M3<R> Ht = dyn_rot_hess<R>(Rm, S, xyz(P.t[k]));
        const M3<R> Hb = dyn_rot_hess<R>(Rm, S, xyz(P.b[k]));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                B.h[3 + i][3 + j] += m.sn * Hn.a[i][j] + m.st * Ht.a[i][j] + m.sb * Hb.a[i][j];
    } else {
        const R sp = P.n[k].w;
        const Q4<R> q1 = q_of(s.q[s.rot[id.w]]), q2 = q_of(s.q[s.rot[P.p5[k]]]);
        const V3<R> qd = minus_s3(q2, q1);
        const Q4<R> qm = plus_s3(q1, sp * qd);
        const M3<R> Rl = mscale(mmul(qmat(qm), S), R(-1));
        const M3<R> gam_inv = inv_right_jac(qd);
        const M3<R> gam = right_jac(sp * qd);
        M3<R> dR;
        R sc;
        if (local == 3) {
            dR = madd(mT(exp_so3(sp * qd)), mmul(gam, mT(gam_inv)), R(1), -sp);
            sc = R(1) - sp;
        } else {
            dR = mscale(mmul(gam, gam_inv), sp);
            sc = sp;
        }
        const M3<R> M = mmul(Rl, dR);
        gn[0] = sc * n.x; gn[1] = sc * n.y; gn[2] = sc * n.z;
#pragma unroll
        for (int j = 0; j < 3; j++) gn[3 + j] = -(n.x * M.a[0][j] + n.y * M.a[1][j] + n.z * M.a[2][j]);
    }
#pragma unroll
    for (int i = 0; i < 6; i++) {
        B.g[i] += m.lnp * gn[i];
#pragma unroll
        for (int j = 0; j < 6; j++) B.h[i][j] += m.kn * gn[i] * gn[j];
    }
}

// CollisionConstraintEnergySolver::updateAfterIteration for contact k
template <typename R>
AVBD_D void dyn_after_iter(DevState<R>& s, int pool, unsigned k) {
    R Cn, Ct, Cb;
    dyn_eval<R>(s, pool, k, Cn, Ct, Cb);
    ContactPoolDev<R>& P = s.cp[pool];
    typename Vec4Of<R>::T kk = P.k[k], lam = P.lam[k];
    uint8_t f = P.flag[k];
    const R mu_s = P.bar[k].w, mu_k = P.cpl[k].w;
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
    P.k[k] = kk;
    P.lam[k] = lam;
    P.flag[k] = f;
}

// CollisionConstraintEnergySolver::updateAfterTimeStep for contact k (at the
// positions of the step start)
template <typename R>
AVBD_D void dyn_after_step(DevState<R>& s, int pool, unsigned k) {
    ContactPoolDev<R>& P = s.cp[pool];
    typename Vec4Of<R>::T kk = P.k[k], lam = P.lam[k];
    uint8_t f = P.flag[k];
    if (lam.x > R(0)) {
        R Cn, Ct, Cb;
        dyn_eval<R>(s, pool, k, Cn, Ct, Cb);
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
    P.k[k] = kk;
    P.lam[k] = lam;
    P.flag[k] = f;
}

// entry layout of the dynamic adjacency: slot << 4 | pool << 3 | local
AVBD_D unsigned dyn_slot(uint32_t en) { return en >> 4; }
AVBD_D int dyn_pool(uint32_t en) { return (en >> 3) & 1; }
AVBD_D unsigned dyn_local(uint32_t en) { return en & 7u; }

}  // namespace avbd
