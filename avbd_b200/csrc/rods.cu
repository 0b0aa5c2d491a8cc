// rods.cu -- oriented-particle (6-DOF) path: rod nodes and rigid bodies.
//
// Reference behaviour followed:
//   _particleRotationInertialUpdate            simulation/VBDSolver.hpp:253-283
//   _solveParticle<6> (6x6 assembly and solve)  simulation/VBDSolver.hpp:450-486
//   Chebyshev on S^3 / angular velocity update  simulation/VBDSolver.hpp:513-566
//   CosseratRodEnergySolver::accumulate         energy/elastic/CosseratRodEnergySolver.hpp:79-159
//   RigidBodyGroundCollisionConstraintSolver    energy/collision/RigidBodyGroundCollisionEnergySolver.hpp:14-183
//   CollisionConstraintEnergySolver (6-DOF)     energy/collision/CollisionConstraintEnergySolver.hpp:60-285
//   HardConstraintEnergySolver + joint           energy/HardConstraintEnergySolver.hpp:42-155,
//                                                energy/joint/OneSidedFixedJointEnergySolver.hpp:16-90
// One thread per oriented vertex: rod nodes have at most two rod elements, one
// ground contact and one joint, so the block is small and the 6x6 system is
// solved by LU with partial pivoting in FP64.
#include "engine.h"
#include "s3math.cuh"
#include "contact_dyn.cuh"

namespace avbd {

namespace {

constexpr double JOINT_K_START = 1e4;  // OneSidedFixedJointEnergyPool.hpp:27
// threads per block of the 6-DOF solve (one node each).  A color of the
// 256-rod workload has ~13 K nodes; 32, 64 and 128 measured the same step
// time there: each node's serial FP64 chain, not the SM spread, bounds it.
constexpr int ROD_BLOCK = 128;

template <typename R>
struct Block6 {
    R g[6];
    R h[6][6];
};

template <typename R>
AVBD_D void b6_zero(Block6<R>& B) {
#pragma unroll
    for (int i = 0; i < 6; i++) {
        B.g[i] = 0;
#pragma unroll
        for (int j = 0; j < 6; j++) B.h[i][j] = 0;
    }
}

template <typename R>
AVBD_D Q4<R> qload(const typename Vec4Of<R>::T* a, unsigned i) { return q_of(a[i]); }

// CosseratRodEnergySolver::accumulate for node `local` of rod r.
template <typename R>
AVBD_D void accumulate_rod(const DevState<R>& s, unsigned r, unsigned local, Block6<R>& B) {
    uint2 id = s.rod_idx[r];
    typename Vec4Of<R>::T K0 = s.rod_K[2 * r], K1 = s.rod_K[2 * r + 1];
    R K[6] = {K0.x, K0.y, K0.z, K0.w, K1.x, K1.y};
    R L = K1.z;
    V3<R> k0 = xyz(s.rod_k0[r]);
    Q4<R> q1 = qload<R>(s.q, s.rot[id.x]), q2 = qload<R>(s.q, s.rot[id.y]);
    V3<R> p1 = xyz(s.x[id.x]), p2 = xyz(s.x[id.y]);
    R il = R(1) / L;
    V3<R> qd = minus_s3(q2, q1);
    Q4<R> qm = plus_s3(q1, R(0.5) * qd);
    V3<R> sh = il * qrot(qconj(qm), p2 - p1) - mk3<R>(0, 0, 1);
    V3<R> be = il * qd - k0;
    R st[6] = {sh.x, sh.y, sh.z, be.x, be.y, be.z};
    M3<R> gi = inv_right_jac(qd);
    V3<R> th = R(0.5) * qd;
    M3<R> eth = exp_so3(th);
    M3<R> gth = right_jac(th);
    M3<R> Rm = qmat(qm);
    V3<R> dpds = il * (p2 - p1);
    M3<R> S = skew(mvec(mT(Rm), dpds));
    M3<R> A, Bm, C;
    if (local == 0) {
        A = mscale(mT(Rm), -il);
        Bm = mmul(S, madd(mT(eth), mmul(gth, mscale(mT(gi), R(-0.5)))));
        C = mscale(mT(gi), -il);
    } else {
        A = mscale(mT(Rm), il);
        Bm = mmul(S, mmul(gth, mscale(gi, R(0.5))));
        C = mscale(gi, il);
    }
    R SG[6][6];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            SG[i][j] = A.a[i][j];
            SG[i][3 + j] = Bm.a[i][j];
            SG[3 + i][j] = 0;
            SG[3 + i][3 + j] = C.a[i][j];
        }
#pragma unroll
    for (int j = 0; j < 6; j++) {
        R g = 0;
#pragma unroll
        for (int i = 0; i < 6; i++) g += st[i] * K[i] * SG[i][j];
        B.g[j] += L * g;
    }
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int b = a; b < 6; b++) {
            R h = 0;
#pragma unroll
            for (int i = 0; i < 6; i++) h += SG[i][a] * K[i] * SG[i][b];
            B.h[a][b] += L * h;
            if (b != a) B.h[b][a] += L * h;
        }
}

// RigidBodyGroundCollisionConstraintSolver::evaluateConstraint for round shapes
// (spheres and rod segments use the exact contact point p - r e_y).
template <typename R>
AVBD_D void rground_eval(V3<R> p, Q4<R> q, typename Vec4Of<R>::T cp, typename Vec4Of<R>::T loc, R& Cn, R& Ct,
                         R& Cb) {
    V3<R> cp_rb = p + qrot(q, xyz(loc));
    V3<R> diff = mk3<R>(cp.x, 0, cp.y) - cp_rb;  // cp_ground - cp_rb, cp_ground.y = 0
    Ct = diff.x;                                  // tangent (1,0,0)
    Cb = diff.z;                                  // binormal (0,0,1)
    Cn = -(p.y - loc.w);                          // n . (cp_ground - (p - r e_y)), n = (0,1,0)
}

// CollisionConstraintEnergySolver::accumulate<6> with the rigid-body ground
// constraint (frame n = e_y, t = e_x, b = e_z, never updated for this energy).
template <typename R>
AVBD_D void accumulate_rground(const DevState<R>& s, unsigned slot, V3<R> p, Q4<R> q, Block6<R>& B) {
    typename Vec4Of<R>::T k = s.rgk[slot], lam = s.rglam[slot], cp = s.rgcp[slot], loc = s.rgloc[slot];
    uint8_t f = s.oflag[slot];
    R Cn, Ct, Cb;
    rground_eval<R>(p, q, cp, loc, Cn, Ct, Cb);
    M3<R> Rm = qmat(q);
    M3<R> RS = mmul(Rm, skew(xyz(loc)));
    // gradients: n -> (-e_y, 0) for round shapes; t -> (-e_x, row 0 of RS); b -> (-e_z, row 2 of RS)
    R gn[6] = {0, -1, 0, 0, 0, 0};
    R gt[6] = {-1, 0, 0, RS.a[0][0], RS.a[0][1], RS.a[0][2]};
    R gb[6] = {0, 0, -1, RS.a[2][0], RS.a[2][1], RS.a[2][2]};
    // rotational Hessian blocks sym(-R^T skew(d) R skew(cp_local)) for d = t, b
    M3<R> S = skew(xyz(loc));
    M3<R> Ht = mmul(mmul(mmul(mT(Rm), skew(mk3<R>(1, 0, 0))), Rm), S);
    M3<R> Hb = mmul(mmul(mmul(mT(Rm), skew(mk3<R>(0, 0, 1))), Rm), S);
    R cc = Cn - R(AVBD_ALPHA) * lam.w;
    R ln = k.x * cc + lam.x;
    R lnp = ln > R(0) ? ln : R(0);
    R lt = k.y * Ct + lam.y, lb = k.z * Cb + lam.z;
    R mag = sqrt(lt * lt + lb * lb);
    R mu = (f & OF_RG_USE_STATIC) ? cp.z : cp.w;
    R mx = mu * lnp;
    if (mag > mx) {
        R sc = mx / (mag + R(1e-8));
        lt *= sc;
        lb *= sc;
    }
    R st = k.y * Ct + lam.y, sb = k.z * Cb + lam.z;  // multipliers of the constraint Hessians
#pragma unroll
    for (int i = 0; i < 6; i++) {
        B.g[i] += lnp * gn[i] + lt * gt[i] + lb * gb[i];
#pragma unroll
        for (int j = 0; j < 6; j++) B.h[i][j] += k.x * gn[i] * gn[j] + k.y * gt[i] * gt[j] + k.z * gb[i] * gb[j];
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            R ht = -R(0.5) * (Ht.a[i][j] + Ht.a[j][i]);
            R hb = -R(0.5) * (Hb.a[i][j] + Hb.a[j][i]);
            B.h[3 + i][3 + j] += st * ht + sb * hb;
        }
}

// OneSidedFixedJointConstraintSolver::evaluateConstraint
template <typename R>
AVBD_D void joint_eval(const DevState<R>& s, unsigned slot, V3<R> p, Q4<R> q, R C[6]) {
    V3<R> jp = p + qrot(q, xyz(s.jpo[slot]));
    Q4<R> jq = qmul(q, q_of(s.jro[slot]));
    V3<R> a = jp - xyz(s.jrp[slot]);
    V3<R> b = minus_s3(jq, q_of(s.jrq[slot]));
    C[0] = a.x; C[1] = a.y; C[2] = a.z; C[3] = b.x; C[4] = b.y; C[5] = b.z;
}

template <typename R>
AVBD_D void joint_load6(const typename Vec4Of<R>::T* a, unsigned slot, R v[6]) {
    typename Vec4Of<R>::T u = a[2 * slot], w = a[2 * slot + 1];
    v[0] = u.x; v[1] = u.y; v[2] = u.z; v[3] = u.w; v[4] = w.x; v[5] = w.y;
}
template <typename R>
AVBD_D void joint_store6(typename Vec4Of<R>::T* a, unsigned slot, const R v[6]) {
    typename Vec4Of<R>::T u, w;
    u.x = v[0]; u.y = v[1]; u.z = v[2]; u.w = v[3];
    w.x = v[4]; w.y = v[5]; w.z = 0; w.w = 0;
    a[2 * slot] = u;
    a[2 * slot + 1] = w;
}

// HardConstraintEnergySolver::accumulate<6> for the joint: the multipliers are
// unbounded (lambda_min/max = lowest/max), so no clamp or k rescale applies to
// finite values; the constraint Hessian is zero (Gauss-Newton).
template <typename R>
AVBD_D void accumulate_joint(const DevState<R>& s, unsigned slot, V3<R> p, Q4<R> q, Block6<R>& B) {
    R Craw[6], k[6], lam[6], cp[6];
    joint_eval<R>(s, slot, p, q, Craw);
    joint_load6<R>(s.jk, slot, k);
    joint_load6<R>(s.jlam, slot, lam);
    joint_load6<R>(s.jcp, slot, cp);
    M3<R> Rm = qmat(q);
    M3<R> dCp = mscale(mmul(Rm, skew(xyz(s.jpo[slot]))), R(-1));
    M3<R> dCR = mmul(inv_right_jac(mk3(Craw[3], Craw[4], Craw[5])), mT(qmat(q_of(s.jro[slot]))));
    R grad[6][6];
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = 0; j < 6; j++) grad[i][j] = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        grad[i][i] = 1;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            grad[i][3 + j] = dCp.a[i][j];
            grad[3 + i][3 + j] = dCR.a[i][j];
        }
    }
#pragma unroll
    for (int ci = 0; ci < 6; ci++) {
        R C = Craw[ci] - R(AVBD_ALPHA) * cp[ci];
        R lp = k[ci] * C + lam[ci];
#pragma unroll
        for (int a = 0; a < 6; a++) {
            B.g[a] += grad[ci][a] * lp;
#pragma unroll
            for (int b = 0; b < 6; b++) B.h[a][b] += k[ci] * grad[ci][a] * grad[ci][b];
        }
    }
}

template <typename R>
AVBD_D void rground_after_iter(DevState<R>& s, unsigned slot, V3<R> p, Q4<R> q) {
    typename Vec4Of<R>::T k = s.rgk[slot], lam = s.rglam[slot], cp = s.rgcp[slot], loc = s.rgloc[slot];
    uint8_t f = s.oflag[slot];
    R Cn, Ct, Cb;
    rground_eval<R>(p, q, cp, loc, Cn, Ct, Cb);
    R cc = Cn - R(AVBD_ALPHA) * lam.w;
    R ln = k.x * cc + lam.x;
    R lt = k.y * Ct + lam.y;
    R lb = k.z * Cb + lam.z;
    if (ln > R(0)) k.x += R(AVBD_BETA) * fabs(cc);
    lam.x = ln > R(0) ? ln : R(0);
    R mag = sqrt(lt * lt + lb * lb);
    bool use_static = f & OF_RG_USE_STATIC;
    R mx = (use_static ? cp.z : cp.w) * lam.x;
    if (mag < mx) {
        k.y += R(AVBD_BETA) * fabs(Ct);
        k.z += R(AVBD_BETA) * fabs(Cb);
        lam.y = lt;
        lam.z = lb;
        f |= OF_RG_UNCLAMPED;
    } else {
        if (use_static) {
            f &= ~OF_RG_USE_STATIC;
            mx = cp.w * ln;
        }
        lam.y = lt / (mag + R(1e-8)) * mx;
        lam.z = lb / (mag + R(1e-8)) * mx;
        f &= ~OF_RG_UNCLAMPED;
    }
    s.rgk[slot] = k;
    s.rglam[slot] = lam;
    s.oflag[slot] = f;
}

template <typename R>
AVBD_D void joint_after_iter(DevState<R>& s, unsigned slot, V3<R> p, Q4<R> q) {
    R C[6], k[6], lam[6], cp[6];
    joint_eval<R>(s, slot, p, q, C);
    joint_load6<R>(s.jk, slot, k);
    joint_load6<R>(s.jlam, slot, lam);
    joint_load6<R>(s.jcp, slot, cp);
#pragma unroll
    for (int i = 0; i < 6; i++) {
        R cc = C[i] - R(AVBD_ALPHA) * cp[i];
        R lp = k[i] * cc + lam[i];
        k[i] += R(AVBD_BETA) * cc;  // signed (HardConstraintEnergySolver.hpp:66)
        lam[i] = lp;
    }
    joint_store6<R>(s.jk, slot, k);
    joint_store6<R>(s.jlam, slot, lam);
}

// ------------------------------------------------------------- kernels

// Step start of oriented particles: energy hooks (rigid-body ground contact
// point + dual decay, joint decay + C_prev), then the inertial prediction of
// position and rotation.
template <typename R>
__global__ void __launch_bounds__(256) k_begin_step_rot(DevState<R> s, R dt, R g) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    uint8_t fl = s.flags[p];
    if (!(fl & VF_ORIENTED)) return;
    unsigned slot = s.rot[p];
    typename Vec4Of<R>::T x4 = s.x[p];
    V3<R> x = xyz(x4);
    Q4<R> q = q_of(s.q[slot]);
    uint8_t f = s.oflag[slot];
    if (f & OF_RGROUND) {
        // RigidBodyGroundCollisionEnergySolver::updateContactPoints
        typename Vec4Of<R>::T cp = s.rgcp[slot], loc = s.rgloc[slot], k = s.rgk[slot], lam = s.rglam[slot];
        cp.x = x.x;
        cp.y = x.z;
        if (f & OF_RG_ROUND) {
            V3<R> l = qrot(qconj(q), mk3<R>(0, -loc.w, 0));
            loc.x = l.x; loc.y = l.y; loc.z = l.z;
        }
        s.rgcp[slot] = cp;
        s.rgloc[slot] = loc;
        // CollisionConstraintEnergySolver::updateAfterTimeStep
        R Cn, Ct, Cb;
        rground_eval<R>(x, q, cp, loc, Cn, Ct, Cb);
        if (lam.x > R(0)) lam.w = Cn;
        if ((f & OF_RG_UNCLAMPED) && !(f & OF_RG_USE_STATIC)) f |= OF_RG_USE_STATIC;
        lam.x *= R(AVBD_ALPHA * AVBD_GAMMA);
        lam.y *= R(AVBD_GAMMA);
        lam.z *= R(AVBD_GAMMA);
        R gk;
        gk = R(AVBD_GAMMA) * k.x; k.x = (gk < k.w) ? k.w : gk;
        gk = R(AVBD_GAMMA) * k.y; k.y = (gk < k.w) ? k.w : gk;
        gk = R(AVBD_GAMMA) * k.z; k.z = (gk < k.w) ? k.w : gk;
        s.rgk[slot] = k;
        s.rglam[slot] = lam;
        s.oflag[slot] = f;
    }
    if (f & OF_JOINT) {
        // HardConstraintEnergySolver::updateAfterTimeStep
        R k[6], lam[6], C[6];
        joint_load6<R>(s.jk, slot, k);
        joint_load6<R>(s.jlam, slot, lam);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            lam[i] = R(AVBD_ALPHA * AVBD_GAMMA) * lam[i];
            R gk = R(AVBD_GAMMA) * k[i];
            k[i] = (R(JOINT_K_START) < gk) ? gk : R(JOINT_K_START);  // k_start.cwiseMax(gamma k)
        }
        joint_eval<R>(s, slot, x, q, C);
        joint_store6<R>(s.jk, slot, k);
        joint_store6<R>(s.jlam, slot, lam);
        joint_store6<R>(s.jcp, slot, C);
    }
    if (fl & VF_FIXED) return;
    // positional inertial update with adaptive initialisation
    V3<R> v = xyz(s.v[p]), vp = xyz(s.vp[p]);
    V3<R> a = (R(1) / dt) * (v - vp);
    V3<R> aext = mk3<R>(0, -g, 0);
    R t = 0;
    if (g > R(1e-12)) {
        R al = dot3(a, aext) / g;
        if (al > g) t = 1;
        else if (al < R(0)) t = 0;
        else t = al / g;
    }
    V3<R> y = (x + dt * v) + (dt * dt) * aext;
    V3<R> xn = x + (dt * v + (dt * dt) * (t * aext));
    typename Vec4Of<R>::T y4 = s.y[p];
    s.y[p] = make4<R>(y, y4.w);
    typename Vec4Of<R>::T o = make4<R>(xn, x4.w);
    s.x[p] = o;
    s.xl[p] = o;
    s.xll[p] = o;
    // rotational inertial update (no external angular acceleration)
    V3<R> w = xyz(s.w[slot]), I = xyz(s.Iv[slot]);
    V3<R> Iw = mk3(I.x * w.x, I.y * w.y, I.z * w.z);
    V3<R> wx = cross3(w, Iw);
    V3<R> acc = mk3(-wx.x / I.x, -wx.y / I.y, -wx.z / I.z);
    V3<R> dqi = dt * w + (dt * dt) * acc;
    s.qy[slot] = q_store(plus_s3_stored(q, dqi));
    Q4<R> qn = plus_s3_stored(q, dt * w);
    s.q[slot] = q_store(qn);
    s.ql[slot] = q_store(qn);
    s.qll[slot] = q_store(qn);
}

enum { RMODE_SOLVE = 0, RMODE_RESIDUAL = 1, RMODE_DEBUG = 2 };

// LANES threads per node.  The rod elements (at most two) and the node's
// dynamic contact terms (triangle-rigid then triangle-rod, each in slot order,
// VBDSolver.hpp:397-446) are spread over the lanes and summed by shuffles;
// the first lane adds the rigid-ground and joint terms and solves.  One lane
// serves the static slabs; the lists of vertices with contacts use 8, since a
// rod node may carry many contacts, each a chain of rotation and Jacobian
// functions.
// FP32 solve of a symmetric positive definite 6x6 block: Jacobi scaling
// (A_s = S A S, S = diag(A)^-1/2) and an LDL^T factorisation of A_s.  A rod
// node's block mixes translational stiffness (EA/L ~ 1e5 N/m) with
// rotational terms (EI/L ~ 1 N m) and has a 2-norm condition number ~2e5;
// scaled, ~2 (at most ~10 on 256 rods of 100 segments).  Returns the pivot ratio
// max(d)/min(d) of the scaled factorisation as the condition estimate
// (infinite when a pivot is not positive); the caller re-solves in FP64
// above its threshold.
AVBD_D float ldlt6_scaled(const float (&A)[6][6], const float (&b)[6], float (&x)[6]) {
    float sc[6], L[6][6], d[6], y[6];
#pragma unroll
    for (int i = 0; i < 6; i++) sc[i] = A[i][i] > 0.f ? rsqrtf(A[i][i]) : 0.f;
    float dmin = 3.402823e38f, dmax = 0.f;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        float dj = A[j][j] * sc[j] * sc[j];
#pragma unroll
        for (int k = 0; k < j; k++) dj -= L[j][k] * L[j][k] * d[k];
        d[j] = dj;
        dmin = fminf(dmin, dj);
        dmax = fmaxf(dmax, dj);
        const float inv = 1.f / dj;
#pragma unroll
        for (int i = j + 1; i < 6; i++) {
            float v = A[i][j] * sc[i] * sc[j];
#pragma unroll
            for (int k = 0; k < j; k++) v -= L[i][k] * L[j][k] * d[k];
            L[i][j] = v * inv;
        }
    }
    if (!(dmin > 0.f)) return 3.402823e38f;
#pragma unroll
    for (int i = 0; i < 6; i++) {  // L y = S b
        float v = b[i] * sc[i];
#pragma unroll
        for (int k = 0; k < i; k++) v -= L[i][k] * y[k];
        y[i] = v;
    }
#pragma unroll
    for (int i = 0; i < 6; i++) y[i] /= d[i];
#pragma unroll
    for (int i = 5; i >= 0; i--) {  // L^T z = y, x = S z
        float v = y[i];
#pragma unroll
        for (int k = i + 1; k < 6; k++) v -= L[k][i] * y[k];
        y[i] = v;
        x[i] = v * sc[i];
    }
    return dmax / dmin;
}

template <typename R, int MODE, int LANES>
__global__ void __launch_bounds__(ROD_BLOCK) k_solve_rod(DevState<R> s, unsigned begin, unsigned count, R dt, double g,
                                                   double* out, SceneTol T, const uint32_t* __restrict__ list,
                                                   double kappa_max, unsigned long long* counters) {
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned gi = tid / LANES, lane = tid % LANES;
    if (LANES == 1 && gi >= count) return;
    // with several lanes no thread returns before the shuffles, which need the whole warp
    bool active = gi < count;
    const unsigned p = active ? (list ? list[gi] : begin + gi) : 0u;
    const uint8_t fl = active ? s.flags[p] : 0;
    if (!(fl & VF_ORIENTED) || (fl & VF_FIXED)) active = false;
    // a recolored vertex is solved from its new color's list, not its slab
    if (MODE == RMODE_SOLVE && active && !list && s.dyn_skip && s.dyn_skip[p]) active = false;
    if (MODE == RMODE_SOLVE && active && T.active && !T.active[T.scene[p]]) active = false;
    if (MODE == RMODE_RESIDUAL && active && T.cand && !T.cand[T.scene[p]]) active = false;
    if (LANES == 1 && !active) return;
    Block6<R> B;
    b6_zero(B);
    if (active) {
        const unsigned re = s.rod_begin[p + 1];
        for (unsigned k = s.rod_begin[p] + lane; k < re; k += LANES) {
            const unsigned e = s.rod_inc[k];
            accumulate_rod<R>(s, e >> 1, e & 1u, B);
        }
        if (s.dyn_begin) {
            const unsigned de = s.dyn_begin[p + 1];
            for (unsigned k = s.dyn_begin[p] + lane; k < de; k += LANES) {
                const uint32_t en = s.dyn_ent[k];
                dyn_accumulate6<R>(s, dyn_pool(en), dyn_slot(en), dyn_local(en), B);
            }
        }
    }
    if constexpr (LANES > 1) {
        // rod and contact blocks are symmetric: the gradient and upper triangle travel
#pragma unroll
        for (int m = LANES / 2; m >= 1; m >>= 1) {
#pragma unroll
            for (int i = 0; i < 6; i++) B.g[i] += __shfl_xor_sync(0xffffffffu, B.g[i], m);
#pragma unroll
            for (int a = 0; a < 6; a++)
#pragma unroll
                for (int b = a; b < 6; b++) B.h[a][b] += __shfl_xor_sync(0xffffffffu, B.h[a][b], m);
        }
#pragma unroll
        for (int a = 0; a < 6; a++)
#pragma unroll
            for (int b = a + 1; b < 6; b++) B.h[b][a] = B.h[a][b];
        if (!active || lane != 0) return;
    }
    const unsigned slot = s.rot[p];
    const V3<R> x = xyz(s.x[p]);
    const Q4<R> q = q_of(s.q[slot]);
    uint8_t f = s.oflag[slot];
    if (f & OF_RGROUND) accumulate_rground<R>(s, slot, x, q, B);
    if (f & OF_JOINT) accumulate_joint<R>(s, slot, x, q, B);
    typename Vec4Of<R>::T y4 = s.y[p];
    R m = y4.w;
    V3<R> I = xyz(s.Iv[slot]);
    R idt2 = R(1) / (dt * dt);
    V3<R> dp = x - xyz(y4);
    V3<R> dr = minus_s3(q, q_of(s.qy[slot]));
    double rhs[6];
    rhs[0] = (double)(-idt2 * m * dp.x) - (double)B.g[0];
    rhs[1] = (double)(-idt2 * m * dp.y) - (double)B.g[1];
    rhs[2] = (double)(-idt2 * m * dp.z) - (double)B.g[2];
    rhs[3] = (double)(-idt2 * (I.x * dr.x)) - (double)B.g[3];
    rhs[4] = (double)(-idt2 * (I.y * dr.y)) - (double)B.g[4];
    rhs[5] = (double)(-idt2 * (I.z * dr.z)) - (double)B.g[5];
    if constexpr (MODE == RMODE_RESIDUAL) {
        double r2 = 0;
        for (int i = 0; i < 6; i++) r2 += rhs[i] * rhs[i];
        if (T.ex) {
            atomicAdd(T.ex + T.scene[p], r2);
        } else {
            double mg = (double)m * g;
            atomicAdd(out, r2);
            atomicAdd(out + 1, mg * mg);
        }
        return;
    }
    if constexpr (MODE == RMODE_DEBUG) {
        for (int i = 0; i < 6; i++) out[i] = B.g[i];
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) out[6 + 6 * i + j] = B.h[i][j];
        return;
    }
    if (T.r2) {
        double r2 = 0;
        for (int i = 0; i < 6; i++) r2 += rhs[i] * rhs[i];
        atomicAdd(T.r2 + T.scene[p], r2);
    }
    double dx[6];
    bool solved = false;
    if constexpr (sizeof(R) == 4) {
        // FP32 mode: scaled FP32 LDL^T, FP64 only above the condition threshold
        float Af[6][6], bf[6], xf[6];
#pragma unroll
        for (int i = 0; i < 6; i++) {
#pragma unroll
            for (int j = 0; j < 6; j++) Af[i][j] = (float)B.h[i][j];
            bf[i] = (float)rhs[i];
        }
        const float mhf = m * idt2;
        Af[0][0] += mhf;
        Af[1][1] += mhf;
        Af[2][2] += mhf;
        Af[3][3] += I.x * idt2;
        Af[4][4] += I.y * idt2;
        Af[5][5] += I.z * idt2;
        const float kap = ldlt6_scaled(Af, bf, xf);
        if (kap <= (float)kappa_max) {
#pragma unroll
            for (int i = 0; i < 6; i++) dx[i] = (double)xf[i];
            solved = true;
        } else if (counters) {
            atomicAdd(counters, 1ull);
        }
    }
    if (!solved) {
        double A[6][6];
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) A[i][j] = (double)B.h[i][j];
        double mh = (double)m * (double)idt2;
        A[0][0] += mh;
        A[1][1] += mh;
        A[2][2] += mh;
        A[3][3] += (double)I.x * (double)idt2;
        A[4][4] += (double)I.y * (double)idt2;
        A[5][5] += (double)I.z * (double)idt2;
        lu_solve_d<6>(A, rhs, dx);
    }
    V3<R> xn = x + mk3<R>((R)dx[0], (R)dx[1], (R)dx[2]);
    if (s.conflicted && s.conflicted[p]) {
        // intra-color conflict: the position is buffered and committed after the
        // color; the rotation update is dropped, as the reference commits
        // positions only (VBDSolver.hpp:108-119,474-479)
        s.buffered[p] = make4<R>(xn, R(0));
        return;
    }
    s.x[p] = make4<R>(xn, R(0));
    s.q[slot] = q_store(plus_s3_stored(q, mk3<R>((R)dx[3], (R)dx[4], (R)dx[5])));
}

// Chebyshev acceleration of oriented particles (position and rotation) fused
// with the dual updates of their rigid-body ground contact and joint.
template <typename R>
__global__ void __launch_bounds__(256) k_chebyshev_rot(DevState<R> s, R omega, unsigned it, SceneTol T) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    uint8_t fl = s.flags[p];
    if (!(fl & VF_ORIENTED)) return;
    if (T.active && !T.active[T.scene[p]]) return;
    if (T.omega) omega = (R)*T.omega;
    if (T.it) it = *T.it;
    unsigned slot = s.rot[p];
    typename Vec4Of<R>::T* h = (it & 1u) ? s.xll : s.xl;  // position history by parity
    typename Vec4Of<R>::T x4 = s.x[p], ll4 = h[p];
    V3<R> xn = omega * (xyz(x4) - xyz(ll4)) + xyz(ll4);
    typename Vec4Of<R>::T o = make4<R>(xn, x4.w);
    s.x[p] = o;
    h[p] = o;
    Q4<R> q = q_of(s.q[slot]), qll = q_of(s.qll[slot]);
    Q4<R> qn = plus_s3_stored(qll, omega * minus_s3(q, qll));
    s.q[slot] = q_store(qn);
    s.qll[slot] = s.ql[slot];
    s.ql[slot] = q_store(qn);
    uint8_t f = s.oflag[slot];
    if (f & OF_RGROUND) rground_after_iter<R>(s, slot, xn, qn);
    if (f & OF_JOINT) joint_after_iter<R>(s, slot, xn, qn);
}

template <typename R>
__global__ void __launch_bounds__(256) k_velocity_rot(DevState<R> s, R inv_dt) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    if (!(s.flags[p] & VF_ORIENTED)) return;
    unsigned slot = s.rot[p];
    typename Vec4Of<R>::T x4 = s.x[p], xp4 = s.xp[p];
    s.vp[p] = s.v[p];
    s.v[p] = make4<R>(inv_dt * (xyz(x4) - xyz(xp4)), R(0));
    s.xp[p] = x4;
    if (!isfinite(x4.x + x4.y + x4.z)) atomicExch(s.err, (int)AVBD_ERR_NAN);
    Q4<R> q = q_of(s.q[slot]);
    s.wp[slot] = s.w[slot];
    s.w[slot] = make4<R>(inv_dt * minus_s3(q, q_of(s.qp[slot])), R(0));
    s.qp[slot] = s.q[slot];
}

// rotations (which 0) or angular velocities (which 1) in external order
template <typename R>
__global__ void k_store_rot(DevState<R> s, int which, double* dst, const uint32_t* inv_map, unsigned n) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned p = inv_map[i];
    if (!(s.flags[p] & VF_ORIENTED)) {
        if (which == 0) { dst[4 * i] = 1; dst[4 * i + 1] = dst[4 * i + 2] = dst[4 * i + 3] = 0; }
        else { dst[3 * i] = dst[3 * i + 1] = dst[3 * i + 2] = 0; }
        return;
    }
    unsigned slot = s.rot[p];
    if (which == 0) {
        typename Vec4Of<R>::T a = s.q[slot];
        dst[4 * i] = a.x; dst[4 * i + 1] = a.y; dst[4 * i + 2] = a.z; dst[4 * i + 3] = a.w;
    } else {
        typename Vec4Of<R>::T a = s.w[slot];
        dst[3 * i] = a.x; dst[3 * i + 1] = a.y; dst[3 * i + 2] = a.z;
    }
}

inline unsigned nblk(unsigned n, unsigned per) { return (n + per - 1) / per; }

}  // namespace

template <typename R>
void launch_begin_step_rot(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    if (s.no == 0) return;
    k_begin_step_rot<R><<<nblk(s.n, 256), 256, 0, st>>>(s, (R)k.dt, (R)k.g);
    count_launch(c);
}

template <typename R>
void launch_solve_rod(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned begin, unsigned count,
                      cudaStream_t st, const SceneTol& T, int mode, double* out, const uint32_t* list) {
    if (count == 0) return;
    // nodes with contacts (lists; the debug pass) take 8 lanes, the static
    // slabs two (a node's rod elements split over a lane pair: 1,289 against
    // 1,225 steps/s with one lane and 893 with eight on 256 rods x 100)
    const double km = k.kappa_max;
    unsigned long long* ctr = c->d_counters;  // [0]: blocks solved in FP64
    if (mode == RMODE_RESIDUAL)
        k_solve_rod<R, RMODE_RESIDUAL, 1><<<nblk(count, ROD_BLOCK), ROD_BLOCK, 0, st>>>(s, begin, count, (R)k.dt, k.g, out, T, list, km, ctr);
    else if (mode == RMODE_DEBUG)
        k_solve_rod<R, RMODE_DEBUG, 8><<<nblk(8 * count, ROD_BLOCK), ROD_BLOCK, 0, st>>>(s, begin, count, (R)k.dt, k.g, out, T, list, km, ctr);
    else if (list)
        k_solve_rod<R, RMODE_SOLVE, 8><<<nblk(8 * count, ROD_BLOCK), ROD_BLOCK, 0, st>>>(s, begin, count, (R)k.dt, k.g, out, T, list, km, ctr);
    else
        k_solve_rod<R, RMODE_SOLVE, 2><<<nblk(2 * count, ROD_BLOCK), ROD_BLOCK, 0, st>>>(s, begin, count, (R)k.dt, k.g, out, T, list, km, ctr);
    count_launch(c);
}

template <typename R>
void launch_chebyshev_rot(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double omega, unsigned it, cudaStream_t st,
                          const SceneTol& T) {
    (void)k;
    if (s.no == 0) return;
    k_chebyshev_rot<R><<<nblk(s.n, 256), 256, 0, st>>>(s, (R)omega, it, T);
    count_launch(c);
}

template <typename R>
void launch_velocity_rot(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    if (s.no == 0) return;
    k_velocity_rot<R><<<nblk(s.n, 256), 256, 0, st>>>(s, (R)(1.0 / k.dt));
    count_launch(c);
}

template <typename R>
void launch_store_rot(const DevState<R>& s, int which, double* dst, const uint32_t* inv_map, unsigned n,
                      cudaStream_t st) {
    if (n == 0) return;
    k_store_rot<R><<<nblk(n, 256), 256, 0, st>>>(s, which, dst, inv_map, n);
}

#define INST(R)                                                                                                 \
    template void launch_begin_step_rot<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t);         \
    template void launch_solve_rod<R>(avbd_ctx*, DevState<R>&, const StepConsts&, unsigned, unsigned,          \
                                      cudaStream_t, const SceneTol&, int, double*, const uint32_t*);           \
    template void launch_chebyshev_rot<R>(avbd_ctx*, DevState<R>&, const StepConsts&, double, unsigned, cudaStream_t,    \
                                          const SceneTol&);                                                     \
    template void launch_velocity_rot<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t);            \
    template void launch_store_rot<R>(const DevState<R>&, int, double*, const uint32_t*, unsigned, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace avbd
