// solve.cu -- per-step kernels of the AVBD solve for positional (3-DOF)
// vertices: step-start energy hooks + inertial prediction, the per-color
// vertex block solve over NeoHookean tets and ground contact, Chebyshev
// acceleration fused with the contact dual update, the velocity update and
// the residual reduction.
//
// Reference behaviour followed:
//   VBDSolver::solve_Parallel step schedule     simulation/VBDSolver.hpp:48-103
//   _particleInertialUpdate                      simulation/VBDSolver.hpp:208-248
//   _solveParticle<3>                            simulation/VBDSolver.hpp:285-511
//   _particleChebyshevAcceleration               simulation/VBDSolver.hpp:513-536
//   _particleVelocityUpdate                      simulation/VBDSolver.hpp:538-566
//   NeoHookeanEnergySolver::accumulate           energy/elastic/NeoHookeanEnergySolver.hpp:121-227
//   NeoHookeanEnergySolver::updateAfterTimeStep  energy/elastic/NeoHookeanEnergySolver.hpp:70-90
//   CollisionConstraintEnergySolver (ground)     energy/collision/CollisionConstraintEnergySolver.hpp:60-285
//   GroundCollisionEnergySolver                  energy/collision/GroundCollisionEnergySolver.hpp:14-91
#include <cuda_bf16.h>

#include "engine.h"
#include "contact_dyn.cuh"

namespace avbd {

template <typename R>
struct Consts {
    R dt, inv_dt, inv_dt2, g, kappa_max;
};

template <typename R>
static Consts<R> mkc(const StepConsts& k) {
    return Consts<R>{(R)k.dt, (R)(1.0 / k.dt), (R)(1.0 / (k.dt * k.dt)), (R)k.g, (R)k.kappa_max};
}

static inline unsigned nblocks(unsigned n, unsigned per) { return (n + per - 1) / per; }

// ----------------------------------------------------------- step start
// Energy hooks of the step start for per-vertex ground contact
// (GroundCollisionEnergySolver::updateContactPoints + CollisionConstraintEnergySolver::
// updateAfterTimeStep) followed by the inertial prediction with adaptive
// initialisation.  Both read the positions at the start of the step; the hook
// runs first, as in the reference (VBDSolver.hpp:54-62).
template <typename R>
__global__ void __launch_bounds__(256) k_begin_step(DevState<R> s, Consts<R> c) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    using V4 = typename Vec4Of<R>::T;
    uint8_t fl = s.flags[p];
    V4 x4 = s.x[p];
    if (fl & VF_GROUND) {
        V4 k = s.gk[p], lam = s.glam[p], cp = s.gcp[p];
        uint8_t gf = s.gflag[p];
        cp.x = x4.x;
        cp.y = x4.z;
        if (lam.x > R(0)) lam.w = -x4.y;
        if ((gf & GF_UNCLAMPED) && !(gf & GF_USE_STATIC)) gf |= GF_USE_STATIC;
        lam.x *= R(AVBD_ALPHA * AVBD_GAMMA);
        lam.y *= R(AVBD_GAMMA);
        lam.z *= R(AVBD_GAMMA);
        R gk;
        gk = R(AVBD_GAMMA) * k.x; k.x = (gk < k.w) ? k.w : gk;
        gk = R(AVBD_GAMMA) * k.y; k.y = (gk < k.w) ? k.w : gk;
        gk = R(AVBD_GAMMA) * k.z; k.z = (gk < k.w) ? k.w : gk;
        s.gk[p] = k;
        s.glam[p] = lam;
        s.gcp[p] = cp;
        s.gflag[p] = gf;
    }
    if (fl & (VF_FIXED | VF_ORIENTED)) return;
    V3<R> x = xyz(x4);
    V3<R> v = xyz(s.v[p]), vp = xyz(s.vp[p]);
    V3<R> a = c.inv_dt * (v - vp);
    V3<R> aext = mk3<R>(0, -c.g, 0);
    R an = c.g;
    R t = 0;
    if (an > R(1e-12)) {
        R al = dot3(a, aext) / an;
        if (al > an) t = 1;
        else if (al < R(0)) t = 0;
        else t = al / an;
    }
    V3<R> at = t * aext;
    R dt2 = c.dt * c.dt;
    V3<R> y = (x + c.dt * v) + dt2 * aext;
    V3<R> xn = x + (c.dt * v + dt2 * at);
    V4 y4 = s.y[p];
    s.y[p] = make4<R>(y, y4.w);
    V4 o = make4<R>(xn, x4.w);
    s.x[p] = o;
    s.xl[p] = o;
    s.xll[p] = o;
}

// E_prev = 1/2 (F_prev^T F_prev - I) of every tet from the previous positions
// (NeoHookeanEnergySolver::updateAfterTimeStep).  Only run when some tet has
// strain-rate damping; without damping E_prev is never read.
template <typename R>
__global__ void __launch_bounds__(256) k_tet_eprev(DevState<R> s) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= s.ntets) return;
    uint4 id = s.tet_idx[t];
    V3<R> x0 = xyz(s.xp[id.x]), x1 = xyz(s.xp[id.y]), x2 = xyz(s.xp[id.z]), x3 = xyz(s.xp[id.w]);
    V3<R> q0 = xyz(s.tet_q[3 * t]), q1 = xyz(s.tet_q[3 * t + 1]), q2 = xyz(s.tet_q[3 * t + 2]);
    V3<R> a = x0 - x3, b = x1 - x3, d = x2 - x3;
    // F = [a b d] Q: column j = a Q0j + b Q1j + d Q2j
    V3<R> F0 = q0.x * a + q1.x * b + q2.x * d;
    V3<R> F1 = q0.y * a + q1.y * b + q2.y * d;
    V3<R> F2 = q0.z * a + q1.z * b + q2.z * d;
    typename Vec4Of<R>::T e0, e1 = s.tet_e[2 * t + 1];
    e0.x = R(0.5) * (dot3(F0, F0) - R(1));
    e0.y = R(0.5) * (dot3(F1, F1) - R(1));
    e0.z = R(0.5) * (dot3(F2, F2) - R(1));
    e0.w = R(0.5) * dot3(F0, F1);
    e1.x = R(0.5) * dot3(F0, F2);
    e1.y = R(0.5) * dot3(F1, F2);
    s.tet_e[2 * t] = e0;
    s.tet_e[2 * t + 1] = e1;
}

// ------------------------------------------------------- vertex block
template <typename R>
AVBD_D IncRec<R> load_rec(const IncRec<R>* p);

template <>
AVBD_D IncRec<float> load_rec<float>(const IncRec<float>* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    float4 a = __ldcs(q), b = __ldcs(q + 1), c = __ldcs(q + 2), d = __ldcs(q + 3);
    IncRec<float> r;
    r.o[0] = __float_as_uint(a.x); r.o[1] = __float_as_uint(a.y); r.o[2] = __float_as_uint(a.z);
    r.tet = __float_as_uint(a.w);
    r.d[0] = b.x; r.d[1] = b.y; r.d[2] = b.z; r.d[3] = b.w;
    r.d[4] = c.x; r.d[5] = c.y; r.d[6] = c.z; r.d[7] = c.w;
    r.d[8] = d.x; r.vlam = d.y; r.vmu = d.z; r.mol = d.w;
    return r;
}
AVBD_D void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
AVBD_D void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

template <>
AVBD_D IncRec<double> load_rec<double>(const IncRec<double>* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const uint4 h = __ldcs(reinterpret_cast<const uint4*>(p));
    IncRec<double> r;
    r.o[0] = h.x; r.o[1] = h.y; r.o[2] = h.z; r.tet = h.w;
    double2 v;
    v = __ldcs(q + 1); r.d[0] = v.x; r.d[1] = v.y;
    v = __ldcs(q + 2); r.d[2] = v.x; r.d[3] = v.y;
    v = __ldcs(q + 3); r.d[4] = v.x; r.d[5] = v.y;
    v = __ldcs(q + 4); r.d[6] = v.x; r.d[7] = v.y;
    v = __ldcs(q + 5); r.d[8] = v.x; r.vlam = v.y;
    v = __ldcs(q + 6); r.vmu = v.x; r.mol = v.y;
    return r;
}

// Accumulated block: gradient in the state precision P, Hessian in HT.  The
// Hessian only shapes the Newton step, never the converged state, so the
// mixed mode keeps it in FP32 while the gradient (which the residual
// measures) is formed in FP64.
template <typename P, typename HT>
struct Block3 {
    P g0 = 0, g1 = 0, g2 = 0;
    HT h00 = 0, h11 = 0, h22 = 0, h01 = 0, h02 = 0, h12 = 0;
};

// One NeoHookean incidence: NeoHookeanEnergySolver::accumulate with the tet
// restated relative to the solved vertex (see IncRec).  P is the precision of
// positions and gradient, RS the stored record scalar, HT the Hessian type.
// The terms from the three edge vectors e_j = x_(o_j) - x_i; `tet` indexes
// the damping state.
template <typename P, typename RS, typename HT, bool DAMP, typename RD>
AVBD_D void accumulate_tet_e(const DevState<P>& s, const RD& r, unsigned tet, V3<P> e1, V3<P> e2, V3<P> e3, P dt,
                             Block3<P, HT>& B) {
    V3<P> d1 = mk3<P>(r.d[0], r.d[1], r.d[2]);
    V3<P> d2 = mk3<P>(r.d[3], r.d[4], r.d[5]);
    V3<P> d3 = mk3<P>(r.d[6], r.d[7], r.d[8]);
    V3<P> dw = mk3<P>(-(d1.x + d2.x + d3.x), -(d1.y + d2.y + d3.y), -(d1.z + d2.z + d3.z));
    // columns of F
    V3<P> F0 = d1.x * e1 + d2.x * e2 + d3.x * e3;
    V3<P> F1 = d1.y * e1 + d2.y * e2 + d3.y * e3;
    V3<P> F2 = d1.z * e1 + d2.z * e2 + d3.z * e3;
    V3<P> c0 = cross3(F1, F2), c1 = cross3(F2, F0), c2 = cross3(F0, F1);
    P J = dot3(F0, c0);
    V3<P> Fc = dw.x * c0 + dw.y * c1 + dw.z * c2;   // cof(F) d
    V3<P> Fd = dw.x * F0 + dw.y * F1 + dw.z * F2;   // F d
    P hyd = (P)r.vlam * ((J - P(1)) - (P)r.mol);     // V lambda (J - mu/lambda - 1)
    P dev = (P)r.vmu;
    P qn2 = dot3(dw, dw);
    B.g0 += hyd * Fc.x + dev * Fd.x;
    B.g1 += hyd * Fc.y + dev * Fd.y;
    B.g2 += hyd * Fc.z + dev * Fd.z;
    const HT vl = (HT)r.vlam, fx = (HT)Fc.x, fy = (HT)Fc.y, fz = (HT)Fc.z;
    const HT dg = (HT)(dev * qn2);
    B.h00 += vl * fx * fx + dg;
    B.h11 += vl * fy * fy + dg;
    B.h22 += vl * fz * fz + dg;
    B.h01 += vl * fx * fy;
    B.h02 += vl * fx * fz;
    B.h12 += vl * fy * fz;
    if constexpr (DAMP) {
        typename Vec4Of<P>::T e0 = s.tet_e[2 * tet], e1v = s.tet_e[2 * tet + 1];
        P vkd = e1v.z;
        if (vkd != P(0)) {
            P idt = P(1) / dt;
            // Edot = (1/2 (F^T F - I) - E_prev) / dt
            P E00 = (P(0.5) * (dot3(F0, F0) - P(1)) - e0.x) * idt;
            P E11 = (P(0.5) * (dot3(F1, F1) - P(1)) - e0.y) * idt;
            P E22 = (P(0.5) * (dot3(F2, F2) - P(1)) - e0.z) * idt;
            P E01 = (P(0.5) * dot3(F0, F1) - e0.w) * idt;
            P E02 = (P(0.5) * dot3(F0, F2) - e1v.x) * idt;
            P E12 = (P(0.5) * dot3(F1, F2) - e1v.y) * idt;
            V3<P> Ed = mk3<P>(E00 * dw.x + E01 * dw.y + E02 * dw.z, E01 * dw.x + E11 * dw.y + E12 * dw.z,
                              E02 * dw.x + E12 * dw.y + E22 * dw.z);
            P damp = P(2) * idt * vkd;
            V3<P> FEd = Ed.x * F0 + Ed.y * F1 + Ed.z * F2;
            B.g0 += damp * FEd.x;
            B.g1 += damp * FEd.y;
            B.g2 += damp * FEd.z;
            HT diag = (HT)(damp * dot3(dw, Ed));
            HT al = (HT)(P(0.5) * damp * idt);
            HT q2 = (HT)qn2;
            // F F^T = sum_c F_c F_c^T
            HT f00 = (HT)(F0.x * F0.x + F1.x * F1.x + F2.x * F2.x);
            HT f11 = (HT)(F0.y * F0.y + F1.y * F1.y + F2.y * F2.y);
            HT f22 = (HT)(F0.z * F0.z + F1.z * F1.z + F2.z * F2.z);
            HT f01 = (HT)(F0.x * F0.y + F1.x * F1.y + F2.x * F2.y);
            HT f02 = (HT)(F0.x * F0.z + F1.x * F1.z + F2.x * F2.z);
            HT f12 = (HT)(F0.y * F0.z + F1.y * F1.z + F2.y * F2.z);
            HT dx = (HT)Fd.x, dy = (HT)Fd.y, dz = (HT)Fd.z;
            B.h00 += diag + al * (f00 * q2 + dx * dx);
            B.h11 += diag + al * (f11 * q2 + dy * dy);
            B.h22 += diag + al * (f22 * q2 + dz * dz);
            B.h01 += al * (f01 * q2 + dx * dy);
            B.h02 += al * (f02 * q2 + dx * dz);
            B.h12 += al * (f12 * q2 + dy * dz);
        }
    }
}

// COH: neighbour positions by coherent loads (the persistent sweep, whose own
// launch writes them); otherwise through the read-only path.
template <typename P, typename RS, typename HT, bool DAMP, bool COH = false>
AVBD_D void accumulate_tet(const DevState<P>& s, const IncRec<RS>& r, V3<P> xi, P dt, Block3<P, HT>& B) {
    V3<P> e1, e2, e3;
    if constexpr (COH) {
        e1 = xyz(s.x[r.o[0]]) - xi;
        e2 = xyz(s.x[r.o[1]]) - xi;
        e3 = xyz(s.x[r.o[2]]) - xi;
    } else {
        e1 = xyz(ld_ro(s.x + r.o[0])) - xi;
        e2 = xyz(ld_ro(s.x + r.o[1])) - xi;
        e3 = xyz(ld_ro(s.x + r.o[2])) - xi;
    }
    accumulate_tet_e<P, RS, HT, DAMP>(s, r, r.tet, e1, e2, e3, dt, B);
}

// Ground contact term of the block (CollisionConstraintEnergySolver::accumulate<3>
// with GroundCollisionConstraintSolver): the Hessian k grad C grad C^T is always
// added, the gradient is gated by the clamped multipliers.
template <typename P, typename HT>
AVBD_D void accumulate_ground(const DevState<P>& s, unsigned p, V3<P> xi, Block3<P, HT>& B) {
    typename Vec4Of<P>::T k = s.gk[p], lam = s.glam[p], cp = s.gcp[p];
    uint8_t gf = s.gflag[p];
    P Cn = -xi.y, Ct = xi.x - cp.x, Cb = xi.z - cp.y;
    P cc = Cn - P(AVBD_ALPHA) * lam.w;
    P ln = k.x * cc + lam.x;
    P lnp = ln > P(0) ? ln : P(0);
    P lt = k.y * Ct + lam.y, lb = k.z * Cb + lam.z;
    P mag = sqrt(lt * lt + lb * lb);
    P mu = (gf & GF_USE_STATIC) ? cp.z : cp.w;
    P mx = mu * lnp;
    if (mag > mx) {
        P sc = mx / (mag + P(1e-8));
        lt = lt * sc;
        lb = lb * sc;
    }
    B.g0 += lt;
    B.g1 += -lnp;
    B.g2 += lb;
    B.h00 += (HT)k.y;
    B.h11 += (HT)k.x;
    B.h22 += (HT)k.z;
}

template <int LANES, typename P, typename HT>
AVBD_D void reduce_block(Block3<P, HT>& B) {
#pragma unroll
    for (int m = LANES / 2; m >= 1; m >>= 1) {
        B.g0 += shfl_xor(B.g0, m);
        B.g1 += shfl_xor(B.g1, m);
        B.g2 += shfl_xor(B.g2, m);
        B.h00 += shfl_xor(B.h00, m);
        B.h11 += shfl_xor(B.h11, m);
        B.h22 += shfl_xor(B.h22, m);
        B.h01 += shfl_xor(B.h01, m);
        B.h02 += shfl_xor(B.h02, m);
        B.h12 += shfl_xor(B.h12, m);
    }
}

enum { MODE_SOLVE = 0, MODE_RESIDUAL = 1, MODE_DEBUG = 2, MODE_FEATURES = 3 };


// Vertex block solve of one color slab: LANES threads per vertex stream the
// vertex's incidence records, each lane accumulating its tets, then a shuffle
// reduction and the 3x3 solve by the group's first lane.  MODE_RESIDUAL
// evaluates |m/h^2 (x-y) + grad| instead of updating; MODE_DEBUG exports the
// accumulated block; MODE_FEATURES writes the learned warm start's 32 BF16
// input features of the vertex (row p of `out`) at the current iterate.
// Resident blocks of 256 threads asked of the compiler: the mixed mode
// (double state, float records) would take 92 registers (2 blocks per SM);
// at 3 blocks (80 registers, ~100 bytes of spill) its vertex solve ran 15 %
// faster over a whole run-to-tolerance step of the 1024-cube batch.  FP32
// fits 4 blocks (64 registers) without spills; FP64 keeps the default.
template <typename P, typename RS>
struct SolveMinBlocks {
    static constexpr int value = sizeof(P) == 4 ? 4 : (sizeof(RS) == 4 ? 3 : 1);
};

// DYN: the instantiation for vertices with dynamic contact energies or a
// color changed by the recoloring, launched over per-color lists; the slab
// launches (DYN false) skip those vertices and carry no dynamic code.
template <typename P, typename RS, typename HT, int LANES, bool DAMP, bool GROUND, int MODE, bool DYN, bool COH = false>
__device__ __forceinline__ void tet_vertex(const DevState<P>& s, const IncRec<RS>* __restrict__ inc, unsigned begin,
                                           unsigned count, unsigned gi, unsigned lane, const Consts<P>& c,
                                           unsigned long long* counters, double* out, const SceneTol& T,
                                           const float4* __restrict__ aux, const uint32_t* __restrict__ list,
                                           double* acc = nullptr) {
    bool active = gi < count;
    unsigned p = list ? (active ? list[gi] : 0u) : begin + (active ? gi : 0);
    uint8_t fl = active ? s.flags[p] : 0;
    if (MODE != MODE_SOLVE && (fl & (VF_FIXED | VF_ORIENTED))) active = false;
    // vertices with dynamic contacts or a new color are solved from their color's list
    if ((MODE == MODE_SOLVE || MODE == MODE_RESIDUAL) && !DYN && s.dyn_skip && active && s.dyn_skip[p])
        active = false;
    // per-scene run-to-tolerance: converged scenes are skipped before any record is read
    if (MODE == MODE_SOLVE && T.active && active && !T.active[T.scene[p]]) active = false;
    if (MODE == MODE_RESIDUAL && T.cand && active && !T.cand[T.scene[p]]) active = false;
    Block3<P, HT> B;
    V3<P> xi = mk3<P>(0, 0, 0);
    // MODE_FEATURES: sum of the other vertices' velocities and of mu/lambda over the incident tets
    float fv0 = 0.f, fv1 = 0.f, fv2 = 0.f, fmol = 0.f, fcnt = 0.f;
    if (active) {
        xi = xyz(s.x[p]);
        unsigned b = s.inc_begin[p], e = s.inc_begin[p + 1];
        // the next record is fetched into L1 while this one is processed (a
        // register copy of it, as a software pipeline, spilled: 192 B of
        // spill in the mixed mode at 3 blocks per SM, 3 % slower), and the
        // record three further on into L2
        unsigned k = b + lane;
        while (k < e) {
            const unsigned kn = k + LANES;
            if (kn < e) prefetch_l1(inc + kn);
            IncRec<RS> r = load_rec<RS>(inc + k);
            if (kn + 3 * LANES < e) prefetch_l2(inc + kn + 3 * LANES);
            accumulate_tet<P, RS, HT, DAMP, COH>(s, r, xi, c.dt, B);
            if constexpr (MODE == MODE_FEATURES) {
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    typename Vec4Of<P>::T vo = s.v[r.o[j]];
                    fv0 += (float)vo.x;
                    fv1 += (float)vo.y;
                    fv2 += (float)vo.z;
                }
                fmol += (float)r.mol;
                fcnt += 1.f;
            }
            k = kn;
        }
    }
    if constexpr (DYN) {
        // dynamic energies (VBDSolver.hpp:397-446): triangle-rigid then
        // triangle-rod contacts, each in slot order, spread over the lanes
        // (a contact term is a chain of rotation and Jacobian functions)
        if (active) {
            const unsigned e = s.dyn_begin[p + 1];
            for (unsigned k = s.dyn_begin[p] + lane; k < e; k += LANES) {
                const uint32_t en = s.dyn_ent[k];
                dyn_accumulate3<P, HT>(s, dyn_pool(en), dyn_slot(en), dyn_local(en), B);
            }
        }
    }
    reduce_block<LANES>(B);
    if constexpr (MODE == MODE_FEATURES) {
#pragma unroll
        for (int m = LANES / 2; m >= 1; m >>= 1) {
            fv0 += shfl_xor(fv0, m);
            fv1 += shfl_xor(fv1, m);
            fv2 += shfl_xor(fv2, m);
            fmol += shfl_xor(fmol, m);
            fcnt += shfl_xor(fcnt, m);
        }
    }
    if (!active || lane != 0) {
        if constexpr (MODE == MODE_RESIDUAL) {
            // keep the warp reduction below well defined
        } else {
            return;
        }
    }
    double r2 = 0.0, mg2 = 0.0;
    if (active && lane == 0) {
        if (GROUND && (fl & VF_GROUND)) accumulate_ground<P, HT>(s, p, xi, B);
        typename Vec4Of<P>::T y4 = s.y[p];
        P m = y4.w;
        P cm = m * c.inv_dt2;
        V3<P> d = xi - xyz(y4);
        if constexpr (MODE == MODE_SOLVE) {
            Sym3<P> A{cm + (P)B.h00, cm + (P)B.h11, cm + (P)B.h22, (P)B.h01, (P)B.h02, (P)B.h12};
            V3<P> rhs = mk3<P>(-cm * d.x - B.g0, -cm * d.y - B.g1, -cm * d.z - B.g2);
            if (T.r2) {  // in-sweep residual: the block RHS just before this vertex's update
                double q = (double)rhs.x * (double)rhs.x + (double)rhs.y * (double)rhs.y +
                           (double)rhs.z * (double)rhs.z;
                if (acc) *acc += q;  // one scene per block: summed over the block
                else atomicAdd(T.r2 + T.scene[p], q);
            }
            V3<P> dx;
            P kappa = solve_sym3<P>(A, rhs, dx);
            if (!(kappa <= c.kappa_max)) {
                double M[3][3] = {{(double)A.a00, (double)A.a01, (double)A.a02},
                                  {(double)A.a01, (double)A.a11, (double)A.a12},
                                  {(double)A.a02, (double)A.a12, (double)A.a22}};
                double bb[3] = {(double)rhs.x, (double)rhs.y, (double)rhs.z}, xx[3];
                lu_solve_d<3>(M, bb, xx);
                dx = mk3<P>((P)xx[0], (P)xx[1], (P)xx[2]);
                atomicAdd(counters, 1ull);
            }
            typename Vec4Of<P>::T o = make4<P>(xi + dx, P(0));
            // an intra-color conflict buffers the update (VBDSolver.hpp:505-509)
            if (DYN && s.conflicted[p]) s.buffered[p] = o;
            else s.x[p] = o;
        } else if constexpr (MODE == MODE_FEATURES) {
            // feature layout of avbd_warmstart_sample (include/avbd.h)
            Sym3<P> A{cm + (P)B.h00, cm + (P)B.h11, cm + (P)B.h22, (P)B.h01, (P)B.h02, (P)B.h12};
            V3<P> rhs = mk3<P>(-cm * d.x - B.g0, -cm * d.y - B.g1, -cm * d.z - B.g2);
            V3<P> dx;
            solve_sym3<P>(A, rhs, dx);
            const float sc = 1.0f / (float)(c.g * c.dt * c.dt);
            const float h = (float)c.dt, icm = 1.0f / (float)cm;
            typename Vec4Of<P>::T v4 = s.v[p];
            const float4* prev = aux;  // MODE_FEATURES: previous-correction rows (may be null)
            const float inv3n = fcnt > 0.f ? 1.0f / (3.0f * fcnt) : 0.f;
            float f[32];
            f[0] = (float)d.x * sc; f[1] = (float)d.y * sc; f[2] = (float)d.z * sc;
            f[3] = (float)v4.x * h * sc; f[4] = (float)v4.y * h * sc; f[5] = (float)v4.z * h * sc;
            // the previous step's converged correction (x_end - x0) / s, kept by k_ws_target
            const float4 pc = prev ? prev[p] : make_float4(0.f, 0.f, 0.f, 0.f);
            f[6] = pc.x; f[7] = pc.y; f[8] = pc.z;
            f[9] = fcnt > 0.f ? (fv0 * inv3n - (float)v4.x) * h * sc : 0.f;
            f[10] = fcnt > 0.f ? (fv1 * inv3n - (float)v4.y) * h * sc : 0.f;
            f[11] = fcnt > 0.f ? (fv2 * inv3n - (float)v4.z) * h * sc : 0.f;
            f[12] = (float)rhs.x * icm * sc; f[13] = (float)rhs.y * icm * sc; f[14] = (float)rhs.z * icm * sc;
            f[15] = (float)dx.x * sc; f[16] = (float)dx.y * sc; f[17] = (float)dx.z * sc;
            f[18] = log1pf(fmaxf(0.f, (float)B.h00 * icm));
            f[19] = log1pf(fmaxf(0.f, (float)B.h11 * icm));
            f[20] = log1pf(fmaxf(0.f, (float)B.h22 * icm));
            f[21] = fcnt > 0.f ? fmol / fcnt : 0.f;
            f[22] = log10f((float)m) + 3.0f;
            f[23] = tanhf((float)xi.y * sc * 0.1f);
            f[24] = (GROUND && (fl & VF_GROUND)) ? (float)s.glam[p].x * icm * sc : 0.f;
            f[25] = fcnt * (1.0f / 24.0f);
            f[26] = tanhf((float)y4.y * sc);
#pragma unroll
            for (int j = 27; j < 32; j++) f[j] = 0.f;
            uint32_t w[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                float a = fminf(fmaxf(f[2 * j], -1e4f), 1e4f), b = fminf(fmaxf(f[2 * j + 1], -1e4f), 1e4f);
                if (!(a == a)) a = 0.f;  // a NaN feature becomes 0
                if (!(b == b)) b = 0.f;
                __nv_bfloat162 hb = __floats2bfloat162_rn(a, b);
                w[j] = *reinterpret_cast<uint32_t*>(&hb);
            }
            uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(out) + (size_t)p * 64);
            dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
            dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
            dst[2] = make_uint4(w[8], w[9], w[10], w[11]);
            dst[3] = make_uint4(w[12], w[13], w[14], w[15]);
        } else if constexpr (MODE == MODE_RESIDUAL) {
            double u0 = (double)cm * (double)d.x + (double)B.g0;
            double u1 = (double)cm * (double)d.y + (double)B.g1;
            double u2 = (double)cm * (double)d.z + (double)B.g2;
            r2 = u0 * u0 + u1 * u1 + u2 * u2;
            double mgv = (double)m * (double)c.g;
            mg2 = mgv * mgv;
        } else {
            out[0] = B.g0; out[1] = B.g1; out[2] = B.g2;
            out[3] = B.h00; out[4] = B.h01; out[5] = B.h02;
            out[6] = B.h01; out[7] = B.h11; out[8] = B.h12;
            out[9] = B.h02; out[10] = B.h12; out[11] = B.h22;
        }
    }
    if constexpr (MODE == MODE_RESIDUAL) {
        if (T.ex) {  // per-scene sums
            if (active && lane == 0) {
                if (acc) *acc += r2;
                else atomicAdd(T.ex + T.scene[p], r2);
            }
            return;
        }
        // FP64 reduction: warp, then one atomic per warp
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) {
            r2 += __shfl_xor_sync(0xffffffffu, r2, m);
            mg2 += __shfl_xor_sync(0xffffffffu, mg2, m);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(out, r2);
            atomicAdd(out + 1, mg2);
        }
    }
}

// ranges: when given, block b serves the vertices [x, x + y) of scene z
// (a piece of one scene's part of a color slab) and returns at once when the
// scene is not iterating (solve) or not a residual candidate (residual):
// with per-scene run-to-tolerance most scenes drop out of the later
// iterations, and a block of them then costs one check.  The block's
// residual terms (in-sweep or exact) are summed in registers and reduced
// over the block: one atomic per piece instead of one per vertex on the
// scene's sum.  Otherwise thread groups map to vertices [begin, begin +
// count) (or to list).
// One piece (at most 512 consecutive solved vertices of one scene in one
// color slab) solved by one block; its residual terms are summed over the
// block.  rg = (first vertex, count, scene).
template <typename P, typename RS, typename HT, int LANES, bool DAMP, bool GROUND, int MODE, bool DYN, bool COH>
__device__ __forceinline__ void solve_piece(const DevState<P>& s, const IncRec<RS>* __restrict__ inc, const uint4 rg,
                                            const Consts<P>& c, unsigned long long* counters, double* out,
                                            const SceneTol& T, const float4* __restrict__ aux,
                                            const uint32_t* __restrict__ list) {
    const unsigned lane = threadIdx.x % LANES;
    const uint8_t* gate = MODE == MODE_SOLVE ? T.active : T.cand;
    if (gate && !gate[rg.z]) return;
    double* sum = MODE == MODE_SOLVE ? T.r2 : (MODE == MODE_RESIDUAL ? T.ex : nullptr);
    SceneTol TB = T;  // gated above, for the whole block
    TB.active = nullptr;
    TB.cand = nullptr;
    double acc = 0.0;
    for (unsigned base = 0; base < rg.y; base += blockDim.x / LANES) {
        // the first records of this thread group's next vertex are fetched
        // into L2 while this one is solved (its first loads are then not
        // DRAM misses)
        const unsigned gn = base + blockDim.x / LANES + threadIdx.x / LANES;
        if (gn < rg.y) {
            const unsigned bn = s.inc_begin[rg.x + gn], en = s.inc_begin[rg.x + gn + 1];
#pragma unroll
            for (unsigned j = 0; j < 4; j++)
                if (bn + lane + j * LANES < en) prefetch_l2(inc + bn + lane + j * LANES);
        }
        tet_vertex<P, RS, HT, LANES, DAMP, GROUND, MODE, DYN, COH>(s, inc, rg.x, rg.y, base + threadIdx.x / LANES,
                                                                   lane, c, counters, out, TB, aux, list,
                                                                   sum ? &acc : nullptr);
    }
    if (sum) {
        __shared__ double part[32];
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (unsigned w = 0; w < (blockDim.x >> 5); w++) t += part[w];
            atomicAdd(sum + rg.z, t);
        }
    }
}

template <typename P, typename RS, typename HT, int LANES, bool DAMP, bool GROUND, int MODE, bool DYN>
__global__ void __launch_bounds__(256, SolveMinBlocks<P, RS>::value) k_solve_tet(DevState<P> s, const IncRec<RS>* __restrict__ inc,
                                                   unsigned begin, unsigned count, Consts<P> c,
                                                   unsigned long long* counters, double* out, SceneTol T,
                                                   const float4* __restrict__ aux, const uint32_t* __restrict__ list,
                                                   const uint4* __restrict__ ranges) {
    if (ranges) {
        solve_piece<P, RS, HT, LANES, DAMP, GROUND, MODE, DYN, false>(s, inc, ranges[blockIdx.x], c, counters, out, T,
                                                                      aux, list);
        return;
    }
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
    tet_vertex<P, RS, HT, LANES, DAMP, GROUND, MODE, DYN>(s, inc, begin, count, tid / LANES, tid % LANES, c, counters,
                                                          out, T, aux, list);
}

// Polls a grid-barrier wait of the persistent sweep may take before it gives
// up (avbd_debug_set_wait_limit lowers it so that tests can make it run out).
__device__ uint32_t g_sweep_wait_polls = AVBD_DEFAULT_WAIT_POLLS;

AVBD_D bool grid_barrier(unsigned* sync, int* err) {
    return grid_barrier_bounded(sync, err, *(volatile uint32_t*)&g_sweep_wait_polls);
}

// The whole sweep of a run-to-tolerance iteration in one cooperative launch:
// for each color in turn the blocks draw its pieces from a shared ticket
// counter (dynamic, so uneven pieces balance), then meet at a grid barrier
// before the next color reads the positions this one wrote.  In color k each
// block draws exactly one ticket past the color's pieces, so color k's tickets
// start at sum over earlier colors of (pieces + blocks).  sync: [ticket,
// arrivals, generation], zeroed before each launch.
template <typename P, typename RS, typename HT, int LANES, bool GROUND>
__global__ void __launch_bounds__(256, SolveMinBlocks<P, RS>::value)
    k_sweep_persistent(DevState<P> s, const IncRec<RS>* __restrict__ inc, Consts<P> c, unsigned long long* counters,
                       SceneTol T, const uint4* __restrict__ ranges, const unsigned* __restrict__ color_off,
                       unsigned ncolors, unsigned* sync) {
    __shared__ unsigned ticket;
    unsigned base = 0;
    for (unsigned col = 0; col < ncolors; col++) {
        const unsigned r0 = color_off[col], np = color_off[col + 1] - r0;
        for (;;) {
            __syncthreads();  // every thread has read the previous ticket
            if (threadIdx.x == 0) ticket = atomicAdd(sync, 1u) - base;
            __syncthreads();
            const unsigned t = ticket;
            if (t >= np) break;
            solve_piece<P, RS, HT, LANES, false, GROUND, MODE_SOLVE, false, true>(s, inc, ranges[r0 + t], c,
                                                                                  counters, nullptr, T, nullptr,
                                                                                  nullptr);
        }
        base += np + gridDim.x;
        if (col + 1 < ncolors && !grid_barrier(sync + 1, s.err)) return;
    }
}

// Chebyshev acceleration of every particle fused with the ground-contact dual
// update that follows it (CollisionConstraintEnergySolver::updateAfterIteration);
// a ground energy reads only its own particle, so the fusion is exact.
template <typename R>
__global__ void __launch_bounds__(256) k_chebyshev_dual(DevState<R> s, R omega, unsigned it, SceneTol T) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    uint8_t fl = s.flags[p];
    if (fl & VF_ORIENTED) return;
    if (T.active && !T.active[T.scene[p]]) return;
    if (T.omega) omega = (R)*T.omega;
    if (T.it) it = *T.it;
    // o_k = omega (x - o_(k-2)) + o_(k-2); o_k replaces o_(k-2) in its buffer
    typename Vec4Of<R>::T* h = (it & 1u) ? s.xll : s.xl;
    typename Vec4Of<R>::T x4 = s.x[p], ll4 = h[p];
    V3<R> x = xyz(x4), ll = xyz(ll4);
    V3<R> xn = omega * (x - ll) + ll;
    typename Vec4Of<R>::T o = make4<R>(xn, x4.w);
    s.x[p] = o;
    h[p] = o;
    if (fl & VF_GROUND) {
        typename Vec4Of<R>::T k = s.gk[p], lam = s.glam[p], cp = s.gcp[p];
        uint8_t gf = s.gflag[p];
        R Cn = -xn.y, Ct = xn.x - cp.x, Cb = xn.z - cp.y;
        R cc = Cn - R(AVBD_ALPHA) * lam.w;
        R ln = k.x * cc + lam.x;
        R lt = k.y * Ct + lam.y;
        R lb = k.z * Cb + lam.z;
        // the penalties grow only in contact: elsewhere k is not stored back
        bool k_grows = ln > R(0);
        if (ln > R(0)) k.x += R(AVBD_BETA) * fabs(cc);
        lam.x = ln > R(0) ? ln : R(0);
        R mag = sqrt(lt * lt + lb * lb);
        bool st = gf & GF_USE_STATIC;
        R mx = (st ? cp.z : cp.w) * lam.x;
        if (mag < mx) {
            k_grows = true;
            k.y += R(AVBD_BETA) * fabs(Ct);
            k.z += R(AVBD_BETA) * fabs(Cb);
            lam.y = lt;
            lam.z = lb;
            gf |= GF_UNCLAMPED;
        } else {
            if (st) {
                gf &= ~GF_USE_STATIC;
                mx = cp.w * ln;
            }
            lam.y = lt / (mag + R(1e-8)) * mx;
            lam.z = lb / (mag + R(1e-8)) * mx;
            gf &= ~GF_UNCLAMPED;
        }
        if (k_grows) s.gk[p] = k;
        s.glam[p] = lam;
        s.gflag[p] = gf;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_velocity(DevState<R> s, R inv_dt) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    if (s.flags[p] & VF_ORIENTED) return;
    typename Vec4Of<R>::T x4 = s.x[p], xp4 = s.xp[p];
    s.vp[p] = s.v[p];
    s.v[p] = make4<R>(inv_dt * (xyz(x4) - xyz(xp4)), R(0));
    s.xp[p] = x4;
    if (!isfinite(x4.x + x4.y + x4.z)) atomicExch(s.err, (int)AVBD_ERR_NAN);
}

// Host FP64 (external order) -> device state.  mode 0: positions only,
// mode 1: positions and every derived position array (ParticlePool::addParticle
// reset), mode 2: velocities (src) and previous velocities (src + 3n),
// mode 3: velocities only.
template <typename R>
__global__ void k_load(DevState<R> s, const double* src, const uint32_t* inv_map, unsigned first, unsigned n,
                       int mode) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned p = inv_map[first + i];
    V3<R> v = mk3<R>((R)src[3 * i], (R)src[3 * i + 1], (R)src[3 * i + 2]);
    if (mode == 2) {
        V3<R> w = mk3<R>((R)src[3 * (n + i)], (R)src[3 * (n + i) + 1], (R)src[3 * (n + i) + 2]);
        s.v[p] = make4<R>(v, R(0));
        s.vp[p] = make4<R>(w, R(0));
        return;
    }
    if (mode == 3) {
        s.v[p] = make4<R>(v, R(0));
        return;
    }
    typename Vec4Of<R>::T o = make4<R>(v, R(0));
    if (mode == 4) {  // a caller's initial guess of the step: solved positional vertices only
        if (s.flags[p] & (VF_FIXED | VF_ORIENTED)) return;
        s.x[p] = o;
        s.xl[p] = o;
        s.xll[p] = o;
        return;
    }
    s.x[p] = o;
    if (mode == 1) {
        typename Vec4Of<R>::T y4 = s.y[p];
        s.y[p] = make4<R>(v, y4.w);
        s.xp[p] = o;
        s.xl[p] = o;
        s.xll[p] = o;
    }
}

// Device state -> host FP64 (external order).  which: 0 x, 1 v, 2 xp.
template <typename R>
__global__ void k_store(DevState<R> s, int which, double* dst, const uint32_t* inv_map, unsigned first, unsigned n) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned p = inv_map[first + i];
    typename Vec4Of<R>::T a = which == 0 ? s.x[p] : which == 1 ? s.v[p] : s.xp[p];
    dst[3 * i] = (double)a.x;
    dst[3 * i + 1] = (double)a.y;
    dst[3 * i + 2] = (double)a.z;
}

// ---------------------------------------------------------------- host
template <typename R>
void launch_begin_step(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    k_begin_step<R><<<nblocks(s.n, 256), 256, 0, st>>>(s, mkc<R>(k));
    count_launch(c);
}

template <typename R>
void launch_tet_eprev(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    (void)k;
    if (s.ntets == 0) return;
    k_tet_eprev<R><<<nblocks(s.ntets, 256), 256, 0, st>>>(s);
    count_launch(c);
}

template <typename P, typename RS, typename HT, int LANES, int MODE, bool DYN = false>
static void solve_dispatch(avbd_ctx* c, DevState<P>& s, const IncRec<RS>* inc, const StepConsts& k, unsigned begin,
                           unsigned count, cudaStream_t st, double* out, const SceneTol& T, const uint32_t* list,
                           const uint4* ranges = nullptr, unsigned nranges = 0) {
    unsigned threads = count * LANES;
    unsigned blocks = ranges ? nranges : nblocks(threads, 256);
    if (blocks == 0) return;
    bool damp = c->damping, ground = !c->ground.empty();
    auto kc = mkc<P>(k);
    auto* ctr = c->d_counters;
    const float4* aux = reinterpret_cast<const float4*>(c->ws_prev_arg);
    if (damp && ground)
        k_solve_tet<P, RS, HT, LANES, true, true, MODE, DYN><<<blocks, 256, 0, st>>>(s, inc, begin, count, kc, ctr, out, T, aux, list, ranges);
    else if (damp)
        k_solve_tet<P, RS, HT, LANES, true, false, MODE, DYN><<<blocks, 256, 0, st>>>(s, inc, begin, count, kc, ctr, out, T, aux, list, ranges);
    else if (ground)
        k_solve_tet<P, RS, HT, LANES, false, true, MODE, DYN><<<blocks, 256, 0, st>>>(s, inc, begin, count, kc, ctr, out, T, aux, list, ranges);
    else
        k_solve_tet<P, RS, HT, LANES, false, false, MODE, DYN><<<blocks, 256, 0, st>>>(s, inc, begin, count, kc, ctr, out, T, aux, list, ranges);
    count_launch(c);
}

// The solve, residual and features passes run with the context's lane count
// (the residual pass spans every vertex every iteration, so its thread count
// matters even when few scenes are candidates); the one-vertex debug pass
// uses 8.
template <typename P, typename RS, typename HT, int MODE>
static void solve_lanes_t(avbd_ctx* c, DevState<P>& s, const IncRec<RS>* inc, const StepConsts& k, unsigned begin,
                          unsigned count, cudaStream_t st, double* out, const SceneTol& T, const uint32_t* list,
                          const uint4* ranges = nullptr, unsigned nranges = 0) {
    if constexpr (MODE == MODE_RESIDUAL) {  // tolerance residual: the sweeps' per-scene pieces, all colors
        if (!list && T.cand && T.ex && c->d_solve_ranges) {
            ranges = c->d_solve_ranges;
            nranges = c->solve_range_off.back();
        }
    }
    if constexpr (MODE == MODE_SOLVE || MODE == MODE_RESIDUAL) {
        if (ranges) {
            const uint4* rg = ranges;
            const unsigned nr = nranges;
            switch (c->lanes) {
                case 1: solve_dispatch<P, RS, HT, 1, MODE>(c, s, inc, k, 0, 0, st, out, T, nullptr, rg, nr); break;
                case 2: solve_dispatch<P, RS, HT, 2, MODE>(c, s, inc, k, 0, 0, st, out, T, nullptr, rg, nr); break;
                case 4: solve_dispatch<P, RS, HT, 4, MODE>(c, s, inc, k, 0, 0, st, out, T, nullptr, rg, nr); break;
                case 16: solve_dispatch<P, RS, HT, 16, MODE>(c, s, inc, k, 0, 0, st, out, T, nullptr, rg, nr); break;
                case 32: solve_dispatch<P, RS, HT, 32, MODE>(c, s, inc, k, 0, 0, st, out, T, nullptr, rg, nr); break;
                default: solve_dispatch<P, RS, HT, 8, MODE>(c, s, inc, k, 0, 0, st, out, T, nullptr, rg, nr); break;
            }
            return;
        }
    }
    if constexpr (MODE == MODE_DEBUG) {
        if (c->dyn) solve_dispatch<P, RS, HT, 8, MODE, true>(c, s, inc, k, begin, count, st, out, T, list);
        else solve_dispatch<P, RS, HT, 8, MODE>(c, s, inc, k, begin, count, st, out, T, list);
    } else if (list) {
        if constexpr (MODE == MODE_SOLVE || MODE == MODE_RESIDUAL)
            solve_dispatch<P, RS, HT, 8, MODE, true>(c, s, inc, k, begin, count, st, out, T, list);
    } else {
        switch (c->lanes) {
            case 1: solve_dispatch<P, RS, HT, 1, MODE>(c, s, inc, k, begin, count, st, out, T, list); break;
            case 2: solve_dispatch<P, RS, HT, 2, MODE>(c, s, inc, k, begin, count, st, out, T, list); break;
            case 4: solve_dispatch<P, RS, HT, 4, MODE>(c, s, inc, k, begin, count, st, out, T, list); break;
            case 16: solve_dispatch<P, RS, HT, 16, MODE>(c, s, inc, k, begin, count, st, out, T, list); break;
            case 32: solve_dispatch<P, RS, HT, 32, MODE>(c, s, inc, k, begin, count, st, out, T, list); break;
            default: solve_dispatch<P, RS, HT, 8, MODE>(c, s, inc, k, begin, count, st, out, T, list); break;
        }
    }
}

// FP32: everything in float.  FP64: everything in double.  Mixed: double
// state and gradient, float records and Hessian.
template <int MODE>
static void solve_lanes(avbd_ctx* c, DevState<float>& s, const StepConsts& k, unsigned begin, unsigned count,
                        cudaStream_t st, double* out, const SceneTol& T, const uint32_t* list = nullptr,
                        const uint4* ranges = nullptr, unsigned nranges = 0) {
    solve_lanes_t<float, float, float, MODE>(c, s, s.inc, k, begin, count, st, out, T, list, ranges, nranges);
}
template <int MODE>
static void solve_lanes(avbd_ctx* c, DevState<double>& s, const StepConsts& k, unsigned begin, unsigned count,
                        cudaStream_t st, double* out, const SceneTol& T, const uint32_t* list = nullptr,
                        const uint4* ranges = nullptr, unsigned nranges = 0) {
    if (c->solver.precision == AVBD_PRECISION_MIXED)
        solve_lanes_t<double, float, float, MODE>(c, s, s.inc32, k, begin, count, st, out, T, list, ranges, nranges);
    else
        solve_lanes_t<double, double, double, MODE>(c, s, s.inc, k, begin, count, st, out, T, list, ranges, nranges);
}

// The persistent sweep (default; AVBD_PERSISTENT=0 at context creation turns
// it off): one cooperative launch per iteration instead of one per color.  Taken for the run-to-tolerance
// sweeps of contexts whose solve runs 2 threads per vertex with no damping,
// no oriented particles and no dynamic contacts (the caller checks the last
// two); returns false, having launched nothing, otherwise.
template <typename P, typename RS, typename HT>
static bool sweep_persistent_t(avbd_ctx* c, DevState<P>& s, const IncRec<RS>* inc, const StepConsts& k,
                               cudaStream_t st, const SceneTol& T) {
    if (!c->persistent || c->lanes != 2 || c->damping || !c->d_solve_ranges || !c->d_solve_range_off ||
        !c->d_sweep_sync || c->num_sms == 0)
        return false;
    const bool ground = !c->ground.empty();
    auto kern = ground ? k_sweep_persistent<P, RS, HT, 2, true> : k_sweep_persistent<P, RS, HT, 2, false>;
    // resident blocks per SM of this context's instantiation, queried once
    // (-1 where the device cannot launch cooperative kernels: per-color
    // launches then)
    if (c->sweep_blocks_per_sm == 0) {
        int per_sm = 0, coop = 0;
        if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device) != cudaSuccess || !coop ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0) != cudaSuccess || per_sm < 1) {
            cudaGetLastError();
            c->sweep_blocks_per_sm = -1;
        } else {
            c->sweep_blocks_per_sm = per_sm;
        }
    }
    if (c->sweep_blocks_per_sm < 1) return false;
    const int per_sm = c->sweep_blocks_per_sm;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)per_sm * c->num_sms);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaMemsetAsync(c->d_sweep_sync, 0, 3 * sizeof(unsigned), st);
    // a failed launch is left in the runtime's last error, which the step checks
    cudaLaunchKernelEx(&cfg, kern, s, inc, mkc<P>(k), c->d_counters, T, (const uint4*)c->d_solve_ranges,
                       (const unsigned*)c->d_solve_range_off, c->num_colors, c->d_sweep_sync);
    count_launch(c);
    return true;
}
static bool sweep_persistent(avbd_ctx* c, DevState<float>& s, const StepConsts& k, cudaStream_t st,
                             const SceneTol& T) {
    return sweep_persistent_t<float, float, float>(c, s, s.inc, k, st, T);
}
static bool sweep_persistent(avbd_ctx* c, DevState<double>& s, const StepConsts& k, cudaStream_t st,
                             const SceneTol& T) {
    if (c->solver.precision == AVBD_PRECISION_MIXED)
        return sweep_persistent_t<double, float, float>(c, s, s.inc32, k, st, T);
    return sweep_persistent_t<double, double, double>(c, s, s.inc, k, st, T);
}

template <typename R>
bool launch_sweep_persistent(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st, const SceneTol& T) {
    return sweep_persistent(c, s, k, st, T);
}

int solve_set_wait_limit(unsigned polls) {
    cudaError_t e = cudaMemcpyToSymbol(g_sweep_wait_polls, &polls, sizeof(polls));
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

template <typename R>
void launch_solve_color(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned begin, unsigned count,
                        cudaStream_t st, const SceneTol& T, const uint32_t* list, const uint4* ranges,
                        unsigned nranges) {
    solve_lanes<MODE_SOLVE>(c, s, k, begin, count, st, nullptr, T, list, ranges, nranges);
}

template <typename R>
void launch_chebyshev_dual(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double omega, unsigned it,
                           cudaStream_t st, const SceneTol& T) {
    (void)k;
    if (s.no == s.n) return;  // every particle oriented: k_chebyshev_rot covers them
    k_chebyshev_dual<R><<<nblocks(s.n, 256), 256, 0, st>>>(s, (R)omega, it, T);
    count_launch(c);
}

template <typename R>
void launch_velocity(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    k_velocity<R><<<nblocks(s.n, 256), 256, 0, st>>>(s, (R)(1.0 / k.dt));
    count_launch(c);
}

template <typename R>
void launch_residual(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double* out2, cudaStream_t st,
                     const SceneTol& T) {
    if (out2) cudaMemsetAsync(out2, 0, 2 * sizeof(double), st);
    solve_lanes<MODE_RESIDUAL>(c, s, k, 0, s.n, st, out2, T);
    if (c->dyn) {  // the positional vertices the slab pass skipped
        const uint32_t* list = nullptr;
        unsigned m = 0;
        dyn_positional_list(c, &list, &m);
        if (m) solve_lanes<MODE_RESIDUAL>(c, s, k, 0, m, st, out2, T, list);
    }
}

// ------------------------------------------- per-scene run-to-tolerance
__global__ void k_tol_init(uint8_t* active, uint8_t* cand, double* r2, double* ex, uint32_t* iters, unsigned S,
                           unsigned long long* maxr, uint32_t* it, double* omega, const double* omega_tab) {
    unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) {
        *maxr = 0ull;
        *it = 0;
        if (omega_tab) *omega = omega_tab[0];
    }
    if (s >= S) return;
    active[s] = 1;
    cand[s] = 0;
    r2[s] = 0;
    ex[s] = 0;
    iters[s] = 0;
}

AVBD_D double scene_R(double r2, double mg2) { return mg2 > 0 ? sqrt(r2) / sqrt(mg2) : sqrt(r2); }

// After a sweep: every active scene counts the iteration and becomes a
// candidate when its in-sweep residual is at the tolerance.
// The in-sweep residual is kept (rin) as the final residual of a scene that
// then stops at the cap without becoming a candidate.
__global__ void k_tol_decide_a(uint8_t* active, uint8_t* cand, double* r2, const double* m2, uint32_t* iters,
                               unsigned S, double tol, double g2, unsigned long long* scene_iterations,
                               double* rin) {
    unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    cand[s] = 0;
    if (active[s]) {
        iters[s]++;
        atomicAdd(scene_iterations, 1ull);
        const double R = scene_R(r2[s], m2[s] * g2);
        rin[s] = R;
        cand[s] = R <= tol;
    }
    r2[s] = 0;
}

AVBD_D unsigned long long ord_enc64(double d) {
    unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

// Candidates whose exact residual is at the tolerance stop; so does every
// scene at the iteration cap.  Counts the scenes still iterating.  maxr[0]
// receives the largest final residual of the step's scenes: the exact one
// where it was evaluated in the stopping iteration, else the in-sweep one of
// a capped scene; maxr[1] counts the capped scenes.
__global__ void k_tol_decide_b(uint8_t* active, uint8_t* cand, double* ex, const double* m2, const uint32_t* iters,
                               unsigned S, double tol, double g2, unsigned max_it, int* n_active,
                               unsigned long long* maxr, const double* rin) {
    unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    if (active[s]) {
        bool done = false;
        double R = rin[s];
        if (cand[s]) {
            R = scene_R(ex[s], m2[s] * g2);
            done = R <= tol;
        }
        if (!done && iters[s] >= max_it) {  // stopped at the cap, unconverged
            done = true;
            atomicAdd(maxr + 1, 1ull);
        }
        if (done) {
            active[s] = 0;
            atomicMax(maxr, ord_enc64(R));
        } else {
            atomicAdd(n_active, 1);
        }
    }
    cand[s] = 0;
    ex[s] = 0;
}

void launch_tol_init(avbd_ctx* c, cudaStream_t st) {
    unsigned S = c->num_scenes;
    k_tol_init<<<nblocks(S, 256), 256, 0, st>>>(c->d_scene_active, c->d_scene_cand, c->d_scene_r2, c->d_scene_ex,
                                                c->d_scene_iters, S, c->d_counters + 2, c->d_tol_it, c->d_tol_omega,
                                                c->d_omega_tab);
    count_launch(c);
}

void launch_tol_decide_a(avbd_ctx* c, double tol, cudaStream_t st) {
    unsigned S = c->num_scenes;
    k_tol_decide_a<<<nblocks(S, 256), 256, 0, st>>>(c->d_scene_active, c->d_scene_cand, c->d_scene_r2,
                                                    c->d_scene_mg2, c->d_scene_iters, S, tol,
                                                    c->params.g_accel * c->params.g_accel, c->d_counters + 1,
                                                    c->d_scene_rin);
    count_launch(c);
}

void launch_tol_decide_b(avbd_ctx* c, double tol, unsigned max_it, cudaStream_t st) {
    unsigned S = c->num_scenes;
    cudaMemsetAsync(c->d_tol_count, 0, sizeof(int), st);
    k_tol_decide_b<<<nblocks(S, 256), 256, 0, st>>>(c->d_scene_active, c->d_scene_cand, c->d_scene_ex,
                                                    c->d_scene_mg2, c->d_scene_iters, S, tol,
                                                    c->params.g_accel * c->params.g_accel, max_it, c->d_tol_count,
                                                    c->d_counters + 2, c->d_scene_rin);
    count_launch(c);
}

// End of one iteration of the device-driven loop: counts it and continues the
// while node while scenes are still iterating.  iters of a scene reach max_it
// within max_it iterations, so n_active is 0 by then; the index bound stops
// the loop at max_it in any case.  Also counts the body's kernel launches.
__global__ void k_tol_loop_next(cudaGraphConditionalHandle h, const int* n_active, uint32_t* it,
                                const double* omega_tab, double* omega, unsigned max_it,
                                unsigned long long body_launches, unsigned long long* launches) {
    const uint32_t i = *it + 1;
    *it = i;
    *launches += body_launches;
    const bool more = *n_active > 0 && i < max_it;
    if (more) *omega = omega_tab[i];
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

void launch_tol_loop_next(avbd_ctx* c, cudaGraphConditionalHandle h, unsigned max_it, unsigned body_launches,
                          cudaStream_t st) {
    k_tol_loop_next<<<1, 1, 0, st>>>(h, c->d_tol_count, c->d_tol_it, c->d_omega_tab, c->d_tol_omega, max_it,
                                     body_launches + 1ull, c->d_counters + 5);
}

__global__ void k_iter_set(uint32_t* it, double* omega, const double* omega_tab) {
    *it = 0;
    *omega = omega_tab[0];
}
__global__ void k_iter_next(uint32_t* it, double* omega, const double* omega_tab, unsigned n) {
    const uint32_t i = *it + 1;
    *it = i;
    if (i < n) *omega = omega_tab[i];
}
void launch_iter_set(avbd_ctx* c, cudaStream_t st) {
    k_iter_set<<<1, 1, 0, st>>>(c->d_tol_it, c->d_tol_omega, c->d_omega_tab);
    count_launch(c);
}
void launch_iter_next(avbd_ctx* c, unsigned n, cudaStream_t st) {
    k_iter_next<<<1, 1, 0, st>>>(c->d_tol_it, c->d_tol_omega, c->d_omega_tab, n);
    count_launch(c);
}

template <typename R>
void launch_debug_block(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned p, double* out, cudaStream_t st) {
    solve_lanes<MODE_DEBUG>(c, s, k, p, 1, st, out, SceneTol());
}

// warm-start features of every solved tet vertex at the current iterate,
// one 64-byte BF16 row per internal vertex
template <typename R>
void launch_features(avbd_ctx* c, DevState<R>& s, const StepConsts& k, void* feat, const float* prev,
                     cudaStream_t st) {
    c->ws_prev_arg = prev;
    solve_lanes<MODE_FEATURES>(c, s, k, 0, s.n, st, reinterpret_cast<double*>(feat), SceneTol());
    c->ws_prev_arg = nullptr;
}

// copy of the solved vertices' warm-start positions (x0)
template <typename R>
__global__ void k_ws_save(const DevState<R> s, typename Vec4Of<R>::T* x0) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < s.n) x0[p] = s.x[p];
}

// target row (x_end - x0) / s, column 3 = 1 for solved tet vertices, else 0
template <typename R>
__global__ void k_ws_target(const DevState<R> s, const typename Vec4Of<R>::T* x0, float inv_s, float4* t) {
    unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n) return;
    if (s.flags[p] & (VF_FIXED | VF_ORIENTED)) {
        t[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    typename Vec4Of<R>::T a = s.x[p], b = x0[p];
    t[p] = make_float4((float)(a.x - b.x) * inv_s, (float)(a.y - b.y) * inv_s, (float)(a.z - b.z) * inv_s, 1.f);
}

template <typename R>
void launch_ws_save(avbd_ctx* c, DevState<R>& s, void* x0, cudaStream_t st) {
    k_ws_save<R><<<nblocks(s.n, 256), 256, 0, st>>>(s, reinterpret_cast<typename Vec4Of<R>::T*>(x0));
    count_launch(c);
}

template <typename R>
void launch_ws_target(avbd_ctx* c, DevState<R>& s, const void* x0, double inv_s, float* t, cudaStream_t st) {
    k_ws_target<R><<<nblocks(s.n, 256), 256, 0, st>>>(s, reinterpret_cast<const typename Vec4Of<R>::T*>(x0),
                                                       (float)inv_s, reinterpret_cast<float4*>(t));
    count_launch(c);
}

template <typename R>
void launch_load_positions(DevState<R>& s, const double* src, const uint32_t* inv_map, unsigned first, unsigned n,
                           int mode, cudaStream_t st) {
    if (n == 0) return;
    k_load<R><<<nblocks(n, 256), 256, 0, st>>>(s, src, inv_map, first, n, mode);
}

template <typename R>
void launch_store_vec(const DevState<R>& s, int which, double* dst, const uint32_t* inv_map, unsigned n,
                      cudaStream_t st) {
    if (n == 0) return;
    k_store<R><<<nblocks(n, 256), 256, 0, st>>>(s, which, dst, inv_map, 0, n);
}

#define INST(R)                                                                                                  \
    template void launch_begin_step<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t);               \
    template void launch_tet_eprev<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t);                \
    template void launch_solve_color<R>(avbd_ctx*, DevState<R>&, const StepConsts&, unsigned, unsigned,         \
                                        cudaStream_t, const SceneTol&, const uint32_t*, const uint4*, unsigned); \
    template bool launch_sweep_persistent<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t,           \
                                             const SceneTol&);                                                  \
    template void launch_chebyshev_dual<R>(avbd_ctx*, DevState<R>&, const StepConsts&, double, unsigned, cudaStream_t,    \
                                           const SceneTol&);                                                    \
    template void launch_velocity<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t);                 \
    template void launch_residual<R>(avbd_ctx*, DevState<R>&, const StepConsts&, double*, cudaStream_t,         \
                                     const SceneTol&);                                                          \
    template void launch_debug_block<R>(avbd_ctx*, DevState<R>&, const StepConsts&, unsigned, double*,          \
                                        cudaStream_t);                                                          \
    template void launch_features<R>(avbd_ctx*, DevState<R>&, const StepConsts&, void*, const float*,           \
                                     cudaStream_t);                                                             \
    template void launch_ws_save<R>(avbd_ctx*, DevState<R>&, void*, cudaStream_t);                               \
    template void launch_ws_target<R>(avbd_ctx*, DevState<R>&, const void*, double, float*, cudaStream_t);       \
    template void launch_load_positions<R>(DevState<R>&, const double*, const uint32_t*, unsigned, unsigned, int, \
                                           cudaStream_t);                                                       \
    template void launch_store_vec<R>(const DevState<R>&, int, double*, const uint32_t*, unsigned, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace avbd
