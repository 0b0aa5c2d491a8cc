// narrow.cu -- narrow phase of the collision stage: the broad phase's
// candidate leaf pairs are mapped to primitives, same-object pairs sharing a
// vertex are skipped; triangle-sphere pairs run the continuous collision
// test of CollisionDetector::_triangleSDF_CCD (collision/CollisionDetector.cpp:
// 689-876; Pelletier-Guenette 2025): alternating golden-section searches in
// time and on the triangle for the first contact of the moving triangle with
// the moving sphere during the step; triangle-rod-segment pairs the
// closest-point test of CollisionDetector::_triangleRod (:601-666) at the
// step-start positions.  One thread per candidate pair.
//
// Compiled without FMA contraction, in FP64, in the reference's operation
// order: detections equal the FP64 oracle's (sin/cos of a rotating sphere may
// differ in the last bit from the host library's).
#include "engine.h"
#include "s3math.cuh"

namespace avbd {
namespace {

using D3 = V3<double>;
using DQ = Q4<double>;

AVBD_D double sdf_sphere(double r, D3 p) { return norm3(p) - r; }
AVBD_D D3 sdf_sphere_grad(D3 p) {
    const double d = norm3(p);
    return d > 1e-8 ? mk3(p.x / d, p.y / d, p.z / d) : mk3(1.0, 0.0, 0.0);
}
// std::min / std::max as the reference evaluates them
AVBD_D double min_ref(double a, double b) { return (b < a) ? b : a; }

AVBD_D double gss_width(double x) { return fabs(x); }
AVBD_D double gss_width(D3 x) { return norm3(x); }
AVBD_D double gss_lerp(double a, double b, double s) { return (1 - s) * a + s * b; }
AVBD_D D3 gss_lerp(D3 a, D3 b, double s) { return (1 - s) * a + s * b; }

// Algorithm::goldenSectionSearch (common/Algorithm.hpp:252-294), bracket
// width 1e-3; at most 64 shrink steps (the width falls by 0.618 per step)
template <typename T, typename F>
AVBD_D T gss(T lo, T hi, F f) {
    const double phi = 1.61803398875, r = 1 / phi, sg = 1 - r, tol = 1e-3;
    double a0 = 0, a1 = sg, a2 = r, a3 = 1;
    T t0 = lo, t1 = gss_lerp(lo, hi, a1), t2 = gss_lerp(lo, hi, a2), t3 = hi;
    double f0 = f(t0), f1 = f(t1), f2 = f(t2), f3 = f(t3);
    for (int guard = 0; gss_width(t3 - t0) > tol && guard < 64; guard++) {
        if (min_ref(f0, f1) < min_ref(f2, f3)) {
            a3 = a2; t3 = t2; f3 = f2;
            a2 = a1; t2 = t1; f2 = f1;
            a1 = r * a2 + sg * a0;
            t1 = gss_lerp(lo, hi, a1);
            f1 = f(t1);
        } else {
            a0 = a1; t0 = t1; f0 = f1;
            a1 = a2; t1 = t2; f1 = f2;
            a2 = r * a1 + sg * a3;
            t2 = gss_lerp(lo, hi, a2);
            f2 = f(t2);
        }
    }
    T tm = gss_lerp(lo, hi, 0.5 * (a0 + a3));
    double fm = f(tm);
    if (f0 < fm && f0 < f3) return t0;
    if (fm < f3) return tm;
    return t3;
}

// Math::barycentricCoordinates (common/Math.hpp:421-438)
AVBD_D D3 barycentric(D3 p, D3 a, D3 b, D3 c) {
    D3 v0 = b - a, v1 = c - a, v2 = p - a;
    double d00 = dot3(v0, v0), d01 = dot3(v0, v1), d11 = dot3(v1, v1), d20 = dot3(v2, v0), d21 = dot3(v2, v1);
    double den = d00 * d11 - d01 * d01;
    double v = (d11 * d20 - d01 * d21) / den;
    double w = (d00 * d21 - d01 * d20) / den;
    return mk3(1 - v - w, v, w);
}

// rotation by the inverse of q, Eigen's inverse (conjugate / |q|^2)
AVBD_D D3 qrot_inv(DQ q, D3 v) {
    const double n2 = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    DQ i{q.w / n2, -q.x / n2, -q.y / n2, -q.z / n2};
    return qrot(i, v);
}

struct Body {
    D3 x, v, w;
    DQ q;
    double r;
    AVBD_D D3 pos(double t) const { return x + t * v; }
    AVBD_D DQ rot(double t) const { return qmul(q, exp_s3(t * w)); }
    AVBD_D D3 to_local(D3 xg, double t) const { return qrot_inv(rot(t), xg - pos(t)); }
    AVBD_D D3 point_vel(D3 xg, double t) const { return v + cross3(qrot(rot(t), w), xg - pos(t)); }
    AVBD_D D3 rel_vel(D3 xg, D3 vg, double t) const { return qrot_inv(rot(t), vg - point_vel(xg, t)); }
};

AVBD_D bool tri_sphere_ccd(const Body& B, const D3 p[3], const D3 vv[3], double dt, double margin, D3& normal,
                           D3& barys, D3& cp_local) {
    double e[3];
#pragma unroll
    for (int k = 0; k < 3; k++) e[k] = dot3(B.rel_vel(p[k], vv[k], 0), sdf_sphere_grad(B.to_local(p[k], 0)));
    double t_start = 0, t_end = dt, t = 0, u, v, w;
    if (e[0] < e[1] && e[0] < e[2]) { u = 1; v = 0; w = 0; }
    else if (e[1] < e[0] && e[1] < e[2]) { u = 0; v = 1; w = 0; }
    else { u = 0; v = 0; w = 1; }
    auto interp = [&](double tt) { return u * (p[0] + tt * vv[0]) + v * (p[1] + tt * vv[1]) + w * (p[2] + tt * vv[2]); };
    auto sd_time = [&](double tt) { return sdf_sphere(B.r, B.to_local(interp(tt), tt)); };
    auto ud_time = [&](double tt) { return fabs(sd_time(tt)); };
    auto sd_point = [&](D3 xl) { return sdf_sphere(B.r, xl); };
    double sd = 0;
    D3 grad = mk3(0.0, 0.0, 0.0), x_ti = mk3(0.0, 0.0, 0.0);
    for (int it = 0; it < 16; it++) {
        const double t_old = t;
        D3 xg = interp(t), vg = u * vv[0] + v * vv[1] + w * vv[2];
        x_ti = B.to_local(xg, t);
        D3 v_ti = B.rel_vel(xg, vg, t);
        sd = sdf_sphere(B.r, x_ti);
        if (sd <= 0) {
            t_end = min_ref(t, t_end);
            t = gss(t_start, t, ud_time);
        } else {
            const double vdg = dot3(v_ti, sdf_sphere_grad(x_ti));
            if (vdg > 0) t = gss(t_start, t, sd_time);
            else t = gss(t, t_end, sd_time);
        }
        xg = interp(t);
        x_ti = B.to_local(xg, t);
        sd = sdf_sphere(B.r, x_ti);
        grad = sdf_sphere_grad(x_ti);
        if (sd <= 0) t_end = min_ref(t, t_end);
        const D3 l1 = B.to_local(p[0] + t * vv[0], t), l2 = B.to_local(p[1] + t * vv[1], t),
                 l3 = B.to_local(p[2] + t * vv[2], t);
        const double s1 = dot3(l1, grad), s2 = dot3(l2, grad), s3 = dot3(l3, grad);
        const D3 sv = (s1 < s2 && s1 < s3) ? l1 : ((s2 < s1 && s2 < s3) ? l2 : l3);
        const D3 x_new = gss(x_ti, sv, sd_point);
        const D3 b = barycentric(x_new, l1, l2, l3);
        u = b.x; v = b.y; w = b.z;
        if (fabs(t_old - t) < 1e-6 && norm3(x_new - x_ti) < 1e-6) break;
    }
    barys = mk3(u, v, w);
    cp_local = x_ti - sd * grad;
    normal = qrot(B.rot(t), grad);
    return sd < margin;
}

// Math::closestPoint_PointTriangle (common/Math.hpp:446-500), Ericson's regions
AVBD_D D3 closest_point_triangle(D3 p, D3 a, D3 b, D3 c) {
    const D3 ab = b - a, ac = c - a, ap = p - a;
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) return a;
    const D3 bp = p - b;
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0 && d4 <= d3) return b;
    const D3 cp = p - c;
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) return c;
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return a + (d1 / (d1 - d3)) * ab;
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return a + (d2 / (d2 - d6)) * ac;
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
    const double den = 1.0 / (va + vb + vc);
    const double v = vb * den, w = vc * den;
    return a + v * ab + w * ac;
}

AVBD_D double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }  // std::clamp

// Math::closestPoint_SegmentSegment (common/Math.hpp:508-560): s on (p1, q1), t on (p2, q2)
AVBD_D void closest_segment_segment(D3 p1, D3 q1, D3 p2, D3 q2, double& s, double& t) {
    const D3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    const double EPS = 1e-8;
    if (a <= EPS && e <= EPS) {
        s = t = 0.0;
        return;
    }
    if (a <= EPS) {
        s = 0.0;
        t = clamp01(f / e);
    } else {
        const double cc = dot3(d1, r);
        if (e <= EPS) {
            t = 0.0;
            s = clamp01(-cc / a);
        } else {
            const double b = dot3(d1, d2);
            const double den = a * e - b * b;
            s = den != 0.0 ? clamp01((b * f - cc * e) / den) : 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) {
                t = 0.0;
                s = clamp01(-cc / a);
            } else if (t > 1.0) {
                t = 1.0;
                s = clamp01((b - cc) / a);
            }
        }
    }
}

// Math::pointInTriangle (common/Math.hpp:562-591)
AVBD_D bool point_in_triangle(D3 p, D3 a, D3 b, D3 c) {
    const D3 v0 = b - a, v1 = c - a, v2 = p - a;
    const double d00 = dot3(v0, v0), d01 = dot3(v0, v1), d11 = dot3(v1, v1), d20 = dot3(v2, v0), d21 = dot3(v2, v1);
    const double den = d00 * d11 - d01 * d01;
    if (fabs(den) < 1e-12) return false;
    const double v = (d11 * d20 - d01 * d21) / den;
    const double w = (d00 * d21 - d01 * d20) / den;
    const double u = 1.0 - v - w;
    return u >= -1e-8 && v >= -1e-8 && w >= -1e-8;
}

// Math::closestPoint_SegmentTriangle (common/Math.hpp:593-681): the crossing
// point, else the closest of the three edge tests and the two end points.
// The edge test measures the distance to the edge point at the segment's
// parameter s, (1-s) q0 + s q1, as the reference does.
AVBD_D void closest_segment_triangle(D3 p0, D3 p1, D3 a, D3 b, D3 c, double& s_out, D3& bary, double& dist) {
    const double EPS = 1e-8;
    const D3 dir = p1 - p0;
    const D3 nrm = cross3(b - a, c - a);
    s_out = 0.0;
    bary = mk3(1.0, 0.0, 0.0);
    dist = 1.7976931348623157e308;  // std::numeric_limits<double>::max()
    if (dot3(nrm, nrm) > EPS) {
        const double den = dot3(nrm, dir);
        if (fabs(den) > EPS) {
            const double s = dot3(nrm, a - p0) / den;
            if (s >= 0.0 && s <= 1.0) {
                const D3 p = p0 + s * dir;
                if (point_in_triangle(p, a, b, c)) {
                    s_out = s;
                    bary = barycentric(p, a, b, c);
                    dist = 0.0;
                    return;
                }
            }
        }
    }
    const D3 q0s[3] = {a, a, b}, q1s[3] = {b, c, c};
    const int i0s[3] = {0, 0, 1}, i1s[3] = {1, 2, 2};
#pragma unroll
    for (int e = 0; e < 3; e++) {
        double s, t;
        closest_segment_segment(p0, p1, q0s[e], q1s[e], s, t);
        const D3 cp = (1 - s) * p0 + s * p1;
        const D3 cq = (1 - s) * q0s[e] + s * q1s[e];
        const D3 dd = cp - cq;
        const double d2 = dot3(dd, dd);
        if (d2 < dist * dist) {
            s_out = s;
            double bb[3] = {0.0, 0.0, 0.0};
            bb[i0s[e]] = 1 - t;
            bb[i1s[e]] = t;
            bary = mk3(bb[0], bb[1], bb[2]);
            dist = sqrt(d2);
        }
    }
    const D3 c0 = closest_point_triangle(p0, a, b, c);
    const D3 e0 = p0 - c0;
    const double d0 = dot3(e0, e0);
    if (d0 < dist * dist) {
        s_out = 0.0;
        bary = barycentric(c0, a, b, c);
        dist = sqrt(d0);
    }
    const D3 c1 = closest_point_triangle(p1, a, b, c);
    const D3 e1 = p1 - c1;
    const double d1 = dot3(e1, e1);
    if (d1 < dist * dist) {
        s_out = 1.0;
        bary = barycentric(c1, a, b, c);
        dist = sqrt(d1);
    }
}

// CollisionDetector::_triangleRod (collision/CollisionDetector.cpp:601-666)
AVBD_D bool tri_rod_contact(const D3 v[3], D3 s1, D3 s2, DQ q1, DQ q2, double radius, double margin, D3& normal,
                            D3& bary, double& s, D3& cp_local) {
    double dist;
    closest_segment_triangle(s1, s2, v[0], v[1], v[2], s, bary, dist);
    if (!(dist < radius + margin)) return false;
    const D3 cl = (1 - s) * s1 + s * s2;
    const D3 ct = bary.x * v[0] + bary.y * v[1] + bary.z * v[2];
    const D3 d = ct - cl;
    const double m = norm3(d);
    normal = m > 1e-8 ? mk3(d.x / m, d.y / m, d.z / m) : mk3(1.0, 0.0, 0.0);
    const DQ qm = plus_s3(q1, s * minus_s3(q2, q1));
    cp_local = qrot_inv(qm, radius * normal);
    return true;
}

// DetectedCollision::generateKey (collision/DetectedCollision.hpp:43-66)
AVBD_D uint64_t collision_key(unsigned type, unsigned a, unsigned b, unsigned code) {
    if (a > b) { unsigned t = a; a = b; b = t; }
    uint64_t k = type & 31u;
    k = (k << 26) | (a & 0x3FFFFFFu);
    k = (k << 26) | (b & 0x3FFFFFFu);
    return (k << 7) | (code & 127u);
}

AVBD_D unsigned prim_np(uint8_t t) { return t == AVBD_SHAPE_TRIANGLE ? 3u : (t == AVBD_SHAPE_ROD_SEGMENT ? 2u : 1u); }

template <typename R>
AVBD_D D3 ld3(const typename Vec4Of<R>::T* a, unsigned i) {
    typename Vec4Of<R>::T v = a[i];
    return mk3((double)v.x, (double)v.y, (double)v.z);
}

template <typename R>
__global__ void __launch_bounds__(128) k_narrow(DevState<R> s, LbvhState L, double dt, double margin, int* err) {
    const unsigned cnt = min(*L.pair_count, L.pair_capacity);
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint2 pr = L.pairs[i];
        unsigned a = L.sorted[pr.x], b = L.sorted[pr.y];
        if (L.obj[a] == L.obj[b]) {  // CollisionDetector::_shouldSkip
            const uint4 ia = L.pidx[a], ib = L.pidx[b];
            const unsigned xa[3] = {ia.x, ia.y, ia.z}, xb[3] = {ib.x, ib.y, ib.z};
            const unsigned na = prim_np(L.type[a]), nbp = prim_np(L.type[b]);
            bool share = false;
            for (unsigned u = 0; u < na; u++)
                for (unsigned v = 0; v < nbp; v++) share |= xa[u] == xb[v];
            if (share) continue;
        }
        if (L.type[a] > L.type[b]) { unsigned t = a; a = b; b = t; }
        if (L.type[a] != AVBD_SHAPE_TRIANGLE) continue;
        if (L.type[b] == AVBD_SHAPE_ROD_SEGMENT) {
            const uint4 it = L.pidx[a], ir = L.pidx[b];
            const D3 v[3] = {ld3<R>(s.x, it.x), ld3<R>(s.x, it.y), ld3<R>(s.x, it.z)};
            const typename Vec4Of<R>::T qa = s.q[s.rot[ir.x]], qb = s.q[s.rot[ir.y]];
            const DQ q1{(double)qa.x, (double)qa.y, (double)qa.z, (double)qa.w};
            const DQ q2{(double)qb.x, (double)qb.y, (double)qb.z, (double)qb.w};
            D3 nrm, bar, cp;
            double sp;
            if (!tri_rod_contact(v, ld3<R>(s.x, ir.x), ld3<R>(s.x, ir.y), q1, q2, L.radius[b], margin, nrm, bar, sp, cp))
                continue;
            const unsigned k = atomicAdd(L.contact_count, 1u);
            if (k >= L.contact_capacity) {
                atomicExch(err, (int)AVBD_ERR_CAPACITY);
                continue;
            }
            L.contact_key[k] = collision_key(3u, a, b, 0u);  // DetectedCollisionType::TriangleRod
            L.contact_idx[k] = make_uint4(it.x, it.y, it.z, ir.x);
            L.contact_idx5[k] = ir.y;
            double* o = L.contact_vec + 10ull * k;
            o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
            o[3] = bar.x; o[4] = bar.y; o[5] = bar.z;
            o[6] = cp.x; o[7] = cp.y; o[8] = cp.z;
            o[9] = sp;
            continue;
        }
        if (L.type[b] != AVBD_SHAPE_SPHERE) continue;
        const uint4 it = L.pidx[a];
        const unsigned rb = L.pidx[b].x, slot = s.rot[rb];
        Body B;
        B.x = ld3<R>(s.x, rb);
        B.v = ld3<R>(s.v, rb);
        B.w = ld3<R>(s.w, slot);
        const typename Vec4Of<R>::T q4 = s.q[slot];
        B.q = DQ{(double)q4.x, (double)q4.y, (double)q4.z, (double)q4.w};
        B.r = L.radius[b];
        const D3 p[3] = {ld3<R>(s.x, it.x), ld3<R>(s.x, it.y), ld3<R>(s.x, it.z)};
        const D3 vv[3] = {ld3<R>(s.v, it.x), ld3<R>(s.v, it.y), ld3<R>(s.v, it.z)};
        D3 nrm, bar, cp;
        if (!tri_sphere_ccd(B, p, vv, dt, margin, nrm, bar, cp)) continue;
        const unsigned k = atomicAdd(L.contact_count, 1u);
        if (k >= L.contact_capacity) {
            atomicExch(err, (int)AVBD_ERR_CAPACITY);
            continue;
        }
        L.contact_key[k] = collision_key(2u, a, b, 0u);  // DetectedCollisionType::TriangleRigid
        L.contact_idx[k] = make_uint4(it.x, it.y, it.z, rb);
        L.contact_idx5[k] = 0;
        double* o = L.contact_vec + 10ull * k;
        o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
        o[3] = bar.x; o[4] = bar.y; o[5] = bar.z;
        o[6] = cp.x; o[7] = cp.y; o[8] = cp.z;
        o[9] = 0.0;
    }
}

}  // namespace

template <typename R>
void launch_narrow(avbd_ctx* c, DevState<R>& s, cudaStream_t st) {
    LbvhState& L = c->lbvh;
    if (!L.contact_capacity) return;
    cudaMemsetAsync(L.contact_count, 0, sizeof(uint32_t), st);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    k_narrow<R><<<4 * sms, 128, 0, st>>>(s, L, c->params.dt, c->params.collision_margin, c->d_error);
    count_launch(c);
}
template void launch_narrow<float>(avbd_ctx*, DevState<float>&, cudaStream_t);
template void launch_narrow<double>(avbd_ctx*, DevState<double>&, cudaStream_t);

}  // namespace avbd
