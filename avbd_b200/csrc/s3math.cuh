// s3math.cuh -- unit-quaternion and SO(3) helpers of the oriented-particle
// (6-DOF) path, restating common/Math.hpp:13-246 of the reference:
// Skew3, Exp_s3 / Log_S3 / Minus_S3 / Plus_S3 (with their small-angle
// branches at 1e-6), Exp_so3 and the right Jacobian of the exponential map
// and its inverse (small-angle branches at 1e-8).  Quaternions are stored
// (w, x, y, z) in the x, y, z, w fields of a 4-vector.
#pragma once

#include "common.cuh"

namespace avbd {

template <typename R>
struct Q4 {
    R w, x, y, z;
};

template <typename R>
struct M3 {
    R a[3][3];
};

template <typename V>
AVBD_HD auto q_of(const V& v) -> Q4<decltype(v.x)> { return {v.x, v.y, v.z, v.w}; }
template <typename R>
AVBD_HD typename Vec4Of<R>::T q_store(Q4<R> q) {
    typename Vec4Of<R>::T r;
    r.x = q.w; r.y = q.x; r.z = q.y; r.w = q.z;
    return r;
}

template <typename R>
AVBD_HD Q4<R> qmul(Q4<R> a, Q4<R> b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
            a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x};
}
template <typename R>
AVBD_HD Q4<R> qconj(Q4<R> q) { return {q.w, -q.x, -q.y, -q.z}; }

// rotation of v by a unit quaternion: v + w t + u x t with t = 2 u x v
template <typename R>
AVBD_HD V3<R> qrot(Q4<R> q, V3<R> v) {
    V3<R> u = mk3(q.x, q.y, q.z);
    V3<R> t = cross3(u, v);
    t = t + t;
    return v + q.w * t + cross3(u, t);
}

template <typename R>
AVBD_HD M3<R> qmat(Q4<R> q) {
    R tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z;
    R twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
    R txx = tx * q.x, txy = ty * q.x, txz = tz * q.x;
    R tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
    M3<R> m;
    m.a[0][0] = 1 - (tyy + tzz); m.a[0][1] = txy - twz;       m.a[0][2] = txz + twy;
    m.a[1][0] = txy + twz;       m.a[1][1] = 1 - (txx + tzz); m.a[1][2] = tyz - twx;
    m.a[2][0] = txz - twy;       m.a[2][1] = tyz + twx;       m.a[2][2] = 1 - (txx + tyy);
    return m;
}

template <typename R>
AVBD_HD M3<R> mzero() {
    M3<R> m;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m.a[i][j] = 0;
    return m;
}
template <typename R>
AVBD_HD M3<R> meye() {
    M3<R> m = mzero<R>();
    m.a[0][0] = m.a[1][1] = m.a[2][2] = 1;
    return m;
}
template <typename R>
AVBD_HD M3<R> mmul(const M3<R>& A, const M3<R>& B) {
    M3<R> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C.a[i][j] = A.a[i][0] * B.a[0][j] + A.a[i][1] * B.a[1][j] + A.a[i][2] * B.a[2][j];
    return C;
}
template <typename R>
AVBD_HD M3<R> mT(const M3<R>& A) {
    M3<R> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C.a[i][j] = A.a[j][i];
    return C;
}
template <typename R>
AVBD_HD M3<R> madd(const M3<R>& A, const M3<R>& B, R sa = 1, R sb = 1) {
    M3<R> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C.a[i][j] = sa * A.a[i][j] + sb * B.a[i][j];
    return C;
}
template <typename R>
AVBD_HD M3<R> mscale(const M3<R>& A, R s) {
    M3<R> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C.a[i][j] = s * A.a[i][j];
    return C;
}
template <typename R>
AVBD_HD V3<R> mvec(const M3<R>& A, V3<R> v) {
    return mk3(A.a[0][0] * v.x + A.a[0][1] * v.y + A.a[0][2] * v.z,
               A.a[1][0] * v.x + A.a[1][1] * v.y + A.a[1][2] * v.z,
               A.a[2][0] * v.x + A.a[2][1] * v.y + A.a[2][2] * v.z);
}
// Math::Skew3 (common/Math.hpp:13-20)
template <typename R>
AVBD_HD M3<R> skew(V3<R> v) {
    M3<R> m = mzero<R>();
    m.a[0][1] = -v.z; m.a[0][2] = v.y;
    m.a[1][0] = v.z;  m.a[1][2] = -v.x;
    m.a[2][0] = -v.y; m.a[2][1] = v.x;
    return m;
}

template <typename R>
AVBD_HD R norm3(V3<R> v) { return sqrt(dot3(v, v)); }

// Math::Exp_s3 (common/Math.hpp:197-222)
template <typename R>
AVBD_HD Q4<R> exp_s3(V3<R> v) {
    R th = norm3(v);
    if (th < R(1e-6)) {
        Q4<R> q{R(1), R(0.5) * v.x, R(0.5) * v.y, R(0.5) * v.z};
        R n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
        return {q.w / n, q.x / n, q.y / n, q.z / n};
    }
    R h = R(0.5) * th;
    R s = sin(h) / th;
    return {cos(h), s * v.x, s * v.y, s * v.z};
}
// Math::Log_S3 (common/Math.hpp:224-236)
template <typename R>
AVBD_HD V3<R> log_s3(Q4<R> q) {
    V3<R> v = mk3(q.x, q.y, q.z);
    R m = norm3(v);
    if (m < R(1e-6)) return R(2) * v;
    R th = R(2) * atan2(m, q.w);
    return (th / m) * v;
}
// Math::Minus_S3 / Plus_S3 (common/Math.hpp:238-246)
template <typename R>
AVBD_HD V3<R> minus_s3(Q4<R> q1, Q4<R> q2) { return log_s3(qmul(qconj(q2), q1)); }
template <typename R>
AVBD_HD Q4<R> plus_s3(Q4<R> q, V3<R> r) { return qmul(q, exp_s3(r)); }

// Plus_S3 for stored rotations.  In FP64 the product of unit quaternions stays
// unit to ~1e-16 per update, as in the reference.  In FP32 the norm would
// random-walk by ~1e-7 per update over thousands of updates a second, and qrot
// of a non-unit q scales the rotated vector (a spurious strain of the stiff rod
// shear terms), so FP32 storage renormalises after every update.
template <typename R>
AVBD_HD Q4<R> plus_s3_stored(Q4<R> q, V3<R> r) {
    Q4<R> o = plus_s3(q, r);
    if constexpr (sizeof(R) == 4) {
        R n = R(1) / sqrt(o.w * o.w + o.x * o.x + o.y * o.y + o.z * o.z);
        o = {o.w * n, o.x * n, o.y * n, o.z * n};
    }
    return o;
}

// Math::ExpMap_RightJacobian (common/Math.hpp:28-38)
template <typename R>
AVBD_HD M3<R> right_jac(V3<R> th) {
    R n = norm3(th);
    M3<R> S = skew(th);
    if (n < R(1e-8)) return madd(meye<R>(), S, R(1), R(-0.5));
    return madd(madd(meye<R>(), S, R(1), -(R(1) - cos(n)) / (n * n)), mmul(S, S), R(1), (n - sin(n)) / (n * n * n));
}
// Math::ExpMap_InvRightJacobian (common/Math.hpp:136-147)
template <typename R>
AVBD_HD M3<R> inv_right_jac(V3<R> th) {
    R n = norm3(th);
    M3<R> S = skew(th);
    if (n < R(1e-8)) return madd(meye<R>(), S, R(1), R(0.5));
    R c = R(1) / (n * n) - (R(1) + cos(n)) / (R(2) * n * sin(n));
    return madd(madd(meye<R>(), S, R(1), R(0.5)), mmul(S, S), R(1), c);
}
// Math::Exp_so3 (common/Math.hpp:149-158)
template <typename R>
AVBD_HD M3<R> exp_so3(V3<R> v) {
    M3<R> S = skew(v);
    R m = norm3(v);
    if (m < R(1e-8)) return madd(meye<R>(), S);
    return madd(madd(meye<R>(), S, R(1), sin(m) / m), mmul(S, S), R(1), (R(1) - cos(m)) / (m * m));
}

}  // namespace avbd
