// common.cuh -- device math shared by the engine's kernels.
//
// All per-vertex state lives in HBM as 16-byte float4 records (FP32 path) or
// 32-byte records of four doubles (FP64 parity path); the templates below let
// one kernel body serve both.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "avbd.h"

#define AVBD_HD __host__ __device__ __forceinline__
#define AVBD_D __device__ __forceinline__

// AVBD constants of the reference (common/common.hpp:13-15).
#define AVBD_BETA 10.0
#define AVBD_GAMMA 0.99
#define AVBD_ALPHA 0.95

struct alignas(32) double4a {
    double x, y, z, w;
};

template <typename R> struct Vec4Of;
template <> struct Vec4Of<float> { using T = float4; };
template <> struct Vec4Of<double> { using T = double4a; };

template <typename R>
struct V3 {
    R x, y, z;
};

template <typename R>
AVBD_HD V3<R> mk3(R a, R b, R c) { return V3<R>{a, b, c}; }

template <typename R> AVBD_HD V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> AVBD_HD V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R> AVBD_HD V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename R> AVBD_HD R dot3(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> AVBD_HD V3<R> cross3(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <typename V> AVBD_D auto xyz(const V& v) -> V3<decltype(v.x)> { return {v.x, v.y, v.z}; }

template <typename R>
AVBD_HD typename Vec4Of<R>::T make4(V3<R> v, R w) {
    typename Vec4Of<R>::T r;
    r.x = v.x; r.y = v.y; r.z = v.z; r.w = w;
    return r;
}

// Streaming (evict-first) 16-byte load for data read once per launch.
AVBD_D float4 ld_stream(const float4* p) { return __ldcs(p); }
AVBD_D double4a ld_stream(const double4a* p) {
    double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    return double4a{a.x, a.y, b.x, b.y};
}
// Read-only-path load for neighbour positions (never written during a launch).
AVBD_D float4 ld_ro(const float4* p) { return __ldg(p); }
AVBD_D double4a ld_ro(const double4a* p) {
    double2 a = __ldg(reinterpret_cast<const double2*>(p));
    double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return double4a{a.x, a.y, b.x, b.y};
}

template <typename T>
AVBD_D T shfl_xor(T v, int mask) { return __shfl_xor_sync(0xffffffffu, v, mask); }

// Symmetric 3x3 stored as (00, 11, 22, 01, 02, 12).
template <typename R>
struct Sym3 {
    R a00, a11, a22, a01, a02, a12;
};

// Solves (A) x = b for a symmetric 3x3 through the adjugate.  Returns the
// condition estimate kappa = |A|_F |adj A|_F / |det A| (infinite when singular).
template <typename R>
AVBD_D R solve_sym3(const Sym3<R>& A, V3<R> b, V3<R>& x) {
    R c00 = A.a11 * A.a22 - A.a12 * A.a12;
    R c01 = A.a02 * A.a12 - A.a01 * A.a22;
    R c02 = A.a01 * A.a12 - A.a02 * A.a11;
    R c11 = A.a00 * A.a22 - A.a02 * A.a02;
    R c12 = A.a01 * A.a02 - A.a00 * A.a12;
    R c22 = A.a00 * A.a11 - A.a01 * A.a01;
    R det = A.a00 * c00 + A.a01 * c01 + A.a02 * c02;
    R inv = R(1) / det;
    x.x = (c00 * b.x + c01 * b.y + c02 * b.z) * inv;
    x.y = (c01 * b.x + c11 * b.y + c12 * b.z) * inv;
    x.z = (c02 * b.x + c12 * b.y + c22 * b.z) * inv;
    R na = A.a00 * A.a00 + A.a11 * A.a11 + A.a22 * A.a22 + R(2) * (A.a01 * A.a01 + A.a02 * A.a02 + A.a12 * A.a12);
    R nc = c00 * c00 + c11 * c11 + c22 * c22 + R(2) * (c01 * c01 + c02 * c02 + c12 * c12);
    return sqrt(na * nc) * fabs(inv);
}

// Dense LU with row pivoting for small N in FP64 (the fallback for
// ill-conditioned blocks and the 6x6 rod blocks).
template <int N>
AVBD_D void lu_solve_d(double (&A)[N][N], double (&b)[N], double (&x)[N]) {
#pragma unroll
    for (int k = 0; k < N; k++) {
        int p = k;
        double best = fabs(A[k][k]);
#pragma unroll
        for (int i = k + 1; i < N; i++) {
            double v = fabs(A[i][k]);
            if (v > best) { best = v; p = i; }
        }
        if (p != k) {
#pragma unroll
            for (int j = 0; j < N; j++) { double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
#pragma unroll
        for (int i = k + 1; i < N; i++) {
            double l = A[i][k] / A[k][k];
            A[i][k] = l;
#pragma unroll
            for (int j = k + 1; j < N; j++) A[i][j] -= l * A[k][j];
            b[i] -= l * b[k];
        }
    }
#pragma unroll
    for (int i = N - 1; i >= 0; i--) {
        double s = b[i];
#pragma unroll
        for (int j = i + 1; j < N; j++) s -= A[i][j] * x[j];
        x[i] = s / A[i][i];
    }

}

// Barrier over every block of a cooperative launch.  sync[0] counts the
// arrivals, sync[1] is the generation: thread 0 of the last block to arrive
// resets the count and advances the generation, the others poll it at most
// `limit` times and then set AVBD_ERR_BARRIER_TIMEOUT in *err.  A block
// returns false when that error (or any other in *err) is set, so that every
// block leaves the kernel; the polls are bounded, so none waits forever.
AVBD_D bool grid_barrier_bounded(unsigned* sync, int* err, unsigned limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = *(volatile unsigned*)(sync + 1);
        int good = 1;
        __threadfence();
        if (atomicAdd(sync, 1u) == gridDim.x - 1) {
            atomicExch(sync, 0u);
            __threadfence();
            atomicAdd(sync + 1, 1u);
        } else {
            unsigned polls = 0;
            while (*(volatile unsigned*)(sync + 1) == gen) {
                if (polls++ >= limit || *(volatile int*)err != 0) {
                    good = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (!good) atomicCAS(err, 0, (int)AVBD_ERR_BARRIER_TIMEOUT);
        ok = good && *(volatile int*)err == 0;
    }
    __syncthreads();
    return ok != 0;
}
