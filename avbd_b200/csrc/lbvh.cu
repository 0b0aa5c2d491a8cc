// lbvh.cu -- collision broad phase on the GPU: swept AABBs, 63-bit Morton
// codes, stable LSD radix sort, Karras radix tree, bottom-up refit and the
// self traversal that yields the candidate leaf pairs.
//
// Reference behaviour followed (bit-exact on identical FP64 inputs):
//   CollisionPrimitivePool::speculativeGlobalBounds  collision/CollisionPrimitivePool.hpp:160-236
//   LBVHBuilder::computeAABB_MortonCode              collision/LBVHBuilder.cpp:98-127
//   LBVHBuilder::morton3D_64 / expandBits21          collision/LBVHBuilder.hpp:65-85
//   Algorithm::radixSort (stable, 8 x 8-bit passes)  common/Algorithm.hpp:22-56
//   LBVHBuilder::constructTree + commonPrefixLen     collision/LBVHBuilder.cpp:181-286, LBVHBuilder.hpp:33-41
//   LBVHBuilder::assembleBVH (refit)                 collision/LBVHBuilder.cpp:410-453
//   LBVHTraversal::traverseSelfIterative             collision/LBVHTraversal.hpp:30-88
// The FP64 arithmetic uses explicit round-to-nearest intrinsics so that no
// multiply-add is fused: p + dt*v is a multiply then an add, as in the
// reference built without FMA contraction.
//
// The self traversal of the reference emits every pair of leaves (a < b)
// whose boxes overlap: a node pair is pruned only when the node boxes are
// disjoint, which implies all leaf pairs below are disjoint too.  The same set
// is produced here by one thread per leaf a walking the tree for leaves b > a.
#include <algorithm>
#include <mutex>

#include "engine.h"
#include "s3math.cuh"

namespace avbd {

static constexpr int RB = 256;  // keys per radix tile (= threads per block)
static constexpr unsigned INVALID = 0xFFFFFFFFu;

AVBD_D unsigned long long ord_enc(double d) {
    unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
AVBD_D double ord_dec(unsigned long long u) {
    return __longlong_as_double((long long)((u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u));
}
AVBD_D double dmin_ref(double a, double b) { return (b < a) ? b : a; }  // std::min(a, b)
AVBD_D double dmax_ref(double a, double b) { return (a < b) ? b : a; }  // std::max(a, b)

template <typename R>
AVBD_D void pos_vel(const DevState<R>& s, unsigned p, double* x, double* v) {
    typename Vec4Of<R>::T a = s.x[p], b = s.v[p];
    x[0] = (double)a.x; x[1] = (double)a.y; x[2] = (double)a.z;
    v[0] = (double)b.x; v[1] = (double)b.y; v[2] = (double)b.z;
}

// |R| v, rows summed left to right
AVBD_D V3<double> abs_mat_vec(const M3<double>& R, V3<double> v) {
    return mk3(fabs(R.a[0][0]) * v.x + fabs(R.a[0][1]) * v.y + fabs(R.a[0][2]) * v.z,
               fabs(R.a[1][0]) * v.x + fabs(R.a[1][1]) * v.y + fabs(R.a[1][2]) * v.z,
               fabs(R.a[2][0]) * v.x + fabs(R.a[2][1]) * v.y + fabs(R.a[2][2]) * v.z);
}

// Swept bounds of every primitive and the scene box (exact min/max through
// order-preserving integer atomics).
template <typename R>
__global__ void __launch_bounds__(256) k_prim_bounds(DevState<R> s, LbvhState L, double dt,
                                                     unsigned long long* box) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    double mn[3] = {1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
    double mx[3] = {-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
    bool valid = i < L.n;
    if (valid) {
        uint4 id = L.pidx[i];
        uint8_t t = L.type[i];
        if (t == AVBD_SHAPE_TRIANGLE) {
            unsigned ids[3] = {id.x, id.y, id.z};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double x[3], v[3];
                pos_vel(s, ids[k], x, v);
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    mn[a] = dmin_ref(mn[a], x[a]);
                    mx[a] = dmax_ref(mx[a], x[a]);
                }
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    double nx = __dadd_rn(x[a], __dmul_rn(dt, v[a]));
                    mn[a] = dmin_ref(mn[a], nx);
                    mx[a] = dmax_ref(mx[a], nx);
                }
            }
        } else if (t == AVBD_SHAPE_SPHERE) {
            // analytic shape: local box [-r, r]^3 rotated into the world at the
            // current and at the predicted pose (CollisionPrimitivePool.hpp:199-231);
            // this file is compiled without FMA contraction, so the expressions
            // below round like the reference's
            const unsigned op = id.x, slot = s.rot[op];
            const double r = L.radius[i];
            const V3<double> lmin = mk3(-r, -r, -r), lmax = mk3(r, r, r);
            const V3<double> ctr = 0.5 * (lmin + lmax), he = 0.5 * (lmax - lmin);
            const typename Vec4Of<R>::T q4 = s.q[slot], w4 = s.w[slot];
            const Q4<double> q{(double)q4.x, (double)q4.y, (double)q4.z, (double)q4.w};
            double x[3], v[3];
            pos_vel(s, op, x, v);
            const V3<double> xp = mk3(x[0], x[1], x[2]), vp = mk3(v[0], v[1], v[2]);
            const V3<double> wc = qrot(q, ctr) + xp;
            const V3<double> we = abs_mat_vec(qmat(q), he);
            const Q4<double> nq = plus_s3(q, dt * mk3((double)w4.x, (double)w4.y, (double)w4.z));
            const V3<double> nwc = qrot(nq, ctr) + xp + dt * vp;
            const V3<double> nwe = abs_mat_vec(qmat(nq), he);
            const double c0[3] = {wc.x, wc.y, wc.z}, e0[3] = {we.x, we.y, we.z};
            const double c1[3] = {nwc.x, nwc.y, nwc.z}, e1[3] = {nwe.x, nwe.y, nwe.z};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                mn[a] = dmin_ref(c0[a] - e0[a], c1[a] - e1[a]);
                mx[a] = dmax_ref(c0[a] + e0[a], c1[a] + e1[a]);
            }
        } else {  // rod segment
            double x1[3], v1[3], x2[3], v2[3];
            pos_vel(s, id.x, x1, v1);
            pos_vel(s, id.y, x2, v2);
            double r = L.radius[i];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                mn[a] = __dsub_rn(dmin_ref(x1[a], x2[a]), r);
                mx[a] = __dadd_rn(dmax_ref(x1[a], x2[a]), r);
                double n1 = __dadd_rn(x1[a], __dmul_rn(dt, v1[a]));
                double n2 = __dadd_rn(x2[a], __dmul_rn(dt, v2[a]));
                mn[a] = dmin_ref(mn[a], __dsub_rn(dmin_ref(n1, n2), r));
                mx[a] = dmax_ref(mx[a], __dadd_rn(dmax_ref(n1, n2), r));
            }
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            L.aabb[6ull * i + a] = mn[a];
            L.aabb[6ull * i + 3 + a] = mx[a];
        }
    }
    // block reduction of the scene box
    unsigned long long e[6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        e[a] = valid ? ord_enc(mn[a]) : ~0ull;
        e[3 + a] = valid ? ord_enc(mx[a]) : 0ull;
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            unsigned long long o = __shfl_xor_sync(0xffffffffu, e[a], m);
            e[a] = o < e[a] ? o : e[a];
            o = __shfl_xor_sync(0xffffffffu, e[3 + a], m);
            e[3 + a] = o > e[3 + a] ? o : e[3 + a];
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            atomicMin(box + a, e[a]);
            atomicMax(box + 3 + a, e[3 + a]);
        }
    }
}

AVBD_D uint64_t expand21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

AVBD_D double clamp_ref(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

__global__ void __launch_bounds__(256) k_morton(LbvhState L, const unsigned long long* box) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    double smin[3], ext[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        smin[a] = ord_dec(box[a]);
        double e = __dsub_rn(ord_dec(box[3 + a]), smin[a]);
        ext[a] = (e < 1e-6) ? 1e-6 : e;  // extent.cwiseMax(1e-6)
    }
    uint64_t code = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        double c = __dmul_rn(__dadd_rn(L.aabb[6ull * i + a], L.aabb[6ull * i + 3 + a]), 0.5);
        double nx = __ddiv_rn(__dsub_rn(c, smin[a]), ext[a]);
        double q = clamp_ref(__dmul_rn(nx, 2097152.0), 0.0, 2097151.0);
        code |= expand21((uint64_t)q) << a;
    }
    L.morton[i] = code;
    L.sorted[i] = i;
}

// ---------------------------------------------------------- radix sort
__global__ void __launch_bounds__(RB) k_radix_count(const uint64_t* __restrict__ keys, unsigned n, int shift,
                                                    uint32_t* __restrict__ hist, unsigned nblk) {
    __shared__ uint32_t bins[256];
    bins[threadIdx.x] = 0;
    __syncthreads();
    unsigned i = blockIdx.x * RB + threadIdx.x;
    if (i < n) atomicAdd(&bins[(keys[i] >> shift) & 255u], 1u);
    __syncthreads();
    hist[(size_t)threadIdx.x * nblk + blockIdx.x] = bins[threadIdx.x];
}

// Exclusive scan of the digit-major histogram (digit d of block b at d*nblk+b).
// One block of 32 warps; warp w owns a contiguous segment and walks it 32
// entries at a time with coalesced loads (the walk's loads do not depend on
// the running carry, so they are in flight together): segment totals, a scan
// of the 32 totals, then the segment's exclusive scan from its offset.
// Integer sums, so the result does not depend on the split.
__global__ void __launch_bounds__(1024) k_radix_scan(uint32_t* hist, unsigned total) {
    __shared__ uint32_t wsum[32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned seg = (total + 31u) / 32u;
    const unsigned b = min(warp * seg, total), e = min(b + seg, total);
    uint32_t s = 0;
#pragma unroll 4
    for (unsigned k = b + lane; k < e; k += 32u) s += hist[k];
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    if (lane == 0) wsum[warp] = s;
    __syncthreads();
    if (warp == 0) {
        const uint32_t t = wsum[lane];
        uint32_t incl = t;
#pragma unroll
        for (int m = 1; m < 32; m <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, m);
            if (lane >= (unsigned)m) incl += u;
        }
        wsum[lane] = incl - t;
    }
    __syncthreads();
    uint32_t carry = wsum[warp];
#pragma unroll 4
    for (unsigned k0 = b; k0 < e; k0 += 32u) {
        const unsigned k = k0 + lane;
        const uint32_t v = k < e ? hist[k] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int m = 1; m < 32; m <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, m);
            if (lane >= (unsigned)m) incl += u;
        }
        if (k < e) hist[k] = carry + incl - v;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// Stable scatter: a key's destination is the global offset of (digit, tile)
// plus the number of equal digits before it in the tile (warps in order,
// lanes in order).
__global__ void __launch_bounds__(RB) k_radix_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                      uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                      unsigned n, int shift, const uint32_t* __restrict__ hist,
                                                      unsigned nblk) {
    __shared__ uint32_t wc[RB / 32][256];
    for (unsigned k = threadIdx.x; k < (RB / 32) * 256; k += RB) (&wc[0][0])[k] = 0;
    __syncthreads();
    unsigned i = blockIdx.x * RB + threadIdx.x;
    bool valid = i < n;
    unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned mask = __ballot_sync(0xffffffffu, valid);
    uint64_t key = valid ? kin[i] : 0;
    uint32_t val = valid ? vin[i] : 0;
    unsigned d = (unsigned)((key >> shift) & 255u);
    unsigned rank = 0;
    if (valid) {
        unsigned peers = __match_any_sync(mask, d);
        rank = __popc(peers & ((1u << lane) - 1u));
        if (rank == 0) wc[warp][d] = __popc(peers);
    }
    __syncthreads();
    {
        unsigned dg = threadIdx.x;  // RB == 256: one digit per thread
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < RB / 32; w++) {
            uint32_t t = wc[w][dg];
            wc[w][dg] = run;
            run += t;
        }
    }
    __syncthreads();
    if (valid) {
        uint32_t dst = hist[(size_t)d * nblk + blockIdx.x] + wc[warp][d] + rank;
        kout[dst] = key;
        vout[dst] = val;
    }
}

// ------------------------------------------------------------ Karras tree
AVBD_D int delta_ref(const uint64_t* keys, const uint32_t* idx, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clzll((long long)((uint64_t)idx[i] ^ (uint64_t)idx[j]));
    return __clzll((long long)(a ^ b));
}

__global__ void __launch_bounds__(256) k_karras(LbvhState L, const uint64_t* keys, uint2* range) {
    int n = (int)L.n;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const uint32_t* idx = L.sorted;
    int d = (delta_ref(keys, idx, n, i, i + 1) - delta_ref(keys, idx, n, i, i - 1) >= 0) ? 1 : -1;
    int dmin = delta_ref(keys, idx, n, i, i - d);
    int lmax = 128;
    while (delta_ref(keys, idx, n, i, i + lmax * d) > dmin) lmax *= 4;
    int l = 0;
    for (unsigned t = lmax; t >= 1; t /= 2)
        if (delta_ref(keys, idx, n, i, i + (l + (int)t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta_ref(keys, idx, n, i, j);
    int s = 0;
    for (int t = (l + 1) / 2; t >= 1; t = (t == 1 ? 0 : (t + 1) / 2)) {
        int ns = s + t;
        if (ns < l && delta_ref(keys, idx, n, i, i + ns * d) > dnode) s = ns;
    }
    int gamma = i + s * d + min(d, 0);
    unsigned g = (unsigned)(i + n);
    unsigned lc = (min(i, j) == gamma) ? (unsigned)gamma : (unsigned)(n + gamma);
    unsigned rc = (max(i, j) == gamma + 1) ? (unsigned)(gamma + 1) : (unsigned)(n + gamma + 1);
    L.left[g] = lc;
    L.right[g] = rc;
    L.parent[lc] = g;
    L.parent[rc] = g;
    range[i] = make_uint2((unsigned)min(i, j), (unsigned)max(i, j));
}

AVBD_D unsigned atomic_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Bottom-up refit with one visit counter per internal node: the second child
// to arrive computes the union (LBVHBuilder::assembleBVH).  min/max are exact,
// so the result does not depend on arrival order.
__global__ void __launch_bounds__(256) k_refit(LbvhState L) {
    unsigned l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= L.n) return;
    const double* b = L.aabb + 6ull * L.sorted[l];
#pragma unroll
    for (int a = 0; a < 6; a++) L.nbounds[6ull * l + a] = b[a];
    L.subtree[l] = 1;
    L.left[l] = INVALID;
    L.right[l] = INVALID;
    unsigned node = L.parent[l];
    while (node != INVALID) {
        // the first child to arrive stops; the second combines both.  The
        // count is an acquire-release RMW at device scope: the first arrival
        // releases its subtree's writes, the second acquires them
        if (atomic_add_acq_rel(&L.visited[node], 1u) == 0) break;
        unsigned a = L.left[node], c = L.right[node];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            L.nbounds[6ull * node + k] = dmin_ref(__ldcg(L.nbounds + 6ull * a + k), __ldcg(L.nbounds + 6ull * c + k));
            L.nbounds[6ull * node + 3 + k] =
                dmax_ref(__ldcg(L.nbounds + 6ull * a + 3 + k), __ldcg(L.nbounds + 6ull * c + 3 + k));
        }
        L.subtree[node] = __ldcg(L.subtree + a) + __ldcg(L.subtree + c);
        node = L.parent[node];
    }
}

AVBD_D bool overlaps(const double* A, const double* B) {
    return A[0] <= B[3] && A[1] <= B[4] && A[2] <= B[5] && A[3] >= B[0] && A[4] >= B[1] && A[5] >= B[2];
}

// One thread per leaf a: every leaf b > a whose box overlaps a's box.
__global__ void __launch_bounds__(128) k_traverse(LbvhState L, const uint2* range, unsigned root, int* err) {
    unsigned a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= L.n || L.n < 2) return;
    double q[6];
#pragma unroll
    for (int k = 0; k < 6; k++) q[k] = L.nbounds[6ull * a + k];
    const unsigned n = L.n;
    unsigned stack[128];
    int sp = 0;
    stack[sp++] = root;
    const unsigned pa = L.sorted[a];
    const uint8_t ta = L.type[pa];
    while (sp > 0) {
        unsigned node = stack[--sp];
        if (node >= n) {
            uint2 rg = range[node - n];
            if (rg.y <= a) continue;
        } else if (node <= a) {
            continue;
        }
        double nb[6];
#pragma unroll
        for (int k = 0; k < 6; k++) nb[k] = L.nbounds[6ull * node + k];
        if (!overlaps(q, nb)) continue;
        if (node < n) {
            unsigned slot = atomicAdd(L.pair_count, 1u);
            if (slot < L.pair_capacity) L.pairs[slot] = make_uint2(a, node);
            else atomicExch(err, (int)AVBD_ERR_CAPACITY);  // a dropped pair would be a missed collision
            // narrow-phase dispatch (CollisionDetector.cpp:166-215): triangle-triangle and
            // rod-rod are no-ops; sphere-sphere and sphere-rod throw "Unsupported collision!"
            uint8_t tb = L.type[L.sorted[node]];
            bool sph = ta == AVBD_SHAPE_SPHERE || tb == AVBD_SHAPE_SPHERE;
            bool tri = ta == AVBD_SHAPE_TRIANGLE || tb == AVBD_SHAPE_TRIANGLE;
            if (sph && !tri) atomicExch(err, (int)AVBD_ERR_UNSUPPORTED_PAIR);
            continue;
        }
        if (sp + 2 > 128) {
            atomicExch(err, (int)AVBD_ERR_CAPACITY);
            return;
        }
        stack[sp++] = L.left[node];
        stack[sp++] = L.right[node];
    }
}

// ---------------------------------------------------------------- host
static inline unsigned nb(unsigned n, unsigned per) { return (n + per - 1) / per; }

int lbvh_allocate(avbd_ctx* c, std::string& err) {
    LbvhState& L = c->lbvh;
    const unsigned n = (unsigned)c->prims.size();
    L.n = n;
    const unsigned nn = 2 * n - 1;
    L.hist_blocks = nb(n, RB);
    L.pair_capacity = c->debug_pair_capacity ? c->debug_pair_capacity : std::max(1024u, 64u * n);
    std::vector<uint8_t> type(n);
    std::vector<uint4> pidx(n);
    std::vector<double> radius(n);
    std::vector<uint32_t> obj(n);
    unsigned spheres = 0, segments = 0, triangles = 0;
    for (unsigned i = 0; i < n; i++) {
        const HostPrim& p = c->prims[i];
        type[i] = p.type;
        obj[i] = p.object_id;
        spheres += p.type == AVBD_SHAPE_SPHERE;
        segments += p.type == AVBD_SHAPE_ROD_SEGMENT;
        triangles += p.type == AVBD_SHAPE_TRIANGLE;
        pidx[i] = make_uint4(c->inv[p.idx[0]], p.type == AVBD_SHAPE_SPHERE ? 0 : c->inv[p.idx[1]],
                             p.type == AVBD_SHAPE_TRIANGLE ? c->inv[p.idx[2]] : 0, 0);
        radius[i] = p.radius;
    }
    auto alloc = [&](void** ptr, size_t bytes) -> bool {
        cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 16);
        if (e != cudaSuccess) {
            err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
            return false;
        }
        c->allocations.push_back(*ptr);
        return true;
    };
    if (!alloc((void**)&L.type, n) || !alloc((void**)&L.pidx, sizeof(uint4) * n) ||
        !alloc((void**)&L.radius, sizeof(double) * n) || !alloc((void**)&L.aabb, sizeof(double) * 6 * n) ||
        !alloc((void**)&L.morton, sizeof(uint64_t) * n) || !alloc((void**)&L.keys_tmp, sizeof(uint64_t) * n) ||
        !alloc((void**)&L.sorted, sizeof(uint32_t) * n) || !alloc((void**)&L.sorted_tmp, sizeof(uint32_t) * n) ||
        !alloc((void**)&L.hist, sizeof(uint32_t) * 256 * L.hist_blocks) ||
        !alloc((void**)&L.left, sizeof(uint32_t) * nn) || !alloc((void**)&L.right, sizeof(uint32_t) * nn) ||
        !alloc((void**)&L.parent, sizeof(uint32_t) * nn) || !alloc((void**)&L.subtree, sizeof(uint32_t) * nn) ||
        !alloc((void**)&L.visited, sizeof(uint32_t) * nn) || !alloc((void**)&L.nbounds, sizeof(double) * 6 * nn) ||
        !alloc((void**)&L.scene_box, sizeof(unsigned long long) * 8) || !alloc((void**)&L.root, sizeof(uint32_t) * 2) ||
        !alloc((void**)&L.pairs, sizeof(uint2) * L.pair_capacity) || !alloc((void**)&L.pair_count, sizeof(uint32_t)) ||
        !alloc((void**)&L.range, sizeof(uint2) * std::max(1u, n - 1)) ||
        !alloc((void**)&L.obj, sizeof(uint32_t) * n))
        return AVBD_ERR_CUDA;
    if (triangles && (spheres || segments)) {  // room for 64 triangle contacts per sphere, 16 per segment
        L.contact_capacity = std::max(1024u, 64u * spheres + 16u * segments);
        if (!alloc((void**)&L.contact_key, sizeof(uint64_t) * L.contact_capacity) ||
            !alloc((void**)&L.contact_idx, sizeof(uint4) * L.contact_capacity) ||
            !alloc((void**)&L.contact_idx5, sizeof(uint32_t) * L.contact_capacity) ||
            !alloc((void**)&L.contact_vec, sizeof(double) * 10 * L.contact_capacity) ||
            !alloc((void**)&L.contact_count, sizeof(uint32_t)))
            return AVBD_ERR_CUDA;
        cudaMemsetAsync(L.contact_count, 0, sizeof(uint32_t), c->stream);
    }
    cudaMemcpyAsync(L.obj, obj.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(L.type, type.data(), n, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(L.pidx, pidx.data(), sizeof(uint4) * n, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(L.radius, radius.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(L.pair_count, 0, sizeof(uint32_t), c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return AVBD_ERR_CUDA;
    }
    return AVBD_OK;
}

template <typename R>
void lbvh_stage(avbd_ctx* c, DevState<R>& s, cudaStream_t st) {
    LbvhState& L = c->lbvh;
    const unsigned n = L.n;
    if (n == 0) return;
    const unsigned nn = 2 * n - 1;
    unsigned long long* box = reinterpret_cast<unsigned long long*>(L.scene_box);
    cudaMemsetAsync(box, 0xFF, 3 * sizeof(unsigned long long), st);
    cudaMemsetAsync(box + 3, 0x00, 3 * sizeof(unsigned long long), st);
    k_prim_bounds<R><<<nb(n, 256), 256, 0, st>>>(s, L, c->params.dt, box);
    k_morton<<<nb(n, 256), 256, 0, st>>>(L, box);
    count_launch(c, 2);
    uint64_t *ka = L.morton, *kb = L.keys_tmp;
    uint32_t *va = L.sorted, *vb = L.sorted_tmp;
    for (int shift = 0; shift < 64; shift += 8) {
        k_radix_count<<<L.hist_blocks, RB, 0, st>>>(ka, n, shift, L.hist, L.hist_blocks);
        k_radix_scan<<<1, 1024, 0, st>>>(L.hist, 256 * L.hist_blocks);
        k_radix_scatter<<<L.hist_blocks, RB, 0, st>>>(ka, va, kb, vb, n, shift, L.hist, L.hist_blocks);
        count_launch(c, 3);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // 8 passes: the sorted keys/values end in the original buffers, but the
    // original codes were overwritten, so keep the sorted codes and restore the
    // per-primitive codes by a scatter through the sorted order.
    // (ka == L.morton holds sorted keys, va == L.sorted holds sorted indices.)
    cudaMemsetAsync(L.parent, 0xFF, sizeof(uint32_t) * nn, st);
    cudaMemsetAsync(L.visited, 0, sizeof(uint32_t) * nn, st);
    cudaMemsetAsync(L.pair_count, 0, sizeof(uint32_t), st);
    if (n > 1) {
        k_karras<<<nb(n - 1, 256), 256, 0, st>>>(L, ka, L.range);
        count_launch(c);
    }
    k_refit<<<nb(n, 256), 256, 0, st>>>(L);
    k_traverse<<<nb(n, 128), 128, 0, st>>>(L, L.range, n > 1 ? n : 0, c->d_error);
    count_launch(c, 2);
    launch_narrow<R>(c, s, st);
}

template void lbvh_stage<float>(avbd_ctx*, DevState<float>&, cudaStream_t);
template void lbvh_stage<double>(avbd_ctx*, DevState<double>&, cudaStream_t);

}  // namespace avbd

// ------------------------------------------------------------- C-ABI
using namespace avbd;

__global__ void k_unsort_codes(const uint64_t* sorted_keys, const uint32_t* sorted_idx, uint64_t* out, unsigned n) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[sorted_idx[i]] = sorted_keys[i];
}

extern "C" int avbd_get_lbvh(avbd_ctx* c, unsigned* num_primitives, uint64_t* morton, unsigned* sorted_order,
                             unsigned* left, unsigned* right, unsigned* parent, unsigned* subtree_size,
                             double* bounds6, unsigned* root) {
    if (!c || !c->finalized) return AVBD_ERR_STATE;
    LbvhState& L = c->lbvh;
    const unsigned n = L.n;
    if (num_primitives) *num_primitives = n;
    if (n == 0) return AVBD_OK;
    const unsigned nn = 2 * n - 1;
    cudaStream_t st = c->stream;
    if (morton) {
        // codes per primitive (CollisionPrimitivePool::morton_code order)
        k_unsort_codes<<<(n + 255) / 256, 256, 0, st>>>(L.morton, L.sorted, L.keys_tmp, n);
        cudaMemcpyAsync(morton, L.keys_tmp, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, st);
    }
    if (sorted_order) cudaMemcpyAsync(sorted_order, L.sorted, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
    if (left) cudaMemcpyAsync(left, L.left, sizeof(uint32_t) * nn, cudaMemcpyDeviceToHost, st);
    if (right) cudaMemcpyAsync(right, L.right, sizeof(uint32_t) * nn, cudaMemcpyDeviceToHost, st);
    if (parent) cudaMemcpyAsync(parent, L.parent, sizeof(uint32_t) * nn, cudaMemcpyDeviceToHost, st);
    if (subtree_size) cudaMemcpyAsync(subtree_size, L.subtree, sizeof(uint32_t) * nn, cudaMemcpyDeviceToHost, st);
    if (bounds6) cudaMemcpyAsync(bounds6, L.nbounds, sizeof(double) * 6 * nn, cudaMemcpyDeviceToHost, st);
    if (root) *root = n > 1 ? n : 0;
    cudaError_t e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? AVBD_OK : AVBD_ERR_CUDA;
}

extern "C" int avbd_get_candidate_pairs(avbd_ctx* c, unsigned capacity, unsigned* pairs2, unsigned* count) {
    if (!c || !c->finalized) return AVBD_ERR_STATE;
    LbvhState& L = c->lbvh;
    if (L.n == 0) {
        if (count) *count = 0;
        return AVBD_OK;
    }
    uint32_t cnt = 0;
    cudaMemcpyAsync(&cnt, L.pair_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    if (count) *count = cnt;
    if (cnt > L.pair_capacity) return AVBD_ERR_CAPACITY;
    if (!pairs2) return AVBD_OK;
    if (capacity < cnt) return AVBD_ERR_CAPACITY;
    std::vector<uint2> h(cnt);
    cudaMemcpyAsync(h.data(), L.pairs, sizeof(uint2) * cnt, cudaMemcpyDeviceToHost, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return AVBD_ERR_CUDA;
    std::sort(h.begin(), h.end(), [](uint2 a, uint2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
    for (uint32_t k = 0; k < cnt; k++) {
        pairs2[2 * k] = h[k].x;
        pairs2[2 * k + 1] = h[k].y;
    }
    return AVBD_OK;
}

// ======================================================= no-alloc variant
//
// Morton codes + stable radix sort of caller-provided primitive boxes, with
// every scratch buffer in file-scope device arrays instead of cudaMalloc.  For
// callers that must not allocate device memory while they run: a host loop
// being recorded into a CUDA graph, a real-time loop with a fixed memory
// budget, or an application whose device memory belongs to another
// framework's allocator.  The arrays are sized for AVBD_NOALLOC_MAX_PRIMITIVES
// primitives (about 6 MiB: two 2 MiB key buffers, a 1 MiB index buffer and a
// 1 MiB digit histogram) and stay resident on every GPU that loads the
// library until the process exits.

namespace {

constexpr unsigned kNoAllocMax = AVBD_NOALLOC_MAX_PRIMITIVES;
constexpr unsigned kNoAllocBlocks = (kNoAllocMax + RB - 1) / RB;

static __device__ __align__(256) uint64_t g_na_keys_a[kNoAllocMax];  // sorted keys end here
static __device__ __align__(256) uint64_t g_na_keys_b[kNoAllocMax];
static __device__ __align__(256) uint32_t g_na_vals_b[kNoAllocMax];
static __device__ __align__(256) uint32_t g_na_hist[256 * kNoAllocBlocks];
static __device__ __align__(256) unsigned long long g_na_box[8];

struct NoAllocScratch {
    uint64_t* keys_a = nullptr;
    uint64_t* keys_b = nullptr;
    uint32_t* vals_b = nullptr;
    uint32_t* hist = nullptr;
    unsigned long long* box = nullptr;
};

// Device addresses of the scratch arrays, resolved once per device with that
// device current (host code cannot use the arrays' names as addresses).
std::mutex g_na_mutex;
NoAllocScratch g_na_addr[64];
bool g_na_ready[64] = {};

int noalloc_scratch(int dev, NoAllocScratch& out) {
    if (dev < 0 || dev >= 64) return AVBD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ready[dev]) {
        NoAllocScratch s;
        if (cudaGetSymbolAddress((void**)&s.keys_a, g_na_keys_a) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.keys_b, g_na_keys_b) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.vals_b, g_na_vals_b) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.hist, g_na_hist) != cudaSuccess ||
            cudaGetSymbolAddress((void**)&s.box, g_na_box) != cudaSuccess)
            return AVBD_ERR_CUDA;
        g_na_addr[dev] = s;
        g_na_ready[dev] = true;
    }
    out = g_na_addr[dev];
    return AVBD_OK;
}

// Scene box of caller-provided boxes (min/max are exact, order-preserving
// integer atomics as in k_prim_bounds).
__global__ void __launch_bounds__(256) k_box_of_aabbs(const double* __restrict__ aabb, unsigned n,
                                                      unsigned long long* box) {
    unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < n;
    unsigned long long e[6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        e[a] = valid ? ord_enc(aabb[6ull * i + a]) : ~0ull;
        e[3 + a] = valid ? ord_enc(aabb[6ull * i + 3 + a]) : 0ull;
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            unsigned long long o = __shfl_xor_sync(0xffffffffu, e[a], m);
            e[a] = o < e[a] ? o : e[a];
            o = __shfl_xor_sync(0xffffffffu, e[3 + a], m);
            e[3 + a] = o > e[3 + a] ? o : e[3 + a];
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            atomicMin(box + a, e[a]);
            atomicMax(box + 3 + a, e[3 + a]);
        }
    }
}

}  // namespace

// Same results as the context path's Morton codes and sorted order
// (LBVHBuilder::computeAABB_MortonCode + Algorithm::radixSort), on boxes the
// caller computed.  Every call shares the scratch arrays, which keep the last
// call's contents; the scene box is cleared at the start of each call.  Calls
// that overlap on the GPU (for example on two streams at once) race on the
// scratch and give wrong results.  The first call on a device resolves the
// scratch addresses and should come before any stream capture.
extern "C" int avbd_lbvh_morton_sort_noalloc(const double* aabb6, unsigned n, uint64_t* morton,
                                             unsigned* sorted_order, void* stream) {
    if (n == 0) return AVBD_OK;
    if (!aabb6 || !morton || !sorted_order) return set_error(AVBD_ERR_INVALID_ARG, "null buffer");
    if (n > kNoAllocMax)
        return set_error(AVBD_ERR_CAPACITY, "more primitives than AVBD_NOALLOC_MAX_PRIMITIVES");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(AVBD_ERR_NO_DEVICE, "no CUDA device");
    NoAllocScratch S;
    if (int rc = noalloc_scratch(dev, S)) return set_error(rc, "cannot resolve the scratch arrays' addresses");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned nblk = (n + RB - 1) / RB;
    // Every call below reports its own status; an error some earlier work
    // left pending is neither consumed nor mistaken for one of these.
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    auto launch = [&](auto kernel, unsigned grid, unsigned block, auto... args) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.stream = st;
        return ok(cudaLaunchKernelEx(&cfg, kernel, args...));
    };
    LbvhState L;
    L.n = n;
    L.aabb = const_cast<double*>(aabb6);
    L.morton = morton;          // per-primitive codes (output)
    L.sorted = sorted_order;    // identity, sorted in place below
    ok(cudaMemsetAsync(S.box, 0xFF, 3 * sizeof(unsigned long long), st)) &&
        ok(cudaMemsetAsync(S.box + 3, 0x00, 3 * sizeof(unsigned long long), st)) &&
        launch(k_box_of_aabbs, (n + 255) / 256, 256, (const double*)aabb6, n, S.box) &&
        launch(k_morton, (n + 255) / 256, 256, L, (const unsigned long long*)S.box) &&
        ok(cudaMemcpyAsync(S.keys_a, morton, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, st));
    uint64_t *ka = S.keys_a, *kb = S.keys_b;
    uint32_t *va = sorted_order, *vb = S.vals_b;
    for (int shift = 0; shift < 64 && e == cudaSuccess; shift += 8) {
        launch(k_radix_count, nblk, RB, (const uint64_t*)ka, n, shift, S.hist, nblk) &&
            launch(k_radix_scan, 1, 1024, S.hist, 256 * nblk) &&
            launch(k_radix_scatter, nblk, RB, (const uint64_t*)ka, (const uint32_t*)va, kb, vb, n, shift,
                   (const uint32_t*)S.hist, nblk);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // eight passes: sorted keys are back in keys_a, the order in sorted_order
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}
