// contacts.cu -- dynamic contacts (triangle-rigid and triangle-rod): the
// contact handling of the collision stage and the per-color solve around it.
//
// Reference behaviour followed:
//   CollisionDetector::detectCollisionsAndRecolor_Parallel   collision/CollisionDetector.cpp:57-128
//   CollisionDetector::_handleDetectedCollisions / _add / _update / _removeCollision
//                                                            collision/CollisionDetector.cpp:265-482
//   TriangleRigidCollisionEnergyPool::addEnergy              energy/collision/TriangleRigidCollisionEnergyPool.hpp:31-62
//   TriangleRodCollisionEnergyPool::addEnergy                energy/collision/TriangleRodCollisionEnergyPool.hpp:29-66
//   CollisionConstraintEnergyPool::addEnergy                 energy/collision/CollisionConstraintEnergyPool.hpp:48-69
//   CollisionConstraintEnergySolver::updateCollisionFrame    energy/collision/CollisionConstraintEnergySolver.hpp:17-53
//   Math::completeOrthonormalBasisGivenNormal                common/Math.hpp:323-327
//   TombstonePool::allocSlot / freeSlot                      common/TombstonePool.hpp:56-103
//   DynamicParticleAdjacency::buildAdjacency                 common/DynamicParticleAdjacency.hpp:33-118
//   ColorList::markParticleDirty / incrementalRecoloring / finalizeConflicts
//                                                            common/ColorList.hpp:365-522
//   VBDSolver::_commitConflictedInColor                      simulation/VBDSolver.hpp:82-87,108-119
//
// Layout.  The narrow phase leaves its detections on the device; the host
// reads them with the pool's multipliers, runs the merge, the tombstone pool,
// the dynamic adjacency and the incremental recoloring in the reference's
// particle numbering (the order the recoloring's "lower index" rule and the
// pool's slot order depend on), then uploads the pool records and, in the
// engine's color-major vertex order, the dynamic adjacency, the conflict
// flags and per-color lists.  The vertex slabs of the static coloring stay in
// place: a vertex with contacts or a color changed by the recoloring is
// skipped by its slab's launch and solved from its color's list by the
// solve's dynamic instantiation; colors beyond the static ones have lists
// only.  The pool is small (tens to thousands of contacts per step), so this
// host pass costs less than one of the step's sweeps.
#include <algorithm>
#include <cmath>

#include "engine.h"
#include "contact_dyn.cuh"

namespace avbd {

struct DynHost {
    // ---- contact pools (FP64 host mirror, reference particle ids):
    // pool[0] triangle-rigid, pool[1] triangle-rod
    struct Rec {
        unsigned p[5];  // triangle x3, rigid body / rod nodes
        double n[3], t[3], b[3], bar[3], cpl[3];
        double s;       // along the rod segment
        double k[4];    // k_n, k_t, k_b, k_start
        double lam[4];  // lam_n, lam_t, lam_b, C_n_prev
        double mu_s, mu_k;
        uint8_t flag;   // ContactFlags
    };
    struct Pool {
        std::vector<Rec> rec;
        std::vector<uint8_t> active;
        std::vector<unsigned> slots;   // free-slot stack
        unsigned top = 0, count = 0, size = 0;
    };
    unsigned cap = 0;  // slots per pool on the device
    Pool pool[2];
    struct Det {
        uint64_t key;
        int pool;       // 0: DetectedCollisionType::TriangleRigid (2), 1: TriangleRod (3)
        unsigned tri[3], p4[2];   // rigid body, or the rod's two nodes
        double n[3], bar[3], cpl[3], s;
        unsigned e_idx;
    };
    std::vector<Det> cur, prev;
    // ---- adjacency and coloring (reference particle ids)
    std::vector<unsigned> p_off, p_nbr;          // static neighbours
    std::vector<unsigned> dyn_off, dnb_off, dnb; // dynamic entries per particle, dynamic neighbours
    std::vector<uint32_t> dyn_ent_ext;           // slot << 4 | pool << 3 | local
    std::vector<unsigned> color, slab_color;
    unsigned num_colors = 0;
    std::vector<unsigned> last_dirty, dirty, next_dirty, touched_frame, cand, touched_conflicted;
    std::vector<uint8_t> conflicted;
    unsigned rounds = 6;  // ColorList::incrementalRecoloring MAX_COLOR_ITERS
    // ---- device-side products (engine vertex order)
    std::vector<unsigned> off3, off6, offc;      // per color: recolored 3-DOF, 6-DOF, conflicted
    std::vector<uint32_t> lists, dyn_begin, dyn_ent;
    std::vector<uint8_t> skip, confl;
    std::vector<uint8_t> skip_dev, confl_dev;    // what the device holds
    uint32_t* d_lists = nullptr;
    unsigned ent_cap = 0;
    bool csr_dirty = true;
    // ---- staging
    std::vector<uint64_t> h_key;
    std::vector<uint4> h_idx;
    std::vector<uint32_t> h_idx5;
    std::vector<double> h_vec;
};

namespace {

constexpr unsigned DIRTY_SENTINEL = 0xFFFFFFFFu;  // ColorList::SENTINEL

void cross3d(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
double dot3d(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Eigen's MatrixBase::unitOrthogonal for a 3-vector (Eigen 3.3+, the
// reference's linear-algebra library; published behaviour: a unit vector
// orthogonal to v, built from (x, y) unless both are negligible next to z at
// dummy precision 1e-12, then from (y, z)).
void unit_orthogonal(const double v[3], double t[3]) {
    const double prec = 1e-12;
    auto negligible = [&](double a, double b) { return std::fabs(a) <= std::fabs(b) * prec; };
    if (!negligible(v[0], v[2]) || !negligible(v[1], v[2])) {
        const double inv = 1.0 / std::sqrt(v[0] * v[0] + v[1] * v[1]);
        t[0] = -v[1] * inv; t[1] = v[0] * inv; t[2] = 0.0;
    } else {
        const double inv = 1.0 / std::sqrt(v[1] * v[1] + v[2] * v[2]);
        t[0] = 0.0; t[1] = -v[2] * inv; t[2] = v[1] * inv;
    }
}

void normal_basis(const double n[3], double t[3], double b[3]) {
    unit_orthogonal(n, t);
    cross3d(n, t, b);
}

// updateCollisionFrame: the tangent is carried over by projection and the
// friction multipliers keep the friction force
void update_frame(DynHost::Rec& e, const double nn[3]) {
    double f[3], tp[3];
    for (int i = 0; i < 3; i++) f[i] = e.lam[1] * e.t[i] + e.lam[2] * e.b[i];
    const double tn = dot3d(e.t, nn);
    for (int i = 0; i < 3; i++) tp[i] = e.t[i] - tn * nn[i];
    const double m = std::sqrt(dot3d(tp, tp));
    if (m > 1e-8) {
        for (int i = 0; i < 3; i++) e.t[i] = tp[i] / m;
        cross3d(nn, e.t, e.b);
    } else {
        normal_basis(nn, e.t, e.b);
    }
    for (int i = 0; i < 3; i++) e.n[i] = nn[i];
    e.lam[1] = dot3d(f, e.t);
    e.lam[2] = dot3d(f, e.b);
}

// TombstonePool: the stack grows on demand; a slot never reached holds its
// own index, as the reference's iota-initialised stack does
int pool_alloc(DynHost::Pool& P, unsigned cap, unsigned& slot) {
    if (P.top == P.slots.size()) P.slots.push_back((unsigned)P.slots.size());
    slot = P.slots[P.top];
    if (slot >= cap) return set_error(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    P.top++;
    if (slot >= P.rec.size()) {
        P.rec.resize(slot + 1);
        P.active.resize(slot + 1, 0);
    }
    P.active[slot] = 1;
    P.count++;
    P.size = std::max(P.size, slot + 1);
    return AVBD_OK;
}
int pool_free(DynHost::Pool& P, unsigned slot) {
    if (slot >= P.active.size() || !P.active[slot]) return set_error(AVBD_ERR_STATE, "freeSlot called on inactive slot");
    P.active[slot] = 0;
    P.count--;
    P.slots[--P.top] = slot;
    return AVBD_OK;
}

void mark_dirty(DynHost& D, unsigned p) {
    if (D.last_dirty[p] != 0) {
        D.last_dirty[p] = 0;
        D.touched_frame.push_back(p);
        D.dirty.push_back(p);
    }
}

// _addCollision: k_start from the smallest mass of the contact's particles,
// frame from the normal, all its particles dirty
int add_contact(avbd_ctx* c, DynHost& D, DynHost::Det& d) {
    const int np = d.pool == POOL_TRI_ROD ? 5 : 4;
    unsigned ps[5] = {d.tri[0], d.tri[1], d.tri[2], d.p4[0], d.p4[1]};
    double mn = c->mass[ps[0]];
    for (int k = 1; k < np; k++) mn = std::min(mn, c->mass[ps[k]]);
    const double ks = mn / (c->params.dt * c->params.dt);
    DynHost::Pool& P = D.pool[d.pool];
    unsigned slot;
    if (int r = pool_alloc(P, D.cap, slot)) return r;
    DynHost::Rec& e = P.rec[slot];
    e = DynHost::Rec{};
    for (int k = 0; k < 5; k++) e.p[k] = k < np ? ps[k] : 0;
    for (int i = 0; i < 3; i++) { e.n[i] = d.n[i]; e.bar[i] = d.bar[i]; e.cpl[i] = d.cpl[i]; }
    e.s = d.s;
    normal_basis(d.n, e.t, e.b);
    e.k[0] = e.k[1] = e.k[2] = e.k[3] = ks;
    e.lam[0] = e.lam[1] = e.lam[2] = e.lam[3] = 0;
    e.mu_s = 0.4;
    e.mu_k = 0.2;
    e.flag = CF_ACTIVE;
    d.e_idx = slot;
    for (int k = 0; k < np; k++) mark_dirty(D, ps[k]);
    D.csr_dirty = true;
    return AVBD_OK;
}

// _updateCollision: new barycentrics, body-frame point (and s), frame update
void update_contact(DynHost& D, const DynHost::Det& d) {
    DynHost::Rec& e = D.pool[d.pool].rec[d.e_idx];
    for (int i = 0; i < 3; i++) { e.cpl[i] = d.cpl[i]; e.bar[i] = d.bar[i]; }
    e.s = d.s;
    update_frame(e, d.n);
}

int remove_contact(DynHost& D, const DynHost::Det& d) {
    DynHost::Pool& P = D.pool[d.pool];
    if (int r = pool_free(P, d.e_idx)) return r;
    P.rec[d.e_idx].flag = 0;
    D.csr_dirty = true;
    return AVBD_OK;
}

// _handleDetectedCollisions: merge of two key-sorted lists; primitives are
// never removed, so equal keys are always the same contact
int handle_detections(avbd_ctx* c, DynHost& D) {
    auto& cur = D.cur;
    auto& prev = D.prev;
    size_t i = 0, j = 0;
    while (i < cur.size() && j < prev.size()) {
        if (cur[i].key < prev[j].key) {
            if (int r = add_contact(c, D, cur[i++])) return r;
        } else if (cur[i].key > prev[j].key) {
            if (int r = remove_contact(D, prev[j++])) return r;
        } else {
            cur[i].e_idx = prev[j].e_idx;
            update_contact(D, cur[i]);
            i++;
            j++;
        }
    }
    for (; i < cur.size(); i++)
        if (int r = add_contact(c, D, cur[i])) return r;
    for (; j < prev.size(); j++)
        if (int r = remove_contact(D, prev[j])) return r;
    return AVBD_OK;
}

// DynamicParticleAdjacency::buildAdjacency over the live slots in slot order
void build_dynamic_adjacency(DynHost& D, unsigned n) {
    D.dyn_off.assign(n + 1, 0);
    D.dnb_off.assign(n + 1, 0);
    for (int pl = 0; pl < 2; pl++) {
        const DynHost::Pool& P = D.pool[pl];
        const int np = pl == POOL_TRI_ROD ? 5 : 4;
        for (unsigned s = 0; s < P.size; s++) {
            if (!P.active[s]) continue;
            for (int k = 0; k < np; k++) {
                D.dyn_off[P.rec[s].p[k] + 1]++;
                D.dnb_off[P.rec[s].p[k] + 1] += np - 1;
            }
        }
    }
    for (unsigned p = 0; p < n; p++) {
        D.dyn_off[p + 1] += D.dyn_off[p];
        D.dnb_off[p + 1] += D.dnb_off[p];
    }
    D.dyn_ent_ext.assign(D.dyn_off[n], 0);
    D.dnb.assign(D.dnb_off[n], 0);
    std::vector<unsigned> ec(D.dyn_off.begin(), D.dyn_off.end() - 1), nc(D.dnb_off.begin(), D.dnb_off.end() - 1);
    for (int pl = 0; pl < 2; pl++) {  // DynamicEnergyType order: triangle-rigid, triangle-rod
        const DynHost::Pool& P = D.pool[pl];
        const unsigned np = pl == POOL_TRI_ROD ? 5 : 4;
        for (unsigned s = 0; s < P.size; s++) {
            if (!P.active[s]) continue;
            const DynHost::Rec& e = P.rec[s];
            for (unsigned k = 0; k < np; k++) {
                const unsigned p = e.p[k];
                D.dyn_ent_ext[ec[p]++] = (s << 4) | ((unsigned)pl << 3) | k;
                for (unsigned k2 = 0; k2 < np; k2++)
                    if (k2 != k) D.dnb[nc[p]++] = e.p[k2];
            }
        }
    }
}

template <typename F>
void for_each_neighbor(const DynHost& D, unsigned p, F&& f) {
    for (unsigned k = D.p_off[p]; k < D.p_off[p + 1]; k++) f(D.p_nbr[k]);
    for (unsigned k = D.dnb_off[p]; k < D.dnb_off[p + 1]; k++) f(D.dnb[k]);
}

int finalize_conflicts(DynHost& D) {
    for (unsigned p : D.dirty)
        for_each_neighbor(D, p, [&](unsigned q) {
            if (D.color[q] == D.color[p]) {
                if (!D.conflicted[p]) { D.conflicted[p] = 1; D.touched_conflicted.push_back(p); }
                if (!D.conflicted[q]) { D.conflicted[q] = 1; D.touched_conflicted.push_back(q); }
            }
        });
    return AVBD_OK;
}

// ColorList::incrementalRecoloring (at most D.rounds rounds, 256 colors)
int incremental_recoloring(DynHost& D) {
    for (unsigned p : D.touched_conflicted) D.conflicted[p] = 0;
    D.touched_conflicted.clear();
    unsigned iter = 0;
    bool overflow = false;
    while (!D.dirty.empty() && iter < D.rounds) {
        for (unsigned p : D.dirty) {
            uint64_t bits[4] = {0, 0, 0, 0};
            bool must = false;
            for_each_neighbor(D, p, [&](unsigned q) {
                const unsigned cq = D.color[q];
                if (cq >= 256) { overflow = true; return; }
                bits[cq / 64] |= 1ull << (cq % 64);
                if (cq == D.color[p] && q < p) must = true;
            });
            if (overflow) return set_error(AVBD_ERR_COLORS, "Ran out of colors!");
            if (must) {
                unsigned cand = UINT32_MAX;
                for (unsigned w = 0; w < 4 && cand == UINT32_MAX; w++)
                    if (~bits[w]) cand = w * 64 + (unsigned)__builtin_ctzll(~bits[w]);
                if (cand == UINT32_MAX) return set_error(AVBD_ERR_COLORS, "Ran out of colors!");
                D.cand[p] = cand;
                if (cand >= D.num_colors) D.num_colors++;
            } else {
                D.cand[p] = D.color[p];
            }
        }
        D.next_dirty.clear();
        for (unsigned p : D.dirty) {
            if (D.cand[p] == D.color[p]) continue;
            D.color[p] = D.cand[p];
            for_each_neighbor(D, p, [&](unsigned q) {
                if (D.last_dirty[q] != iter + 1) {
                    D.last_dirty[q] = iter + 1;
                    D.touched_frame.push_back(q);
                    D.next_dirty.push_back(q);
                }
            });
        }
        D.dirty.swap(D.next_dirty);
        iter++;
    }
    if (!D.dirty.empty()) finalize_conflicts(D);
    for (unsigned p : D.touched_frame) D.last_dirty[p] = DIRTY_SENTINEL;
    D.touched_frame.clear();
    for (unsigned p : D.dirty) D.last_dirty[p] = 0;
    return AVBD_OK;
}

// Lists of the engine's vertex order: per color the positional and oriented
// vertices that have contacts or a color changed by the recoloring (solved by
// the dynamic instantiation of the solve) and the conflicted vertices to
// commit; skip and conflict flags per vertex.
void build_lists(avbd_ctx* c, DynHost& D) {
    const unsigned n = (unsigned)c->perm.size(), nc = D.num_colors;
    std::vector<unsigned> c3(nc, 0), c6(nc, 0), cc(nc, 0);
    D.skip.assign(n, 0);
    D.confl.assign(n, 0);
    for (unsigned i = 0; i < n; i++) {
        const unsigned e = c->perm[i];
        if (D.conflicted[e]) {
            D.confl[i] = 1;
            cc[D.color[e]]++;
        }
        if (D.color[e] == D.slab_color[i] && D.dyn_off[e + 1] == D.dyn_off[e]) continue;
        D.skip[i] = 1;
        if (c->fixed[e]) continue;
        if (c->rot[e] != UINT32_MAX) c6[D.color[e]]++;
        else c3[D.color[e]]++;
    }
    D.off3.assign(nc + 1, 0);
    D.off6.assign(nc + 1, 0);
    D.offc.assign(nc + 1, 0);
    unsigned run = 0;
    for (unsigned k = 0; k < nc; k++) { D.off3[k] = run; run += c3[k]; }
    D.off3[nc] = run;
    for (unsigned k = 0; k < nc; k++) { D.off6[k] = run; run += c6[k]; }
    D.off6[nc] = run;
    for (unsigned k = 0; k < nc; k++) { D.offc[k] = run; run += cc[k]; }
    D.offc[nc] = run;
    D.lists.assign(run, 0);
    std::vector<unsigned> u3(D.off3.begin(), D.off3.end() - 1), u6(D.off6.begin(), D.off6.end() - 1),
        uc(D.offc.begin(), D.offc.end() - 1);
    for (unsigned i = 0; i < n; i++) {
        const unsigned e = c->perm[i];
        if (D.confl[i]) D.lists[uc[D.color[e]]++] = i;
        if (!D.skip[i] || c->fixed[e]) continue;
        if (c->rot[e] != UINT32_MAX) D.lists[u6[D.color[e]]++] = i;
        else D.lists[u3[D.color[e]]++] = i;
    }
}

// the step-start hook of every live contact of both pools: thread i < size0
// serves pool 0 slot i, the rest pool 1
template <typename R>
__global__ void k_contact_after_step(DevState<R> s, unsigned size0, unsigned size1) {
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    int pool = 0;
    if (k >= size0) {
        k -= size0;
        pool = 1;
        if (k >= size1) return;
    }
    if (!(s.cp[pool].flag[k] & CF_ACTIVE)) return;
    dyn_after_step<R>(s, pool, k);
}

template <typename R>
__global__ void k_contact_after_iter(DevState<R> s, unsigned size0, unsigned size1, SceneTol T) {
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    int pool = 0;
    if (k >= size0) {
        k -= size0;
        pool = 1;
        if (k >= size1) return;
    }
    if (!(s.cp[pool].flag[k] & CF_ACTIVE)) return;
    if (T.active && !T.active[T.scene[s.cp[pool].p[k].w]]) return;
    dyn_after_iter<R>(s, pool, k);
}

// _commitConflictedInColor: buffered positions of the color's conflicted
// vertices.  A fixed conflicted vertex never writes its buffer (the reference
// then copies an uninitialised buffer); it keeps its position here.
template <typename R>
__global__ void k_commit_conflicted(DevState<R> s, const uint32_t* __restrict__ list, unsigned count, SceneTol T) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned p = list[i];
    if (s.flags[p] & VF_FIXED) return;
    if (T.active && !T.active[T.scene[p]]) return;
    s.x[p] = s.buffered[p];
}

unsigned nblk(unsigned n, unsigned per) { return (n + per - 1) / per; }

template <typename R>
int alloc_state(avbd_ctx* c, DevState<R>& s, DynHost& D, std::string& err) {
    using V4 = typename Vec4Of<R>::T;
    const unsigned n = s.n, cap = D.cap;
    auto alloc = [&](void** p, size_t bytes) {
        *p = nullptr;
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 1);
        if (e != cudaSuccess) {
            err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
            return false;
        }
        c->allocations.push_back(*p);
        return true;
    };
    D.ent_cap = 4 * cap + 5 * cap;  // entries of a full triangle-rigid and a full triangle-rod pool
    for (int pl = 0; pl < 2; pl++) {
        ContactPoolDev<R>& P = s.cp[pl];
        if (!alloc((void**)&P.p, sizeof(uint4) * cap) || !alloc((void**)&P.p5, sizeof(uint32_t) * cap) ||
            !alloc((void**)&P.n, sizeof(V4) * cap) || !alloc((void**)&P.t, sizeof(V4) * cap) ||
            !alloc((void**)&P.b, sizeof(V4) * cap) || !alloc((void**)&P.bar, sizeof(V4) * cap) ||
            !alloc((void**)&P.cpl, sizeof(V4) * cap) || !alloc((void**)&P.k, sizeof(V4) * cap) ||
            !alloc((void**)&P.lam, sizeof(V4) * cap) || !alloc((void**)&P.flag, cap))
            return AVBD_ERR_CUDA;
        P.cap = cap;
        cudaMemsetAsync(P.flag, 0, cap, c->stream);
    }
    if (!alloc((void**)&s.dyn_begin, sizeof(uint32_t) * (n + 1)) ||
        !alloc((void**)&s.dyn_ent, sizeof(uint32_t) * D.ent_cap) || !alloc((void**)&s.dyn_skip, n) ||
        !alloc((void**)&s.conflicted, n) || !alloc((void**)&s.buffered, sizeof(V4) * n) ||
        !alloc((void**)&D.d_lists, sizeof(uint32_t) * 2 * (size_t)n))
        return AVBD_ERR_CUDA;
    cudaStream_t st = c->stream;
    cudaMemsetAsync(s.dyn_begin, 0, sizeof(uint32_t) * (n + 1), st);
    cudaMemsetAsync(s.dyn_skip, 0, n, st);
    cudaMemsetAsync(s.conflicted, 0, n, st);
    cudaMemsetAsync(s.buffered, 0, sizeof(V4) * n, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return AVBD_ERR_CUDA;
    }
    return AVBD_OK;
}

#define DYN_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return set_error(AVBD_ERR_CUDA, cudaGetErrorString(e_));     \
    } while (0)

// reads the device's k / lam / flag of slots [0, size) of one pool into the host mirror
template <typename R>
int download_pool(const ContactPoolDev<R>& S, DynHost::Pool& D, cudaStream_t st) {
    using V4 = typename Vec4Of<R>::T;
    if (D.size == 0) return AVBD_OK;
    std::vector<V4> k(D.size), lam(D.size);
    std::vector<uint8_t> f(D.size);
    DYN_CUDA(cudaMemcpyAsync(k.data(), S.k, sizeof(V4) * D.size, cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaMemcpyAsync(lam.data(), S.lam, sizeof(V4) * D.size, cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaMemcpyAsync(f.data(), S.flag, D.size, cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    for (unsigned i = 0; i < D.size; i++) {
        if (!D.active[i]) continue;
        DynHost::Rec& e = D.rec[i];
        e.k[0] = k[i].x; e.k[1] = k[i].y; e.k[2] = k[i].z; e.k[3] = k[i].w;
        e.lam[0] = lam[i].x; e.lam[1] = lam[i].y; e.lam[2] = lam[i].z; e.lam[3] = lam[i].w;
        e.flag = f[i];
    }
    return AVBD_OK;
}

template <typename R>
int upload_pool(avbd_ctx* c, ContactPoolDev<R>& S, const DynHost::Pool& D, cudaStream_t st) {
    using V4 = typename Vec4Of<R>::T;
    const unsigned m = D.size;
    if (m == 0) return AVBD_OK;
    std::vector<uint4> p(m);
    std::vector<uint32_t> p5(m, 0);
    std::vector<V4> vn(m), vt(m), vb(m), vbar(m), vcpl(m), vk(m), vlam(m);
    std::vector<uint8_t> f(m);
    auto v4 = [](const double a[3], double w) {
        V4 o;
        o.x = (R)a[0]; o.y = (R)a[1]; o.z = (R)a[2]; o.w = (R)w;
        return o;
    };
    for (unsigned i = 0; i < m; i++) {
        const DynHost::Rec& e = D.rec[i];
        if (!D.active[i]) {
            f[i] = 0;
            p[i] = make_uint4(0, 0, 0, 0);
            continue;
        }
        p[i] = make_uint4(c->inv[e.p[0]], c->inv[e.p[1]], c->inv[e.p[2]], c->inv[e.p[3]]);
        p5[i] = c->inv[e.p[4]];
        vn[i] = v4(e.n, e.s);
        vt[i] = v4(e.t, 0);
        vb[i] = v4(e.b, 0);
        vbar[i] = v4(e.bar, e.mu_s);
        vcpl[i] = v4(e.cpl, e.mu_k);
        vk[i] = v4(e.k, e.k[3]);
        vlam[i] = v4(e.lam, e.lam[3]);
        f[i] = e.flag;
    }
    DYN_CUDA(cudaMemcpyAsync(S.p, p.data(), sizeof(uint4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.p5, p5.data(), sizeof(uint32_t) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.n, vn.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.t, vt.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.b, vb.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.bar, vbar.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.cpl, vcpl.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.k, vk.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.lam, vlam.data(), sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.flag, f.data(), m, cudaMemcpyHostToDevice, st));
    // the host vectors are pageable: the copies complete before the call returns
    DYN_CUDA(cudaStreamSynchronize(st));
    return AVBD_OK;
}

}  // namespace

int dyn_create(avbd_ctx* c, const std::vector<unsigned>& p_off, const std::vector<unsigned>& p_nbr,
               std::string& err) {
    dyn_destroy(c);
    const unsigned n = (unsigned)c->perm.size();
    DynHost* D = new DynHost();
    // a merge may add this stage's contacts before it frees the last stage's,
    // so each pool holds up to twice the narrow phase's capacity
    D->cap = 2 * c->lbvh.contact_capacity;
    D->p_off = p_off;
    D->p_nbr = p_nbr;
    D->color = c->color;
    D->num_colors = c->num_colors;
    D->slab_color.assign(n, 0);
    for (unsigned k = 0; k < c->num_colors; k++)
        for (unsigned i = c->color_begin[k]; i < c->color_begin[k + 1]; i++) D->slab_color[i] = k;
    D->last_dirty.assign(n, DIRTY_SENTINEL);
    D->cand.assign(n, 0);
    D->conflicted.assign(n, 0);
    D->skip_dev.assign(n, 0);
    D->confl_dev.assign(n, 0);
    D->dyn_off.assign(n + 1, 0);
    D->dnb_off.assign(n + 1, 0);
    D->off3.assign(D->num_colors + 1, 0);
    D->off6.assign(D->num_colors + 1, 0);
    D->offc.assign(D->num_colors + 1, 0);
    c->dyn = D;
    const bool d64 = c->solver.precision != AVBD_PRECISION_FP32;
    int rc = d64 ? alloc_state<double>(c, c->d, *D, err) : alloc_state<float>(c, c->f, *D, err);
    if (rc) dyn_destroy(c);
    return rc;
}

void dyn_destroy(avbd_ctx* c) {
    delete c->dyn;
    c->dyn = nullptr;
}

unsigned dyn_num_colors(const avbd_ctx* c) { return c->dyn ? c->dyn->num_colors : c->num_colors; }

void dyn_positional_list(const avbd_ctx* c, const uint32_t** list, unsigned* count) {
    const DynHost& D = *c->dyn;
    *list = D.d_lists + D.off3.front();
    *count = D.off3.back() - D.off3.front();
}

int dyn_coloring(const avbd_ctx* c, unsigned* colors) {
    const auto& col = c->dyn ? c->dyn->color : c->color;
    std::copy(col.begin(), col.end(), colors);
    return AVBD_OK;
}

template <typename R>
int dyn_manage(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    (void)k;
    DynHost& D = *c->dyn;
    LbvhState& L = c->lbvh;
    // detections of the narrow phase and the pools' multipliers
    uint32_t cnt = 0, pairs = 0;
    DYN_CUDA(cudaMemcpyAsync(&cnt, L.contact_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaMemcpyAsync(&pairs, L.pair_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    for (int pl = 0; pl < 2; pl++)
        if (int r = download_pool<R>(s.cp[pl], D.pool[pl], st)) return r;
    DYN_CUDA(cudaStreamSynchronize(st));
    if (pairs > L.pair_capacity)
        return set_error(AVBD_ERR_CAPACITY, "broad-phase candidate pairs exceed the pair buffer's capacity");
    if (cnt > L.contact_capacity)
        return set_error(AVBD_ERR_CAPACITY, "narrow-phase contacts exceed the contact buffer's capacity");
    D.h_key.resize(cnt);
    D.h_idx.resize(cnt);
    D.h_idx5.resize(cnt);
    D.h_vec.resize(10ull * cnt);
    if (cnt) {
        DYN_CUDA(cudaMemcpyAsync(D.h_key.data(), L.contact_key, sizeof(uint64_t) * cnt, cudaMemcpyDeviceToHost, st));
        DYN_CUDA(cudaMemcpyAsync(D.h_idx.data(), L.contact_idx, sizeof(uint4) * cnt, cudaMemcpyDeviceToHost, st));
        DYN_CUDA(cudaMemcpyAsync(D.h_idx5.data(), L.contact_idx5, sizeof(uint32_t) * cnt, cudaMemcpyDeviceToHost, st));
        DYN_CUDA(cudaMemcpyAsync(D.h_vec.data(), L.contact_vec, sizeof(double) * 10 * cnt, cudaMemcpyDeviceToHost, st));
        DYN_CUDA(cudaStreamSynchronize(st));
    }
    D.prev.swap(D.cur);
    D.cur.resize(cnt);
    for (uint32_t i = 0; i < cnt; i++) {
        DynHost::Det& d = D.cur[i];
        d.key = D.h_key[i];
        d.pool = (d.key >> 59) == 3u ? POOL_TRI_ROD : POOL_TRI_RIGID;  // DetectedCollisionType in the top 5 bits
        d.tri[0] = c->perm[D.h_idx[i].x];
        d.tri[1] = c->perm[D.h_idx[i].y];
        d.tri[2] = c->perm[D.h_idx[i].z];
        d.p4[0] = c->perm[D.h_idx[i].w];
        d.p4[1] = d.pool == POOL_TRI_ROD ? c->perm[D.h_idx5[i]] : 0u;
        for (int j = 0; j < 3; j++) {
            d.n[j] = D.h_vec[10ull * i + j];
            d.bar[j] = D.h_vec[10ull * i + 3 + j];
            d.cpl[j] = D.h_vec[10ull * i + 6 + j];
        }
        d.s = D.h_vec[10ull * i + 9];
        d.e_idx = 0;
    }
    // the narrow phase appends in any order; the reference radix-sorts by key
    std::sort(D.cur.begin(), D.cur.end(), [](const DynHost::Det& a, const DynHost::Det& b) { return a.key < b.key; });
    if (int r = handle_detections(c, D)) return r;
    const unsigned n = (unsigned)c->perm.size();
    build_dynamic_adjacency(D, n);
    if (int r = incremental_recoloring(D)) return r;
    build_lists(c, D);

    // uploads: pool records, dynamic adjacency (engine order), flags, lists
    for (int pl = 0; pl < 2; pl++)
        if (int r = upload_pool<R>(c, s.cp[pl], D.pool[pl], st)) return r;
    if (D.csr_dirty) {
        D.dyn_begin.assign(n + 1, 0);
        for (unsigned i = 0; i < n; i++) {
            const unsigned e = c->perm[i];
            D.dyn_begin[i + 1] = D.dyn_begin[i] + (D.dyn_off[e + 1] - D.dyn_off[e]);
        }
        D.dyn_ent.resize(D.dyn_begin[n]);
        for (unsigned i = 0; i < n; i++) {
            const unsigned e = c->perm[i];
            std::copy(D.dyn_ent_ext.begin() + D.dyn_off[e], D.dyn_ent_ext.begin() + D.dyn_off[e + 1],
                      D.dyn_ent.begin() + D.dyn_begin[i]);
        }
        if (D.dyn_begin[n] > D.ent_cap) return set_error(AVBD_ERR_CAPACITY, "dynamic adjacency exceeds its capacity");
        DYN_CUDA(cudaMemcpyAsync(s.dyn_begin, D.dyn_begin.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, st));
        if (D.dyn_begin[n])
            DYN_CUDA(cudaMemcpyAsync(s.dyn_ent, D.dyn_ent.data(), sizeof(uint32_t) * D.dyn_begin[n],
                                     cudaMemcpyHostToDevice, st));
        D.csr_dirty = false;
    }
    if (D.skip != D.skip_dev) {
        DYN_CUDA(cudaMemcpyAsync(s.dyn_skip, D.skip.data(), n, cudaMemcpyHostToDevice, st));
        D.skip_dev = D.skip;
    }
    if (D.confl != D.confl_dev) {
        DYN_CUDA(cudaMemcpyAsync(s.conflicted, D.confl.data(), n, cudaMemcpyHostToDevice, st));
        D.confl_dev = D.confl;
    }
    if (!D.lists.empty())
        DYN_CUDA(cudaMemcpyAsync(D.d_lists, D.lists.data(), sizeof(uint32_t) * D.lists.size(), cudaMemcpyHostToDevice,
                                 st));
    DYN_CUDA(cudaStreamSynchronize(st));
    // the contacts' step-start hook, at the positions of the step start
    const unsigned s0 = D.pool[0].size, s1 = D.pool[1].size;
    if (s0 + s1) {
        k_contact_after_step<R><<<nblk(s0 + s1, 128), 128, 0, st>>>(s, s0, s1);
        count_launch(c);
    }
    return AVBD_OK;
}

template <typename R>
void dyn_solve_color(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned col, cudaStream_t st,
                     const SceneTol& T) {
    DynHost& D = *c->dyn;
    if (col < c->num_colors) {
        if (c->color_solve[col]) launch_solve_color<R>(c, s, k, c->color_begin[col], c->color_solve[col], st, T);
        if (c->color_orient[col])
            launch_solve_rod<R>(c, s, k, c->color_begin[col] + c->color_solve[col], c->color_orient[col], st, T, 0,
                                nullptr);
    }
    if (col >= D.num_colors) return;
    const unsigned n3 = D.off3[col + 1] - D.off3[col], n6 = D.off6[col + 1] - D.off6[col];
    const unsigned ncf = D.offc[col + 1] - D.offc[col];
    if (n3) launch_solve_color<R>(c, s, k, 0, n3, st, T, D.d_lists + D.off3[col]);
    if (n6) launch_solve_rod<R>(c, s, k, 0, n6, st, T, 0, nullptr, D.d_lists + D.off6[col]);
    if (ncf) {
        k_commit_conflicted<R><<<nblk(ncf, 128), 128, 0, st>>>(s, D.d_lists + D.offc[col], ncf, T);
        count_launch(c);
    }
}

template <typename R>
void launch_contact_after_iter(avbd_ctx* c, DevState<R>& s, cudaStream_t st, const SceneTol& T) {
    if (!c->dyn) return;
    const unsigned s0 = c->dyn->pool[0].size, s1 = c->dyn->pool[1].size;
    if (!(s0 + s1)) return;
    k_contact_after_iter<R><<<nblk(s0 + s1, 128), 128, 0, st>>>(s, s0, s1, T);
    count_launch(c);
}

}  // namespace avbd

// ============================================================ C-ABI queries
using namespace avbd;

extern "C" {

int avbd_dynamic_info(avbd_ctx* c, unsigned out[8]) {
    if (!c || !out) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    std::fill(out, out + 8, 0u);
    if (!c->dyn) return AVBD_OK;
    const DynHost& D = *c->dyn;
    out[0] = D.pool[0].count;
    out[1] = D.pool[0].size;
    out[2] = D.num_colors;
    out[3] = (unsigned)D.touched_conflicted.size();
    out[4] = (unsigned)D.dirty.size();
    out[5] = (unsigned)D.dyn_ent_ext.size();
    out[6] = D.pool[1].count;
    out[7] = D.pool[1].size;
    return AVBD_OK;
}

// pool `pl` by slot into p (np per slot), active, data (24 or 25 per slot)
static int get_pool(avbd_ctx* c, int pl, unsigned capacity, unsigned* p, uint8_t* active, double* data,
                    unsigned* size) {
    if (!c || !size) return set_error(AVBD_ERR_INVALID_ARG, "null argument");
    *size = 0;
    if (!c->dyn) return AVBD_OK;
    DynHost::Pool& D = c->dyn->pool[pl];
    if (cudaSetDevice(c->device) != cudaSuccess) return set_error(AVBD_ERR_CUDA, "cudaSetDevice");
    const bool d64 = c->solver.precision != AVBD_PRECISION_FP32;
    if (int r = d64 ? download_pool<double>(c->d.cp[pl], D, c->stream) : download_pool<float>(c->f.cp[pl], D, c->stream))
        return r;
    const int np = pl == POOL_TRI_ROD ? 5 : 4, nd = pl == POOL_TRI_ROD ? 25 : 24;
    *size = D.size;
    for (unsigned i = 0; i < D.size && i < capacity; i++) {
        const DynHost::Rec& e = D.rec[i];
        if (p)
            for (int k = 0; k < np; k++) p[np * i + k] = e.p[k];
        if (active) active[i] = D.active[i];
        if (data) {
            double* o = data + (size_t)nd * i;
            for (int j = 0; j < 3; j++) {
                o[j] = e.n[j];
                o[3 + j] = e.t[j];
                o[6 + j] = e.b[j];
                o[9 + j] = e.bar[j];
                o[12 + j] = e.cpl[j];
            }
            int q = 15;
            if (pl == POOL_TRI_ROD) o[q++] = e.s;  // the rod record carries s before k
            o[q] = e.k[3];
            o[q + 1] = e.k[0];
            o[q + 2] = e.k[1];
            o[q + 3] = e.k[2];
            for (int j = 0; j < 4; j++) o[q + 4 + j] = e.lam[j];
            o[q + 8] = ((e.flag & CF_USE_STATIC) ? 1 : 0) + ((e.flag & CF_UNCLAMPED) ? 2 : 0);
        }
    }
    return AVBD_OK;
}

int avbd_get_contact_pool(avbd_ctx* c, unsigned capacity, unsigned* p4, uint8_t* active, double* data24,
                          unsigned* size) {
    return get_pool(c, POOL_TRI_RIGID, capacity, p4, active, data24, size);
}

int avbd_get_rod_contact_pool(avbd_ctx* c, unsigned capacity, unsigned* p5, uint8_t* active, double* data25,
                              unsigned* size) {
    return get_pool(c, POOL_TRI_ROD, capacity, p5, active, data25, size);
}

int avbd_debug_set_pair_capacity(avbd_ctx* c, unsigned capacity) {
    if (!c) return set_error(AVBD_ERR_INVALID_ARG, "null context");
    if (c->finalized) return set_error(AVBD_ERR_STATE, "the pair capacity is fixed at avbd_finalize");
    c->debug_pair_capacity = capacity;
    return AVBD_OK;
}

int avbd_debug_set_recolor_rounds(avbd_ctx* c, unsigned rounds) {
    if (!c) return set_error(AVBD_ERR_INVALID_ARG, "null context");
    if (!c->dyn) return set_error(AVBD_ERR_STATE, "no dynamic contacts (finalize a context with triangles and spheres or rod segments)");
    c->dyn->rounds = rounds;
    return AVBD_OK;
}

}  // extern "C"

namespace avbd {

#define INST(R)                                                                                                \
    template int dyn_manage<R>(avbd_ctx*, DevState<R>&, const StepConsts&, cudaStream_t);                     \
    template void dyn_solve_color<R>(avbd_ctx*, DevState<R>&, const StepConsts&, unsigned, cudaStream_t,      \
                                     const SceneTol&);                                                         \
    template void launch_contact_after_iter<R>(avbd_ctx*, DevState<R>&, cudaStream_t, const SceneTol&);
INST(float)
INST(double)
#undef INST

}  // namespace avbd
