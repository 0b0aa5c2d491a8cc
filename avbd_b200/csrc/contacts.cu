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
// reads them with the pool's multipliers and runs the key-ordered merge and
// the tombstone pool (slots are popped and pushed in key order), then
// uploads the pool records and the particles to mark dirty.  On the device:
// the dynamic adjacency when contacts came or went (engine vertex order for
// the solve, reference particle numbering for the recoloring), the
// incremental recoloring in the reference's numbering (its "lower index"
// rule depends on it), the conflicts and the per-color lists in the engine's
// color-major vertex order; the color count and list offsets come back to
// the host, which launches the stage's sweeps.  The vertex slabs of the
// static coloring stay in place: a vertex with contacts or a color changed by
// the recoloring is skipped by its slab's launch and solved from its color's
// list by the solve's dynamic instantiation; colors beyond the static ones
// have lists only.
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
    // ---- dynamic adjacency (built on the device when contacts come or go)
    unsigned num_entries = 0;                    // dynamic entries (slot << 4 | pool << 3 | local)
    uint32_t *d_cnt_eng = nullptr, *d_cnt_ext = nullptr;  // per-vertex counts, then fill cursors
    std::vector<uint32_t> marks;                 // particles of this stage's new contacts (to mark dirty)
    unsigned rounds = 6;  // ColorList::incrementalRecoloring MAX_COLOR_ITERS
    // ---- coloring on the device (reference particle ids): colors, the
    // dirty set (two lists by round parity), last-dirty labels, conflicts
    unsigned num_colors = 0;                     // after the last recoloring
    unsigned dirty_count = 0, conflicted_count = 0;
    uint32_t *d_color = nullptr, *d_cand = nullptr, *d_last_dirty = nullptr;
    uint32_t *d_dirty0 = nullptr, *d_dirty1 = nullptr;
    uint8_t* d_touched = nullptr;
    uint32_t* d_confl_ext = nullptr;
    uint32_t *d_p_off = nullptr, *d_p_nbr = nullptr, *d_dnb_off = nullptr, *d_dnb = nullptr;
    uint32_t *d_marks = nullptr, *d_slab = nullptr;
    uint32_t* d_ctr = nullptr;                   // RC_* counters
    uint32_t* d_lc = nullptr;                    // per-color list counts and cursors
    uint32_t* d_summary = nullptr;               // RC_SUMMARY words for the host
    uint32_t* h_summary = nullptr;               // pinned copy
    unsigned dnb_cap = 0, marks_cap = 0;
    unsigned coop_blocks = 0;                    // grid of the cooperative rounds kernel (0: one block)
    uint8_t* stage[2] = {nullptr, nullptr};      // pinned staging of each pool's upload
    size_t stage_cap[2] = {0, 0};
    // ---- per-color lists (engine vertex order) on the device
    std::vector<unsigned> off3, off6, offc;      // per color: recolored 3-DOF, 6-DOF, conflicted
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

// ColorList::markParticleDirty: recorded here, applied on the device before
// the recoloring (k_rc_mark)
void mark_dirty(DynHost& D, unsigned p) { D.marks.push_back(p); }

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

// ---------------------------------------------- recoloring on the device
// ColorList::incrementalRecoloring, finalizeConflicts and the per-color
// work lists (common/ColorList.hpp:381-522) over reference particle ids.
// A round computes every dirty particle's candidate from the current colors
// and only then applies them (the reference's rounds are Jacobi-style), so
// one kernel per half-round gives the reference's colors exactly; the dirty
// set, its last-dirty labels and the conflicts are sets, so the order in
// which threads append to them changes nothing.
enum : unsigned {
    RC_CNT0 = 0, RC_CNT1 = 1, RC_CUR = 2, RC_NCONFL = 3, RC_NCOLORS = 4, RC_ERR = 5,
    RC_SYNC = 6,   // two words: the cooperative kernel's grid barrier
    RC_BERR = 8,   // its status (AVBD_ERR_BARRIER_TIMEOUT)
    RC_NENT = 9,   // dynamic entries of the current adjacency
    RC_AERR = 10,  // the adjacency outgrew its buffers
    RC_NCTR = 12
};
constexpr unsigned RC_MAXC = 256;  // colors (ColorList's bitset)
// summary for the host: [num_colors, dirty count, conflicted count, error,
// off3[0..256], off6[0..256], offc[0..256], dynamic entries]
constexpr unsigned RC_SUMMARY = 4 + 3 * (RC_MAXC + 1) + 1;

struct RcDev {
    uint32_t *color, *cand, *last_dirty, *dirty0, *dirty1, *ctr;
    uint8_t* touched;
    uint32_t* confl;
    const uint32_t *p_off, *p_nbr, *dnb_off, *dnb;
};

// the lane's share of p's neighbours: static ones, then dynamic ones,
// every 32nd from `lane`
template <typename F>
AVBD_D void rc_neighbors_lane(const RcDev& R, unsigned p, unsigned lane, F&& f) {
    const unsigned s0 = R.p_off[p], ds = R.p_off[p + 1] - s0;
    const unsigned d0 = R.dnb_off[p], dd = R.dnb_off[p + 1] - d0;
    for (unsigned k = lane; k < ds + dd; k += 32) f(k < ds ? R.p_nbr[s0 + k] : R.dnb[d0 + k - ds]);
}

// the conflicts of the last stage are cleared, then this stage's new
// contacts' particles join the dirty set (those already in it keep label 0)
AVBD_D void rc_mark(const RcDev& R, const uint32_t* __restrict__ marks, unsigned nmarks, unsigned t0, unsigned dt) {
    const unsigned cur = R.ctr[RC_CUR];
    uint32_t* list = cur ? R.dirty1 : R.dirty0;
    for (unsigned j = t0; j < nmarks; j += dt) {
        const unsigned p = marks[j];
        if (atomicExch(R.last_dirty + p, 0u) != 0u) {
            R.touched[p] = 1;
            list[atomicAdd(R.ctr + cur, 1u)] = p;
        }
    }
}

// half-round 1: a dirty particle sharing its color with a lower-numbered
// neighbour takes the smallest color no neighbour holds (one warp per
// particle, the neighbours' color bits or-reduced over the lanes)
AVBD_D void rc_cand(const RcDev& R, unsigned cur, unsigned warp, unsigned nwarps, unsigned lane) {
    const unsigned cnt = R.ctr[cur];
    const uint32_t* list = cur ? R.dirty1 : R.dirty0;
    for (unsigned j = warp; j < cnt; j += nwarps) {  // one warp per dirty particle
        const unsigned p = list[j], cp = R.color[p];
        uint32_t bits[RC_MAXC / 32] = {0, 0, 0, 0, 0, 0, 0, 0};
        bool must = false, over = false;
        rc_neighbors_lane(R, p, lane, [&](unsigned q) {
            const unsigned cq = R.color[q];
            if (cq >= RC_MAXC) {
                over = true;
                return;
            }
            bits[cq >> 5] |= 1u << (cq & 31u);
            if (cq == cp && q < p) must = true;
        });
#pragma unroll
        for (unsigned w = 0; w < RC_MAXC / 32; w++) bits[w] = __reduce_or_sync(0xffffffffu, bits[w]);
        must = __any_sync(0xffffffffu, must);
        over = __any_sync(0xffffffffu, over);
        if (lane != 0) continue;
        unsigned cand = cp;
        if (over) {
            atomicExch(R.ctr + RC_ERR, 1u);
        } else if (must) {
            cand = RC_MAXC;
            for (unsigned w = 0; w < RC_MAXC / 32 && cand == RC_MAXC; w++)
                if (~bits[w]) cand = w * 32 + (unsigned)__ffs((int)~bits[w]) - 1u;
            if (cand == RC_MAXC) {
                atomicExch(R.ctr + RC_ERR, 1u);
                cand = cp;
            } else {
                atomicMax(R.ctr + RC_NCOLORS, cand + 1u);  // cand <= num_colors: one new color at most
            }
        }
        R.cand[p] = cand;
    }
}

// half-round 2: candidates applied; every neighbour of a changed particle
// joins the next round's dirty set, once per round (label = round + 1)
AVBD_D void rc_apply(const RcDev& R, unsigned cur, unsigned label, unsigned warp, unsigned nwarps, unsigned lane) {
    const unsigned cnt = R.ctr[cur];
    const uint32_t* list = cur ? R.dirty1 : R.dirty0;
    uint32_t* next = cur ? R.dirty0 : R.dirty1;
    for (unsigned j = warp; j < cnt; j += nwarps) {
        const unsigned p = list[j], cand = R.cand[p];
        if (cand == R.color[p]) continue;  // the same answer on every lane of the warp
        __syncwarp();                       // every lane has read the old color
        if (lane == 0) R.color[p] = cand;
        rc_neighbors_lane(R, p, lane, [&](unsigned q) {
            if (atomicExch(R.last_dirty + q, label) != label) {
                R.touched[q] = 1;
                next[atomicAdd(R.ctr + (cur ^ 1u), 1u)] = q;
            }
        });
    }
}

// finalizeConflicts: particles still dirty after the last round and their
// same-colored neighbours are conflicted
AVBD_D void rc_conflicts(const RcDev& R, unsigned cur, unsigned warp, unsigned nwarps, unsigned lane) {
    const unsigned cnt = R.ctr[cur];
    const uint32_t* list = cur ? R.dirty1 : R.dirty0;
    for (unsigned j = warp; j < cnt; j += nwarps) {
        const unsigned p = list[j], cp = R.color[p];
        rc_neighbors_lane(R, p, lane, [&](unsigned q) {
            if (R.color[q] != cp) return;
            if (atomicExch(R.confl + p, 1u) == 0u) atomicAdd(R.ctr + RC_NCONFL, 1u);
            if (atomicExch(R.confl + q, 1u) == 0u) atomicAdd(R.ctr + RC_NCONFL, 1u);
        });
    }
}

// labels written this stage go back to the sentinel ...
AVBD_D void rc_settle(const RcDev& R, unsigned n, unsigned t0, unsigned dt) {
    for (unsigned p = t0; p < n; p += dt)
        if (R.touched[p]) {
            R.touched[p] = 0;
            R.last_dirty[p] = DIRTY_SENTINEL;
        }
}
// ... and the particles still dirty carry label 0 into the next stage
AVBD_D void rc_keep(const RcDev& R, unsigned t0, unsigned dt) {
    const unsigned cur = R.ctr[RC_CUR], cnt = R.ctr[cur];
    const uint32_t* list = cur ? R.dirty1 : R.dirty0;
    for (unsigned j = t0; j < cnt; j += dt)
        R.last_dirty[list[j]] = 0;
}

// Per-color lists in the engine's vertex order: a vertex with dynamic
// entries or a color other than its slab's is skipped by the slab launch and
// solved from its color's list (positional or oriented; fixed vertices are
// skipped and not listed); conflicted vertices are listed for the commit.
// lc: counts [3][256] then cursors [3][256].
struct RcLists {
    const uint32_t *perm, *slab, *dyn_begin;
    const uint8_t* flags;
    uint8_t *skip, *confl_eng;
    uint32_t *lc, *lists, *summary;
    unsigned n;
};

AVBD_D void rc_count(const RcDev& R, const RcLists& L, unsigned t0, unsigned dt) {
    const uint32_t *perm = L.perm, *slab = L.slab, *dyn_begin = L.dyn_begin;
    const uint8_t* flags = L.flags;
    uint8_t *skip = L.skip, *confl_eng = L.confl_eng;
    uint32_t* lc = L.lc;
    for (unsigned i = t0; i < L.n; i += dt) {
        const unsigned e = perm[i], ce = R.color[e];
        const uint8_t cf = R.confl[e] ? 1 : 0;
        confl_eng[i] = cf;
        if (cf) atomicAdd(lc + 2 * RC_MAXC + ce, 1u);
        const bool sk = ce != slab[i] || dyn_begin[i + 1] != dyn_begin[i];
        skip[i] = sk ? 1 : 0;
        if (!sk || (flags[i] & VF_FIXED)) continue;
        atomicAdd(lc + ((flags[i] & VF_ORIENTED) ? RC_MAXC : 0u) + ce, 1u);
    }
}

// offsets: all positional lists, then all oriented, then all conflicted;
// the summary the host reads back
AVBD_D void rc_offsets(const RcDev& R, const RcLists& L) {
    uint32_t *lc = L.lc, *summary = L.summary;
    const unsigned nc = min(R.ctr[RC_NCOLORS], RC_MAXC);
    unsigned run = 0;
    for (unsigned t = 0; t < 3; t++) {
        uint32_t* off = summary + 4 + t * (RC_MAXC + 1);
        for (unsigned k = 0; k < nc; k++) {
            off[k] = run;
            lc[3 * RC_MAXC + t * RC_MAXC + k] = run;
            run += lc[t * RC_MAXC + k];
        }
        off[nc] = run;
    }
    summary[4 + 3 * (RC_MAXC + 1)] = R.ctr[RC_NENT];
    summary[0] = R.ctr[RC_NCOLORS];
    summary[1] = R.ctr[R.ctr[RC_CUR]];
    summary[2] = R.ctr[RC_NCONFL];
    summary[3] = R.ctr[RC_ERR] ? 1u : (R.ctr[RC_BERR] ? 2u : (R.ctr[RC_AERR] ? 3u : 0u));
}

AVBD_D void rc_fill(const RcDev& R, const RcLists& L, unsigned t0, unsigned dt) {
    const uint32_t* perm = L.perm;
    const uint8_t *skip = L.skip, *confl_eng = L.confl_eng, *flags = L.flags;
    uint32_t *lc = L.lc, *lists = L.lists;
    for (unsigned i = t0; i < L.n; i += dt) {
        const unsigned ce = R.color[perm[i]];
        if (confl_eng[i]) lists[atomicAdd(lc + 3 * RC_MAXC + 2 * RC_MAXC + ce, 1u)] = i;
        if (!skip[i] || (flags[i] & VF_FIXED)) continue;
        lists[atomicAdd(lc + 3 * RC_MAXC + ((flags[i] & VF_ORIENTED) ? RC_MAXC : 0u) + ce, 1u)] = i;
    }
}

// the passes over every vertex as grid-wide kernels ...
#define RC_GRID blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x
__global__ void k_rc_settle(RcDev R, unsigned n) { rc_settle(R, n, RC_GRID); }
__global__ void k_rc_offsets(RcDev R, RcLists L) {
    if (blockIdx.x == 0 && threadIdx.x == 0) rc_offsets(R, L);
}
__global__ void k_rc_fill(RcDev R, RcLists L) { rc_fill(R, L, RC_GRID); }
#undef RC_GRID

// ... and the phases over the dirty set (the particles of new contacts and
// their neighbourhoods): the conflicts and list counts cleared, the marks,
// every round (candidates, then their application), the conflicts.  Round r
// reads the dirty list cur ^ (r & 1) and appends to the other, whose count
// its candidate phase has zeroed (nobody reads it then).  Either as one
// cooperative launch over the SMs, the phases separated by bounded grid
// barriers, or, where the device cannot launch cooperatively, in one block,
// separated by block barriers.
__device__ uint32_t g_rc_wait_polls = AVBD_DEFAULT_WAIT_POLLS;

template <bool COOP>
__global__ void __launch_bounds__(COOP ? 256 : 1024) k_rc_rounds(RcDev R, uint32_t* lc, unsigned n,
                                                                  const uint32_t* __restrict__ marks,
                                                                  unsigned nmarks, unsigned rounds) {
    const unsigned t0 = COOP ? blockIdx.x * blockDim.x + threadIdx.x : threadIdx.x;
    const unsigned dt = COOP ? gridDim.x * blockDim.x : blockDim.x;
    const unsigned warp = t0 >> 5, nwarps = dt >> 5, lane = threadIdx.x & 31u;
    const unsigned limit = *(volatile uint32_t*)&g_rc_wait_polls;
    unsigned* sync = R.ctr + RC_SYNC;
    int* berr = reinterpret_cast<int*>(R.ctr + RC_BERR);
    auto barrier = [&]() -> bool {
        if constexpr (COOP) return grid_barrier_bounded(sync, berr, limit);
        __syncthreads();
        return true;
    };
    // an adjacency that outgrew its buffers is not read (the stage reports
    // AVBD_ERR_CAPACITY); every block returns here, before any barrier
    if (R.ctr[RC_AERR]) return;
    const unsigned cur0 = R.ctr[RC_CUR];
    for (unsigned p = t0; p < n; p += dt) R.confl[p] = 0;  // the last stage's conflicts
    for (unsigned k = t0; k < 6 * RC_MAXC; k += dt) lc[k] = 0;
    if (t0 == 0) R.ctr[RC_NCONFL] = 0;
    if (!barrier()) return;
    rc_mark(R, marks, nmarks, t0, dt);
    if (!barrier()) return;
    for (unsigned it = 0; it < rounds; it++) {
        const unsigned cur = cur0 ^ (it & 1u);
        if (t0 == 0) R.ctr[cur ^ 1u] = 0;
        rc_cand(R, cur, warp, nwarps, lane);
        if (!barrier()) return;
        rc_apply(R, cur, it + 1, warp, nwarps, lane);
        if (!barrier()) return;
    }
    const unsigned cur = cur0 ^ (rounds & 1u);
    if (t0 == 0) R.ctr[RC_CUR] = cur;
    rc_conflicts(R, cur, warp, nwarps, lane);
}

// the list counts, with the carried-over labels of the still-dirty particles
// set by block 0 (after the settle kernel, independent of the counts)
__global__ void k_rc_count_keep(RcDev R, RcLists L) {
    if (blockIdx.x == 0) rc_keep(R, threadIdx.x, blockDim.x);
    rc_count(R, L, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ------------------------------------------- dynamic adjacency on the device
// DynamicParticleAdjacency::buildAdjacency (common/DynamicParticleAdjacency.hpp:33-118)
// over the live slots of both pools: per engine vertex the entries of its
// contacts in the reference's order (pool 0 then pool 1, ascending slot) for
// the solve, whose block sums follow it; per reference particle the other
// particles of its contacts for the recoloring (a set: any order).
// Counts, one exclusive scan each, a fill through per-vertex cursors, then
// each engine vertex's few entries sorted by (pool, slot).
template <typename R>
AVBD_D void adj_slot(const ContactPoolDev<R>& P, unsigned pl, unsigned s, unsigned (&ids)[5], unsigned& np) {
    const uint4 q = P.p[s];
    np = pl ? 5u : 4u;
    ids[0] = q.x;
    ids[1] = q.y;
    ids[2] = q.z;
    ids[3] = q.w;
    ids[4] = pl ? P.p5[s] : 0u;
}

template <typename R>
__global__ void k_adj_count(DevState<R> s, unsigned size0, unsigned size1, const uint32_t* __restrict__ perm,
                            uint32_t* cnt_eng, uint32_t* cnt_ext) {
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned pl = 0;
    if (k >= size0) {
        k -= size0;
        pl = 1;
        if (k >= size1) return;
    }
    const ContactPoolDev<R>& P = s.cp[pl];
    if (!(P.flag[k] & CF_ACTIVE)) return;
    unsigned ids[5], np;
    adj_slot(P, pl, k, ids, np);
    for (unsigned j = 0; j < np; j++) {
        atomicAdd(cnt_eng + ids[j], 1u);
        atomicAdd(cnt_ext + perm[ids[j]], np - 1u);
    }
}

// exclusive scan of n + 1 counts (the last is 0) into off, the counts become
// the fill cursors; one block, a warp per contiguous segment (as the radix
// sort's histogram scan); total into *total
__global__ void __launch_bounds__(1024) k_adj_scan(uint32_t* cnt, uint32_t* off, unsigned n1, uint32_t* total) {
    __shared__ uint32_t wsum[32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned seg = (n1 + 31u) / 32u;
    const unsigned b = min(warp * seg, n1), e = min(b + seg, n1);
    uint32_t t = 0;
    for (unsigned k = b + lane; k < e; k += 32u) t += cnt[k];
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) t += __shfl_xor_sync(0xffffffffu, t, m);
    if (lane == 0) wsum[warp] = t;
    __syncthreads();
    if (warp == 0) {
        const uint32_t v = wsum[lane];
        uint32_t incl = v;
#pragma unroll
        for (int m = 1; m < 32; m <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, m);
            if (lane >= (unsigned)m) incl += u;
        }
        wsum[lane] = incl - v;
        if (lane == 31 && total) *total = incl;
    }
    __syncthreads();
    uint32_t carry = wsum[warp];
    for (unsigned k0 = b; k0 < e; k0 += 32u) {
        const unsigned k = k0 + lane;
        const uint32_t v = k < e ? cnt[k] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int m = 1; m < 32; m <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, m);
            if (lane >= (unsigned)m) incl += u;
        }
        if (k < e) {
            off[k] = carry + incl - v;
            cnt[k] = carry + incl - v;  // the cursor of vertex k
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
}

template <typename R>
__global__ void k_adj_fill(DevState<R> s, unsigned size0, unsigned size1, const uint32_t* __restrict__ perm,
                           uint32_t* cur_eng, uint32_t* cur_ext, uint32_t* dnb, unsigned ent_cap, unsigned dnb_cap,
                           uint32_t* err) {
    unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned pl = 0;
    if (k >= size0) {
        k -= size0;
        pl = 1;
        if (k >= size1) return;
    }
    const ContactPoolDev<R>& P = s.cp[pl];
    if (!(P.flag[k] & CF_ACTIVE)) return;
    unsigned ids[5], np;
    adj_slot(P, pl, k, ids, np);
    for (unsigned j = 0; j < np; j++) {
        const unsigned pos = atomicAdd(cur_eng + ids[j], 1u);
        if (pos < ent_cap) s.dyn_ent[pos] = (k << 4) | (pl << 3) | j;
        else atomicExch(err, 1u);
        const unsigned e = perm[ids[j]];
        for (unsigned j2 = 0; j2 < np; j2++) {
            if (j2 == j) continue;
            const unsigned q = atomicAdd(cur_ext + e, 1u);
            if (q < dnb_cap) dnb[q] = perm[ids[j2]];
            else atomicExch(err, 1u);
        }
    }
}

// each engine vertex's entries in (pool, slot) order
template <typename R>
__global__ void k_adj_order(DevState<R> s, unsigned n, unsigned ent_cap) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned b = s.dyn_begin[i], e = min(s.dyn_begin[i + 1], ent_cap);
    for (unsigned a = b + 1; a < e; a++) {  // insertion sort: a few entries per vertex
        const uint32_t v = s.dyn_ent[a];
        const uint32_t key = ((v >> 3) & 1u) << 28 | (v >> 4);
        unsigned j = a;
        while (j > b) {
            const uint32_t w = s.dyn_ent[j - 1];
            if ((((w >> 3) & 1u) << 28 | (w >> 4)) <= key) break;
            s.dyn_ent[j] = w;
            j--;
        }
        s.dyn_ent[j] = v;
    }
}

RcDev rc_dev(DynHost& D) {
    return RcDev{D.d_color, D.d_cand, D.d_last_dirty, D.d_dirty0, D.d_dirty1, D.d_ctr,
                 D.d_touched, D.d_confl_ext, D.d_p_off, D.d_p_nbr, D.d_dnb_off, D.d_dnb};
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
    // the recoloring's state; a dynamic entry has at most 4 other particles
    D.dnb_cap = 4 * D.ent_cap;
    D.marks_cap = 5 * cap;
    if (!alloc((void**)&D.d_color, sizeof(uint32_t) * n) || !alloc((void**)&D.d_cand, sizeof(uint32_t) * n) ||
        !alloc((void**)&D.d_last_dirty, sizeof(uint32_t) * n) || !alloc((void**)&D.d_dirty0, sizeof(uint32_t) * n) ||
        !alloc((void**)&D.d_dirty1, sizeof(uint32_t) * n) || !alloc((void**)&D.d_touched, n) ||
        !alloc((void**)&D.d_confl_ext, sizeof(uint32_t) * n) || !alloc((void**)&D.d_dnb_off, sizeof(uint32_t) * (n + 1)) ||
        !alloc((void**)&D.d_dnb, sizeof(uint32_t) * D.dnb_cap) || !alloc((void**)&D.d_marks, sizeof(uint32_t) * D.marks_cap) ||
        !alloc((void**)&D.d_slab, sizeof(uint32_t) * n) || !alloc((void**)&D.d_ctr, sizeof(uint32_t) * RC_NCTR) ||
        !alloc((void**)&D.d_lc, sizeof(uint32_t) * 6 * RC_MAXC) || !alloc((void**)&D.d_summary, sizeof(uint32_t) * RC_SUMMARY) ||
        !alloc((void**)&D.d_cnt_eng, sizeof(uint32_t) * (n + 1)) || !alloc((void**)&D.d_cnt_ext, sizeof(uint32_t) * (n + 1)))
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

// The pool's records by slot (engine particle ids, state precision) into a
// pinned staging area that persists across stages, then copied to the device
// asynchronously: the next stage reuses the area only after its own
// synchronisation, which follows these copies on the stream.
template <typename R>
int upload_pool(avbd_ctx* c, ContactPoolDev<R>& S, const DynHost::Pool& D, DynHost& H, int pl, cudaStream_t st) {
    using V4 = typename Vec4Of<R>::T;
    const unsigned m = D.size;
    if (m == 0) return AVBD_OK;
    const size_t need = (size_t)m * (7 * sizeof(V4) + sizeof(uint4) + sizeof(uint32_t) + 1);
    if (H.stage_cap[pl] < need) {
        DYN_CUDA(cudaStreamSynchronize(st));  // copies from the old area are done
        if (H.stage[pl]) cudaFreeHost(H.stage[pl]);
        H.stage[pl] = nullptr;
        H.stage_cap[pl] = 0;
        DYN_CUDA(cudaMallocHost((void**)&H.stage[pl], 2 * need));
        H.stage_cap[pl] = 2 * need;
    }
    uint8_t* base = H.stage[pl];
    V4* vn = reinterpret_cast<V4*>(base);
    V4 *vt = vn + m, *vb = vt + m, *vbar = vb + m, *vcpl = vbar + m, *vk = vcpl + m, *vlam = vk + m;
    uint4* p = reinterpret_cast<uint4*>(vlam + m);
    uint32_t* p5 = reinterpret_cast<uint32_t*>(p + m);
    uint8_t* f = reinterpret_cast<uint8_t*>(p5 + m);
    auto v4 = [](const double a[3], double w) {
        V4 o;
        o.x = (R)a[0]; o.y = (R)a[1]; o.z = (R)a[2]; o.w = (R)w;
        return o;
    };
    const double z3[3] = {0, 0, 0};
    const V4 zero = v4(z3, 0);
    for (unsigned i = 0; i < m; i++) {
        const DynHost::Rec& e = D.rec[i];
        if (!D.active[i]) {
            f[i] = 0;
            p[i] = make_uint4(0, 0, 0, 0);
            p5[i] = 0;
            vn[i] = vt[i] = vb[i] = vbar[i] = vcpl[i] = vk[i] = vlam[i] = zero;
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
    DYN_CUDA(cudaMemcpyAsync(S.p, p, sizeof(uint4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.p5, p5, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.n, vn, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.t, vt, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.b, vb, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.bar, vbar, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.cpl, vcpl, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.k, vk, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.lam, vlam, sizeof(V4) * m, cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemcpyAsync(S.flag, f, m, cudaMemcpyHostToDevice, st));
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
    D->num_colors = c->num_colors;
    D->off3.assign(D->num_colors + 1, 0);
    D->off6.assign(D->num_colors + 1, 0);
    D->offc.assign(D->num_colors + 1, 0);
    c->dyn = D;
    const bool d64 = c->solver.precision != AVBD_PRECISION_FP32;
    int rc = d64 ? alloc_state<double>(c, c->d, *D, err) : alloc_state<float>(c, c->f, *D, err);
    if (rc) {
        dyn_destroy(c);
        return rc;
    }
    // the set-up coloring, the static neighbours and each engine vertex's
    // slab color go to the device once; no particle is dirty yet
    std::vector<uint32_t> slab(n, 0), ctr(RC_NCTR, 0);
    for (unsigned k = 0; k < c->num_colors; k++)
        for (unsigned i = c->color_begin[k]; i < c->color_begin[k + 1]; i++) slab[i] = k;
    ctr[RC_NCOLORS] = c->num_colors;
    int coop = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device) == cudaSuccess && coop &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rc_rounds<true>, 256, 0) == cudaSuccess && per_sm > 0)
        D->coop_blocks = c->num_sms;  // one block per SM: always co-resident
    cudaGetLastError();
    cudaStream_t st = c->stream;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return bytes == 0 || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    };
    auto dalloc = [&](uint32_t** q, size_t count) {
        *q = nullptr;
        if (cudaMalloc((void**)q, sizeof(uint32_t) * (count ? count : 1)) != cudaSuccess) return false;
        c->allocations.push_back((void*)*q);
        return true;
    };
    bool ok = cudaMallocHost((void**)&D->h_summary, sizeof(uint32_t) * RC_SUMMARY) == cudaSuccess &&
              dalloc(&D->d_p_off, n + 1) && dalloc(&D->d_p_nbr, p_nbr.size());
    ok = ok && up(D->d_color, c->color.data(), sizeof(uint32_t) * n) && up(D->d_slab, slab.data(), sizeof(uint32_t) * n) &&
         up(D->d_ctr, ctr.data(), sizeof(uint32_t) * RC_NCTR) &&
         up(D->d_p_off, p_off.data(), sizeof(uint32_t) * (n + 1)) &&
         up(D->d_p_nbr, p_nbr.data(), sizeof(uint32_t) * p_nbr.size()) &&
         cudaMemsetAsync(D->d_last_dirty, 0xFF, sizeof(uint32_t) * n, st) == cudaSuccess &&
         cudaMemsetAsync(D->d_touched, 0, n, st) == cudaSuccess &&
         cudaMemsetAsync(D->d_confl_ext, 0, sizeof(uint32_t) * n, st) == cudaSuccess &&
         cudaMemsetAsync(D->d_dnb_off, 0, sizeof(uint32_t) * (n + 1), st) == cudaSuccess &&
         cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
        if (err.empty()) err = "recoloring state: CUDA call failed";
        dyn_destroy(c);
        return AVBD_ERR_CUDA;
    }
    return AVBD_OK;
}

void dyn_destroy(avbd_ctx* c) {
    if (c->dyn) {
        if (c->dyn->h_summary || c->dyn->stage[0] || c->dyn->stage[1]) cudaStreamSynchronize(c->stream);
        if (c->dyn->h_summary) cudaFreeHost(c->dyn->h_summary);
        for (uint8_t* b : c->dyn->stage)
            if (b) cudaFreeHost(b);
    }
    delete c->dyn;
    c->dyn = nullptr;
}

unsigned dyn_num_colors(const avbd_ctx* c) { return c->dyn ? c->dyn->num_colors : c->num_colors; }

void dyn_positional_list(const avbd_ctx* c, const uint32_t** list, unsigned* count) {
    const DynHost& D = *c->dyn;
    *list = D.d_lists + D.off3.front();
    *count = D.off3.back() - D.off3.front();
}

int contacts_set_wait_limit(unsigned polls) {
    cudaError_t e = cudaMemcpyToSymbol(g_rc_wait_polls, &polls, sizeof(polls));
    return e == cudaSuccess ? AVBD_OK : set_error(AVBD_ERR_CUDA, cudaGetErrorString(e));
}

int dyn_coloring(const avbd_ctx* c, unsigned* colors) {
    if (!c->dyn) {
        std::copy(c->color.begin(), c->color.end(), colors);
        return AVBD_OK;
    }
    const size_t n = c->color.size();
    DYN_CUDA(cudaMemcpyAsync(colors, c->dyn->d_color, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    DYN_CUDA(cudaStreamSynchronize(c->stream));
    return AVBD_OK;
}

// The recoloring, the conflicts and the per-color lists of one stage on the
// device (after the merge's marks and the dynamic adjacency are uploaded),
// then the per-color list offsets, the color count and the error flag read
// back: the host needs them to launch the stage's sweeps.
int dyn_recolor_device(avbd_ctx* c, const uint32_t* dyn_begin, const uint8_t* flags, uint8_t* skip,
                       uint8_t* confl_eng, cudaStream_t st) {
    DynHost& D = *c->dyn;
    const unsigned n = (unsigned)c->perm.size();
    const RcDev R = rc_dev(D);
    const unsigned nm = (unsigned)D.marks.size();
    if (nm > D.marks_cap) return set_error(AVBD_ERR_CAPACITY, "dirty marks exceed their capacity");
    if (nm) DYN_CUDA(cudaMemcpyAsync(D.d_marks, D.marks.data(), sizeof(uint32_t) * nm, cudaMemcpyHostToDevice, st));
    D.marks.clear();
    const RcLists L{c->d_perm, D.d_slab, dyn_begin, flags, skip, confl_eng, D.d_lc, D.d_lists, D.d_summary, n};
    const unsigned gb = nblk(n, 256);
    if (D.coop_blocks) {
        DYN_CUDA(cudaMemsetAsync(D.d_ctr + RC_SYNC, 0, sizeof(uint32_t) * 3, st));  // barrier and its status
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(D.coop_blocks);
        cfg.blockDim = dim3(256);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        DYN_CUDA(cudaLaunchKernelEx(&cfg, k_rc_rounds<true>, R, D.d_lc, n, (const uint32_t*)D.d_marks, nm, D.rounds));
    } else {
        k_rc_rounds<false><<<1, 1024, 0, st>>>(R, D.d_lc, n, D.d_marks, nm, D.rounds);
    }
    k_rc_settle<<<gb, 256, 0, st>>>(R, n);
    k_rc_count_keep<<<gb, 256, 0, st>>>(R, L);
    k_rc_offsets<<<1, 32, 0, st>>>(R, L);
    k_rc_fill<<<gb, 256, 0, st>>>(R, L);
    count_launch(c, 5);
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaMemcpyAsync(D.h_summary, D.d_summary, sizeof(uint32_t) * RC_SUMMARY, cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    const uint32_t* h = D.h_summary;
    if (h[3] == 2)
        return set_error(AVBD_ERR_BARRIER_TIMEOUT, "a grid-barrier wait of the recoloring gave up");
    if (h[3] == 3) return set_error(AVBD_ERR_CAPACITY, "dynamic adjacency exceeds its capacity");
    D.num_entries = h[4 + 3 * (RC_MAXC + 1)];
    if (h[3]) return set_error(AVBD_ERR_COLORS, "Ran out of colors!");
    D.num_colors = std::min(h[0], RC_MAXC);
    D.dirty_count = h[1];
    D.conflicted_count = h[2];
    const unsigned nc = D.num_colors;
    D.off3.assign(h + 4, h + 4 + nc + 1);
    D.off6.assign(h + 4 + (RC_MAXC + 1), h + 4 + (RC_MAXC + 1) + nc + 1);
    D.offc.assign(h + 4 + 2 * (RC_MAXC + 1), h + 4 + 2 * (RC_MAXC + 1) + nc + 1);
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

    // uploads: pool records, dynamic adjacency (engine order for the solve,
    // reference order for the recoloring)
    for (int pl = 0; pl < 2; pl++)
        if (int r = upload_pool<R>(c, s.cp[pl], D.pool[pl], D, pl, st)) return r;
    if (D.csr_dirty) {  // contacts came or went: the dynamic adjacency anew, on the device
        const unsigned s0 = D.pool[0].size, s1 = D.pool[1].size;
        DYN_CUDA(cudaMemsetAsync(D.d_cnt_eng, 0, sizeof(uint32_t) * (n + 1), st));
        DYN_CUDA(cudaMemsetAsync(D.d_cnt_ext, 0, sizeof(uint32_t) * (n + 1), st));
        DYN_CUDA(cudaMemsetAsync(D.d_ctr + RC_AERR, 0, sizeof(uint32_t), st));
        if (s0 + s1) k_adj_count<R><<<nblk(s0 + s1, 128), 128, 0, st>>>(s, s0, s1, c->d_perm, D.d_cnt_eng, D.d_cnt_ext);
        k_adj_scan<<<1, 1024, 0, st>>>(D.d_cnt_eng, s.dyn_begin, n + 1, D.d_ctr + RC_NENT);
        k_adj_scan<<<1, 1024, 0, st>>>(D.d_cnt_ext, D.d_dnb_off, n + 1, nullptr);
        if (s0 + s1)
            k_adj_fill<R><<<nblk(s0 + s1, 128), 128, 0, st>>>(s, s0, s1, c->d_perm, D.d_cnt_eng, D.d_cnt_ext, D.d_dnb,
                                                             D.ent_cap, D.dnb_cap, D.d_ctr + RC_AERR);
        k_adj_order<R><<<nblk(n, 256), 256, 0, st>>>(s, n, D.ent_cap);
        count_launch(c, 6);
        D.csr_dirty = false;
    }
    if (int r = dyn_recolor_device(c, s.dyn_begin, s.flags, s.dyn_skip, s.conflicted, st)) return r;
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
    out[3] = D.conflicted_count;
    out[4] = D.dirty_count;
    out[5] = D.num_entries;
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
