// capi.cu -- the C-ABI of include/avbd.h: context lifetime, set-up staging,
// finalize (adjacency, coloring, HBM layout) and the step driver.
//
// Device layout chosen at finalize:
//   * particles are renumbered color-major (internal order): every color is a
//     contiguous slab [solved positional | oriented | fixed], so a color phase
//     reads and writes its vertices' x, y and contact state with unit stride;
//   * every solved vertex owns a contiguous run of 64-byte NeoHookean
//     incidence records in slab order, streamed once per color phase;
//   * one CUDA graph holds a whole fixed-iteration step.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <thread>
#include <type_traits>

#include "engine.h"

using namespace avbd;

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

// AVBD_TRACE=1 prints the set-up stages to stderr.
static void trace(const char* what) {
    static int on = -1;
    if (on < 0) on = getenv("AVBD_TRACE") != nullptr;
    if (on) fprintf(stderr, "[avbd] %s\n", what);
}

#define CUDA_OR_FAIL(x)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess) return fail(AVBD_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace avbd {
void count_launch(avbd_ctx* c, unsigned k) { c->stats.kernel_launches += k; }
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}

// FP64 and mixed keep the particle state in double precision.
static bool use64(const avbd_ctx* c) { return c->solver.precision != AVBD_PRECISION_FP32; }

template <typename T>
static int dalloc(avbd_ctx* c, T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) return fail(AVBD_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    c->allocations.push_back((void*)*p);
    return AVBD_OK;
}

static void free_device(avbd_ctx* c) {
    if (c->graph) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    if (c->dyn_graph) {
        cudaGraphExecDestroy(c->dyn_graph);
        c->dyn_graph = nullptr;
    }
    for (void* p : c->allocations) cudaFree(p);
    c->allocations.clear();
    dyn_destroy(c);
    c->f = DevState<float>();
    c->d = DevState<double>();
    c->lbvh = LbvhState();
    c->d_residual = nullptr;
    c->d_h2d = nullptr;
    c->h2d_cap = 0;
    c->d_counters = nullptr;
    c->d_perm = nullptr;
    c->d_inv = nullptr;
    c->d_error = nullptr;
    c->d_scene = nullptr;
    c->d_scene_active = nullptr;
    c->d_scene_cand = nullptr;
    c->d_scene_r2 = nullptr;
    c->d_scene_ex = nullptr;
    c->d_scene_rin = nullptr;
    c->d_scene_mg2 = nullptr;
    c->d_scene_iters = nullptr;
    c->d_tol_count = nullptr;
    c->d_tol_it = nullptr;
    c->d_tol_omega = nullptr;
    c->d_omega_tab = nullptr;
    c->omega_tab_n = 0;
    c->graph_tol = false;
    c->d_solve_ranges = nullptr;
    c->solve_range_off.clear();
    mlp_device_free(c->ws_mlp);
    c->ws_mlp = nullptr;
    c->d_ws_feat = c->d_ws_x0 = nullptr;
    c->d_ws_target = nullptr;
    c->ws_mode = 0;
    c->d_ws_guess = nullptr;
    c->ws_guess_pending = false;
    c->ws_recorded = false;
    c->finalized = false;
    c->graph_dirty = true;
}

static int check_ctx(avbd_ctx* c) {
    if (!c) return fail(AVBD_ERR_INVALID_ARG, "null context");
    return AVBD_OK;
}

static int staging_only(avbd_ctx* c) {
    if (c->finalized) {
        // adding after finalize invalidates the device layout; it is rebuilt at the next finalize
        free_device(c);
    }
    return AVBD_OK;
}

extern "C" {

const char* avbd_last_error_string(void) { return g_err.c_str(); }
const char* avbd_version(void) { return "avbd-b200 0.1 (sm_100a)"; }

int avbd_create(avbd_ctx** out, int device, unsigned particles_capacity, unsigned oriented_capacity,
                unsigned energies_capacity, unsigned primitives_capacity, unsigned sdf_capacity) {
    if (!out) return fail(AVBD_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(AVBD_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(AVBD_ERR_INVALID_ARG, "bad device index");
    CUDA_OR_FAIL(cudaSetDevice(device));
    avbd_ctx* c = new avbd_ctx();
    c->device = device;
    c->cap_particles = particles_capacity;
    c->cap_oriented = oriented_capacity;
    c->cap_energies = energies_capacity;
    c->cap_prims = primitives_capacity;
    c->cap_sdf = sdf_capacity;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return fail(AVBD_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    c->stream = c->own_stream;
    if (const char* g = getenv("AVBD_GRAPH")) c->use_graph = atoi(g) != 0;  // 0: no CUDA graphs
    // condition threshold above which a block is re-solved in FP64 (0: always)
    if (const char* km = getenv("AVBD_KAPPA_MAX")) c->kappa_max = atof(km);
    // the sweeps of run-to-tolerance steps as one persistent cooperative launch
    // per iteration (default; 0 launches each color separately)
    if (const char* ps = getenv("AVBD_PERSISTENT")) c->persistent = atoi(ps) != 0;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess) c->num_sms = (unsigned)sms;
    *out = c;
    return AVBD_OK;
}

int avbd_destroy(avbd_ctx* c) {
    if (!c) return AVBD_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_device(c);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return AVBD_OK;
}

int avbd_set_stream(avbd_ctx* c, void* s) {
    if (int r = check_ctx(c)) return r;
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    c->graph_dirty = true;
    return AVBD_OK;
}

int avbd_set_params(avbd_ctx* c, const avbd_params* p) {
    if (int r = check_ctx(c)) return r;
    if (!p || !(p->dt > 0)) return fail(AVBD_ERR_INVALID_ARG, "dt must be positive");
    c->params = *p;
    c->graph_dirty = true;
    return AVBD_OK;
}

int avbd_set_solver(avbd_ctx* c, const avbd_solver_params* s) {
    if (int r = check_ctx(c)) return r;
    if (!s) return fail(AVBD_ERR_INVALID_ARG, "null solver params");
    if (s->precision != AVBD_PRECISION_FP32 && s->precision != AVBD_PRECISION_FP64 &&
        s->precision != AVBD_PRECISION_MIXED)
        return fail(AVBD_ERR_INVALID_ARG, "unknown precision");
    if (c->finalized && s->precision != c->solver.precision) free_device(c);
    c->solver = *s;
    c->graph_dirty = true;
    return AVBD_OK;
}

int avbd_begin_scene(avbd_ctx* c, unsigned* scene_index) {
    if (int r = check_ctx(c)) return r;
    staging_only(c);
    unsigned n = (unsigned)c->mass.size();
    if (c->scene_begin.back() != n) c->scene_begin.push_back(n);
    if (scene_index) *scene_index = (unsigned)c->scene_begin.size() - 1;
    return AVBD_OK;
}

int avbd_particles_add(avbd_ctx* c, unsigned n, const double* pos, const double* mass, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (n && (!pos || !mass)) return fail(AVBD_ERR_INVALID_ARG, "null positions/masses");
    if (c->mass.size() + n > c->cap_particles) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    staging_only(c);
    if (first) *first = (unsigned)c->mass.size();
    c->x.insert(c->x.end(), pos, pos + 3ull * n);
    c->v.insert(c->v.end(), 3ull * n, 0.0);
    c->vp.insert(c->vp.end(), 3ull * n, 0.0);
    c->mass.insert(c->mass.end(), mass, mass + n);
    c->fixed.insert(c->fixed.end(), n, 0);
    c->rot.insert(c->rot.end(), n, UINT32_MAX);
    return AVBD_OK;
}

int avbd_particles_add_oriented(avbd_ctx* c, unsigned n, const double* pos, const double* rot, const double* mass,
                                const double* inertia, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (n && (!rot || !inertia)) return fail(AVBD_ERR_INVALID_ARG, "null rotations/inertias");
    unsigned no = (unsigned)c->inertia.size() / 3;
    if (no + n > c->cap_oriented) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    unsigned f0 = 0;
    if (int r = avbd_particles_add(c, n, pos, mass, &f0)) return r;
    for (unsigned i = 0; i < n; i++) c->rot[f0 + i] = no + i;
    c->q.insert(c->q.end(), rot, rot + 4ull * n);
    c->inertia.insert(c->inertia.end(), inertia, inertia + 3ull * n);
    if (first) *first = f0;
    return AVBD_OK;
}

int avbd_particles_set_fixed(avbd_ctx* c, unsigned n, const unsigned* slots, const uint8_t* fixed) {
    if (int r = check_ctx(c)) return r;
    for (unsigned i = 0; i < n; i++)
        if (slots[i] >= c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "particle index out of range");
    staging_only(c);
    for (unsigned i = 0; i < n; i++) c->fixed[slots[i]] = fixed ? fixed[i] : 1;
    return AVBD_OK;
}

int avbd_num_particles(avbd_ctx* c, unsigned* n) {
    if (int r = check_ctx(c)) return r;
    *n = (unsigned)c->mass.size();
    return AVBD_OK;
}

// ------------------------------------------------------------- energies
int avbd_neo_hookean_add(avbd_ctx* c, unsigned n, const unsigned* idx, const double* lam, const double* mu,
                         const double* kd, const double* Q, const double* V, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (c->nh.size() + n > c->cap_energies) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    size_t np = c->mass.size();
    for (size_t i = 0; i < 4ull * n; i++)
        if (idx[i] >= np) return fail(AVBD_ERR_INVALID_ARG, "tet particle index out of range");
    staging_only(c);
    if (first) *first = (unsigned)c->nh.size();
    for (unsigned i = 0; i < n; i++) {
        HostNH e;
        for (int k = 0; k < 4; k++) e.idx[k] = idx[4 * i + k];
        e.lambda = lam[i];
        e.mu = mu[i];
        e.kd = kd[i];
        for (int k = 0; k < 9; k++) e.Q[k] = Q[9 * i + k];
        e.V = V[i];
        c->nh.push_back(e);
    }
    return AVBD_OK;
}

int avbd_ground_collision_add(avbd_ctx* c, unsigned n, const unsigned* p, const double* ks, const double* ms,
                              const double* mk, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (c->ground.size() + n > c->cap_energies) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    for (unsigned i = 0; i < n; i++)
        if (p[i] >= c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "particle index out of range");
    staging_only(c);
    if (first) *first = (unsigned)c->ground.size();
    for (unsigned i = 0; i < n; i++) c->ground.push_back(HostGround{p[i], ks[i], ms[i], mk[i]});
    return AVBD_OK;
}

int avbd_cosserat_rod_add(avbd_ctx* c, unsigned n, const unsigned* idx, const double* K, const double* L,
                          const double* kappa, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (c->rods.size() + n > c->cap_energies) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    for (size_t i = 0; i < 2ull * n; i++)
        if (idx[i] >= c->mass.size() || c->rot[idx[i]] == UINT32_MAX)
            return fail(AVBD_ERR_INVALID_ARG, "rod element needs oriented particles");
    staging_only(c);
    if (first) *first = (unsigned)c->rods.size();
    for (unsigned i = 0; i < n; i++) {
        HostRod e;
        e.idx[0] = idx[2 * i];
        e.idx[1] = idx[2 * i + 1];
        for (int k = 0; k < 6; k++) e.K[k] = K[6 * i + k];
        e.L = L[i];
        for (int k = 0; k < 3; k++) e.kappa[k] = kappa[3 * i + k];
        c->rods.push_back(e);
    }
    return AVBD_OK;
}

int avbd_rigid_body_ground_collision_add(avbd_ctx* c, unsigned n, const unsigned* p, const uint8_t* shape,
                                         const double* radius, const double* cp, const double* ks, const double* ms,
                                         const double* mk, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (c->rground.size() + n > c->cap_energies) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    for (unsigned i = 0; i < n; i++)
        if (p[i] >= c->mass.size() || c->rot[p[i]] == UINT32_MAX)
            return fail(AVBD_ERR_INVALID_ARG, "rigid-body ground contact needs an oriented particle");
    staging_only(c);
    if (first) *first = (unsigned)c->rground.size();
    for (unsigned i = 0; i < n; i++) {
        HostRGround e;
        e.p = p[i];
        e.shape = shape[i];
        e.radius = radius[i];
        for (int k = 0; k < 3; k++) e.cp[k] = cp[3 * i + k];
        e.k_start = ks[i];
        e.mu_s = ms[i];
        e.mu_k = mk[i];
        c->rground.push_back(e);
    }
    return AVBD_OK;
}

int avbd_one_sided_fixed_joint_add(avbd_ctx* c, unsigned n, const unsigned* p, const double* po, const double* ro,
                                   const double* rp, const double* rq, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (c->joints.size() + n > c->cap_energies) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    for (unsigned i = 0; i < n; i++)
        if (p[i] >= c->mass.size() || c->rot[p[i]] == UINT32_MAX)
            return fail(AVBD_ERR_INVALID_ARG, "joint needs an oriented particle");
    staging_only(c);
    if (first) *first = (unsigned)c->joints.size();
    for (unsigned i = 0; i < n; i++) {
        HostJoint e;
        e.p = p[i];
        for (int k = 0; k < 3; k++) { e.po[k] = po[3 * i + k]; e.rp[k] = rp[3 * i + k]; }
        for (int k = 0; k < 4; k++) { e.ro[k] = ro[4 * i + k]; e.rq[k] = rq[4 * i + k]; }
        c->joints.push_back(e);
    }
    return AVBD_OK;
}

static int add_prims(avbd_ctx* c, unsigned n, uint8_t type, const unsigned* idx, int k, const double* radius,
                     double rconst, const unsigned* obj, unsigned objconst, unsigned* first) {
    if (int r = check_ctx(c)) return r;
    if (c->prims.size() + n > c->cap_prims) return fail(AVBD_ERR_CAPACITY, "Pool has exceeded capacity");
    for (size_t i = 0; i < (size_t)k * n; i++)
        if (idx[i] >= c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "primitive particle index out of range");
    staging_only(c);
    if (first) *first = (unsigned)c->prims.size();
    for (unsigned i = 0; i < n; i++) {
        HostPrim p{};
        p.type = type;
        for (int j = 0; j < k; j++) p.idx[j] = idx[k * i + j];
        p.object_id = obj ? obj[i] : objconst;
        p.radius = radius ? radius[i] : rconst;
        c->prims.push_back(p);
    }
    return AVBD_OK;
}

int avbd_collision_add_triangles(avbd_ctx* c, unsigned n, const unsigned* idx, unsigned object_id, unsigned* first) {
    return add_prims(c, n, AVBD_SHAPE_TRIANGLE, idx, 3, nullptr, 0.0, nullptr, object_id, first);
}
int avbd_collision_add_rod_segments(avbd_ctx* c, unsigned n, const unsigned* idx, double radius, unsigned object_id,
                                    unsigned* first) {
    return add_prims(c, n, AVBD_SHAPE_ROD_SEGMENT, idx, 2, nullptr, radius, nullptr, object_id, first);
}
int avbd_collision_add_spheres(avbd_ctx* c, unsigned n, const unsigned* p, const double* radius,
                               const unsigned* object_id, unsigned* first) {
    for (unsigned i = 0; i < n; i++)
        if (p[i] >= c->mass.size() || c->rot[p[i]] == UINT32_MAX)
            return fail(AVBD_ERR_INVALID_ARG, "sphere primitive needs an oriented particle");
    return add_prims(c, n, AVBD_SHAPE_SPHERE, p, 1, radius, 0.0, object_id, 0, first);
}

}  // extern "C"

// ============================================================== finalize

namespace {

// Vertex-vertex adjacency of the static energies (StaticParticleAdjacency::
// buildAdjacency, common/StaticParticleAdjacency.hpp:42-133): the distinct
// other particles of every energy a particle belongs to.
void build_neighbors(avbd_ctx* c, const std::vector<unsigned>& inc_off, const std::vector<uint32_t>& inc_tet,
                     std::vector<unsigned>& p_off, std::vector<unsigned>& p_nbr) {
    const unsigned n = (unsigned)c->mass.size();
    // rod neighbours
    std::vector<std::vector<unsigned>> rodn;
    if (!c->rods.empty()) {
        rodn.resize(n);
        for (auto& e : c->rods) {
            rodn[e.idx[0]].push_back(e.idx[1]);
            rodn[e.idx[1]].push_back(e.idx[0]);
        }
    }
    std::vector<unsigned> deg(n, 0);
    std::vector<std::vector<unsigned>> lists;
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 20000) nt = 1;
    std::vector<std::vector<unsigned>> chunk_nbr(nt);
    std::vector<std::vector<unsigned>> chunk_deg(nt);
    auto work = [&](unsigned t) {
        unsigned b = (unsigned)((uint64_t)n * t / nt), e = (unsigned)((uint64_t)n * (t + 1) / nt);
        std::vector<unsigned> tmp;
        auto& out = chunk_nbr[t];
        auto& dg = chunk_deg[t];
        for (unsigned p = b; p < e; p++) {
            tmp.clear();
            for (unsigned k = inc_off[p]; k < inc_off[p + 1]; k++) {
                const HostNH& h = c->nh[inc_tet[k]];
                for (int j = 0; j < 4; j++)
                    if (h.idx[j] != p) tmp.push_back(h.idx[j]);
            }
            if (!rodn.empty())
                for (unsigned q : rodn[p]) if (q != p) tmp.push_back(q);
            std::sort(tmp.begin(), tmp.end());
            tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
            dg.push_back((unsigned)tmp.size());
            out.insert(out.end(), tmp.begin(), tmp.end());
        }
    };
    if (nt == 1) work(0);
    else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; t++) th.emplace_back(work, t);
        for (auto& t : th) t.join();
    }
    p_off.assign(n + 1, 0);
    size_t total = 0;
    for (unsigned t = 0; t < nt; t++) total += chunk_nbr[t].size();
    p_nbr.clear();
    p_nbr.reserve(total);
    unsigned p = 0;
    for (unsigned t = 0; t < nt; t++) {
        for (unsigned d : chunk_deg[t]) { p_off[p + 1] = p_off[p] + d; p++; }
        p_nbr.insert(p_nbr.end(), chunk_nbr[t].begin(), chunk_nbr[t].end());
    }
}

template <typename R, typename RS>
int upload_state(avbd_ctx* c, DevState<R>& s, const std::vector<unsigned>& inc_off,
                 const std::vector<uint32_t>& inc_tet, const std::vector<uint16_t>& inc_local,
                 const std::vector<int>& ground_of) {
    using V4 = typename Vec4Of<R>::T;
    const unsigned n = (unsigned)c->mass.size();
    s.n = n;
    std::vector<V4> x(n), y(n), v(n), vp(n);
    std::vector<uint8_t> flags(n, 0);
    for (unsigned i = 0; i < n; i++) {
        unsigned e = c->perm[i];
        V3<R> xe = mk3<R>((R)c->x[3 * e], (R)c->x[3 * e + 1], (R)c->x[3 * e + 2]);
        x[i] = make4<R>(xe, R(0));
        y[i] = make4<R>(xe, (R)c->mass[e]);
        v[i] = make4<R>(mk3<R>((R)c->v[3 * e], (R)c->v[3 * e + 1], (R)c->v[3 * e + 2]), R(0));
        vp[i] = make4<R>(mk3<R>((R)c->vp[3 * e], (R)c->vp[3 * e + 1], (R)c->vp[3 * e + 2]), R(0));
        uint8_t f = 0;
        if (c->fixed[e]) f |= VF_FIXED;
        if (c->rot[e] != UINT32_MAX) f |= VF_ORIENTED;
        if (ground_of[e] >= 0) f |= VF_GROUND;
        flags[i] = f;
    }
    // incidence records in internal order; only solved positional vertices get records
    std::vector<uint32_t> begin(n + 1, 0);
    for (unsigned i = 0; i < n; i++) {
        unsigned e = c->perm[i];
        bool solved = !(flags[i] & (VF_FIXED | VF_ORIENTED));
        begin[i + 1] = begin[i] + (solved ? inc_off[e + 1] - inc_off[e] : 0);
    }
    const size_t nrec = begin[n];
    // algorithmic bytes of each color's solve launch, and of each scene's
    // part of it (the pieces a run-to-tolerance sweep launches per scene)
    c->color_bytes.assign(c->num_colors, 0.0);
    {
        const double V4B = sizeof(V4), RECB = sizeof(IncRec<RS>);
        const double ground_b = c->ground.empty() ? 0.0 : 3 * V4B + 1;
        std::vector<unsigned> sb = c->scene_begin;
        if (sb.back() != n) sb.push_back(n);
        const unsigned S = (unsigned)sb.size() - 1;
        c->color_scene_bytes.assign((size_t)c->num_colors * S, 0.0);
        for (unsigned col = 0; col < c->num_colors; col++) {
            double b = 0;
            for (unsigned i = c->color_begin[col]; i < c->color_begin[col] + c->color_solve[col]; i++) {
                double bi = 3 * V4B + 2 * sizeof(uint32_t) + 1 + RECB * (begin[i + 1] - begin[i]);
                if (flags[i] & VF_GROUND) bi += ground_b;
                b += bi;
                const unsigned sc = (unsigned)(std::upper_bound(sb.begin(), sb.end(), c->perm[i]) - sb.begin()) - 1;
                c->color_scene_bytes[(size_t)col * S + sc] += bi;
            }
            c->color_bytes[col] = b;
        }
    }
    std::vector<IncRec<RS>> rec(nrec);
    {
        unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        if (n < 20000) nt = 1;
        auto work = [&](unsigned t) {
            unsigned b = (unsigned)((uint64_t)n * t / nt), en = (unsigned)((uint64_t)n * (t + 1) / nt);
            for (unsigned i = b; i < en; i++) {
                unsigned e = c->perm[i];
                if (begin[i + 1] == begin[i]) continue;
                size_t w = begin[i];
                for (unsigned k = inc_off[e]; k < inc_off[e + 1]; k++, w++) {
                    const HostNH& h = c->nh[inc_tet[k]];
                    unsigned loc = inc_local[k];
                    double D[4][3];
                    for (int j = 0; j < 3; j++) {
                        D[0][j] = h.Q[0 * 3 + j];
                        D[1][j] = h.Q[1 * 3 + j];
                        D[2][j] = h.Q[2 * 3 + j];
                        D[3][j] = -(h.Q[j] + h.Q[3 + j] + h.Q[6 + j]);
                    }
                    IncRec<RS>& r = rec[w];
                    int o = 0;
                    for (int j = 0; j < 4; j++) {
                        if ((unsigned)j == loc) continue;
                        r.o[o] = c->inv[h.idx[j]];
                        r.d[3 * o] = (RS)D[j][0];
                        r.d[3 * o + 1] = (RS)D[j][1];
                        r.d[3 * o + 2] = (RS)D[j][2];
                        o++;
                    }
                    r.tet = inc_tet[k];
                    r.vlam = (RS)(h.V * h.lambda);
                    r.vmu = (RS)(h.V * h.mu);
                    r.mol = (RS)(h.mu / h.lambda);
                }
            }
        };
        if (nt == 1) work(0);
        else {
            std::vector<std::thread> th;
            for (unsigned t = 0; t < nt; t++) th.emplace_back(work, t);
            for (auto& t : th) t.join();
        }
    }
    int rc;
    if ((rc = dalloc(c, &s.x, n)) || (rc = dalloc(c, &s.y, n)) || (rc = dalloc(c, &s.xp, n)) ||
        (rc = dalloc(c, &s.xl, n)) || (rc = dalloc(c, &s.xll, n)) || (rc = dalloc(c, &s.v, n)) ||
        (rc = dalloc(c, &s.vp, n)) || (rc = dalloc(c, &s.flags, n)) || (rc = dalloc(c, &s.inc_begin, n + 1)))
        return rc;
    IncRec<RS>* d_rec = nullptr;
    if ((rc = dalloc(c, &d_rec, nrec))) return rc;
    if constexpr (std::is_same<R, RS>::value) s.inc = d_rec;
    else s.inc32 = d_rec;
    cudaStream_t st = c->stream;
    CUDA_OR_FAIL(cudaMemcpyAsync(s.x, x.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.y, y.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.xp, x.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.xl, x.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.xll, x.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.v, v.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.vp, vp.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.flags, flags.data(), n, cudaMemcpyHostToDevice, st));
    if (nrec) CUDA_OR_FAIL(cudaMemcpyAsync(d_rec, rec.data(), sizeof(IncRec<RS>) * nrec, cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaMemcpyAsync(s.inc_begin, begin.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, st));

    // ground contact, one record per particle (internal order)
    if (!c->ground.empty()) {
        std::vector<V4> gk(n), glam(n), gcp(n);
        std::vector<uint8_t> gfl(n, 0);
        for (unsigned i = 0; i < n; i++) {
            int gi = ground_of[c->perm[i]];
            if (gi < 0) {
                gk[i] = make4<R>(mk3<R>(0, 0, 0), R(0));
                glam[i] = gk[i];
                gcp[i] = gk[i];
                continue;
            }
            const HostGround& g = c->ground[gi];
            gk[i] = make4<R>(mk3<R>((R)g.k_start, (R)g.k_start, (R)g.k_start), (R)g.k_start);
            glam[i] = make4<R>(mk3<R>(0, 0, 0), R(0));
            gcp[i] = make4<R>(mk3<R>(0, 0, (R)g.mu_s), (R)g.mu_k);
        }
        if ((rc = dalloc(c, &s.gk, n)) || (rc = dalloc(c, &s.glam, n)) || (rc = dalloc(c, &s.gcp, n)) ||
            (rc = dalloc(c, &s.gflag, n)))
            return rc;
        CUDA_OR_FAIL(cudaMemcpyAsync(s.gk, gk.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
        CUDA_OR_FAIL(cudaMemcpyAsync(s.glam, glam.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
        CUDA_OR_FAIL(cudaMemcpyAsync(s.gcp, gcp.data(), sizeof(V4) * n, cudaMemcpyHostToDevice, st));
        CUDA_OR_FAIL(cudaMemcpyAsync(s.gflag, gfl.data(), n, cudaMemcpyHostToDevice, st));
    }
    // per-tet data for strain-rate damping
    s.ntets = 0;
    if (c->damping) {
        const unsigned nt = (unsigned)c->nh.size();
        std::vector<uint4> ti(nt);
        std::vector<V4> tq(3ull * nt), te(2ull * nt);
        for (unsigned t = 0; t < nt; t++) {
            const HostNH& h = c->nh[t];
            ti[t] = make_uint4(c->inv[h.idx[0]], c->inv[h.idx[1]], c->inv[h.idx[2]], c->inv[h.idx[3]]);
            for (int r = 0; r < 3; r++)
                tq[3 * t + r] = make4<R>(mk3<R>((R)h.Q[3 * r], (R)h.Q[3 * r + 1], (R)h.Q[3 * r + 2]), R(0));
            te[2 * t] = make4<R>(mk3<R>(0, 0, 0), R(0));
            te[2 * t + 1] = make4<R>(mk3<R>(0, 0, (R)(h.V * h.kd)), R(0));
        }
        if ((rc = dalloc(c, &s.tet_idx, nt)) || (rc = dalloc(c, &s.tet_q, 3ull * nt)) ||
            (rc = dalloc(c, &s.tet_e, 2ull * nt)))
            return rc;
        CUDA_OR_FAIL(cudaMemcpyAsync(s.tet_idx, ti.data(), sizeof(uint4) * nt, cudaMemcpyHostToDevice, st));
        CUDA_OR_FAIL(cudaMemcpyAsync(s.tet_q, tq.data(), sizeof(V4) * 3 * nt, cudaMemcpyHostToDevice, st));
        CUDA_OR_FAIL(cudaMemcpyAsync(s.tet_e, te.data(), sizeof(V4) * 2 * nt, cudaMemcpyHostToDevice, st));
        s.ntets = nt;
    }
    // oriented particles: rotation slots in internal order, rods, rigid-body
    // ground contact and joints (RotationPool::addParticle initial state)
    s.no = 0;
    {
        std::vector<uint32_t> rot(n, UINT32_MAX);
        std::vector<unsigned> ext_slot_of(c->inertia.size() / 3, UINT32_MAX);
        unsigned no = 0;
        for (unsigned i = 0; i < n; i++) {
            unsigned e = c->perm[i];
            if (c->rot[e] != UINT32_MAX) {
                rot[i] = no;
                ext_slot_of[c->rot[e]] = no;
                no++;
            }
        }
        if (no > 0) {
            auto qv = [](const double* q) {
                V4 r;
                r.x = (R)q[0]; r.y = (R)q[1]; r.z = (R)q[2]; r.w = (R)q[3];
                return r;
            };
            std::vector<V4> q(no), Iv(no), zero(no), rgk(no), rglam(no), rgcp(no), rgloc(no);
            std::vector<V4> jk(2ull * no), jlam(2ull * no), jcp(2ull * no), jpo(no), jro(no), jrp(no), jrq(no);
            std::vector<uint8_t> oflag(no, 0);
            V4 z = make4<R>(mk3<R>(0, 0, 0), R(0));
            for (unsigned i = 0; i < n; i++) {
                if (rot[i] == UINT32_MAX) continue;
                unsigned e = c->perm[i], es = c->rot[e], sl = rot[i];
                q[sl] = qv(&c->q[4ull * es]);
                Iv[sl] = make4<R>(mk3<R>((R)c->inertia[3ull * es], (R)c->inertia[3ull * es + 1],
                                         (R)c->inertia[3ull * es + 2]), R(0));
                zero[sl] = z;
                rgk[sl] = rglam[sl] = rgcp[sl] = rgloc[sl] = z;
                jk[2 * sl] = jk[2 * sl + 1] = jlam[2 * sl] = jlam[2 * sl + 1] = jcp[2 * sl] = jcp[2 * sl + 1] = z;
                jpo[sl] = jro[sl] = jrp[sl] = jrq[sl] = z;
            }
            for (auto& g : c->rground) {
                unsigned sl = rot[c->inv[g.p]];
                R ks = (R)g.k_start;
                rgk[sl] = make4<R>(mk3<R>(ks, ks, ks), ks);
                rgcp[sl] = make4<R>(mk3<R>(0, 0, (R)g.mu_s), (R)g.mu_k);
                rgloc[sl] = make4<R>(mk3<R>((R)g.cp[0], (R)g.cp[1], (R)g.cp[2]), (R)g.radius);
                oflag[sl] |= OF_RGROUND | OF_RG_ROUND;
            }
            for (auto& j : c->joints) {
                unsigned sl = rot[c->inv[j.p]];
                V4 k4 = make4<R>(mk3<R>(R(1e4), R(1e4), R(1e4)), R(1e4));
                jk[2 * sl] = k4;
                jk[2 * sl + 1] = make4<R>(mk3<R>(R(1e4), R(1e4), 0), R(0));
                jpo[sl] = make4<R>(mk3<R>((R)j.po[0], (R)j.po[1], (R)j.po[2]), R(0));
                jro[sl] = qv(j.ro);
                jrp[sl] = make4<R>(mk3<R>((R)j.rp[0], (R)j.rp[1], (R)j.rp[2]), R(0));
                jrq[sl] = qv(j.rq);
                oflag[sl] |= OF_JOINT;
            }
            // rods and the per-vertex CSR of their incidences (slot order)
            const unsigned nr = (unsigned)c->rods.size();
            std::vector<uint2> ridx(nr);
            std::vector<V4> rK(2ull * nr), rk0(nr);
            std::vector<uint32_t> rb(n + 1, 0);
            for (unsigned r = 0; r < nr; r++) {
                const HostRod& h = c->rods[r];
                ridx[r] = make_uint2(c->inv[h.idx[0]], c->inv[h.idx[1]]);
                rK[2 * r] = make4<R>(mk3<R>((R)h.K[0], (R)h.K[1], (R)h.K[2]), (R)h.K[3]);
                rK[2 * r + 1] = make4<R>(mk3<R>((R)h.K[4], (R)h.K[5], (R)h.L), R(0));
                rk0[r] = make4<R>(mk3<R>((R)h.kappa[0], (R)h.kappa[1], (R)h.kappa[2]), R(0));
                rb[ridx[r].x + 1]++;
                rb[ridx[r].y + 1]++;
            }
            for (unsigned i = 0; i < n; i++) rb[i + 1] += rb[i];
            std::vector<uint32_t> rinc(std::max(1u, rb[n]));
            {
                std::vector<uint32_t> cr(rb.begin(), rb.end() - 1);
                for (unsigned r = 0; r < nr; r++) {
                    rinc[cr[ridx[r].x]++] = (r << 1) | 0u;
                    rinc[cr[ridx[r].y]++] = (r << 1) | 1u;
                }
            }
            // algorithmic bytes of the 6-DOF solve of each color: own state
            // (x, q, y, qy, inertia; flags, slot, CSR bounds), per rod element
            // its index, record and the other node's x and q, the contact and
            // joint records, and the x and q writes
            {
                const double V4B = sizeof(V4);
                for (unsigned col = 0; col < c->num_colors; col++) {
                    const unsigned b0 = c->color_begin[col] + c->color_solve[col];
                    for (unsigned i = b0; i < b0 + c->color_orient[col]; i++) {
                        if (flags[i] & VF_FIXED) continue;
                        const unsigned sl = rot[i];
                        double b = 7 * V4B + 2 + 3 * sizeof(uint32_t);
                        b += (rb[i + 1] - rb[i]) * (sizeof(uint32_t) + sizeof(uint2) + 5 * V4B);
                        if (oflag[sl] & OF_RGROUND) b += 4 * V4B;
                        if (oflag[sl] & OF_JOINT) b += 10 * V4B;
                        c->color_bytes[col] += b;
                    }
                }
            }
            if ((rc = dalloc(c, &s.rot, n)) || (rc = dalloc(c, &s.q, no)) || (rc = dalloc(c, &s.qy, no)) ||
                (rc = dalloc(c, &s.qp, no)) || (rc = dalloc(c, &s.ql, no)) || (rc = dalloc(c, &s.qll, no)) ||
                (rc = dalloc(c, &s.w, no)) || (rc = dalloc(c, &s.wp, no)) || (rc = dalloc(c, &s.Iv, no)) ||
                (rc = dalloc(c, &s.rgk, no)) || (rc = dalloc(c, &s.rglam, no)) || (rc = dalloc(c, &s.rgcp, no)) ||
                (rc = dalloc(c, &s.rgloc, no)) || (rc = dalloc(c, &s.jk, 2ull * no)) ||
                (rc = dalloc(c, &s.jlam, 2ull * no)) || (rc = dalloc(c, &s.jcp, 2ull * no)) ||
                (rc = dalloc(c, &s.jpo, no)) || (rc = dalloc(c, &s.jro, no)) || (rc = dalloc(c, &s.jrp, no)) ||
                (rc = dalloc(c, &s.jrq, no)) || (rc = dalloc(c, &s.oflag, no)) ||
                (rc = dalloc(c, &s.rod_begin, n + 1)) || (rc = dalloc(c, &s.rod_inc, rinc.size())) ||
                (rc = dalloc(c, &s.rod_idx, std::max(1u, nr))) || (rc = dalloc(c, &s.rod_K, std::max(2u, 2 * nr))) ||
                (rc = dalloc(c, &s.rod_k0, std::max(1u, nr))))
                return rc;
            auto up = [&](void* d, const void* h, size_t bytes) {
                return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st);
            };
            const size_t qb = sizeof(V4) * no;
            CUDA_OR_FAIL(up(s.rot, rot.data(), sizeof(uint32_t) * n));
            CUDA_OR_FAIL(up(s.q, q.data(), qb));
            CUDA_OR_FAIL(up(s.qy, q.data(), qb));
            CUDA_OR_FAIL(up(s.qp, q.data(), qb));
            CUDA_OR_FAIL(up(s.ql, q.data(), qb));
            CUDA_OR_FAIL(up(s.qll, q.data(), qb));
            CUDA_OR_FAIL(up(s.w, zero.data(), qb));
            CUDA_OR_FAIL(up(s.wp, zero.data(), qb));
            CUDA_OR_FAIL(up(s.Iv, Iv.data(), qb));
            CUDA_OR_FAIL(up(s.rgk, rgk.data(), qb));
            CUDA_OR_FAIL(up(s.rglam, rglam.data(), qb));
            CUDA_OR_FAIL(up(s.rgcp, rgcp.data(), qb));
            CUDA_OR_FAIL(up(s.rgloc, rgloc.data(), qb));
            CUDA_OR_FAIL(up(s.jk, jk.data(), 2 * qb));
            CUDA_OR_FAIL(up(s.jlam, jlam.data(), 2 * qb));
            CUDA_OR_FAIL(up(s.jcp, jcp.data(), 2 * qb));
            CUDA_OR_FAIL(up(s.jpo, jpo.data(), qb));
            CUDA_OR_FAIL(up(s.jro, jro.data(), qb));
            CUDA_OR_FAIL(up(s.jrp, jrp.data(), qb));
            CUDA_OR_FAIL(up(s.jrq, jrq.data(), qb));
            CUDA_OR_FAIL(up(s.oflag, oflag.data(), no));
            CUDA_OR_FAIL(up(s.rod_begin, rb.data(), sizeof(uint32_t) * (n + 1)));
            CUDA_OR_FAIL(up(s.rod_inc, rinc.data(), sizeof(uint32_t) * rinc.size()));
            if (nr) {
                CUDA_OR_FAIL(up(s.rod_idx, ridx.data(), sizeof(uint2) * nr));
                CUDA_OR_FAIL(up(s.rod_K, rK.data(), sizeof(V4) * 2 * nr));
                CUDA_OR_FAIL(up(s.rod_k0, rk0.data(), sizeof(V4) * nr));
            }
            s.no = no;
            s.nrods = nr;
            (void)ext_slot_of;
        }
    }
    s.err = c->d_error;
    CUDA_OR_FAIL(cudaStreamSynchronize(st));
    return AVBD_OK;
}

}  // namespace

static int autotune(avbd_ctx* c);

extern "C" int avbd_finalize(avbd_ctx* c) {
    if (int r = check_ctx(c)) return r;
    CUDA_OR_FAIL(cudaSetDevice(c->device));
    free_device(c);
    const unsigned n = (unsigned)c->mass.size();
    if (n == 0) return fail(AVBD_ERR_STATE, "no particles");
    for (auto& g : c->ground)
        if (c->rot[g.p] != UINT32_MAX)
            return fail(AVBD_ERR_UNSUPPORTED, "ground energy on an oriented particle (use rigid-body ground)");
    // a rod segment's contact frame interpolates its nodes' rotations
    // (CollisionDetector::_triangleRod, collision/CollisionDetector.cpp:637-640)
    for (auto& pr : c->prims)
        if (pr.type == AVBD_SHAPE_ROD_SEGMENT && (c->rot[pr.idx[0]] == UINT32_MAX || c->rot[pr.idx[1]] == UINT32_MAX))
            return fail(AVBD_ERR_INVALID_ARG, "rod segment primitive on a positional particle");
    for (auto& g : c->rground)
        if (g.shape != AVBD_SHAPE_SPHERE && g.shape != AVBD_SHAPE_ROD_SEGMENT)
            return fail(AVBD_ERR_UNSUPPORTED, "rigid-body ground contact needs a sphere or rod-segment shape");
    {
        std::vector<uint8_t> seen_rg(n, 0), seen_j(n, 0);
        for (auto& g : c->rground) {
            if (seen_rg[g.p]++) return fail(AVBD_ERR_UNSUPPORTED, "more than one rigid-body ground energy on a particle");
        }
        for (auto& j : c->joints) {
            if (seen_j[j.p]++) return fail(AVBD_ERR_UNSUPPORTED, "more than one joint on a particle");
        }
    }

    // scenes: [scene_begin[s], scene_begin[s+1])
    std::vector<unsigned> sb = c->scene_begin;
    if (sb.back() != n) sb.push_back(n);
    std::vector<unsigned> scene_of(n);
    for (size_t s = 0; s + 1 < sb.size(); s++)
        for (unsigned p = sb[s]; p < sb[s + 1]; p++) scene_of[p] = (unsigned)s;

    // NeoHookean incidences per particle, in pool-slot order
    // (StaticParticleAdjacency::buildAdjacency scatter, common/StaticParticleAdjacency.hpp:100-118)
    std::vector<unsigned> inc_off(n + 1, 0);
    c->damping = false;
    for (auto& h : c->nh) {
        for (int k = 0; k < 4; k++)
            if (c->rot[h.idx[k]] != UINT32_MAX)
                return fail(AVBD_ERR_INVALID_ARG, "NeoHookean energy on an oriented particle");
        for (int k = 0; k < 4; k++) inc_off[h.idx[k] + 1]++;
        if (h.kd != 0) c->damping = true;
        unsigned s0 = scene_of[h.idx[0]];
        for (int k = 1; k < 4; k++)
            if (scene_of[h.idx[k]] != s0) return fail(AVBD_ERR_INVALID_ARG, "energy spans two scenes");
        if (!(h.lambda != 0)) return fail(AVBD_ERR_INVALID_ARG, "NeoHookean lambda must be non-zero");
    }
    for (unsigned p = 0; p < n; p++) inc_off[p + 1] += inc_off[p];
    std::vector<uint32_t> inc_tet(inc_off[n]);
    std::vector<uint16_t> inc_local(inc_off[n]);
    {
        std::vector<unsigned> cur(inc_off.begin(), inc_off.end() - 1);
        for (unsigned t = 0; t < c->nh.size(); t++)
            for (int k = 0; k < 4; k++) {
                unsigned p = c->nh[t].idx[k];
                inc_tet[cur[p]] = t;
                inc_local[cur[p]] = (uint16_t)k;
                cur[p]++;
            }
    }
    std::vector<int> ground_of(n, -1);
    for (unsigned g = 0; g < c->ground.size(); g++) {
        unsigned p = c->ground[g].p;
        if (ground_of[p] >= 0)
            return fail(AVBD_ERR_UNSUPPORTED, "more than one ground energy on a particle");
        ground_of[p] = (int)g;
    }

    // coloring
    std::vector<unsigned> p_off, p_nbr;
    trace("finalize: adjacency");
    build_neighbors(c, inc_off, inc_tet, p_off, p_nbr);
    trace("finalize: dsatur");
    for (unsigned p = 0; p < n; p++)
        if (p_off[p + 1] - p_off[p] > 0xFFFFu) return fail(AVBD_ERR_UNSUPPORTED, "vertex degree above 65535");
    {
        std::string err;
        int rc = gpu_dsatur(p_off, p_nbr, sb, c->color, c->num_colors, c->stream, err);
        if (rc) return fail(rc, err);
    }

    trace("finalize: permutation");
    // color-major permutation: [solved positional | oriented | fixed] per color
    const unsigned nc = c->num_colors;
    std::vector<unsigned> cnt(3ull * nc, 0);
    auto cls = [&](unsigned e) -> int {
        if (c->fixed[e]) return 2;
        if (c->rot[e] != UINT32_MAX) return 1;
        return 0;
    };
    for (unsigned e = 0; e < n; e++) cnt[3ull * c->color[e] + cls(e)]++;
    c->color_begin.assign(nc + 1, 0);
    c->color_solve.assign(nc, 0);
    c->color_orient.assign(nc, 0);
    std::vector<unsigned> cur(3ull * nc);
    unsigned run = 0;
    for (unsigned k = 0; k < nc; k++) {
        c->color_begin[k] = run;
        c->color_solve[k] = cnt[3ull * k];
        c->color_orient[k] = cnt[3ull * k + 1];
        for (int t = 0; t < 3; t++) { cur[3ull * k + t] = run; run += cnt[3ull * k + t]; }
    }
    c->color_begin[nc] = run;
    c->max_color_solve = *std::max_element(c->color_solve.begin(), c->color_solve.end());
    c->perm.assign(n, 0);
    c->inv.assign(n, 0);
    for (unsigned e = 0; e < n; e++) {
        unsigned i = cur[3ull * c->color[e] + cls(e)]++;
        c->perm[i] = e;
    }
    // within a slab: scene by scene (locality of the neighbour gathers), and
    // inside a scene by descending incidence count (threads of a warp then run
    // loops of similar length)
    for (unsigned k = 0; k < nc; k++) {
        auto first = c->perm.begin() + c->color_begin[k];
        std::stable_sort(first, first + c->color_solve[k], [&](unsigned a, unsigned b) {
            if (scene_of[a] != scene_of[b]) return scene_of[a] < scene_of[b];
            return inc_off[a + 1] - inc_off[a] > inc_off[b + 1] - inc_off[b];
        });
    }
    for (unsigned i = 0; i < n; i++) c->inv[c->perm[i]] = i;

    trace("finalize: device buffers");
    // device buffers
    int rc;
    if ((rc = dalloc(c, &c->d_counters, 8)) || (rc = dalloc(c, &c->d_residual, 4)) ||
        (rc = dalloc(c, &c->d_perm, n)) || (rc = dalloc(c, &c->d_inv, n)) || (rc = dalloc(c, &c->d_error, 1)))
        return rc;
    CUDA_OR_FAIL(cudaMemsetAsync(c->d_counters, 0, 8 * sizeof(unsigned long long), c->stream));
    CUDA_OR_FAIL(cudaMemsetAsync(c->d_error, 0, sizeof(int), c->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(c->d_perm, c->perm.data(), sizeof(unsigned) * n, cudaMemcpyHostToDevice, c->stream));
    CUDA_OR_FAIL(cudaMemcpyAsync(c->d_inv, c->inv.data(), sizeof(unsigned) * n, cudaMemcpyHostToDevice, c->stream));
    if (c->solver.precision == AVBD_PRECISION_MIXED)
        rc = upload_state<double, float>(c, c->d, inc_off, inc_tet, inc_local, ground_of);
    else if (use64(c))
        rc = upload_state<double, double>(c, c->d, inc_off, inc_tet, inc_local, ground_of);
    else
        rc = upload_state<float, float>(c, c->f, inc_off, inc_tet, inc_local, ground_of);
    if (rc) return rc;
    // per-scene run-to-tolerance state
    {
        const unsigned S = (unsigned)sb.size() - 1;
        c->num_scenes = S;
        std::vector<uint32_t> sid(n);
        for (unsigned i = 0; i < n; i++) sid[i] = scene_of[c->perm[i]];
        std::vector<double> mg2(S, 0.0);
        for (unsigned e = 0; e < n; e++)
            if (!c->fixed[e]) {
                mg2[scene_of[e]] += c->mass[e] * c->mass[e];  // sum of m^2; g^2 is applied per step
            }
        if ((rc = dalloc(c, &c->d_scene, n)) || (rc = dalloc(c, &c->d_scene_active, S)) ||
            (rc = dalloc(c, &c->d_scene_cand, S)) || (rc = dalloc(c, &c->d_scene_r2, S)) ||
            (rc = dalloc(c, &c->d_scene_ex, S)) || (rc = dalloc(c, &c->d_scene_rin, S)) || (rc = dalloc(c, &c->d_scene_mg2, S)) ||
            (rc = dalloc(c, &c->d_scene_iters, S)) || (rc = dalloc(c, &c->d_tol_count, 1)) ||
            (rc = dalloc(c, &c->d_tol_it, 1)) || (rc = dalloc(c, &c->d_tol_omega, 1)))
            return rc;
        CUDA_OR_FAIL(cudaMemcpyAsync(c->d_scene, sid.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, c->stream));
        // the solved part of each color slab is ordered scene by scene
        std::vector<uint4> ranges;
        for (unsigned k = 0; k < nc; k++) {
            unsigned b = c->color_begin[k];
            const unsigned e = b + c->color_solve[k];
            while (b < e) {
                unsigned q = b;
                while (q < e && sid[q] == sid[b]) q++;
                ranges.push_back(make_uint4(b, q - b, sid[b], 0));
                b = q;
            }
        }
        // pieces of at most solve_chunk vertices for the sweeps (AVBD_SOLVE_CHUNK
        // overrides; 0 launches whole slabs): 256 for the persistent sweep,
        // whose blocks draw pieces by ticket (a finer grain shortens each
        // color's tail at its grid barrier), 512 for one block per piece
        c->solve_chunk = c->persistent ? 256 : 512;
        if (const char* env = getenv("AVBD_SOLVE_CHUNK")) c->solve_chunk = (unsigned)atoi(env);
        c->solve_range_off.assign(nc + 1, 0);
        std::vector<uint4> pieces;
        if (c->solve_chunk) {
            unsigned r = 0;
            for (unsigned k = 0; k < nc; k++) {
                c->solve_range_off[k] = (unsigned)pieces.size();
                for (; r < ranges.size() && ranges[r].x < c->color_begin[k] + c->color_solve[k]; r++)
                    for (unsigned o = 0; o < ranges[r].y; o += c->solve_chunk)
                        pieces.push_back(make_uint4(ranges[r].x + o, std::min(c->solve_chunk, ranges[r].y - o),
                                                    ranges[r].z, 0));
            }
            c->solve_range_off[nc] = (unsigned)pieces.size();
        }
        if (!pieces.empty()) {
            if ((rc = dalloc(c, &c->d_solve_ranges, pieces.size()))) return rc;
            CUDA_OR_FAIL(cudaMemcpyAsync(c->d_solve_ranges, pieces.data(), sizeof(uint4) * pieces.size(),
                                         cudaMemcpyHostToDevice, c->stream));
            if (c->persistent) {
                if ((rc = dalloc(c, &c->d_solve_range_off, nc + 1)) || (rc = dalloc(c, &c->d_sweep_sync, 3)))
                    return rc;
                CUDA_OR_FAIL(cudaMemcpyAsync(c->d_solve_range_off, c->solve_range_off.data(),
                                             sizeof(uint32_t) * (nc + 1), cudaMemcpyHostToDevice, c->stream));
            }
        }
        CUDA_OR_FAIL(cudaMemcpyAsync(c->d_scene_mg2, mg2.data(), sizeof(double) * S, cudaMemcpyHostToDevice, c->stream));
        CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    }
    trace("finalize: lbvh");
    if (!c->prims.empty()) {
        std::string err;
        if (int r2 = lbvh_allocate(c, err)) return fail(r2, err);
        if (c->lbvh.contact_capacity)  // triangles with spheres or rod segments: dynamic contacts
            if (int r2 = dyn_create(c, p_off, p_nbr, err)) return fail(r2, err);
    }
    c->stats.num_colors = nc;
    c->stats.num_scenes = (unsigned)sb.size() - 1;
    trace("finalize: autotune");
    if (int r3 = autotune(c)) return r3;
    c->finalized = true;
    c->graph_dirty = true;
    return AVBD_OK;
}

// ================================================================== step

namespace {

double omega_at(unsigned i, double rho, double prev) {
    // Chebyshev schedule (simulation/VBDSolver.hpp:69-74)
    if (i > 2) return 4 / (4 - rho * rho * prev);
    if (i == 2) return 2 / (2 - rho * rho);
    return 1;
}

// Collision stage and step-start hooks + inertial prediction.  With dynamic
// contacts the collision stage ends on the host (contact pool, recoloring),
// which synchronizes the stream.
template <typename R>
int enqueue_begin(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    if (!c->prims.empty()) lbvh_stage<R>(c, s, st);
    if (c->dyn)
        if (int r = dyn_manage<R>(c, s, k, st)) return r;
    if (c->damping) launch_tet_eprev<R>(c, s, k, st);
    launch_begin_step<R>(c, s, k, st);
    launch_begin_step_rot<R>(c, s, k, st);
    if (c->ws_guess_pending) {  // the caller's initial guess replaces the inertial one, once
        launch_load_positions<R>(s, c->d_ws_guess, c->d_inv, 0, (unsigned)c->mass.size(), 4, st);
        count_launch(c);
        c->ws_guess_pending = false;
    }
    if (c->ws_mode) {
        // learned warm start: features at the inertial guess x0, then either
        // x0 += s MLP(features) or (recording) a copy of x0 for the targets
        launch_features<R>(c, s, k, c->d_ws_feat, c->d_ws_target, st);
        launch_ws_save<R>(c, s, c->d_ws_x0, st);
        if (c->ws_mode == 2) {
            mlp_apply_state<R>(*c->ws_mlp, c->d_ws_feat, s.n, s.x, s.xl, s.xll, s.flags, k.g * k.dt * k.dt,
                               c->ws_kappa, c->d_counters + 4, st);
            count_launch(c);
        }
    }
    return AVBD_OK;
}

// One Gauss-Seidel sweep: per color, the positional (3-DOF) slab then the
// oriented (6-DOF) slab; both are independent sets within the color.
template <typename R>
void enqueue_sweep(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st, const SceneTol& T) {
    if (c->dyn) {  // recolored vertices and conflicts of the dynamic contacts
        const unsigned nc = dyn_num_colors(c);
        for (unsigned col = 0; col < nc; col++) dyn_solve_color<R>(c, s, k, col, st, T);
        return;
    }
    // the persistent sweep covers tet-only contexts (no 6-DOF slabs between the colors)
    if (T.active && c->persistent && s.no == 0 && launch_sweep_persistent<R>(c, s, k, st, T)) return;
    for (unsigned col = 0; col < c->num_colors; col++) {
        if (c->color_solve[col] && T.active && c->d_solve_ranges) {  // run-to-tolerance: per-scene pieces
            const unsigned r0 = c->solve_range_off[col], r1 = c->solve_range_off[col + 1];
            launch_solve_color<R>(c, s, k, 0, 0, st, T, nullptr, c->d_solve_ranges + r0, r1 - r0);
        } else if (c->color_solve[col])
            launch_solve_color<R>(c, s, k, c->color_begin[col], c->color_solve[col], st, T);
        if (c->color_orient[col])
            launch_solve_rod<R>(c, s, k, c->color_begin[col] + c->color_solve[col], c->color_orient[col], st, T, 0,
                                nullptr);
    }
}

template <typename R>
void enqueue_chebyshev(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double omega, unsigned it, cudaStream_t st,
                       const SceneTol& T) {
    launch_chebyshev_dual<R>(c, s, k, omega, it, st, T);
    launch_chebyshev_rot<R>(c, s, k, omega, it, st, T);
    if (c->dyn) launch_contact_after_iter<R>(c, s, st, T);
}

template <typename R>
void enqueue_velocity(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    launch_velocity<R>(c, s, k, st);
    launch_velocity_rot<R>(c, s, k, st);
    if (c->ws_mode) {  // (x_end - x0) / (g h^2): the target, and a feature of the next step
        launch_ws_target<R>(c, s, c->d_ws_x0, 1.0 / (k.g * k.dt * k.dt), c->d_ws_target, st);
        c->ws_recorded = true;
    }
}

// Residual pass over all particles (positional and oriented blocks).
template <typename R>
void enqueue_residual(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double* out2, cudaStream_t st,
                      const SceneTol& T) {
    launch_residual<R>(c, s, k, out2, st, T);
    if (s.no) launch_solve_rod<R>(c, s, k, 0, s.n, st, T, 1, out2);
}

template <typename R>
void enqueue_iteration(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double omega, unsigned it, cudaStream_t st) {
    enqueue_sweep<R>(c, s, k, st, SceneTol());
    enqueue_chebyshev<R>(c, s, k, omega, it, st, SceneTol());
}

template <typename R>
int enqueue_step_fixed(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    if (int r = enqueue_begin<R>(c, s, k, st)) return r;
    double omega = 1;
    for (unsigned i = 0; i < c->solver.solver_iters; i++) {
        omega = omega_at(i, c->solver.iter_acceleration, omega);
        enqueue_iteration<R>(c, s, k, omega, i, st);
    }
    enqueue_velocity<R>(c, s, k, st);
    return AVBD_OK;
}

int ensure_omega_table(avbd_ctx* c, unsigned n, cudaStream_t st);

// A fixed-iteration step with dynamic contacts: the step start runs the
// host contact management (so the step as a whole cannot be one graph), then
// one iteration -- the sweep over the step's colors and contact lists,
// Chebyshev with the contact dual updates, the index advance -- is recorded
// as a graph whose iteration index and Chebyshev weight live in device
// memory, and replayed solver_iters times: the same kernels with the same
// arguments as the host loop's, a few microseconds of host time per
// iteration instead of one launch call per kernel.  The executable graph is
// updated in place while the launch sequence keeps its shape.
template <typename R>
int step_fixed_dyn_graph(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st) {
    if (int r = enqueue_begin<R>(c, s, k, st)) return r;
    const unsigned n = c->solver.solver_iters;
    if (n > 0) {
        if (int r = ensure_omega_table(c, n, st)) return r;
        SceneTol T;
        T.omega = c->d_tol_omega;
        T.it = c->d_tol_it;
        const unsigned long long before = c->stats.kernel_launches;
        cudaGraph_t g = nullptr;
        CUDA_OR_FAIL(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue_sweep<R>(c, s, k, st, SceneTol());
        enqueue_chebyshev<R>(c, s, k, 1.0, 0, st, T);
        launch_iter_next(c, n, st);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        const unsigned long long per_iter = c->stats.kernel_launches - before;
        c->stats.kernel_launches = before;
        if (e != cudaSuccess) return fail(AVBD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        if (c->dyn_graph) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(c->dyn_graph, g, &info) != cudaSuccess) {
                cudaGetLastError();  // a changed shape: instantiated anew below
                cudaGraphExecDestroy(c->dyn_graph);
                c->dyn_graph = nullptr;
            }
        }
        if (!c->dyn_graph) {
            e = cudaGraphInstantiate(&c->dyn_graph, g, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                c->dyn_graph = nullptr;
                return fail(AVBD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            }
        }
        cudaGraphDestroy(g);
        launch_iter_set(c, st);
        for (unsigned i = 0; i < n; i++) CUDA_OR_FAIL(cudaGraphLaunch(c->dyn_graph, st));
        c->stats.kernel_launches += per_iter * n;
    }
    enqueue_velocity<R>(c, s, k, st);
    return AVBD_OK;
}

StepConsts consts(avbd_ctx* c) { return StepConsts{c->params.dt, c->params.g_accel, c->kappa_max}; }

// Picks the threads-per-vertex of the tet solve (1, 2, 4, 8, 16 or 32) by timing one
// sweep of every color slab with each choice on the context's own data.
// Positions are snapshotted and restored, so the state is untouched.
// AVBD_LANES=<n> in the environment forces a choice.
template <typename R>
int autotune_impl(avbd_ctx* c, DevState<R>& s) {
    const char* env = getenv("AVBD_LANES");
    if (env) {
        int l = atoi(env);
        if (l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32) c->lanes = l;
        return AVBD_OK;
    }
    unsigned long long solved = 0;
    for (unsigned v : c->color_solve) solved += v;
    c->lanes = 8;
    if (solved < 50000) return AVBD_OK;
    using V4 = typename Vec4Of<R>::T;
    V4* snap = nullptr;
    CUDA_OR_FAIL(cudaMalloc(&snap, sizeof(V4) * s.n));
    cudaStream_t st = c->stream;
    CUDA_OR_FAIL(cudaMemcpyAsync(snap, s.x, sizeof(V4) * s.n, cudaMemcpyDeviceToDevice, st));
    StepConsts k = consts(c);
    cudaEvent_t a, b;
    CUDA_OR_FAIL(cudaEventCreate(&a));
    CUDA_OR_FAIL(cudaEventCreate(&b));
    const unsigned long long launches0 = c->stats.kernel_launches;
    int best = 8;
    float best_ms = 1e30f;
    for (int l : {1, 2, 4, 8, 16}) {
        c->lanes = l;
        for (int rep = 0; rep < 2; rep++) {  // rep 0 warms up, rep 1 is timed
            if (rep == 1) CUDA_OR_FAIL(cudaEventRecord(a, st));
            for (unsigned col = 0; col < c->num_colors; col++) {
                if (!c->color_solve[col]) continue;
                if (c->solver.residual_tolerance > 0 && c->d_solve_ranges) {  // the launches a step will use
                    const unsigned r0 = c->solve_range_off[col], r1 = c->solve_range_off[col + 1];
                    launch_solve_color<R>(c, s, k, 0, 0, st, SceneTol(), nullptr, c->d_solve_ranges + r0, r1 - r0);
                } else {
                    launch_solve_color<R>(c, s, k, c->color_begin[col], c->color_solve[col], st);
                }
            }
            if (rep == 1) CUDA_OR_FAIL(cudaEventRecord(b, st));
        }
        CUDA_OR_FAIL(cudaEventSynchronize(b));
        float ms = 0;
        CUDA_OR_FAIL(cudaEventElapsedTime(&ms, a, b));
        if (getenv("AVBD_TRACE")) fprintf(stderr, "[avbd] autotune: %d threads per vertex: %.3f ms per sweep\n", l, ms);
        if (ms < best_ms) {
            best_ms = ms;
            best = l;
        }
        CUDA_OR_FAIL(cudaMemcpyAsync(s.x, snap, sizeof(V4) * s.n, cudaMemcpyDeviceToDevice, st));
    }
    CUDA_OR_FAIL(cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long), st));
    CUDA_OR_FAIL(cudaStreamSynchronize(st));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(snap);
    c->lanes = best;
    c->stats.kernel_launches = launches0;
    if (getenv("AVBD_TRACE")) fprintf(stderr, "[avbd] autotune: %d threads per vertex (%.3f ms per sweep)\n", best, best_ms);
    return AVBD_OK;
}

// Chebyshev weights omega(0..n-1) of the context's rho in device memory (for
// the device-driven loops), computed on the host by the recurrence the host
// loop uses; rebuilt only when n grows or rho changes.
int ensure_omega_table(avbd_ctx* c, unsigned n, cudaStream_t st) {
    const double rho = c->solver.iter_acceleration;
    if (c->omega_tab_n >= n && c->omega_tab_rho == rho) return AVBD_OK;
    if (c->omega_tab_n < n) {
        if (c->d_omega_tab) {
            CUDA_OR_FAIL(cudaStreamSynchronize(st));
            cudaFree(c->d_omega_tab);
            c->allocations.erase(std::find(c->allocations.begin(), c->allocations.end(), (void*)c->d_omega_tab));
            c->d_omega_tab = nullptr;
            c->omega_tab_n = 0;
        }
        if (int r = dalloc(c, &c->d_omega_tab, n)) return r;
        c->omega_tab_n = n;
    }
    std::vector<double> tab(c->omega_tab_n);
    double w = 1;
    for (unsigned i = 0; i < c->omega_tab_n; i++) tab[i] = w = omega_at(i, rho, w);
    CUDA_OR_FAIL(cudaMemcpyAsync(c->d_omega_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st));
    CUDA_OR_FAIL(cudaStreamSynchronize(st));
    c->omega_tab_rho = rho;
    return AVBD_OK;
}

// Records the run-to-tolerance step as one CUDA graph: the step start, a
// conditional while node whose body is one iteration (sweep, Chebyshev,
// in-sweep decision, candidates' exact residual, stop decision, loop
// control), then the velocity update.  The iteration index and its Chebyshev
// weight live in device memory, so a step needs no host round trip; the loop
// runs the iterations of the host-driven loop, in the same order, with the
// same weights.
template <typename R>
int build_tol_graph(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st, unsigned max_it, double tol,
                    const SceneTol& solveT, const SceneTol& resT) {
    if (int r = ensure_omega_table(c, max_it, st)) return r;

    SceneTol loopT = solveT;
    loopT.omega = c->d_tol_omega;
    loopT.it = c->d_tol_it;
    const unsigned long long before = c->stats.kernel_launches;
    cudaGraph_t g = nullptr;
    CUDA_OR_FAIL(cudaGraphCreate(&g, 0));
    auto abandon = [&](const char* what, cudaError_t e) {
        cudaGraph_t partial = nullptr;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
            cudaStreamEndCapture(st, &partial);
        cudaGraphDestroy(g);
        c->stats.kernel_launches = before;
        return fail(AVBD_ERR_CUDA, std::string(what) + cudaGetErrorString(e));
    };
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    // step start and the per-scene bookkeeping
    cudaError_t e = cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    enqueue_begin<R>(c, s, k, st);  // no host step without dynamic contacts: cannot fail
    launch_tol_init(c, st);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &ndeps);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    std::vector<cudaGraphNode_t> tail(deps, deps + ndeps);
    e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    // the iteration loop
    cudaGraphConditionalHandle h;
    e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return abandon("conditional handle: ", e);
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t loop;
    e = cudaGraphAddNode(&loop, g, tail.data(), tail.size(), &np);
    if (e != cudaSuccess) return abandon("conditional node: ", e);
    cudaGraph_t body = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    const unsigned long long body0 = c->stats.kernel_launches;
    enqueue_sweep<R>(c, s, k, st, loopT);
    enqueue_chebyshev<R>(c, s, k, 1.0, 0, st, loopT);
    launch_tol_decide_a(c, tol, st);
    enqueue_residual<R>(c, s, k, nullptr, st, resT);
    launch_tol_decide_b(c, tol, max_it, st);
    const unsigned body_launches = (unsigned)(c->stats.kernel_launches - body0);
    launch_tol_loop_next(c, h, max_it, body_launches, st);
    e = cudaStreamEndCapture(st, &body);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    // step end
    e = cudaStreamBeginCaptureToGraph(st, g, &loop, nullptr, 1, mode);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    enqueue_velocity<R>(c, s, k, st);
    e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return abandon("graph capture: ", e);
    e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        c->graph = nullptr;
        c->stats.kernel_launches = before;
        return fail(AVBD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    // launches counted per graph launch on the host; the loop body's are
    // counted on the device by the loop control kernel
    c->launches_per_step = c->stats.kernel_launches - before - body_launches;
    c->stats.kernel_launches = before;
    c->graph_tol = true;
    c->graph_dirty = false;
    return AVBD_OK;
}

template <typename R>
int step_impl(avbd_ctx* c, DevState<R>& s, unsigned n_steps) {
    StepConsts k = consts(c);
    cudaStream_t st = c->stream;
    // a step with dynamic contacts runs host work between its launches: no graph
    bool capturable = c->use_graph && !c->dyn && !c->ws_guess_pending && st != nullptr &&
                            st != cudaStreamLegacy && st != cudaStreamPerThread;
    const bool tol_mode = c->solver.residual_tolerance > 0;
    if (c->graph && (c->graph_dirty || c->graph_tol != tol_mode || !capturable)) {
        cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
    }
    if (tol_mode) {
        // Run-to-tolerance, scene by scene: a scene iterates until its own
        // residual R_s <= tol (or max_iters), exactly as it would alone in a
        // context.  The in-sweep residual the solve accumulates for free marks
        // candidate scenes; only those pay for the exact post-iteration
        // residual that decides the stop.  Converged scenes are skipped by the
        // solve, Chebyshev and dual kernels.  The iteration loop runs on the
        // device (a conditional while node of the step's graph); without a
        // graph, one host read per iteration (the count of scenes still
        // iterating) ends it.
        const unsigned max_it = c->solver.max_iters ? c->solver.max_iters : 1000;
        const double tol = c->solver.residual_tolerance;
        SceneTol solveT{c->d_scene, c->d_scene_active, nullptr, c->d_scene_r2, nullptr};
        SceneTol resT{c->d_scene, nullptr, c->d_scene_cand, nullptr, c->d_scene_ex};
        int gr = AVBD_OK;
        if (capturable && !c->graph) {
            gr = build_tol_graph<R>(c, s, k, st, max_it, tol, solveT, resT);
            if (gr != AVBD_OK && c->persistent) {
                // a graph that cannot hold the cooperative launch: the
                // host-driven loop runs the same kernels from now on
                cudaGetLastError();
                c->use_graph = false;
                capturable = false;
                trace("persistent sweep: step graph not built, host-driven iteration loop");
            } else if (gr != AVBD_OK) {
                return gr;
            }
        }
        if (capturable) {
            for (unsigned t = 0; t < n_steps; t++) {
                CUDA_OR_FAIL(cudaGraphLaunch(c->graph, st));
                c->stats.kernel_launches += c->launches_per_step;
            }
            CUDA_OR_FAIL(cudaGetLastError());
            return AVBD_OK;
        }
        for (unsigned t = 0; t < n_steps; t++) {
            if (int r = enqueue_begin<R>(c, s, k, st)) return r;
            launch_tol_init(c, st);
            double omega = 1;
            for (unsigned it = 0; it < max_it; it++) {
                omega = omega_at(it, c->solver.iter_acceleration, omega);
                enqueue_sweep<R>(c, s, k, st, solveT);
                enqueue_chebyshev<R>(c, s, k, omega, it, st, solveT);
                launch_tol_decide_a(c, tol, st);
                enqueue_residual<R>(c, s, k, nullptr, st, resT);
                launch_tol_decide_b(c, tol, max_it, st);
                int n_active = 0;
                CUDA_OR_FAIL(cudaMemcpyAsync(&n_active, c->d_tol_count, sizeof(int), cudaMemcpyDeviceToHost, st));
                CUDA_OR_FAIL(cudaStreamSynchronize(st));
                if (n_active == 0) break;
            }
            enqueue_velocity<R>(c, s, k, st);
        }
        CUDA_OR_FAIL(cudaGetLastError());
        return AVBD_OK;
    }
    if (capturable && !c->graph) {
        unsigned long long before = c->stats.kernel_launches;
        cudaGraph_t g;
        CUDA_OR_FAIL(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue_step_fixed<R>(c, s, k, st);  // no host step without dynamic contacts: cannot fail
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) return fail(AVBD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(AVBD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        c->launches_per_step = c->stats.kernel_launches - before;
        c->stats.kernel_launches = before;
        c->graph_tol = false;
        c->graph_dirty = false;
    }
    // a step with dynamic contacts replays a one-iteration graph after its
    // host part (where graphs are allowed and the stream can be captured)
    const bool dyn_graph = c->dyn && c->use_graph && !c->ws_guess_pending && st != nullptr &&
                           st != cudaStreamLegacy && st != cudaStreamPerThread;
    for (unsigned t = 0; t < n_steps; t++) {
        if (capturable) {
            CUDA_OR_FAIL(cudaGraphLaunch(c->graph, st));
            c->stats.kernel_launches += c->launches_per_step;
        } else if (dyn_graph) {
            if (int r = step_fixed_dyn_graph<R>(c, s, k, st)) return r;
        } else {
            if (int r = enqueue_step_fixed<R>(c, s, k, st)) return r;
        }
        c->host_iterations += (unsigned long long)c->solver.solver_iters * c->num_scenes;
    }
    CUDA_OR_FAIL(cudaGetLastError());
    return AVBD_OK;
}

}  // namespace

static int autotune(avbd_ctx* c) {
    return use64(c) ? autotune_impl<double>(c, c->d) : autotune_impl<float>(c, c->f);
}

namespace {

int device_error(avbd_ctx* c) {
    int h = 0;
    if (!c->d_error) return AVBD_OK;
    CUDA_OR_FAIL(cudaMemcpyAsync(&h, c->d_error, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    if (h == AVBD_ERR_NAN) return fail(h, "non-finite particle state");
    if (h == AVBD_ERR_UNSUPPORTED_PAIR) return fail(h, "Unsupported collision!");
    if (h == AVBD_ERR_CAPACITY)
        return fail(h, "a device buffer overflowed (candidate pairs, narrow-phase contacts or the traversal stack)");
    if (h == AVBD_ERR_COLORS) return fail(h, "Ran out of colors (more than 256)");
    if (h == AVBD_ERR_BARRIER_TIMEOUT) {
        // the launch gave up as a whole (every block left the kernel); the
        // step's results are invalid, the context stays usable
        CUDA_OR_FAIL(cudaMemsetAsync(c->d_error, 0, sizeof(int), c->stream));
        CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
        return fail(h, "a grid-barrier wait of the persistent sweep gave up");
    }
    if (h) return fail(h, "device-side error");
    if (c->ws_mlp) return mlp_device_error(c->ws_mlp, c->stream);
    return AVBD_OK;
}

}  // namespace

extern "C" {

int avbd_step(avbd_ctx* c, unsigned n_steps) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "avbd_finalize must run before avbd_step");
    CUDA_OR_FAIL(cudaSetDevice(c->device));
    return use64(c) ? step_impl<double>(c, c->d, n_steps) : step_impl<float>(c, c->f, n_steps);
}

int avbd_synchronize(avbd_ctx* c) {
    if (int r = check_ctx(c)) return r;
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return device_error(c);
}

int avbd_collision_stage(avbd_ctx* c) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (c->prims.empty()) return AVBD_OK;
    if (use64(c)) lbvh_stage<double>(c, c->d, c->stream);
    else lbvh_stage<float>(c, c->f, c->stream);
    CUDA_OR_FAIL(cudaGetLastError());
    return avbd_synchronize(c);
}

int avbd_get_stats(avbd_ctx* c, avbd_stats* out) {
    if (int r = check_ctx(c)) return r;
    if (!out) return fail(AVBD_ERR_INVALID_ARG, "null stats");
    unsigned long long loop_launches = 0;  // launched by device-driven iteration loops
    if (c->finalized) {
        unsigned long long h[6] = {0, 0, 0, 0, 0, 0};
        CUDA_OR_FAIL(cudaMemcpyAsync(h, c->d_counters, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        if (c->lbvh.pair_count) {
            uint32_t pc = 0;
            CUDA_OR_FAIL(cudaMemcpyAsync(&pc, c->lbvh.pair_count, sizeof(pc), cudaMemcpyDeviceToHost, c->stream));
            CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
            c->stats.candidate_pairs = pc;
        }
        CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
        c->stats.fp64_fallbacks = h[0];
        c->stats.iterations = c->host_iterations + h[1];
        c->stats.capped_scene_steps = h[3];
        c->stats.warmstart_applied = h[4];
        loop_launches = h[5];
        if (c->solver.residual_tolerance > 0 && h[2]) {
            // largest final per-scene residual of the last step (order-preserving encoding)
            unsigned long long u = h[2];
            u = (u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
            double r;
            std::memcpy(&r, &u, sizeof(r));
            c->stats.last_residual = r;
        }
    }
    *out = c->stats;
    out->kernel_launches += loop_launches;
    return AVBD_OK;
}

// ----------------------------------------------------------- state I/O
static int ensure_h2d(avbd_ctx* c, size_t doubles) {
    if (c->h2d_cap >= doubles) return AVBD_OK;
    if (c->d_h2d) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->d_h2d);
        c->allocations.erase(std::find(c->allocations.begin(), c->allocations.end(), (void*)c->d_h2d));
        c->d_h2d = nullptr;
    }
    if (int r = dalloc(c, &c->d_h2d, doubles)) return r;
    c->h2d_cap = doubles;
    return AVBD_OK;
}

static int load_dev(avbd_ctx* c, const double* src, unsigned first, unsigned n, int mode) {
    size_t nd = mode == 2 ? 6ull * n : 3ull * n;
    if (int r = ensure_h2d(c, nd)) return r;
    if (mode == 2) {
        CUDA_OR_FAIL(cudaMemcpyAsync(c->d_h2d, src, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
        CUDA_OR_FAIL(cudaMemcpyAsync(c->d_h2d + 3ull * n, src + 3ull * n, sizeof(double) * 3 * n,
                                     cudaMemcpyHostToDevice, c->stream));
    } else {
        CUDA_OR_FAIL(cudaMemcpyAsync(c->d_h2d, src, sizeof(double) * nd, cudaMemcpyHostToDevice, c->stream));
    }
    if (use64(c)) launch_load_positions<double>(c->d, c->d_h2d, c->d_inv, first, n, mode, c->stream);
    else launch_load_positions<float>(c->f, c->d_h2d, c->d_inv, first, n, mode, c->stream);
    CUDA_OR_FAIL(cudaGetLastError());
    return AVBD_OK;
}

int avbd_set_positions(avbd_ctx* c, unsigned first, unsigned n, const double* pos) {
    if (int r = check_ctx(c)) return r;
    if ((size_t)first + n > c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "range out of bounds");
    std::copy(pos, pos + 3ull * n, c->x.begin() + 3ull * first);
    if (!c->finalized) return AVBD_OK;
    return load_dev(c, pos, first, n, 1);
}

int avbd_set_velocities(avbd_ctx* c, unsigned first, unsigned n, const double* v, const double* vp) {
    if (int r = check_ctx(c)) return r;
    if ((size_t)first + n > c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "range out of bounds");
    if (!vp) vp = v;
    std::copy(v, v + 3ull * n, c->v.begin() + 3ull * first);
    std::copy(vp, vp + 3ull * n, c->vp.begin() + 3ull * first);
    if (!c->finalized) return AVBD_OK;
    std::vector<double> both(6ull * n);
    std::copy(v, v + 3ull * n, both.begin());
    std::copy(vp, vp + 3ull * n, both.begin() + 3ull * n);
    int r = load_dev(c, both.data(), first, n, 2);
    if (r) return r;
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return AVBD_OK;
}

// Per-step drop-in upload of the host-owned state: positions and velocities
// of all particles (velocities also become the previous velocities' source
// only through the step itself).
int avbd_set_state(avbd_ctx* c, const double* pos, const double* vel) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    unsigned n = (unsigned)c->mass.size();
    if (pos)
        if (int r = load_dev(c, pos, 0, n, 0)) return r;
    if (vel) {
        size_t nd = 3ull * n;
        if (int r = ensure_h2d(c, 2 * nd)) return r;
        (void)nd;
        // velocities only: reuse mode 2 with previous velocities read back unchanged is not needed;
        // the state upload overwrites v and keeps v_prev on the device
        CUDA_OR_FAIL(cudaMemcpyAsync(c->d_h2d, vel, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
        if (use64(c)) launch_load_positions<double>(c->d, c->d_h2d, c->d_inv, 0, n, 3, c->stream);
        else launch_load_positions<float>(c->f, c->d_h2d, c->d_inv, 0, n, 3, c->stream);
        CUDA_OR_FAIL(cudaGetLastError());
    }
    return AVBD_OK;
}

static int get_vec(avbd_ctx* c, int which, unsigned first, unsigned n, double* out) {
    if (int r = check_ctx(c)) return r;
    if ((size_t)first + n > c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "range out of bounds");
    if (!c->finalized) {
        const std::vector<double>& src = which == 0 ? c->x : c->v;
        std::copy(src.begin() + 3ull * first, src.begin() + 3ull * (first + n), out);
        return AVBD_OK;
    }
    if (int r = ensure_h2d(c, 3ull * n)) return r;
    if (use64(c)) launch_store_vec<double>(c->d, which, c->d_h2d, c->d_inv + first, n, c->stream);
    else launch_store_vec<float>(c->f, which, c->d_h2d, c->d_inv + first, n, c->stream);
    CUDA_OR_FAIL(cudaGetLastError());
    CUDA_OR_FAIL(cudaMemcpyAsync(out, c->d_h2d, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return device_error(c);
}

int avbd_get_positions(avbd_ctx* c, unsigned first, unsigned n, double* out) { return get_vec(c, 0, first, n, out); }
int avbd_get_velocities(avbd_ctx* c, unsigned first, unsigned n, double* out) { return get_vec(c, 1, first, n, out); }

// Rotations (which 0, 4 doubles (w,x,y,z) per particle) or angular velocities
// (which 1, 3 doubles) of particles [first, first+n); positional particles
// report the identity / zero.
static int get_rot(avbd_ctx* c, int which, unsigned first, unsigned n, double* out) {
    if (int r = check_ctx(c)) return r;
    if ((size_t)first + n > c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "range out of bounds");
    const unsigned stride = which == 0 ? 4 : 3;
    if (!c->finalized) {
        for (unsigned i = 0; i < n; i++) {
            unsigned e = first + i;
            for (unsigned k = 0; k < stride; k++) out[stride * i + k] = (which == 0 && k == 0) ? 1.0 : 0.0;
            if (which == 0 && c->rot[e] != UINT32_MAX)
                for (int k = 0; k < 4; k++) out[4 * i + k] = c->q[4ull * c->rot[e] + k];
        }
        return AVBD_OK;
    }
    if (int r = ensure_h2d(c, 4ull * n)) return r;
    if (use64(c)) launch_store_rot<double>(c->d, which, c->d_h2d, c->d_inv + first, n, c->stream);
    else launch_store_rot<float>(c->f, which, c->d_h2d, c->d_inv + first, n, c->stream);
    CUDA_OR_FAIL(cudaGetLastError());
    CUDA_OR_FAIL(cudaMemcpyAsync(out, c->d_h2d, sizeof(double) * stride * n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return device_error(c);
}

int avbd_get_rotations(avbd_ctx* c, unsigned first, unsigned n, double* out) { return get_rot(c, 0, first, n, out); }

int avbd_get_angular_velocities(avbd_ctx* c, unsigned first, unsigned n, double* w) {
    return get_rot(c, 1, first, n, w);
}

int avbd_get_coloring(avbd_ctx* c, unsigned* colors, unsigned* num_colors) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    // the recolored colors when the context has dynamic contacts
    if (colors) dyn_coloring(c, colors);
    if (num_colors) *num_colors = dyn_num_colors(c);
    return AVBD_OK;
}

int avbd_debug_block(avbd_ctx* c, unsigned p, double* G, double* H, int* dof) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (p >= c->mass.size()) return fail(AVBD_ERR_INVALID_ARG, "particle index out of range");
    double h[42] = {0};
    double* out = nullptr;
    if (int r = ensure_h2d(c, 42)) return r;
    out = c->d_h2d;
    CUDA_OR_FAIL(cudaMemsetAsync(out, 0, 42 * sizeof(double), c->stream));
    StepConsts k = consts(c);
    const bool oriented = c->rot[p] != UINT32_MAX;
    const unsigned ip = c->inv[p];
    if (oriented) {
        if (use64(c)) launch_solve_rod<double>(c, c->d, k, ip, 1, c->stream, SceneTol(), 2, out);
        else launch_solve_rod<float>(c, c->f, k, ip, 1, c->stream, SceneTol(), 2, out);
    } else {
        if (use64(c)) launch_debug_block<double>(c, c->d, k, ip, out, c->stream);
        else launch_debug_block<float>(c, c->f, k, ip, out, c->stream);
    }
    CUDA_OR_FAIL(cudaGetLastError());
    CUDA_OR_FAIL(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    const int d = oriented ? 6 : 3;
    for (int i = 0; i < d; i++) G[i] = h[i];
    for (int i = 0; i < d * d; i++) H[i] = h[d + i];
    if (dof) *dof = d;
    return AVBD_OK;
}

}  // extern "C"

namespace {

// One run-to-tolerance step with the launches the timed step uses (the
// per-scene pieces of every color slab, converged scenes gated out), driven
// from the host like the graph-less path, with CUDA events around every
// color's sweep launch.  Bytes: the algorithmic bytes of the scenes still
// iterating when each sweep starts.
template <typename R>
int profile_step_impl(avbd_ctx* c, DevState<R>& s, double* solve_ms, double* solve_bytes, unsigned* launches,
                      unsigned* iterations) {
    StepConsts k = consts(c);
    cudaStream_t st = c->stream;
    const unsigned max_it = c->solver.max_iters ? c->solver.max_iters : 1000;
    const double tol = c->solver.residual_tolerance;
    const unsigned S = c->num_scenes, nc = c->num_colors;
    SceneTol solveT{c->d_scene, c->d_scene_active, nullptr, c->d_scene_r2, nullptr};
    SceneTol resT{c->d_scene, nullptr, c->d_scene_cand, nullptr, c->d_scene_ex};
    std::vector<uint8_t> act(S);
    std::vector<cudaEvent_t> ev(2ull * nc);
    for (auto& e : ev) CUDA_OR_FAIL(cudaEventCreate(&e));
    double ms = 0, bytes = 0;
    unsigned nl = 0, it = 0;
    int rc = enqueue_begin<R>(c, s, k, st);
    if (!rc) launch_tol_init(c, st);
    double omega = 1;
    for (; !rc && it < max_it; it++) {
        omega = omega_at(it, c->solver.iter_acceleration, omega);
        if (cudaMemcpyAsync(act.data(), c->d_scene_active, S, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = fail(AVBD_ERR_CUDA, "profile: scene flags");
            break;
        }
        // the persistent sweep: one launch (and its 12-byte sync reset) timed
        // for all colors
        bool persist = false;
        if (c->persistent && s.no == 0) {
            cudaEventRecord(ev[0], st);
            persist = launch_sweep_persistent<R>(c, s, k, st, solveT);
            cudaEventRecord(ev[1], st);
        }
        for (unsigned col = 0; col < nc; col++) {
            if (!persist) cudaEventRecord(ev[2 * col], st);
            if (c->color_solve[col]) {
                if (!persist) {
                    const unsigned r0 = c->solve_range_off[col], r1 = c->solve_range_off[col + 1];
                    launch_solve_color<R>(c, s, k, 0, 0, st, solveT, nullptr, c->d_solve_ranges + r0, r1 - r0);
                    nl++;
                }
                for (unsigned sc = 0; sc < S; sc++)
                    if (act[sc]) bytes += c->color_scene_bytes[(size_t)col * S + sc];
            }
            if (!persist) cudaEventRecord(ev[2 * col + 1], st);
            if (c->color_orient[col])
                launch_solve_rod<R>(c, s, k, c->color_begin[col] + c->color_solve[col], c->color_orient[col], st,
                                    solveT, 0, nullptr);
        }
        if (persist) nl++;
        enqueue_chebyshev<R>(c, s, k, omega, it, st, solveT);
        launch_tol_decide_a(c, tol, st);
        enqueue_residual<R>(c, s, k, nullptr, st, resT);
        launch_tol_decide_b(c, tol, max_it, st);
        int n_active = 0;
        if (cudaMemcpyAsync(&n_active, c->d_tol_count, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = fail(AVBD_ERR_CUDA, "profile: iteration count");
            break;
        }
        for (unsigned col = 0; col < (persist ? 1u : nc); col++) {
            float t = 0;
            if (cudaEventElapsedTime(&t, ev[2 * col], ev[2 * col + 1]) == cudaSuccess) ms += t;
        }
        if (n_active == 0) {
            it++;
            break;
        }
    }
    if (!rc) enqueue_velocity<R>(c, s, k, st);
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    CUDA_OR_FAIL(cudaGetLastError());
    CUDA_OR_FAIL(cudaStreamSynchronize(st));
    if (solve_ms) *solve_ms = ms;
    if (solve_bytes) *solve_bytes = bytes;
    if (launches) *launches = nl;
    if (iterations) *iterations = it;
    return AVBD_OK;
}

}  // namespace

extern "C" {

int avbd_profile_step(avbd_ctx* c, double* solve_ms, double* solve_bytes, unsigned* launches,
                      unsigned* iterations) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (c->solver.residual_tolerance <= 0 || !c->d_solve_ranges || c->dyn)
        return fail(AVBD_ERR_STATE, "avbd_profile_step profiles run-to-tolerance steps of contexts without dynamic "
                                    "contacts");
    CUDA_OR_FAIL(cudaSetDevice(c->device));
    int rc = use64(c) ? profile_step_impl<double>(c, c->d, solve_ms, solve_bytes, launches, iterations)
                      : profile_step_impl<float>(c, c->f, solve_ms, solve_bytes, launches, iterations);
    if (rc) return rc;
    return device_error(c);
}

int avbd_profile_solve(avbd_ctx* c, unsigned iterations, double* solve_ms, double* solve_bytes,
                       unsigned* launches) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    StepConsts k = consts(c);
    const unsigned nc = c->num_colors;
    std::vector<cudaEvent_t> ev(2ull * nc * iterations);
    for (auto& e : ev) CUDA_OR_FAIL(cudaEventCreate(&e));
    double bytes = 0;
    unsigned nl = 0;
    double omega = 1;
    for (unsigned it = 0; it < iterations; it++) {
        omega = omega_at(it, c->solver.iter_acceleration, omega);
        for (unsigned col = 0; col < nc; col++) {
            cudaEvent_t a = ev[2ull * (it * nc + col)], b = ev[2ull * (it * nc + col) + 1];
            CUDA_OR_FAIL(cudaEventRecord(a, c->stream));
            if (c->color_solve[col]) {
                if (use64(c)) launch_solve_color<double>(c, c->d, k, c->color_begin[col], c->color_solve[col], c->stream);
                else launch_solve_color<float>(c, c->f, k, c->color_begin[col], c->color_solve[col], c->stream);
                nl++;
            }
            if (c->color_orient[col]) {
                unsigned b0 = c->color_begin[col] + c->color_solve[col];
                if (use64(c)) launch_solve_rod<double>(c, c->d, k, b0, c->color_orient[col], c->stream, SceneTol(), 0, nullptr);
                else launch_solve_rod<float>(c, c->f, k, b0, c->color_orient[col], c->stream, SceneTol(), 0, nullptr);
                nl++;
            }
            bytes += c->color_bytes[col];
            CUDA_OR_FAIL(cudaEventRecord(b, c->stream));
        }
        if (use64(c)) enqueue_chebyshev<double>(c, c->d, k, omega, it, c->stream, SceneTol());
        else enqueue_chebyshev<float>(c, c->f, k, omega, it, c->stream, SceneTol());
    }
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    double ms = 0;
    for (size_t i = 0; i < ev.size(); i += 2) {
        float t = 0;
        CUDA_OR_FAIL(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
        ms += t;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (solve_ms) *solve_ms = ms;
    if (solve_bytes) *solve_bytes = bytes;
    if (launches) *launches = nl;
    return device_error(c);
}

}  // extern "C"

namespace {

// The narrow phase's detections of one DetectedCollisionType (2
// triangle-sphere, 3 triangle-rod) in ascending key order.
struct Detections {
    std::vector<uint64_t> key;
    std::vector<uint4> idx;
    std::vector<uint32_t> idx5;
    std::vector<double> vec;   // 10 per detection
};

int read_detections(avbd_ctx* c, unsigned type, Detections& out) {
    const LbvhState& L = c->lbvh;
    if (!L.contact_capacity) return AVBD_OK;
    uint32_t n = 0;
    CUDA_OR_FAIL(cudaMemcpyAsync(&n, L.contact_count, sizeof(n), cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    if (n > L.contact_capacity) return fail(AVBD_ERR_CAPACITY, "more contacts than the contact buffer holds");
    std::vector<uint64_t> k(n);
    std::vector<uint4> ix(n);
    std::vector<uint32_t> ix5(n);
    std::vector<double> v(10ull * n);
    if (n) {
        CUDA_OR_FAIL(cudaMemcpyAsync(k.data(), L.contact_key, 8ull * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_OR_FAIL(cudaMemcpyAsync(ix.data(), L.contact_idx, 16ull * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_OR_FAIL(cudaMemcpyAsync(ix5.data(), L.contact_idx5, 4ull * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_OR_FAIL(cudaMemcpyAsync(v.data(), L.contact_vec, 80ull * n, cudaMemcpyDeviceToHost, c->stream));
        CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    }
    // ascending key, as CollisionDetector::_handleDetectedCollisions orders them
    std::vector<uint32_t> ord;
    for (uint32_t j = 0; j < n; j++)
        if ((k[j] >> 59) == type) ord.push_back(j);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return k[a] < k[b]; });
    for (uint32_t o : ord) {
        out.key.push_back(k[o]);
        out.idx.push_back(make_uint4(c->perm[ix[o].x], c->perm[ix[o].y], c->perm[ix[o].z], c->perm[ix[o].w]));
        out.idx5.push_back(type == 3 ? c->perm[ix5[o]] : 0u);
        out.vec.insert(out.vec.end(), v.begin() + 10ull * o, v.begin() + 10ull * o + 10);
    }
    return AVBD_OK;
}

}  // namespace

extern "C" {

int avbd_get_contacts(avbd_ctx* c, unsigned capacity, uint64_t* keys, unsigned* idx4, double* vec9,
                      unsigned* count) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (!count) return fail(AVBD_ERR_INVALID_ARG, "null count");
    *count = 0;
    Detections D;
    if (int r = read_detections(c, 2, D)) return r;
    *count = (unsigned)D.key.size();
    for (size_t j = 0; j < D.key.size() && j < capacity; j++) {
        if (keys) keys[j] = D.key[j];
        if (idx4) {
            idx4[4 * j] = D.idx[j].x;
            idx4[4 * j + 1] = D.idx[j].y;
            idx4[4 * j + 2] = D.idx[j].z;
            idx4[4 * j + 3] = D.idx[j].w;
        }
        if (vec9) std::copy(D.vec.begin() + 10 * j, D.vec.begin() + 10 * j + 9, vec9 + 9 * j);
    }
    return device_error(c);
}

int avbd_get_rod_contacts(avbd_ctx* c, unsigned capacity, uint64_t* keys, unsigned* idx5, double* vec10,
                          unsigned* count) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (!count) return fail(AVBD_ERR_INVALID_ARG, "null count");
    *count = 0;
    Detections D;
    if (int r = read_detections(c, 3, D)) return r;
    *count = (unsigned)D.key.size();
    for (size_t j = 0; j < D.key.size() && j < capacity; j++) {
        if (keys) keys[j] = D.key[j];
        if (idx5) {
            idx5[5 * j] = D.idx[j].x;
            idx5[5 * j + 1] = D.idx[j].y;
            idx5[5 * j + 2] = D.idx[j].z;
            idx5[5 * j + 3] = D.idx[j].w;
            idx5[5 * j + 4] = D.idx5[j];
        }
        if (vec10) std::copy(D.vec.begin() + 10 * j, D.vec.begin() + 10 * j + 10, vec10 + 10 * j);
    }
    return device_error(c);
}

int avbd_set_warmstart(avbd_ctx* c, int mode, const float* params) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (mode < 0 || mode > 2) return fail(AVBD_ERR_INVALID_ARG, "warm-start mode must be 0, 1 or 2");
    if (mode == 2 && !params) return fail(AVBD_ERR_INVALID_ARG, "mode 2 needs the MLP parameters");
    if (mode == 2 && !(c->params.g_accel > 0)) return fail(AVBD_ERR_UNSUPPORTED, "the warm start needs g > 0");
    const size_t n = c->mass.size();
    if (mode && !c->d_ws_feat) {
        const size_t v4 = use64(c) ? sizeof(double4a) : sizeof(float4);
        uint8_t *f = nullptr, *x0 = nullptr;
        float4* t = nullptr;
        if (int rc = dalloc(c, &f, 64 * n)) return rc;
        if (int rc = dalloc(c, &x0, v4 * n)) return rc;
        if (int rc = dalloc(c, &t, n)) return rc;
        CUDA_OR_FAIL(cudaMemsetAsync(f, 0, 64 * n, c->stream));
        CUDA_OR_FAIL(cudaMemsetAsync(t, 0, sizeof(float4) * n, c->stream));
        c->d_ws_feat = f;
        c->d_ws_x0 = x0;
        c->d_ws_target = reinterpret_cast<float*>(t);
    }
    if (mode == 2)
        if (int rc = mlp_device_upload(&c->ws_mlp, c->device, params, c->stream)) return rc;
    // AVBD_WS_KAPPA overrides the relative error assumed by the acceptance test
    if (const char* kap = getenv("AVBD_WS_KAPPA")) c->ws_kappa = (float)atof(kap);
    c->ws_mode = mode;
    c->ws_recorded = false;
    c->graph_dirty = true;
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return AVBD_OK;
}

int avbd_set_initial_guess(avbd_ctx* c, const double* positions) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (!positions) {
        c->ws_guess_pending = false;
        return AVBD_OK;
    }
    const size_t n = c->mass.size();
    if (!c->d_ws_guess)
        if (int rc = dalloc(c, &c->d_ws_guess, 3 * n)) return rc;
    CUDA_OR_FAIL(cudaMemcpyAsync(c->d_ws_guess, positions, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    c->ws_guess_pending = true;
    return AVBD_OK;
}

int avbd_warmstart_sample(avbd_ctx* c, void* features, float* targets, unsigned* rows) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    if (rows) *rows = (unsigned)c->mass.size();
    if (!features && !targets) return AVBD_OK;
    if (!c->ws_recorded) return fail(AVBD_ERR_STATE, "no recorded step (set warm-start mode 1 and step)");
    const size_t n = c->mass.size();
    if (features)
        CUDA_OR_FAIL(cudaMemcpyAsync(features, c->d_ws_feat, 64 * n, cudaMemcpyDeviceToDevice, c->stream));
    if (targets)
        CUDA_OR_FAIL(cudaMemcpyAsync(targets, c->d_ws_target, 16 * n, cudaMemcpyDeviceToDevice, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return device_error(c);
}

int avbd_get_scene_iterations(avbd_ctx* c, unsigned* iterations) {
    if (int r = check_ctx(c)) return r;
    if (!iterations) return fail(AVBD_ERR_INVALID_ARG, "null output");
    if (!c->finalized || !c->d_scene_iters) return fail(AVBD_ERR_STATE, "no run-to-tolerance step has run");
    CUDA_OR_FAIL(cudaMemcpyAsync(iterations, c->d_scene_iters, sizeof(uint32_t) * c->num_scenes,
                                 cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    return AVBD_OK;
}

int avbd_residual(avbd_ctx* c, double* residual) {
    if (int r = check_ctx(c)) return r;
    if (!c->finalized) return fail(AVBD_ERR_STATE, "finalize first");
    StepConsts k = consts(c);
    if (use64(c)) enqueue_residual<double>(c, c->d, k, c->d_residual, c->stream, SceneTol());
    else enqueue_residual<float>(c, c->f, k, c->d_residual, c->stream, SceneTol());
    double h[2];
    CUDA_OR_FAIL(cudaMemcpyAsync(h, c->d_residual, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUDA_OR_FAIL(cudaStreamSynchronize(c->stream));
    *residual = h[1] > 0 ? std::sqrt(h[0]) / std::sqrt(h[1]) : std::sqrt(h[0]);
    return AVBD_OK;
}

}  // extern "C"
