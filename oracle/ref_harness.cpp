// TEST INFRASTRUCTURE: a C-ABI driver of the reference implementation itself.
//
// Compiled by oracle/Makefile (target _ref/libavbd_ref.so) from the
// reference's unmodified sources -- simulation/VBDSolver.hpp,
// simulation/SimulationExecutor.hpp, energy/**, common/*.hpp,
// collision/{CollisionDetector,LBVHBuilder,LBVH}.cpp -- with the project's
// Eigen-API shim (oracle/eigen_shim) standing in for Eigen.  It builds a
// Sim::SimulationContext directly, as Simulation::setup does
// (simulation/Simulation.cpp:50-91), filling the pools through their own
// addEnergy / addParticle methods, and steps it with
// Sim::SimulationExecutor::timeStep() (simulation/SimulationExecutor.hpp:
// 107-115).  Only tests/ (to pin the FP64 restatement in oracle/avbd_oracle.cpp
// to the reference) and the CPU legs of bench.py load it.
//
// The argument layouts match the restatement's orc_* entry points, so one
// Python scene description feeds both: quaternions (w, x, y, z), Q row-major,
// Cosserat stiffness (6), joint offsets and references per joint.
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <streambuf>

#include "simulation/SimulationContext.hpp"
#include "simulation/SimulationExecutor.hpp"
#include "collision/LBVHTraversal.hpp"

namespace {

thread_local std::string g_err;

// discards what the reference prints while it steps (the joint solver prints
// every constraint evaluation, OneSidedFixedJointEnergySolver.hpp:33,58)
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
    std::streamsize xsputn(const char*, std::streamsize n) override { return n; }
};

// std::cout is one object per process: contexts stepping on several threads
// share one muted period (the first to enter swaps the buffer, the last to
// leave restores it).
struct MuteCout {
    static std::mutex& mu() {
        static std::mutex m;
        return m;
    }
    static NullBuf nb;
    static int depth;
    static std::streambuf* old;
    MuteCout() {
        std::lock_guard<std::mutex> g(mu());
        if (depth++ == 0) old = std::cout.rdbuf(&nb);
    }
    ~MuteCout() {
        std::lock_guard<std::mutex> g(mu());
        if (--depth == 0) std::cout.rdbuf(old);
    }
};
NullBuf MuteCout::nb;
int MuteCout::depth = 0;
std::streambuf* MuteCout::old = nullptr;

struct Ref {
    std::unique_ptr<Sim::SimulationContext> ctx;
    std::unique_ptr<Sim::SimulationExecutor> exec;
    unsigned iters = 10;
    double rho = 0.5;
    unsigned threads = 1;
    bool finalized = false;
    std::vector<std::pair<unsigned, unsigned>> pairs;
};

Quaternion quat(const double* q) { return Quaternion(q[0], q[1], q[2], q[3]); }
Vec3r v3(const double* p) { return Vec3r(p[0], p[1], p[2]); }

#define REF_TRY(body)                          \
    try {                                      \
        body;                                  \
        return 0;                              \
    } catch (const std::exception& e) {        \
        g_err = e.what();                      \
        return 1;                              \
    }

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// SimulationContext(particles, oriented, energies, primitives, sdf)
// (simulation/SimulationContext.hpp:46-59); `threads` worker threads for the
// executor (all contexts of a process must use the same count: the
// reference keeps it in a process-wide static, WorkerThreadContext.hpp:15).
void* ref_create(unsigned particles, unsigned oriented, unsigned energies, unsigned prims, unsigned sdf,
                 unsigned threads) {
    Ref* r = new Ref();
    r->ctx = std::make_unique<Sim::SimulationContext>(std::max(particles, 1u), std::max(oriented, 1u),
                                                      std::max(energies, 1u), std::max(prims, 1u),
                                                      std::max(sdf, 1u));
    r->ctx->params.dt = 1.0 / 60.0;
    r->ctx->params.end_time = 1e9;
    r->ctx->params.g_accel = 9.81;
    r->ctx->params.viewer_refresh_time_ms = 1000.0 / 30.0;
    r->ctx->params.collision_margin = 1e-3;
    r->threads = std::max(threads, 1u);
    return r;
}

void ref_destroy(void* h) { delete (Ref*)h; }

void ref_set_params(void* h, double dt, double g, double margin) {
    Ref& r = *(Ref*)h;
    r.ctx->params.dt = dt;
    r.ctx->params.g_accel = g;
    r.ctx->params.collision_margin = margin;
}

void ref_set_solver(void* h, unsigned iters, double rho) {
    Ref& r = *(Ref*)h;
    r.iters = iters;
    r.rho = rho;
}

unsigned ref_particles_add(void* h, unsigned n, const double* pos, const double* mass) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned s = r.ctx->particles.addParticle(v3(pos + 3 * i), mass[i]);
        if (i == 0) first = s;
    }
    return first;
}

unsigned ref_particles_add_oriented(void* h, unsigned n, const double* pos, const double* q, const double* mass,
                                    const double* inertia) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned s = r.ctx->particles.addOrientedParticle(v3(pos + 3 * i), quat(q + 4 * i), mass[i],
                                                          v3(inertia + 3 * i));
        if (i == 0) first = s;
    }
    return first;
}

void ref_set_fixed(void* h, unsigned n, const unsigned* idx, const uint8_t* f) {
    Ref& r = *(Ref*)h;
    for (unsigned i = 0; i < n; i++) r.ctx->particles.fixed[idx[i]] = f[i];
}

void ref_set_velocities(void* h, unsigned first, unsigned n, const double* v, const double* vp) {
    Ref& r = *(Ref*)h;
    for (unsigned i = 0; i < n; i++) {
        r.ctx->particles.velocities[first + i] = v3(v + 3 * i);
        r.ctx->particles.previous_velocities[first + i] = v3((vp ? vp : v) + 3 * i);
    }
}

void ref_set_angular_velocities(void* h, unsigned first, unsigned n, const double* w) {
    Ref& r = *(Ref*)h;
    for (unsigned i = 0; i < n; i++)
        if (r.ctx->particles.isOriented(first + i)) r.ctx->particles.angularVelocity(first + i) = v3(w + 3 * i);
}

unsigned ref_neo_hookean_add(void* h, unsigned n, const unsigned* idx, const double* lam, const double* mu,
                             const double* kd, const double* Q, const double* V) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        Mat3r q;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) q(a, b) = Q[9 * i + 3 * a + b];
        Vec4u id(idx[4 * i], idx[4 * i + 1], idx[4 * i + 2], idx[4 * i + 3]);
        unsigned s = r.ctx->energies.neo_hookean.addEnergy(id, lam[i], mu[i], kd[i], q, V[i]);
        if (i == 0) first = s;
    }
    return first;
}

unsigned ref_cosserat_rod_add(void* h, unsigned n, const unsigned* idx, const double* K, const double* L,
                              const double* kappa) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        Vec6r k;
        for (int a = 0; a < 6; a++) k(a) = K[6 * i + a];
        unsigned s = r.ctx->energies.cosserat_rod.addEnergy(Vec2u(idx[2 * i], idx[2 * i + 1]), k, L[i],
                                                            v3(kappa + 3 * i));
        if (i == 0) first = s;
    }
    return first;
}

unsigned ref_ground_add(void* h, unsigned n, const unsigned* p, const double* ks, const double* ms,
                        const double* mk) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned s = r.ctx->energies.ground_collision.addEnergy(p[i], ks[i], ms[i], mk[i]);
        if (i == 0) first = s;
    }
    return first;
}

// shape: 0 triangle (unused), 1 rod segment, 2 sphere (CollisionGeometryType)
unsigned ref_rigid_ground_add(void* h, unsigned n, const unsigned* p, const uint8_t* shape, const double* radius,
                              const double* cpl, const double* ks, const double* ms, const double* mk) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        Collision::CollisionShapeParams sp{};
        sp.type = static_cast<Collision::CollisionGeometryType>(shape[i]);
        if (sp.type == Collision::CollisionGeometryType::Sphere) sp.sphere.radius = radius[i];
        else sp.rod.radius = radius[i];
        unsigned s = r.ctx->energies.rigid_body_ground_collision.addEnergy(p[i], sp, v3(cpl + 3 * i), ks[i], ms[i],
                                                                           mk[i]);
        if (i == 0) first = s;
    }
    return first;
}

unsigned ref_joint_add(void* h, unsigned n, const unsigned* p, const double* po, const double* ro,
                       const double* rp, const double* rq) {
    Ref& r = *(Ref*)h;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned s = r.ctx->energies.one_sided_fixed_joint.addEnergy(p[i], v3(po + 3 * i), quat(ro + 4 * i),
                                                                     v3(rp + 3 * i), quat(rq + 4 * i));
        if (i == 0) first = s;
    }
    return first;
}

// Collision primitives filled as CollisionPrimitivePool::addObject does
// (collision/CollisionPrimitivePool.cpp:38-88), one call per primitive list.
unsigned ref_add_triangles(void* h, unsigned n, const unsigned* idx, unsigned obj) {
    auto& cp = ((Ref*)h)->ctx->collision_pool;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned slot = cp.allocSlot();
        if (i == 0) first = slot;
        cp.type[slot] = Collision::CollisionGeometryType::Triangle;
        for (int k = 0; k < 3; k++) cp.particle_indices[slot][k] = idx[3 * i + k];
        cp.num_particles[slot] = 3;
        cp.object_id[slot] = obj;
    }
    return first;
}

unsigned ref_add_rod_segments(void* h, unsigned n, const unsigned* idx, double radius, unsigned obj) {
    auto& cp = ((Ref*)h)->ctx->collision_pool;
    unsigned ps = cp.shape_params_pool.allocSlot();
    cp.shape_params_pool.shape_params[ps].type = Collision::CollisionGeometryType::RodSegment;
    cp.shape_params_pool.shape_params[ps].rod.radius = radius;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned slot = cp.allocSlot();
        if (i == 0) first = slot;
        cp.type[slot] = Collision::CollisionGeometryType::RodSegment;
        cp.particle_indices[slot][0] = idx[2 * i];
        cp.particle_indices[slot][1] = idx[2 * i + 1];
        cp.particle_indices[slot][2] = ps;
        cp.num_particles[slot] = 2;
        cp.object_id[slot] = obj;
    }
    return first;
}

unsigned ref_add_spheres(void* h, unsigned n, const unsigned* p, const double* radius, const unsigned* obj) {
    auto& cp = ((Ref*)h)->ctx->collision_pool;
    unsigned first = 0;
    for (unsigned i = 0; i < n; i++) {
        unsigned ps = cp.shape_params_pool.allocSlot();
        cp.shape_params_pool.shape_params[ps].type = Collision::CollisionGeometryType::Sphere;
        cp.shape_params_pool.shape_params[ps].sphere.radius = radius[i];
        unsigned slot = cp.allocSlot();
        if (i == 0) first = slot;
        cp.type[slot] = Collision::CollisionGeometryType::Sphere;
        cp.particle_indices[slot][0] = p[i];
        cp.particle_indices[slot][1] = ps;
        cp.num_particles[slot] = 1;
        cp.object_id[slot] = obj[i];
    }
    return first;
}

// Simulation::setup's last three calls (simulation/Simulation.cpp:86-89),
// then the executor with its worker threads.
int ref_finalize(void* h) {
    Ref& r = *(Ref*)h;
    REF_TRY({
        auto& c = *r.ctx;
        c.static_adjacency.buildAdjacency(c.particles, c.energies);
        c.dynamic_adjacency.buildAdjacency(c.particles, c.energies);
        c.coloring.buildInitialColorList(c.static_adjacency, c.dynamic_adjacency, c.particles.totalSize());
        r.exec = std::make_unique<Sim::SimulationExecutor>(r.ctx.get(), r.iters, r.rho, r.threads);
        r.finalized = true;
    });
}

// The iteration count of the following steps.  VBDSolver takes it at
// construction (simulation/VBDSolver.hpp:37-42), so the executor is built
// again; its collision detector then starts without the previous step's
// detections, which matters only to scenes with dynamic contacts.
int ref_set_iterations(void* h, unsigned iters) {
    Ref& r = *(Ref*)h;
    if (!r.finalized) {
        g_err = "finalize first";
        return 1;
    }
    if (iters == r.iters) return 0;
    REF_TRY({
        r.iters = iters;
        r.exec.reset();
        r.exec = std::make_unique<Sim::SimulationExecutor>(r.ctx.get(), r.iters, r.rho, r.threads);
    });
}

int ref_step(void* h, unsigned n) {
    Ref& r = *(Ref*)h;
    if (!r.finalized) {
        g_err = "finalize first";
        return 1;
    }
    MuteCout mute;
    REF_TRY({
        for (unsigned s = 0; s < n; s++) r.exec->timeStep();
    });
}

// wall time (seconds) of n steps: the reference arm of the CPU baseline
double ref_time_steps(void* h, unsigned n) {
    Ref& r = *(Ref*)h;
    if (!r.finalized) return -1.0;
    MuteCout mute;
    auto t0 = std::chrono::steady_clock::now();
    try {
        for (unsigned s = 0; s < n; s++) r.exec->timeStep();
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1.0;
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

unsigned ref_num_particles(void* h) { return ((Ref*)h)->ctx->particles.totalSize(); }

void ref_get_positions(void* h, double* out) {
    auto& P = ((Ref*)h)->ctx->particles;
    for (unsigned i = 0; i < P.totalSize(); i++)
        for (int k = 0; k < 3; k++) out[3 * i + k] = P.positions[i](k);
}

void ref_get_velocities(void* h, double* out) {
    auto& P = ((Ref*)h)->ctx->particles;
    for (unsigned i = 0; i < P.totalSize(); i++)
        for (int k = 0; k < 3; k++) out[3 * i + k] = P.velocities[i](k);
}

void ref_get_rotations(void* h, double* out) {
    auto& P = ((Ref*)h)->ctx->particles;
    for (unsigned i = 0; i < P.totalSize(); i++) {
        Quaternion q = P.isOriented(i) ? P.rotation(i) : Quaternion::Identity();
        out[4 * i] = q.w();
        out[4 * i + 1] = q.x();
        out[4 * i + 2] = q.y();
        out[4 * i + 3] = q.z();
    }
}

void ref_get_angular_velocities(void* h, double* out) {
    auto& P = ((Ref*)h)->ctx->particles;
    for (unsigned i = 0; i < P.totalSize(); i++)
        for (int k = 0; k < 3; k++) out[3 * i + k] = P.isOriented(i) ? P.angularVelocity(i)(k) : 0.0;
}

void ref_get_coloring(void* h, unsigned* colors, unsigned* num_colors) {
    auto& c = *((Ref*)h)->ctx;
    for (unsigned i = 0; i < c.particles.totalSize(); i++) colors[i] = c.coloring.color[i];
    *num_colors = c.coloring.num_colors;
}

// Collision stage state after the last step: the primitive pool's Morton
// codes and sorted order, the LBVH arrays (leaves [0, n), internal nodes
// [n, 2n-1)), and the candidate leaf pairs the reference's own
// LBVHTraversal::traverseSelfIterative (collision/LBVHTraversal.hpp:30-88)
// finds in that tree, ascending.  n is the pool's totalSize().
unsigned ref_num_primitives(void* h) { return ((Ref*)h)->ctx->collision_pool.totalSize(); }

unsigned ref_collect_pairs(void* h) {
    Ref& r = *(Ref*)h;
    auto& c = *r.ctx;
    r.pairs.clear();
    if (c.collision_pool.totalSize() > 1) {
        Collision::LBVHTraversal t;
        t.traverseSelfIterative(c.lbvh, c.lbvh.root, c.lbvh.root, r.pairs);
        std::sort(r.pairs.begin(), r.pairs.end());
    }
    return (unsigned)r.pairs.size();
}

void ref_get_lbvh(void* h, uint64_t* morton, unsigned* sorted, unsigned* left, unsigned* right, unsigned* parent,
                  unsigned* subtree, double* bounds, unsigned* root, unsigned* pairs) {
    Ref& r = *(Ref*)h;
    auto& c = *r.ctx;
    const unsigned n = c.collision_pool.totalSize();
    const unsigned nn = 2 * n - 1;
    for (unsigned i = 0; i < n; i++) {
        if (morton) morton[i] = c.collision_pool.morton_code[i];
        if (sorted) sorted[i] = c.collision_pool.sorted_order[i];
    }
    const auto& L = c.lbvh;
    for (unsigned k = 0; k < nn && k < L.parent.size(); k++) {
        if (left) left[k] = L.left[k];
        if (right) right[k] = L.right[k];
        if (parent) parent[k] = L.parent[k];
        if (subtree) subtree[k] = L.subtree_size[k];
        if (bounds) {
            const double b[6] = {L.min_x[k], L.min_y[k], L.min_z[k], L.max_x[k], L.max_y[k], L.max_z[k]};
            std::memcpy(bounds + 6 * k, b, sizeof(b));
        }
    }
    if (root) *root = L.root;
    if (pairs)
        for (size_t k = 0; k < r.pairs.size(); k++) {
            pairs[2 * k] = r.pairs[k].first;
            pairs[2 * k + 1] = r.pairs[k].second;
        }
}

// Dynamic contact state, the layout of orc_dynamic_info: [0] live
// triangle-rigid contacts, [1] their pool's totalSize(), [2] colors,
// [3] conflicted particles, [4] particles still dirty, [5] dynamic adjacency
// entries, [6] live triangle-rod contacts, [7] their pool's totalSize()
void ref_dynamic_info(void* h, unsigned* out) {
    auto& c = *((Ref*)h)->ctx;
    const auto& trc = c.energies.triangle_rigid_collision;
    const auto& trd = c.energies.triangle_rod_collision;
    out[0] = trc.count;
    out[1] = trc.totalSize();
    out[2] = c.coloring.num_colors;
    out[3] = (unsigned)c.coloring.conflicted_by_color_entries.size();
    out[4] = (unsigned)c.coloring.dirty.size();
    out[5] = (unsigned)c.dynamic_adjacency.e_entries.size();
    out[6] = trd.count;
    out[7] = trd.totalSize();
}

// Triangle-rigid pool by slot, the layout of orc_get_trc: particles (4),
// active flag, and 24 doubles: n, t, b, barys, cp_local, k_start, k_n, k_t,
// k_b, lam_n, lam_t, lam_b, C_n_prev, use_static + 2 unclamped
void ref_get_trc(void* h, unsigned* p4, uint8_t* active, double* data) {
    auto& pool = ((Ref*)h)->ctx->energies.triangle_rigid_collision;
    for (unsigned s = 0; s < pool.totalSize(); s++) {
        const auto& e = pool.data[s];
        if (p4)
            for (int k = 0; k < 4; k++) p4[4 * s + k] = e.particle_indices(k);
        if (active) active[s] = pool.active[s];
        if (data) {
            double* d = data + 24 * s;
            const Vec3r v[5] = {e.normal, e.tangent, e.binormal, e.barys, e.cp_rb_local};
            for (int i = 0; i < 5; i++)
                for (int j = 0; j < 3; j++) d[3 * i + j] = v[i](j);
            d[15] = e.k_start; d[16] = e.k_n; d[17] = e.k_t; d[18] = e.k_b;
            d[19] = e.lambda_n; d[20] = e.lambda_t; d[21] = e.lambda_b; d[22] = e.C_n_prev;
            d[23] = (e.use_static ? 1 : 0) + (e.unclamped_lambda_tb ? 2 : 0);
        }
    }
}

// Triangle-rod pool by slot, the layout of orc_get_trd: particles (5),
// active flag, and 25 doubles: n, t, b, barys, cp_local, s, k_start, k_n,
// k_t, k_b, lam_n, lam_t, lam_b, C_n_prev, flags
void ref_get_trd(void* h, unsigned* p5, uint8_t* active, double* data) {
    auto& pool = ((Ref*)h)->ctx->energies.triangle_rod_collision;
    for (unsigned s = 0; s < pool.totalSize(); s++) {
        const auto& e = pool.data[s];
        if (p5)
            for (int k = 0; k < 5; k++) p5[5 * s + k] = e.particle_indices(k);
        if (active) active[s] = pool.active[s];
        if (data) {
            double* d = data + 25 * s;
            const Vec3r v[5] = {e.normal, e.tangent, e.binormal, e.barys, e.cp_rod_local};
            for (int i = 0; i < 5; i++)
                for (int j = 0; j < 3; j++) d[3 * i + j] = v[i](j);
            d[15] = e.s;
            d[16] = e.k_start; d[17] = e.k_n; d[18] = e.k_t; d[19] = e.k_b;
            d[20] = e.lambda_n; d[21] = e.lambda_t; d[22] = e.lambda_b; d[23] = e.C_n_prev;
            d[24] = (e.use_static ? 1 : 0) + (e.unclamped_lambda_tb ? 2 : 0);
        }
    }
}

void ref_get_conflicted(void* h, uint8_t* out) {
    auto& c = *((Ref*)h)->ctx;
    for (unsigned p = 0; p < c.particles.totalSize(); p++) out[p] = c.coloring.is_conflicted[p];
}

// Block gradient and Hessian of particle p at the current state, through
// the reference's own accumulate functions for every static energy the
// particle takes part in (the loop of VBDSolver::_solveParticle,
// simulation/VBDSolver.hpp:293-447, without the solve), 3 or 6 DOF.
int ref_debug_block(void* h, unsigned p, double* G, double* H, int* dof) {
    auto& c = *((Ref*)h)->ctx;
    const Real dt = c.params.dt;
    REF_TRY({
        auto run = [&]<int DOF>() {
            Vec3r_or_Vec6r<DOF> grad = Vec3r_or_Vec6r<DOF>::Zero();
            Mat3r_or_Mat6r<DOF> hess = Mat3r_or_Mat6r<DOF>::Zero();
            const auto& off = c.static_adjacency.e_offsets[p];
            const unsigned adj_end = c.static_adjacency.e_offsets[p + 1][0];
            const unsigned ntypes = static_cast<unsigned>(StaticEnergyType::count);
            Energy::ForEachStaticEnergy([&]<StaticEnergyType E>() {
                const unsigned t = static_cast<unsigned>(E);
                const unsigned b = off[t], e = (t + 1 == ntypes) ? adj_end : off[t + 1];
                using Solver = typename SolverFor<E>::type;
                const auto& pool = c.energies.template get<E>();
                for (unsigned k = b; k < e; k++) {
                    const auto& en = c.static_adjacency.e_entries[k];
                    if constexpr (Solver::SupportsPositional && Solver::SupportsOriented)
                        Solver::template accumulate<DOF>(en.energy_idx, pool, c.particles, en.local_vertex_idx, hess,
                                                         grad, dt);
                    else if constexpr ((DOF == 6 && Solver::SupportsOriented) ||
                                       (DOF == 3 && Solver::SupportsPositional))
                        Solver::accumulate(en.energy_idx, pool, c.particles, en.local_vertex_idx, hess, grad, dt);
                }
            });
            for (int i = 0; i < DOF; i++) {
                G[i] = grad(i);
                for (int j = 0; j < DOF; j++) H[DOF * i + j] = hess(i, j);
            }
            *dof = DOF;
        };
        MuteCout mute;
        if (c.particles.isOriented(p)) run.template operator()<6>();
        else run.template operator()<3>();
    });
}

}  // extern "C"
