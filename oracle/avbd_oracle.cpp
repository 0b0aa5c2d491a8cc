// avbd_oracle.cpp -- FP64 CPU restatement of smtobin/avbd's per-step solve.
//
// TEST INFRASTRUCTURE.  This file is the checker, never the product: only the
// tests, the smoke check and bench.py's CPU-baseline leg load it.  The engine
// under avbd_b200/ never links, calls or falls back to it.
//
// What it restates (each function cites the reference file:line it follows):
//   * VBDSolver::solve_Parallel step schedule, inertial / Chebyshev / velocity
//     updates and the per-vertex 3x3 / 6x6 block solve
//     (simulation/VBDSolver.hpp:48-566);
//   * NeoHookean, Cosserat rod, ground, rigid-body-ground and one-sided fixed
//     joint energies with their AVBD dual updates (energy/**);
//   * static adjacency, DSATUR coloring and the work list
//     (common/StaticParticleAdjacency.hpp:42-133, common/ColorList.hpp:149-363);
//   * swept AABBs, 63-bit Morton codes, stable LSD radix sort, Karras tree,
//     refit and self traversal (collision/*).
//
// Parity status: PINNED to the reference implementation itself.  The
// reference's hot-path sources compile unmodified against the project's
// Eigen-API shim (oracle/eigen_shim, oracle/Makefile -> oracle/_ref), and
// tests/test_ref_pinning.py replays the reference's outputs
// (tests/golden/reference_outputs.npz, written by
// tests/golden/make_reference_golden.py) through this file: DSATUR colors,
// Morton codes, sorted order, LBVH topology and bounds, candidate pairs and
// contact-pool slots identical; positions within 1e-12 .. 1e-9 of the
// bounding-box diagonal after 1-100 steps (the shim's LU and sums round
// differently from Eigen's).  It is also pinned to what the reference's own
// tests hold: the finite-difference checks of
// test/test_neohookean_accumulate.cpp, test_cosserat_accumulate.cpp and
// test_one_sided_fixed_joint_accumulate.cpp (same inputs, same FD scheme,
// test/finite_difference.hpp), and the Karras-2012 radix-tree example of
// test/test_lbvh.cpp:38-47.  Build flags disable FMA contraction
// (-ffp-contract=off) so that the FP64 Morton codes are reproducible
// operation by operation.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <queue>
#include <stdexcept>
#include <string>
#include <vector>
#include <array>
#include <chrono>
#include <atomic>
#include <functional>
#include <thread>

namespace orc {

// ----------------------------------------------------------------- math
struct V3 {
    double x = 0, y = 0, z = 0;
    V3() {}
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    double& operator[](int i) { return (&x)[i]; }
    double operator[](int i) const { return (&x)[i]; }
};
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
static inline V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline double sqnorm(V3 a) { return dot(a, a); }
static inline double norm(V3 a) { return std::sqrt(sqnorm(a)); }

struct M3 {
    double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    static M3 zero() { return M3(); }
    static M3 eye() { M3 m; m.a[0][0] = m.a[1][1] = m.a[2][2] = 1; return m; }
    V3 row(int r) const { return {a[r][0], a[r][1], a[r][2]}; }
    V3 col(int c) const { return {a[0][c], a[1][c], a[2][c]}; }
    M3 T() const { M3 m; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) m.a[i][j] = a[j][i]; return m; }
};
static inline M3 operator*(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double s = 0;
            for (int k = 0; k < 3; k++) s += A.a[i][k] * B.a[k][j];
            C.a[i][j] = s;
        }
    return C;
}
static inline V3 operator*(const M3& A, V3 v) {
    return {A.a[0][0] * v.x + A.a[0][1] * v.y + A.a[0][2] * v.z,
            A.a[1][0] * v.x + A.a[1][1] * v.y + A.a[1][2] * v.z,
            A.a[2][0] * v.x + A.a[2][1] * v.y + A.a[2][2] * v.z};
}
static inline M3 operator*(double s, const M3& A) {
    M3 C; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) C.a[i][j] = s * A.a[i][j]; return C;
}
static inline M3 operator+(const M3& A, const M3& B) {
    M3 C; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) C.a[i][j] = A.a[i][j] + B.a[i][j]; return C;
}
static inline M3 operator-(const M3& A, const M3& B) {
    M3 C; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) C.a[i][j] = A.a[i][j] - B.a[i][j]; return C;
}
static inline M3 outer(V3 u, V3 v) {
    M3 C; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) C.a[i][j] = u[i] * v[j]; return C;
}
static inline double det(const M3& F) { return dot(F.col(0), cross(F.col(1), F.col(2))); }

// Math::Skew3 (common/Math.hpp:13-20)
static inline M3 skew(V3 v) {
    M3 m;
    m.a[0][1] = -v.z; m.a[0][2] = v.y;
    m.a[1][0] = v.z;  m.a[1][2] = -v.x;
    m.a[2][0] = -v.y; m.a[2][1] = v.x;
    return m;
}

struct Q4 { double w = 1, x = 0, y = 0, z = 0; };
static inline Q4 qmul(Q4 a, Q4 b) {   // Hamilton product
    Q4 r;
    r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    r.y = a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z;
    r.z = a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x;
    return r;
}
static inline Q4 qconj(Q4 q) { return {q.w, -q.x, -q.y, -q.z}; }
static inline V3 qvec(Q4 q) { return {q.x, q.y, q.z}; }
// rotation of a vector by a unit quaternion: v + 2w (u x v) + u x (2 u x v)
static inline V3 qrot(Q4 q, V3 v) {
    V3 u = qvec(q);
    V3 uv = cross(u, v);
    uv = uv + uv;
    return v + q.w * uv + cross(u, uv);
}
static inline M3 qmat(Q4 q) {   // rotation matrix of a unit quaternion
    double tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z;
    double twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
    double txx = tx * q.x, txy = ty * q.x, txz = tz * q.x;
    double tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
    M3 R;
    R.a[0][0] = 1 - (tyy + tzz); R.a[0][1] = txy - twz;       R.a[0][2] = txz + twy;
    R.a[1][0] = txy + twz;       R.a[1][1] = 1 - (txx + tzz); R.a[1][2] = tyz - twx;
    R.a[2][0] = txz - twy;       R.a[2][1] = tyz + twx;       R.a[2][2] = 1 - (txx + tyy);
    return R;
}
static inline Q4 qnormalize(Q4 q) {
    double n = std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    return {q.w / n, q.x / n, q.y / n, q.z / n};
}

// Math::Exp_s3 (common/Math.hpp:197-222)
static inline Q4 exp_s3(V3 v) {
    double th = norm(v);
    if (th < 1e-6) {
        Q4 q{1.0, 0.5 * v.x, 0.5 * v.y, 0.5 * v.z};
        return qnormalize(q);
    }
    double h = 0.5 * th, s = std::sin(h) / th;
    return {std::cos(h), s * v.x, s * v.y, s * v.z};
}
// Math::Log_S3 (common/Math.hpp:224-236)
static inline V3 log_s3(Q4 q) {
    V3 v = qvec(q);
    double m = norm(v);
    if (m < 1e-6) return 2.0 * v;
    double th = 2 * std::atan2(m, q.w);
    return (th / m) * v;
}
// Math::Minus_S3 / Plus_S3 (common/Math.hpp:238-246)
static inline V3 minus_s3(Q4 q1, Q4 q2) { return log_s3(qmul(qconj(q2), q1)); }
static inline Q4 plus_s3(Q4 q, V3 r) { return qmul(q, exp_s3(r)); }

// Math::ExpMap_RightJacobian (common/Math.hpp:28-38)
static inline M3 right_jac(V3 th) {
    double n = norm(th);
    M3 S = skew(th);
    if (n < 1e-8) return M3::eye() - 0.5 * S;
    return M3::eye() - ((1 - std::cos(n)) / (n * n)) * S + ((n - std::sin(n)) / (n * n * n)) * (S * S);
}
// Math::ExpMap_InvRightJacobian (common/Math.hpp:136-147)
static inline M3 inv_right_jac(V3 th) {
    double n = norm(th);
    M3 S = skew(th);
    if (n < 1e-8) return M3::eye() + 0.5 * S;
    return M3::eye() + 0.5 * S + (1 / (n * n) - (1 + std::cos(n)) / (2 * n * std::sin(n))) * (S * S);
}
// Math::Exp_so3 (common/Math.hpp:149-158)
static inline M3 exp_so3(V3 v) {
    M3 S = skew(v);
    double m = norm(v);
    if (m < 1e-8) return M3::eye() + S;
    return M3::eye() + (std::sin(m) / m) * S + ((1 - std::cos(m)) / (m * m)) * (S * S);
}

// Dense LU with partial (row) pivoting, the factorisation behind
// Mat3r/Mat6r::partialPivLu().solve (simulation/VBDSolver.hpp:472,498).
template <int N>
static void lu_solve(double A[N][N], const double* b_in, double* x) {
    double b[N];
    for (int i = 0; i < N; i++) b[i] = b_in[i];
    for (int k = 0; k < N; k++) {
        int p = k;
        double best = std::fabs(A[k][k]);
        for (int i = k + 1; i < N; i++)
            if (std::fabs(A[i][k]) > best) { best = std::fabs(A[i][k]); p = i; }
        if (p != k) {
            for (int j = 0; j < N; j++) std::swap(A[k][j], A[p][j]);
            std::swap(b[k], b[p]);
        }
        for (int i = k + 1; i < N; i++) {
            double l = A[i][k] / A[k][k];
            A[i][k] = l;
            for (int j = k + 1; j < N; j++) A[i][j] -= l * A[k][j];
            b[i] -= l * b[k];
        }
    }
    for (int i = N - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < N; j++) s -= A[i][j] * x[j];
        x[i] = s / A[i][i];
    }
}

// AVBD constants (common/common.hpp:13-15)
static constexpr double BETA = 10;
static constexpr double GAMMA = 0.99;
static constexpr double ALPHA = 0.95;

// Worker pool: the caller is worker 0, the other workers wait on a generation
// counter and split every range statically, the execution model of
// SimulationExecutor (simulation/SimulationExecutor.hpp:107-139) and
// WorkerThreadContext::computeStartEnd (common/WorkerThreadContext.hpp:48-53).
// Waits spin briefly, then block in the kernel (atomic wait/notify), so idle
// pools of oracles that are alive but not stepping take no CPU time.
struct Pool {
    int nt = 1;
    std::vector<std::thread> th;
    std::atomic<unsigned> gen{0};
    std::atomic<int> done{0};
    std::atomic<bool> stop{false};
    const std::function<void(int)>* job = nullptr;

    void start(int n) {
        shutdown();
        nt = n < 1 ? 1 : n;
        stop = false;
        for (int t = 1; t < nt; t++) th.emplace_back([this, t] { worker(t); });
    }
    // Waiters announce themselves (seq_cst, Dekker-style against the
    // counter's update) so that a hot run issues no wake-up system call.
    static constexpr int kSpins = 1 << 16;
    std::atomic<int> sleepers{0};
    std::atomic<bool> caller_sleeps{false};
    void worker(int t) {
        unsigned seen = gen.load();
        for (;;) {
            unsigned g;
            int spins = 0;
            while ((g = gen.load(std::memory_order_acquire)) == seen) {
                if (++spins > kSpins) {
                    sleepers.fetch_add(1);
                    gen.wait(seen);
                    sleepers.fetch_sub(1);
                    spins = 0;
                }
            }
            seen = g;
            if (stop.load()) return;
            (*job)(t);
            if (done.fetch_add(1) + 1 == nt - 1 && caller_sleeps.load()) done.notify_one();
        }
    }
    void wake() {
        gen.fetch_add(1);
        if (sleepers.load() > 0) gen.notify_all();
    }
    void run(const std::function<void(int)>& f) {
        if (nt == 1) { f(0); return; }
        job = &f;
        done.store(0);
        wake();
        f(0);
        int d, spins = 0;
        while ((d = done.load(std::memory_order_acquire)) != nt - 1) {
            if (++spins > kSpins) {
                caller_sleeps.store(true);
                done.wait(d);
                caller_sleeps.store(false);
                spins = 0;
            }
        }
    }
    template <typename F>
    void parallel_for(long lo, long hi, F&& fn) {
        long n = hi - lo;
        if (n <= 0) return;
        if (nt == 1 || n < 64) { for (long i = lo; i < hi; i++) fn(i); return; }
        std::function<void(int)> f = [&](int t) {
            long b = lo + n * t / nt, e = lo + n * (t + 1) / nt;
            for (long i = b; i < e; i++) fn(i);
        };
        run(f);
    }
    void shutdown() {
        if (th.empty()) return;
        stop = true;
        wake();
        for (auto& t : th) t.join();
        th.clear();
    }
    ~Pool() { shutdown(); }
};

// ------------------------------------------------------------ the state
enum StaticType : uint8_t { NEO_HOOKEAN = 0, COSSERAT_ROD = 1, GROUND = 2, RIGID_GROUND = 3, JOINT = 4, NTYPES = 5 };

// CollisionConstraintEnergyInfo (energy/collision/CollisionConstraintEnergyPool.hpp:9-30)
struct Contact {
    double k_start = 0, k_n = 0, k_t = 0, k_b = 0;
    double lam_n = 0, lam_t = 0, lam_b = 0, cn_prev = 0;
    V3 n, t, b;
    bool use_static = false, unclamped = false;
    double mu_s = 0, mu_k = 0;
};
struct Ground : Contact { unsigned p = 0; double cp_x = 0, cp_z = 0; };
struct RGround : Contact { unsigned p = 0; V3 cp_local, cp_ground; int shape = 2; double radius = 0; };
struct NH { unsigned idx[4]; double lambda, mu, kd; M3 Q; double V; M3 Eprev; };
struct Rod { unsigned idx[2]; double K[6]; double L; V3 kappa0; };
struct Joint {
    unsigned p = 0;
    double k[6], lam[6], cprev[6];
    V3 pos_off; Q4 rot_off; V3 ref_p; Q4 ref_q;
};
// TriangleRigidCollisionEnergyInfo (energy/collision/TriangleRigidCollisionEnergyPool.hpp:10-16):
// p[0..2] the triangle's vertices, p[3] the rigid body
struct TriRigid : Contact { unsigned p[4]; V3 barys, cp_local; };
// TriangleRodCollisionEnergyInfo (energy/collision/TriangleRodCollisionEnergyPool.hpp:9-15):
// p[0..2] the triangle's vertices, p[3], p[4] the rod segment's nodes
struct TriRod : Contact { unsigned p[5]; V3 barys, cp_local; double s = 0; };

// TombstonePool::allocSlot / freeSlot (common/TombstonePool.hpp:56-103).  The
// stack grows on demand; a slot never reached holds its own index, as the
// reference's iota-initialised stack does.  freeSlot's lowering of
// highest_index runs while the freed slot is still active, so it never
// lowers; the live slots are always a subset of [0, size()).
struct SlotPool {
    std::vector<uint8_t> active;
    std::vector<unsigned> slots;
    unsigned top = 0, count = 0;
    unsigned size() const { return (unsigned)active.size(); }
    unsigned alloc() {
        if (top == slots.size()) slots.push_back((unsigned)slots.size());
        unsigned slot = slots[top++];
        if (slot >= active.size()) active.resize(slot + 1, 0);
        active[slot] = 1;
        count++;
        return slot;
    }
    void free(unsigned slot) {
        if (slot >= active.size() || !active[slot]) throw std::runtime_error("freeSlot called on inactive slot");
        active[slot] = 0;
        count--;
        slots[--top] = slot;
    }
};
enum DynamicType : uint8_t { DYN_TRI_RIGID = 0, DYN_TRI_ROD = 1 };   // DynamicEnergyType order
struct DynEnt { uint8_t type; unsigned slot; uint16_t local; };
struct Prim { uint8_t type; unsigned idx[3]; uint8_t np; unsigned object_id; double radius; };
struct Entry { uint8_t type; unsigned idx; uint16_t local; };

struct Ctx {
    // SimulationParams / VBDSolver arguments
    double dt = 1e-3, g = 9.81, margin = 1e-3;
    unsigned iters = 1; double rho = 0.5;
    double tol = 0; unsigned max_iters = 0;
    int nthreads = 1;
    Pool pool;
    std::string err;

    // ParticlePool (common/ParticlePool.hpp:76-111)
    std::vector<V3> x, xb, y, xp, xl, xll, v, vp;
    std::vector<double> m;
    std::vector<uint8_t> fixed;
    std::vector<unsigned> rot;              // rotation_idx, UINT_MAX if positional
    // RotationPool (common/ParticlePool.hpp:7-68)
    std::vector<Q4> q, qb, qy, qp, ql, qll;
    std::vector<V3> w, wp, I;
    std::vector<unsigned> scene_of;         // scene index of each particle
    unsigned num_scenes = 1;
    // run-to-tolerance bookkeeping: every scene iterates until its own residual
    // reaches the tolerance, as it would in a context of its own
    std::vector<double> sweep_r2;           // in-sweep block residual of each particle
    std::vector<uint8_t> scene_active;
    std::vector<double> scene_mg2;
    std::vector<unsigned> scene_iters;      // iterations of the last step, per scene

    // energy pools
    std::vector<NH> nh;
    std::vector<Rod> rods;
    std::vector<Ground> ground;
    std::vector<RGround> rground;
    std::vector<Joint> joints;
    double joint_k_start = 1e4;

    // static adjacency (common/StaticParticleAdjacency.hpp:17-34)
    std::vector<unsigned> e_off;            // (np+1)*NTYPES, end of p = e_off[(p+1)*NTYPES]
    std::vector<Entry> entries;
    std::vector<unsigned> p_off, p_nbr;
    // ColorList (common/ColorList.hpp:62-78)
    std::vector<unsigned> color;
    unsigned num_colors = 0;
    std::vector<unsigned> color_offsets, work_list;

    // collision
    std::vector<Prim> prims;
    std::vector<double> aabb;               // 6 per primitive
    std::vector<uint64_t> morton;
    std::vector<unsigned> sorted;
    std::vector<unsigned> left, right, parent, subtree, leaf_count;
    std::vector<double> nbounds;            // 6 per node
    unsigned root = 0;
    std::vector<std::pair<unsigned, unsigned>> pairs;
    // detected triangle-sphere contacts of the last collision stage, ascending key
    // type 2 (TriangleRigid): rb = sphere particle; type 3 (TriangleRod): rod[2], s
    struct Detected {
        uint64_t key; unsigned type = 2; unsigned tri[3], rb = 0, rod[2] = {0, 0};
        V3 normal, barys, cp_local; double s = 0; unsigned e_idx = 0;
    };
    std::vector<Detected> detected;                 // narrow-phase output of the last stage
    std::vector<Detected> contacts, prev_contacts;  // managed detections with their pool slots

    // TriangleRigid / TriangleRodCollisionEnergyPool, each over a TombstonePool
    std::vector<TriRigid> trc;
    SlotPool trc_pool;
    std::vector<TriRod> trd;
    SlotPool trd_pool;
    // DynamicParticleAdjacency (common/DynamicParticleAdjacency.hpp:17-118)
    std::vector<unsigned> dyn_off;          // np + 1
    std::vector<DynEnt> dyn_ent;            // per particle by type, then slot
    std::vector<unsigned> dnb_off, dnb;
    // ColorList incremental recoloring state (common/ColorList.hpp:62-90)
    std::vector<unsigned> last_dirty, dirty, next_dirty, touched_frame, cand_color, touched_conflicted;
    std::vector<uint8_t> conflicted;
    std::vector<unsigned> conf_off, conf_list;   // conflicted particles per color
    std::vector<V3> buffered;               // buffered positions of conflicted particles
    unsigned recolor_rounds = 6;            // incrementalRecoloring's MAX_COLOR_ITERS

    // statistics
    double last_residual = -1;
    unsigned long long iterations = 0;
    bool finalized = false;

    unsigned np() const { return (unsigned)x.size(); }
    bool oriented(unsigned p) const { return rot[p] != UINT32_MAX; }
};

// -------------------------------------------------------------- energies
// NeoHookeanEnergySolver::computeF (energy/elastic/NeoHookeanEnergySolver.hpp:96-109)
static inline M3 computeF(V3 v1, V3 v2, V3 v3, V3 v4, const M3& Q) {
    M3 X;
    V3 c0 = v1 - v4, c1 = v2 - v4, c2 = v3 - v4;
    for (int i = 0; i < 3; i++) { X.a[i][0] = c0[i]; X.a[i][1] = c1[i]; X.a[i][2] = c2[i]; }
    return X * Q;
}

// NeoHookeanEnergySolver::energy (energy/elastic/NeoHookeanEnergySolver.hpp:20-53)
static double nh_energy(const Ctx& c, const NH& e, double dt) {
    M3 F = computeF(c.x[e.idx[0]], c.x[e.idx[1]], c.x[e.idx[2]], c.x[e.idx[3]], e.Q);
    M3 FtF = F.T() * F;
    M3 E = 0.5 * (FtF - M3::eye());
    M3 Ed = (1 / dt) * (E - e.Eprev);
    double sq = 0;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) sq += Ed.a[i][j] * Ed.a[i][j];
    double damp = e.V * e.kd * sq;
    double f = det(F) - e.mu / e.lambda - 1;
    double hyd = 0.5 * e.lambda * e.V * f * f;
    double dev = 0.5 * e.mu * e.V * (FtF.a[0][0] + FtF.a[1][1] + FtF.a[2][2] - 3);
    return hyd + dev + damp;
}

// NeoHookeanEnergySolver::updateAfterTimeStep (energy/elastic/NeoHookeanEnergySolver.hpp:70-90)
static void nh_after_step(Ctx& c, NH& e) {
    M3 F = computeF(c.xp[e.idx[0]], c.xp[e.idx[1]], c.xp[e.idx[2]], c.xp[e.idx[3]], e.Q);
    e.Eprev = 0.5 * (F.T() * F - M3::eye());
}

// NeoHookeanEnergySolver::accumulate (energy/elastic/NeoHookeanEnergySolver.hpp:121-227)
static void nh_accumulate(const Ctx& c, const NH& e, unsigned local, double H[3][3], double G[3], double dt) {
    M3 F = computeF(c.x[e.idx[0]], c.x[e.idx[1]], c.x[e.idx[2]], c.x[e.idx[3]], e.Q);
    V3 c0 = cross(F.col(1), F.col(2));
    V3 c1 = cross(F.col(2), F.col(0));
    V3 c2 = cross(F.col(0), F.col(1));
    double detF = dot(F.col(0), c0);
    V3 qi; double sign;
    if (local < 3) { qi = e.Q.row(local); sign = 1.0; }
    else { qi = e.Q.row(0) + e.Q.row(1) + e.Q.row(2); sign = -1.0; }
    V3 Fqi = F * qi;
    V3 Fc = qi.x * c0 + qi.y * c1 + qi.z * c2;
    double hyd = e.V * e.lambda * (detF - e.mu / e.lambda - 1);
    double dev = e.V * e.mu;
    M3 FtF = F.T() * F;
    double qn2 = sqnorm(qi);
    double damp = 2 / dt * e.V * e.kd;
    V3 g = (sign * hyd) * Fc + (sign * dev) * Fqi;
    M3 Ed = 0.5 * FtF;
    for (int i = 0; i < 3; i++) Ed.a[i][i] -= 0.5;
    Ed = (1 / dt) * (Ed - e.Eprev);
    g += (sign * damp) * (F * (Ed * qi));
    for (int i = 0; i < 3; i++) G[i] += g[i];
    double qEq = dot(qi, Ed * qi);
    M3 FFt = F * F.T();
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double h = e.V * e.lambda * Fc[i] * Fc[j];
            if (i == j) h += e.V * e.mu * qn2 + damp * qEq;
            h += (0.5 * damp / dt) * (FFt.a[i][j] * qn2 + Fqi[i] * Fqi[j]);
            H[i][j] += h;
        }
}

// CosseratRodEnergySolver strain and Jacobians
// (energy/elastic/CosseratRodEnergySolver.hpp:20-159)
static void rod_strain(const Ctx& c, const Rod& e, double strain[6], Q4* qmid_out = nullptr, V3* qdiff_out = nullptr) {
    Q4 q1 = c.q[c.rot[e.idx[0]]], q2 = c.q[c.rot[e.idx[1]]];
    V3 p1 = c.x[e.idx[0]], p2 = c.x[e.idx[1]];
    V3 qd = minus_s3(q2, q1);
    Q4 qm = plus_s3(q1, 0.5 * qd);
    double il = 1.0 / e.L;
    V3 sh = il * qrot(qconj(qm), p2 - p1) - V3(0, 0, 1);
    V3 be = il * qd - e.kappa0;
    for (int i = 0; i < 3; i++) { strain[i] = sh[i]; strain[3 + i] = be[i]; }
    if (qmid_out) *qmid_out = qm;
    if (qdiff_out) *qdiff_out = qd;
}

static double rod_energy(const Ctx& c, const Rod& e) {
    double s[6];
    rod_strain(c, e, s);
    double E = 0;
    for (int i = 0; i < 6; i++) E += s[i] * e.K[i] * s[i];
    return 0.5 * e.L * E;
}

static void rod_accumulate(const Ctx& c, const Rod& e, unsigned local, double H[6][6], double G[6]) {
    double s[6]; Q4 qm; V3 qd;
    rod_strain(c, e, s, &qm, &qd);
    V3 p1 = c.x[e.idx[0]], p2 = c.x[e.idx[1]];
    double il = 1.0 / e.L;
    M3 gi = inv_right_jac(qd);
    V3 th = 0.5 * qd;
    M3 eth = exp_so3(th);
    M3 gth = right_jac(th);
    M3 R = qmat(qm);
    V3 dpds = il * (p2 - p1);
    M3 S = skew(R.T() * dpds);
    double SG[6][6] = {};
    M3 A, B, C;
    if (local == 0) {
        M3 dth = (-0.5) * gi.T();
        M3 dthds = (-il) * gi.T();
        A = (-il) * R.T();
        B = S * (eth.T() + gth * dth);
        C = dthds;
    } else {
        M3 dth = 0.5 * gi;
        M3 dthds = il * gi;
        A = il * R.T();
        B = S * gth * dth;
        C = dthds;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { SG[i][j] = A.a[i][j]; SG[i][3 + j] = B.a[i][j]; SG[3 + i][3 + j] = C.a[i][j]; }
    for (int j = 0; j < 6; j++) {
        double g = 0;
        for (int i = 0; i < 6; i++) g += s[i] * e.K[i] * SG[i][j];
        G[j] += e.L * g;
    }
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) {
            double h = 0;
            for (int i = 0; i < 6; i++) h += SG[i][a] * e.K[i] * SG[i][b];
            H[a][b] += e.L * h;
        }
}

// GroundCollisionConstraintSolver::evaluateConstraint (energy/collision/GroundCollisionEnergySolver.hpp:14-25)
static void ground_eval(const Ctx& c, const Ground& e, double& Cn, double& Ct, double& Cb) {
    V3 p = c.x[e.p];
    Cn = -p.y; Ct = p.x - e.cp_x; Cb = p.z - e.cp_z;
}

// RigidBodyGroundCollisionConstraintSolver::evaluateConstraint
// (energy/collision/RigidBodyGroundCollisionEnergySolver.hpp:14-54)
static void rground_eval(const Ctx& c, const RGround& e, double& Cn, double& Ct, double& Cb) {
    V3 p = c.x[e.p];
    Q4 q = c.q[c.rot[e.p]];
    V3 cp_rb = p + qrot(q, e.cp_local);
    V3 diff = e.cp_ground - cp_rb;
    Ct = dot(e.t, diff); Cb = dot(e.b, diff);
    if (e.shape == 2 || e.shape == 1) {
        V3 cpg = p - V3(0, e.radius, 0);
        Cn = dot(e.n, e.cp_ground - cpg);
    } else {
        Cn = dot(e.n, diff);
    }
}

// CollisionConstraintEnergySolver::updateAfterIteration
// (energy/collision/CollisionConstraintEnergySolver.hpp:60-134)
static void contact_after_iter(Contact& e, double Cn, double Ct, double Cb) {
    double cc = Cn - ALPHA * e.cn_prev;
    double ln = e.k_n * cc + e.lam_n;
    double lt = e.k_t * Ct + e.lam_t;
    double lb = e.k_b * Cb + e.lam_b;
    if (ln > 0) e.k_n += BETA * std::fabs(cc);
    e.lam_n = std::max(0.0, ln);
    double mag = std::sqrt(lt * lt + lb * lb);
    double mu = e.use_static ? e.mu_s : e.mu_k;
    double mx = mu * e.lam_n;
    if (mag < mx) {
        e.k_t += BETA * std::fabs(Ct);
        e.k_b += BETA * std::fabs(Cb);
        e.lam_t = lt; e.lam_b = lb;
        e.unclamped = true;
    } else {
        if (e.use_static) { e.use_static = false; mx = e.mu_k * ln; }
        e.lam_t = lt / (mag + 1e-8) * mx;
        e.lam_b = lb / (mag + 1e-8) * mx;
        e.unclamped = false;
    }
}

// CollisionConstraintEnergySolver::updateAfterTimeStep
// (energy/collision/CollisionConstraintEnergySolver.hpp:141-167)
static void contact_after_step(Contact& e, double Cn_if_needed) {
    if (e.lam_n > 0) e.cn_prev = Cn_if_needed;
    if (e.unclamped && !e.use_static) e.use_static = true;
    e.lam_n *= ALPHA * GAMMA;
    e.lam_t *= GAMMA;
    e.lam_b *= GAMMA;
    e.k_n = std::max(GAMMA * e.k_n, e.k_start);
    e.k_t = std::max(GAMMA * e.k_t, e.k_start);
    e.k_b = std::max(GAMMA * e.k_b, e.k_start);
}

// CollisionConstraintEnergySolver::accumulate<DOF>
// (energy/collision/CollisionConstraintEnergySolver.hpp:179-285).  gn/gt/gb are
// the constraint gradients (DOF entries), hn/ht/hb the constraint Hessians.
template <int DOF>
static void contact_accumulate(const Contact& e, double Cn, double Ct, double Cb,
                               const double* gn, const double* gt, const double* gb,
                               const double (*hn)[DOF], const double (*ht)[DOF], const double (*hb)[DOF],
                               double H[DOF][DOF], double G[DOF]) {
    double cc = Cn - ALPHA * e.cn_prev;
    double lnp = std::max(0.0, e.k_n * cc + e.lam_n);
    double lt = e.k_t * Ct + e.lam_t, lb = e.k_b * Cb + e.lam_b;
    double mag = std::sqrt(lt * lt + lb * lb);
    double mu = e.use_static ? e.mu_s : e.mu_k;
    double mx = mu * lnp;
    if (mag > mx) {
        double nn = std::sqrt(lt * lt + lb * lb);
        lt = lt / (nn + 1e-8) * mx;
        lb = lb / (nn + 1e-8) * mx;
    }
    double sn = e.k_n * cc + e.lam_n, st = e.k_t * Ct + e.lam_t, sb = e.k_b * Cb + e.lam_b;
    for (int i = 0; i < DOF; i++) {
        G[i] += lnp * gn[i] + lt * gt[i] + lb * gb[i];
        for (int j = 0; j < DOF; j++) {
            double h = 0;
            h += sn * (hn ? hn[i][j] : 0.0) + e.k_n * gn[i] * gn[j];
            h += st * (ht ? ht[i][j] : 0.0) + e.k_t * gt[i] * gt[j];
            h += sb * (hb ? hb[i][j] : 0.0) + e.k_b * gb[i] * gb[j];
            H[i][j] += h;
        }
    }
}

// GroundCollisionConstraintSolver::constraintGradientHessian
// (energy/collision/GroundCollisionEnergySolver.hpp:27-60)
template <int DOF>
static void ground_accumulate(const Ctx& c, const Ground& e, double H[DOF][DOF], double G[DOF]) {
    double Cn, Ct, Cb;
    ground_eval(c, e, Cn, Ct, Cb);
    double gn[DOF] = {}, gt[DOF] = {}, gb[DOF] = {};
    gn[1] = -1; gt[0] = 1; gb[2] = 1;
    contact_accumulate<DOF>(e, Cn, Ct, Cb, gn, gt, gb, nullptr, nullptr, nullptr, H, G);
}

// RigidBodyGroundCollisionConstraintSolver::constraintGradientHessian
// (energy/collision/RigidBodyGroundCollisionEnergySolver.hpp:56-140)
static void rground_accumulate(const Ctx& c, const RGround& e, double H[6][6], double G[6]) {
    double Cn, Ct, Cb;
    rground_eval(c, e, Cn, Ct, Cb);
    Q4 q = c.q[c.rot[e.p]];
    M3 R = qmat(q);
    M3 S = skew(e.cp_local);
    M3 RS = R * S;
    double gn[6] = {}, gt[6] = {}, gb[6] = {};
    double hn[6][6] = {}, ht[6][6] = {}, hb[6][6] = {};
    auto rot_grad = [&](V3 d, double* g) {  // d^T (R S) as a column
        for (int j = 0; j < 3; j++) g[3 + j] = d.x * RS.a[0][j] + d.y * RS.a[1][j] + d.z * RS.a[2][j];
    };
    auto rot_hess = [&](V3 d, double h[6][6]) {
        M3 Hd = (-1.0) * (R.T() * skew(d) * R * S);
        M3 Hs = 0.5 * (Hd + Hd.T());
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) h[3 + i][3 + j] = Hs.a[i][j];
    };
    for (int i = 0; i < 3; i++) gn[i] = -e.n[i];
    if (!(e.shape == 2 || e.shape == 1)) { rot_grad(e.n, gn); rot_hess(e.n, hn); }
    for (int i = 0; i < 3; i++) { gt[i] = -e.t[i]; gb[i] = -e.b[i]; }
    rot_grad(e.t, gt); rot_grad(e.b, gb);
    rot_hess(e.t, ht); rot_hess(e.b, hb);
    contact_accumulate<6>(e, Cn, Ct, Cb, gn, gt, gb, hn, ht, hb, H, G);
}

// TriangleRigidCollisionConstraintSolver::evaluateConstraint
// (energy/collision/TriangleRigidCollisionEnergySolver.hpp:14-41)
static void trc_eval(const Ctx& c, const TriRigid& e, double& Cn, double& Ct, double& Cb) {
    V3 cp_tri = e.barys.x * c.x[e.p[0]] + e.barys.y * c.x[e.p[1]] + e.barys.z * c.x[e.p[2]];
    V3 cp_rb = c.x[e.p[3]] + qrot(c.q[c.rot[e.p[3]]], e.cp_local);
    V3 d = cp_rb - cp_tri;
    Cn = dot(e.n, d); Ct = dot(e.t, d); Cb = dot(e.b, d);
}

// TriangleRigidCollisionConstraintSolver::constraintGradientHessian
// (energy/collision/TriangleRigidCollisionEnergySolver.hpp:43-118) inside
// CollisionConstraintEnergySolver::accumulate<DOF>.  A triangle vertex (DOF 3)
// has gradients -bary (n, t, b) and no constraint Hessian.  The rigid body
// (DOF 6) has the normal's gradient (n, -(R S)^T n) with S = skew(cp_local),
// zero tangent and binormal gradients (the reference overwrites them), and
// rotational Hessian blocks sym(R^T skew(d) R S) for d = n, t, b.
template <int DOF>
static void trc_accumulate(const Ctx& c, const TriRigid& e, unsigned local, double H[DOF][DOF], double G[DOF]) {
    double Cn, Ct, Cb;
    trc_eval(c, e, Cn, Ct, Cb);
    double gn[DOF] = {}, gt[DOF] = {}, gb[DOF] = {};
    if constexpr (DOF == 6) {
        M3 R = qmat(c.q[c.rot[e.p[3]]]);
        M3 S = skew(e.cp_local);
        M3 RS = R * S;
        double hn[6][6] = {}, ht[6][6] = {}, hb[6][6] = {};
        for (int i = 0; i < 3; i++) gn[i] = e.n[i];
        for (int j = 0; j < 3; j++) gn[3 + j] = -(e.n.x * RS.a[0][j] + e.n.y * RS.a[1][j] + e.n.z * RS.a[2][j]);
        auto rot_hess = [&](V3 d, double h[6][6]) {
            M3 Hd = R.T() * skew(d) * R * S;
            M3 Hs = 0.5 * (Hd + Hd.T());
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) h[3 + i][3 + j] = Hs.a[i][j];
        };
        rot_hess(e.n, hn); rot_hess(e.t, ht); rot_hess(e.b, hb);
        contact_accumulate<6>(e, Cn, Ct, Cb, gn, gt, gb, hn, ht, hb, (double(*)[6])H, G);
    } else {
        if (local >= 3) throw std::runtime_error("TriangleRigidCollisionEnergySolver::constraintGradientHessian local_idx out of bounds!");
        double br = e.barys[local];
        for (int i = 0; i < 3; i++) { gn[i] = -br * e.n[i]; gt[i] = -br * e.t[i]; gb[i] = -br * e.b[i]; }
        contact_accumulate<DOF>(e, Cn, Ct, Cb, gn, gt, gb, nullptr, nullptr, nullptr, H, G);
    }
}

// TriangleRodCollisionConstraintSolver::evaluateConstraint
// (energy/collision/TriangleRodCollisionEnergySolver.hpp:14-50): the rod point
// is p_mid + q_mid cp_local, with p_mid and q_mid interpolated at s along the
// segment (q_mid = q1 (+) s (q2 (-) q1))
static void trd_eval(const Ctx& c, const TriRod& e, double& Cn, double& Ct, double& Cb) {
    V3 cp_tri = e.barys.x * c.x[e.p[0]] + e.barys.y * c.x[e.p[1]] + e.barys.z * c.x[e.p[2]];
    Q4 q1 = c.q[c.rot[e.p[3]]], q2 = c.q[c.rot[e.p[4]]];
    Q4 qm = plus_s3(q1, e.s * minus_s3(q2, q1));
    V3 pm = (1 - e.s) * c.x[e.p[3]] + e.s * c.x[e.p[4]];
    V3 d = (pm + qrot(qm, e.cp_local)) - cp_tri;
    Cn = dot(e.n, d); Ct = dot(e.t, d); Cb = dot(e.b, d);
}

// TriangleRodCollisionConstraintSolver::constraintGradientHessian
// (energy/collision/TriangleRodCollisionEnergySolver.hpp:52-149).  Triangle
// vertices as for the rigid contact.  Rod node 3 / 4: translation gradient
// (1 - s) n / s n; rotation gradient -n^T (-R S) dR_s/dR with
// dR_s/dR = Exp(s dq)^T - s J_r(s dq) J_r^-1(dq)^T for node 3 and
// s J_r(s dq) J_r^-1(dq) for node 4 (dq = q2 (-) q1, R = R(q_mid),
// S = skew(cp_local)); tangent and binormal gradients and all constraint
// Hessians are zero (Gauss-Newton).
template <int DOF>
static void trd_accumulate(const Ctx& c, const TriRod& e, unsigned local, double H[DOF][DOF], double G[DOF]) {
    double Cn, Ct, Cb;
    trd_eval(c, e, Cn, Ct, Cb);
    double gn[DOF] = {}, gt[DOF] = {}, gb[DOF] = {};
    if constexpr (DOF == 6) {
        Q4 q1 = c.q[c.rot[e.p[3]]], q2 = c.q[c.rot[e.p[4]]];
        V3 qd = minus_s3(q2, q1);
        Q4 qm = plus_s3(q1, e.s * qd);
        M3 R = qmat(qm);
        M3 Rl = (-1.0) * (R * skew(e.cp_local));
        M3 gam_inv = inv_right_jac(qd);
        M3 gam = right_jac(e.s * qd);
        M3 dR;
        double sc;
        if (local == 3) {
            dR = exp_so3(e.s * qd).T() - e.s * (gam * gam_inv.T());
            sc = 1 - e.s;
        } else if (local == 4) {
            dR = e.s * (gam * gam_inv);
            sc = e.s;
        } else {
            throw std::runtime_error("TriangleRigidCollisionEnergySolver::constraintGradientHessian local_idx out of bounds!");
        }
        M3 M = Rl * dR;
        for (int i = 0; i < 3; i++) gn[i] = sc * e.n[i];
        for (int j = 0; j < 3; j++) gn[3 + j] = -(e.n.x * M.a[0][j] + e.n.y * M.a[1][j] + e.n.z * M.a[2][j]);
        contact_accumulate<6>(e, Cn, Ct, Cb, gn, gt, gb, nullptr, nullptr, nullptr, (double(*)[6])H, G);
    } else {
        if (local >= 3) throw std::runtime_error("TriangleRigidCollisionEnergySolver::constraintGradientHessian local_idx out of bounds!");
        double br = e.barys[local];
        for (int i = 0; i < 3; i++) { gn[i] = -br * e.n[i]; gt[i] = -br * e.t[i]; gb[i] = -br * e.b[i]; }
        contact_accumulate<DOF>(e, Cn, Ct, Cb, gn, gt, gb, nullptr, nullptr, nullptr, H, G);
    }
}

// OneSidedFixedJointConstraintSolver::evaluateConstraint
// (energy/joint/OneSidedFixedJointEnergySolver.hpp:16-34)
static void joint_eval(const Ctx& c, const Joint& e, double C[6]) {
    V3 p = c.x[e.p];
    Q4 q = c.q[c.rot[e.p]];
    V3 jp = p + qrot(q, e.pos_off);
    Q4 jq = qmul(q, e.rot_off);
    V3 a = jp - e.ref_p;
    V3 b = minus_s3(jq, e.ref_q);
    for (int i = 0; i < 3; i++) { C[i] = a[i]; C[3 + i] = b[i]; }
}

// HardConstraintEnergySolver::energy (energy/HardConstraintEnergySolver.hpp:17-35)
static double joint_energy(const Ctx& c, const Joint& e) {
    double C[6]; joint_eval(c, e, C);
    double E = 0;
    for (int i = 0; i < 6; i++) E += 0.5 * e.k[i] * C[i] * C[i] + e.lam[i] * C[i];
    return E;
}

// HardConstraintEnergySolver::accumulate<6> with
// OneSidedFixedJointConstraintSolver::constraintGradientHessian
// (energy/HardConstraintEnergySolver.hpp:100-155, energy/joint/OneSidedFixedJointEnergySolver.hpp:36-90)
static void joint_accumulate(const Ctx& c, const Joint& e, double H[6][6], double G[6]) {
    double Craw[6]; joint_eval(c, e, Craw);
    Q4 q = c.q[c.rot[e.p]];
    M3 R = qmat(q);
    M3 dCp = (-1.0) * (R * skew(e.pos_off));
    V3 th(Craw[3], Craw[4], Craw[5]);
    M3 dCR = inv_right_jac(th) * qmat(e.rot_off).T();
    double grad[6][6] = {};
    for (int i = 0; i < 3; i++) {
        grad[i][i] = 1;
        for (int j = 0; j < 3; j++) { grad[i][3 + j] = dCp.a[i][j]; grad[3 + i][3 + j] = dCR.a[i][j]; }
    }
    const double lmin = std::numeric_limits<double>::lowest(), lmax = std::numeric_limits<double>::max();
    for (int ci = 0; ci < 6; ci++) {
        double C = Craw[ci] - ALPHA * e.cprev[ci];
        double lu = e.k[ci] * C + e.lam[ci];
        double lp = std::max(lmin, std::min(lmax, lu));
        double ks = e.k[ci];
        if (lu < lmin && std::fabs(C) > 1e-12) ks = std::fabs((lmin - e.lam[ci]) / C);
        else if (lu > lmax && std::fabs(C) > 1e-12) ks = std::fabs((lmax - e.lam[ci]) / C);
        for (int a = 0; a < 6; a++) {
            G[a] += grad[ci][a] * lp;
            for (int b = 0; b < 6; b++) H[a][b] += ks * grad[ci][a] * grad[ci][b];
        }
    }
}

// HardConstraintEnergySolver::updateAfterIteration (energy/HardConstraintEnergySolver.hpp:42-72)
static void joint_after_iter(const Ctx& c, Joint& e) {
    double C[6]; joint_eval(c, e, C);
    const double lmin = std::numeric_limits<double>::lowest(), lmax = std::numeric_limits<double>::max();
    for (int ci = 0; ci < 6; ci++) {
        double cc = C[ci] - ALPHA * e.cprev[ci];
        double lp = e.k[ci] * cc + e.lam[ci];
        if (lp > lmin && lp < lmax) e.k[ci] += BETA * cc;
        e.lam[ci] = std::max(lmin, std::min(lmax, lp));
    }
}

// HardConstraintEnergySolver::updateAfterTimeStep (energy/HardConstraintEnergySolver.hpp:79-88)
static void joint_after_step(const Ctx& c, Joint& e, double k_start) {
    for (int i = 0; i < 6; i++) {
        e.lam[i] = ALPHA * GAMMA * e.lam[i];
        e.k[i] = std::max(k_start, GAMMA * e.k[i]);
    }
    joint_eval(c, e, e.cprev);
}

// ------------------------------------------------------- vertex block
// Gradient / Hessian accumulation of VBDSolver::_solveParticle<DOF>
// (simulation/VBDSolver.hpp:293-447): static energies in type order, each in
// pool-slot order.
template <int DOF>
static void accumulate_block(const Ctx& c, unsigned p, double H[DOF][DOF], double G[DOF]) {
    for (int i = 0; i < DOF; i++) { G[i] = 0; for (int j = 0; j < DOF; j++) H[i][j] = 0; }
    unsigned beg = c.e_off[p * NTYPES], end = c.e_off[(p + 1) * NTYPES];
    for (unsigned k = beg; k < end; k++) {
        const Entry& en = c.entries[k];
        switch (en.type) {
            case NEO_HOOKEAN:
                if (DOF == 3) nh_accumulate(c, c.nh[en.idx], en.local, (double(*)[3])H, G, c.dt);
                break;
            case COSSERAT_ROD:
                if (DOF == 6) rod_accumulate(c, c.rods[en.idx], en.local, (double(*)[6])H, G);
                break;
            case GROUND:
                ground_accumulate<DOF>(c, c.ground[en.idx], H, G);
                break;
            case RIGID_GROUND:
                if (DOF == 6) rground_accumulate(c, c.rground[en.idx], (double(*)[6])H, G);
                break;
            case JOINT:
                if (DOF == 6) joint_accumulate(c, c.joints[en.idx], (double(*)[6])H, G);
                break;
        }
    }
    // dynamic energies (VBDSolver.hpp:397-446): triangle-rigid, then
    // triangle-rod contacts, each in slot order
    if (!c.dyn_off.empty())
        for (unsigned k = c.dyn_off[p]; k < c.dyn_off[p + 1]; k++) {
            const DynEnt& en = c.dyn_ent[k];
            if (en.type == DYN_TRI_RIGID) trc_accumulate<DOF>(c, c.trc[en.slot], en.local, H, G);
            else trd_accumulate<DOF>(c, c.trd[en.slot], en.local, H, G);
        }
}

// VBDSolver::_solveParticle<DOF> assembly and solve (simulation/VBDSolver.hpp:449-510)
static void solve_particle(Ctx& c, unsigned p) {
    if (c.fixed[p]) return;
    if (!c.scene_active.empty() && !c.scene_active[c.scene_of[p]]) return;
    double dt = c.dt;
    if (c.oriented(p)) {
        double H[6][6], G[6];
        accumulate_block<6>(c, p, H, G);
        unsigned r = c.rot[p];
        double mass = c.m[p];
        V3 Iv = c.I[r];
        V3 a = (-1 / (dt * dt) * mass) * (c.x[p] - c.y[p]);
        V3 ms = minus_s3(c.q[r], c.qy[r]);
        double rhs[6];
        for (int i = 0; i < 3; i++) { rhs[i] = a[i] - G[i]; rhs[3 + i] = -1 / (dt * dt) * (Iv[i] * ms[i]) - G[3 + i]; }
        for (int i = 0; i < 3; i++) { H[i][i] += mass / (dt * dt); H[3 + i][3 + i] += Iv[i] / (dt * dt); }
        if (!c.sweep_r2.empty()) {
            double s = 0;
            for (int i = 0; i < 6; i++) s += rhs[i] * rhs[i];
            c.sweep_r2[p] = s;
        }
        double dx[6];
        lu_solve<6>(H, rhs, dx);
        if (!c.conflicted.empty() && c.conflicted[p]) {
            // intra-color conflict: the update is buffered; _commitConflictedInColor
            // later copies the position only, so the rotation update is dropped
            c.buffered[p] = c.x[p] + V3(dx[0], dx[1], dx[2]);
        } else {
            c.x[p] += V3(dx[0], dx[1], dx[2]);
            c.q[r] = plus_s3(c.q[r], V3(dx[3], dx[4], dx[5]));
        }
    } else {
        double H[3][3], G[3];
        accumulate_block<3>(c, p, H, G);
        double mass = c.m[p];
        V3 d = c.x[p] - c.y[p];
        double rhs[3];
        for (int i = 0; i < 3; i++) rhs[i] = -mass / (dt * dt) * d[i] - G[i];
        for (int i = 0; i < 3; i++) H[i][i] += mass / (dt * dt);
        if (!c.sweep_r2.empty()) c.sweep_r2[p] = rhs[0] * rhs[0] + rhs[1] * rhs[1] + rhs[2] * rhs[2];
        double dx[3];
        lu_solve<3>(H, rhs, dx);
        if (!c.conflicted.empty() && c.conflicted[p]) c.buffered[p] = c.x[p] + V3(dx[0], dx[1], dx[2]);
        else c.x[p] += V3(dx[0], dx[1], dx[2]);
    }
}

// Block residual r_p = |m/h^2 (x - y) + g_p| (the negated RHS of
// simulation/VBDSolver.hpp:462-464,493) for the current iterate.
static double block_residual_sq(const Ctx& c, unsigned p) {
    double dt = c.dt;
    if (c.oriented(p)) {
        double H[6][6], G[6];
        accumulate_block<6>(c, p, H, G);
        unsigned r = c.rot[p];
        V3 a = (c.m[p] / (dt * dt)) * (c.x[p] - c.y[p]);
        V3 ms = minus_s3(c.q[r], c.qy[r]);
        double s = 0;
        for (int i = 0; i < 3; i++) {
            double u = a[i] + G[i], w = c.I[r][i] / (dt * dt) * ms[i] + G[3 + i];
            s += u * u + w * w;
        }
        return s;
    }
    double H[3][3], G[3];
    accumulate_block<3>(c, p, H, G);
    V3 a = (c.m[p] / (dt * dt)) * (c.x[p] - c.y[p]);
    double s = 0;
    for (int i = 0; i < 3; i++) { double u = a[i] + G[i]; s += u * u; }
    return s;
}

static double residual(Ctx& c) {
    double num = 0, den = 0;
    for (unsigned p = 0; p < c.np(); p++) {
        if (c.fixed[p]) continue;
        num += block_residual_sq(c, p);
        double mg = c.m[p] * c.g;
        den += mg * mg;
    }
    return den > 0 ? std::sqrt(num) / std::sqrt(den) : std::sqrt(num);
}

// ----------------------------------------------------- step schedule
// VBDSolver::_particleInertialUpdate (simulation/VBDSolver.hpp:208-248)
static void inertial(Ctx& c, unsigned p) {
    if (c.fixed[p]) return;
    double dt = c.dt;
    V3 aext(0, -c.g, 0);
    V3 a = (c.v[p] - c.vp[p]) / dt;
    V3 at;
    double an = norm(aext);
    if (an > 1e-12) {
        double al = dot(a, aext) / an;
        double t;
        if (al > an) t = 1;
        else if (al < 0) t = 0;
        else t = al / an;
        at = t * aext;
    }
    c.y[p] = c.x[p] + dt * c.v[p] + (dt * dt) * aext;
    c.x[p] += dt * c.v[p] + (dt * dt) * at;
    c.xl[p] = c.x[p];
    c.xll[p] = c.x[p];
    if (c.oriented(p)) {
        // VBDSolver::_particleRotationInertialUpdate (simulation/VBDSolver.hpp:253-283)
        unsigned r = c.rot[p];
        V3 w = c.w[r], Iv = c.I[r];
        V3 Iw(Iv.x * w.x, Iv.y * w.y, Iv.z * w.z);
        V3 wx = cross(w, Iw);
        V3 acc(-(1 / Iv.x) * wx.x, -(1 / Iv.y) * wx.y, -(1 / Iv.z) * wx.z);
        V3 dqi = dt * w + (dt * dt) * acc;
        c.qy[r] = plus_s3(c.q[r], dqi);
        c.q[r] = plus_s3(c.q[r], dt * w);
        c.ql[r] = c.q[r];
        c.qll[r] = c.q[r];
    }
}

// VBDSolver::_particleChebyshevAcceleration (simulation/VBDSolver.hpp:513-536)
static void chebyshev(Ctx& c, unsigned p, double omega) {
    c.x[p] = omega * (c.x[p] - c.xll[p]) + c.xll[p];
    if (c.oriented(p)) {
        unsigned r = c.rot[p];
        c.q[r] = plus_s3(c.qll[r], omega * minus_s3(c.q[r], c.qll[r]));
    }
    c.xll[p] = c.xl[p];
    c.xl[p] = c.x[p];
    if (c.oriented(p)) {
        unsigned r = c.rot[p];
        c.qll[r] = c.ql[r];
        c.ql[r] = c.q[r];
    }
}

// VBDSolver::_particleVelocityUpdate (simulation/VBDSolver.hpp:538-566)
static void velocity(Ctx& c, unsigned p) {
    double dt = c.dt;
    c.vp[p] = c.v[p];
    c.v[p] = (c.x[p] - c.xp[p]) / dt;
    c.xp[p] = c.x[p];
    if (c.oriented(p)) {
        unsigned r = c.rot[p];
        c.wp[r] = c.w[r];
        c.w[r] = minus_s3(c.q[r], c.qp[r]) / dt;
        c.qp[r] = c.q[r];
    }
}

// Energy hooks run at the start of each step, in EnergyRegistry order
// (energy/EnergyRegistry.hpp:100-109, simulation/VBDSolver.hpp:54-58).
static void after_time_step(Ctx& c) {
    c.pool.parallel_for(0, (long)c.nh.size(), [&](long e) { nh_after_step(c, c.nh[e]); });
    // GroundCollisionEnergySolver::updateContactPoints + updateAfterTimeStep
    // (energy/collision/GroundCollisionEnergySolver.hpp:81-91)
    c.pool.parallel_for(0, (long)c.ground.size(), [&](long i) {
        Ground& e = c.ground[i];
        e.cp_x = c.x[e.p].x;
        e.cp_z = c.x[e.p].z;
        double Cn, Ct, Cb;
        ground_eval(c, e, Cn, Ct, Cb);
        contact_after_step(e, Cn);
    });
    // RigidBodyGroundCollisionEnergySolver::updateContactPoints
    // (energy/collision/RigidBodyGroundCollisionEnergySolver.hpp:161-183)
    for (auto& e : c.rground) {
        e.cp_ground.x = c.x[e.p].x;
        e.cp_ground.z = c.x[e.p].z;
        if (e.shape == 2 || e.shape == 1)
            e.cp_local = qrot(qconj(c.q[c.rot[e.p]]), V3(0, -e.radius, 0));
        double Cn, Ct, Cb;
        rground_eval(c, e, Cn, Ct, Cb);
        contact_after_step(e, Cn);
    }
    // TriangleRigidCollisionEnergySolver::updateAfterTimeStep over the live slots
    for (unsigned i = 0; i < c.trc_pool.size(); i++) {
        if (!c.trc_pool.active[i]) continue;
        double Cn, Ct, Cb;
        trc_eval(c, c.trc[i], Cn, Ct, Cb);
        contact_after_step(c.trc[i], Cn);
    }
    for (unsigned i = 0; i < c.trd_pool.size(); i++) {
        if (!c.trd_pool.active[i]) continue;
        double Cn, Ct, Cb;
        trd_eval(c, c.trd[i], Cn, Ct, Cb);
        contact_after_step(c.trd[i], Cn);
    }
    for (auto& e : c.joints) joint_after_step(c, e, c.joint_k_start);
}

static inline bool scene_on(const Ctx& c, unsigned p) {
    return c.scene_active.empty() || c.scene_active[c.scene_of[p]];
}

static void after_iteration(Ctx& c) {
    c.pool.parallel_for(0, (long)c.ground.size(), [&](long i) {
        if (!scene_on(c, c.ground[i].p)) return;
        double Cn, Ct, Cb;
        ground_eval(c, c.ground[i], Cn, Ct, Cb);
        contact_after_iter(c.ground[i], Cn, Ct, Cb);
    });
    for (auto& e : c.rground) {
        if (!scene_on(c, e.p)) continue;
        double Cn, Ct, Cb;
        rground_eval(c, e, Cn, Ct, Cb);
        contact_after_iter(e, Cn, Ct, Cb);
    }
    for (unsigned i = 0; i < c.trc_pool.size(); i++) {
        if (!c.trc_pool.active[i] || !scene_on(c, c.trc[i].p[3])) continue;
        double Cn, Ct, Cb;
        trc_eval(c, c.trc[i], Cn, Ct, Cb);
        contact_after_iter(c.trc[i], Cn, Ct, Cb);
    }
    for (unsigned i = 0; i < c.trd_pool.size(); i++) {
        if (!c.trd_pool.active[i] || !scene_on(c, c.trd[i].p[3])) continue;
        double Cn, Ct, Cb;
        trd_eval(c, c.trd[i], Cn, Ct, Cb);
        contact_after_iter(c.trd[i], Cn, Ct, Cb);
    }
    for (auto& e : c.joints)
        if (scene_on(c, e.p)) joint_after_iter(c, e);
}

static void collision_stage(Ctx& c, bool manage);

// VBDSolver::solve_Parallel (simulation/VBDSolver.hpp:48-103) preceded by the
// collision stage of SimulationExecutor::_workerTimeStep
// (simulation/SimulationExecutor.hpp:142-156).
static void time_step(Ctx& c) {
    if (!c.prims.empty()) collision_stage(c, true);
    after_time_step(c);
    long n = (long)c.np();
    c.pool.parallel_for(0, n, [&](long p) { inertial(c, (unsigned)p); });
    double omega = 1;
    const bool tol_mode = c.tol > 0;
    unsigned max_it = tol_mode ? c.max_iters : c.iters;
    const unsigned S = c.num_scenes;
    if (tol_mode) {
        // Each scene iterates until its own residual R_s <= tol (or max_iters).
        // The in-sweep residual (every block's RHS just before its update) is
        // the trigger; the exact post-iteration residual confirms the stop.
        c.scene_active.assign(S, 1);
        c.scene_iters.assign(S, 0);
        c.sweep_r2.assign(c.np(), 0.0);
        c.scene_mg2.assign(S, 0.0);
        for (unsigned p = 0; p < c.np(); p++)
            if (!c.fixed[p]) c.scene_mg2[c.scene_of[p]] += (c.m[p] * c.g) * (c.m[p] * c.g);
    }
    unsigned it = 0;
    for (; it < max_it; it++) {
        if (it > 2) omega = 4 / (4 - c.rho * c.rho * omega);
        else if (it == 2) omega = 2 / (2 - c.rho * c.rho);
        else omega = 1;
        if (tol_mode) {
            bool any = false;
            for (unsigned s = 0; s < S; s++) any |= c.scene_active[s] != 0;
            if (!any) break;
        }
        for (unsigned col = 0; col < c.num_colors; col++) {
            c.pool.parallel_for(c.color_offsets[col], c.color_offsets[col + 1],
                                [&](long k) { solve_particle(c, c.work_list[k]); });
            // VBDSolver::_commitConflictedInColor (simulation/VBDSolver.hpp:82-87,108-119).
            // A fixed conflicted particle never writes its buffer; the reference
            // then copies an uninitialised buffer, here it keeps its position.
            if (col + 1 < c.conf_off.size())
                for (unsigned k = c.conf_off[col]; k < c.conf_off[col + 1]; k++) {
                    unsigned q = c.conf_list[k];
                    if (!c.fixed[q] && scene_on(c, q)) c.x[q] = c.buffered[q];
                }
        }
        c.pool.parallel_for(0, n, [&](long p) {
            if (scene_on(c, (unsigned)p)) chebyshev(c, (unsigned)p, omega);
        });
        after_iteration(c);
        if (tol_mode) {
            std::vector<double> r2(S, 0.0), ex(S, 0.0);
            for (unsigned p = 0; p < c.np(); p++)
                if (!c.fixed[p] && c.scene_active[c.scene_of[p]]) r2[c.scene_of[p]] += c.sweep_r2[p];
            std::vector<uint8_t> cand(S, 0);
            for (unsigned s = 0; s < S; s++) {
                if (!c.scene_active[s]) continue;
                c.scene_iters[s]++;
                double R = c.scene_mg2[s] > 0 ? std::sqrt(r2[s]) / std::sqrt(c.scene_mg2[s]) : std::sqrt(r2[s]);
                cand[s] = R <= c.tol;
            }
            for (unsigned p = 0; p < c.np(); p++)
                if (!c.fixed[p] && cand[c.scene_of[p]]) ex[c.scene_of[p]] += block_residual_sq(c, p);
            c.last_residual = 0;
            for (unsigned s = 0; s < S; s++) {
                if (!c.scene_active[s]) continue;
                if (cand[s]) {
                    double R = c.scene_mg2[s] > 0 ? std::sqrt(ex[s]) / std::sqrt(c.scene_mg2[s]) : std::sqrt(ex[s]);
                    if (R <= c.tol) c.scene_active[s] = 0;
                    c.last_residual = std::max(c.last_residual, R);
                }
                if (c.scene_iters[s] >= max_it) c.scene_active[s] = 0;
            }
        }
    }
    if (tol_mode) {
        for (unsigned s = 0; s < S; s++) c.iterations += c.scene_iters[s];
        c.scene_active.clear();
        c.sweep_r2.clear();
    } else {
        c.iterations += (unsigned long long)it * S;
    }
    c.pool.parallel_for(0, n, [&](long p) { velocity(c, (unsigned)p); });
}

// ------------------------------------------------- adjacency / coloring
// StaticParticleAdjacency::buildAdjacency (common/StaticParticleAdjacency.hpp:42-133):
// entries grouped per particle by type, then by pool slot; neighbour sets are
// the distinct other particles of every shared static energy.
static void build_adjacency(Ctx& c) {
    unsigned n = c.np();
    std::vector<unsigned> val((size_t)n * NTYPES, 0);
    std::vector<std::vector<unsigned>> nb(n);
    auto visit = [&](uint8_t type, const unsigned* idx, int k) {
        for (int a = 0; a < k; a++) {
            val[(size_t)idx[a] * NTYPES + type]++;
            for (int b = 0; b < k; b++) if (a != b) nb[idx[a]].push_back(idx[b]);
        }
    };
    for (auto& e : c.nh) visit(NEO_HOOKEAN, e.idx, 4);
    for (auto& e : c.rods) visit(COSSERAT_ROD, e.idx, 2);
    for (auto& e : c.ground) visit(GROUND, &e.p, 1);
    for (auto& e : c.rground) visit(RIGID_GROUND, &e.p, 1);
    for (auto& e : c.joints) visit(JOINT, &e.p, 1);
    c.e_off.assign((size_t)(n + 1) * NTYPES, 0);
    unsigned run = 0;
    for (unsigned p = 0; p < n; p++)
        for (int t = 0; t < NTYPES; t++) { c.e_off[(size_t)p * NTYPES + t] = run; run += val[(size_t)p * NTYPES + t]; }
    for (int t = 0; t < NTYPES; t++) c.e_off[(size_t)n * NTYPES + t] = run;
    c.entries.assign(run, Entry{});
    std::vector<unsigned> cur(c.e_off.begin(), c.e_off.end());
    auto scatter = [&](uint8_t type, const unsigned* idx, int k, unsigned slot) {
        for (int a = 0; a < k; a++) c.entries[cur[(size_t)idx[a] * NTYPES + type]++] = Entry{type, slot, (uint16_t)a};
    };
    for (unsigned s = 0; s < c.nh.size(); s++) scatter(NEO_HOOKEAN, c.nh[s].idx, 4, s);
    for (unsigned s = 0; s < c.rods.size(); s++) scatter(COSSERAT_ROD, c.rods[s].idx, 2, s);
    for (unsigned s = 0; s < c.ground.size(); s++) scatter(GROUND, &c.ground[s].p, 1, s);
    for (unsigned s = 0; s < c.rground.size(); s++) scatter(RIGID_GROUND, &c.rground[s].p, 1, s);
    for (unsigned s = 0; s < c.joints.size(); s++) scatter(JOINT, &c.joints[s].p, 1, s);
    c.p_off.assign(n + 1, 0);
    c.p_nbr.clear();
    for (unsigned p = 0; p < n; p++) {
        auto& v = nb[p];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        c.p_off[p + 1] = c.p_off[p] + (unsigned)v.size();
        c.p_nbr.insert(c.p_nbr.end(), v.begin(), v.end());
    }
}

// ColorList::greedyColor2 -- DSATUR, verbatim O(V^2) selection
// (common/ColorList.hpp:149-241).
static void dsatur_reference(Ctx& c) {
    unsigned n = c.np();
    const unsigned UNC = UINT32_MAX;
    c.color.assign(n, UNC);
    std::vector<unsigned> sat(n, 0);
    unsigned ncol = 0;
    std::vector<char> used;
    for (unsigned it = 0; it < n; it++) {
        unsigned best = UNC;
        for (unsigned j = 0; j < n; j++) {
            if (c.color[j] != UNC) continue;
            if (best == UNC) best = j;
            unsigned db = c.p_off[best + 1] - c.p_off[best];
            unsigned dj = c.p_off[j + 1] - c.p_off[j];
            if (sat[j] > sat[best]) best = j;
            else if (sat[j] == sat[best] && dj > db) best = j;
        }
        used.assign(ncol + 1, 0);
        for (unsigned e = c.p_off[best]; e < c.p_off[best + 1]; e++) {
            unsigned nbh = c.p_nbr[e];
            if (c.color[nbh] != UNC) used[c.color[nbh]] = 1;
        }
        unsigned col = 0;
        while (col < used.size() && used[col]) col++;
        c.color[best] = col;
        ncol = std::max(ncol, col + 1);
        for (unsigned e = c.p_off[best]; e < c.p_off[best + 1]; e++) {
            unsigned u = c.p_nbr[e];
            if (c.color[u] != UNC) continue;
            std::vector<char> seen(ncol, 0);
            unsigned cnt = 0;
            for (unsigned k = c.p_off[u]; k < c.p_off[u + 1]; k++) {
                unsigned w = c.p_nbr[k];
                if (c.color[w] != UNC && !seen[c.color[w]]) { seen[c.color[w]] = 1; cnt++; }
            }
            sat[u] = cnt;
        }
    }
    c.num_colors = ncol;
}

// Same selection rule as dsatur_reference -- maximise (saturation, degree),
// ties to the lowest index -- kept in a lazy max-heap so that large scenes
// finish in O((V+E) log V).  Produces the identical coloring.
static void dsatur_fast(Ctx& c) {
    unsigned n = c.np();
    const unsigned UNC = UINT32_MAX;
    c.color.assign(n, UNC);
    std::vector<unsigned> sat(n, 0);
    std::vector<std::array<uint64_t, 4>> seen(n, {0, 0, 0, 0});
    std::priority_queue<std::tuple<unsigned, unsigned, unsigned>> pq;  // (sat, deg, ~idx)
    for (unsigned p = 0; p < n; p++) pq.push({0u, c.p_off[p + 1] - c.p_off[p], ~p});
    unsigned ncol = 0;
    while (!pq.empty()) {
        auto [s, d, ni] = pq.top();
        pq.pop();
        unsigned v = ~ni;
        if (c.color[v] != UNC || s != sat[v]) continue;
        uint64_t used[5] = {0, 0, 0, 0, 0};
        for (unsigned e = c.p_off[v]; e < c.p_off[v + 1]; e++) {
            unsigned w = c.p_nbr[e];
            if (c.color[w] != UNC) used[c.color[w] >> 6] |= 1ull << (c.color[w] & 63);
        }
        unsigned col = 0;
        while (col < 320 && (used[col >> 6] >> (col & 63) & 1)) col++;
        if (col >= 256) throw std::runtime_error("Ran out of colors!");
        c.color[v] = col;
        ncol = std::max(ncol, col + 1);
        for (unsigned e = c.p_off[v]; e < c.p_off[v + 1]; e++) {
            unsigned u = c.p_nbr[e];
            if (c.color[u] != UNC) continue;
            uint64_t& word = seen[u][col >> 6];
            if (!(word >> (col & 63) & 1)) {
                word |= 1ull << (col & 63);
                sat[u]++;
                pq.push({sat[u], c.p_off[u + 1] - c.p_off[u], ~u});
            }
        }
    }
    c.num_colors = ncol;
}

// ColorList::rebuildWorkList (common/ColorList.hpp:345-363)
static void rebuild_work_list(Ctx& c) {
    unsigned n = c.np();
    std::vector<unsigned> cnt(c.num_colors, 0);
    for (unsigned p = 0; p < n; p++) cnt[c.color[p]]++;
    c.color_offsets.assign(c.num_colors + 1, 0);
    for (unsigned k = 0; k < c.num_colors; k++) c.color_offsets[k + 1] = c.color_offsets[k] + cnt[k];
    c.work_list.assign(n, 0);
    std::vector<unsigned> cur(c.color_offsets.begin(), c.color_offsets.end() - 1);
    for (unsigned p = 0; p < n; p++) c.work_list[cur[c.color[p]]++] = p;
}

// ----------------------------------------------------------------- LBVH
static inline double dmin_(double a, double b) { return (b < a) ? b : a; }  // std::min
static inline double dmax_(double a, double b) { return (a < b) ? b : a; }  // std::max

// CollisionPrimitivePool::speculativeGlobalBounds (collision/CollisionPrimitivePool.hpp:160-236)
static void spec_bounds(const Ctx& c, const Prim& pr, double* bx) {
    double mn[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(), std::numeric_limits<double>::max()};
    double mx[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest()};
    auto expand = [&](V3 p) { for (int i = 0; i < 3; i++) { mn[i] = dmin_(mn[i], p[i]); mx[i] = dmax_(mx[i], p[i]); } };
    const double dt = c.dt;
    if (pr.type == 0) {
        for (int k = 0; k < 3; k++) {
            V3 p = c.x[pr.idx[k]];
            expand(p);
            V3 dv = dt * c.v[pr.idx[k]];
            expand(p + dv);
        }
    } else if (pr.type == 1) {
        V3 p1 = c.x[pr.idx[0]], p2 = c.x[pr.idx[1]];
        double r = pr.radius;
        for (int i = 0; i < 3; i++) { mn[i] = dmin_(p1[i], p2[i]) - r; mx[i] = dmax_(p1[i], p2[i]) + r; }
        V3 n1 = p1 + dt * c.v[pr.idx[0]], n2 = p2 + dt * c.v[pr.idx[1]];
        for (int i = 0; i < 3; i++) { mn[i] = dmin_(mn[i], dmin_(n1[i], n2[i]) - r); mx[i] = dmax_(mx[i], dmax_(n1[i], n2[i]) + r); }
    } else {
        // sphere: local bounds [-r, r]^3 centred on the particle (collision/SDF.hpp)
        unsigned op = pr.idx[0];
        double r = pr.radius;
        V3 lmin(-r, -r, -r), lmax(r, r, r);
        V3 ctr = 0.5 * (lmin + lmax);
        V3 he = 0.5 * (lmax - lmin);
        Q4 q = c.q[c.rot[op]];
        V3 wc = qrot(q, ctr) + c.x[op];
        M3 R = qmat(q);
        M3 A; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) A.a[i][j] = std::fabs(R.a[i][j]);
        V3 we = A * he;
        for (int i = 0; i < 3; i++) { mn[i] = wc[i] - we[i]; mx[i] = wc[i] + we[i]; }
        Q4 nq = plus_s3(q, dt * c.w[c.rot[op]]);
        V3 nwc = qrot(nq, ctr) + c.x[op] + dt * c.v[op];
        M3 NR = qmat(nq);
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) A.a[i][j] = std::fabs(NR.a[i][j]);
        V3 nwe = A * he;
        for (int i = 0; i < 3; i++) { mn[i] = dmin_(mn[i], nwc[i] - nwe[i]); mx[i] = dmax_(mx[i], nwc[i] + nwe[i]); }
    }
    for (int i = 0; i < 3; i++) { bx[i] = mn[i]; bx[3 + i] = mx[i]; }
}

// LBVHBuilder::expandBits21 / morton3D_64 (collision/LBVHBuilder.hpp:65-85)
static inline uint64_t expand21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
static inline uint64_t morton64(double nx, double ny, double nz) {
    double x = std::clamp(nx * 2097152.0, 0.0, 2097151.0);
    double y = std::clamp(ny * 2097152.0, 0.0, 2097151.0);
    double z = std::clamp(nz * 2097152.0, 0.0, 2097151.0);
    return expand21((uint64_t)x) | (expand21((uint64_t)y) << 1) | (expand21((uint64_t)z) << 2);
}

// LBVHBuilder::constructTree (collision/LBVHBuilder.cpp:181-286)
static void construct_tree(Ctx& c, unsigned nprim) {
    int n = (int)nprim;
    unsigned nn = 2 * nprim - 1;
    const unsigned INV = UINT32_MAX;
    c.left.assign(nn, INV); c.right.assign(nn, INV); c.parent.assign(nn, INV);
    c.leaf_count.assign(nn, 0); c.subtree.assign(nn, 0);
    // LBVHBuilder::commonPrefixLen (collision/LBVHBuilder.hpp:33-41): equal
    // codes fall back to the primitive indices
    auto delta = [&](int i, int j) -> int {
        if (j < 0 || j >= n) return -1;
        unsigned si = c.sorted[i], sj = c.sorted[j];
        uint64_t a = c.morton[si], b = c.morton[sj];
        if (a == b) {
            uint64_t x = (uint64_t)si ^ (uint64_t)sj;
            return 64 + (x ? __builtin_clzll(x) : 64);
        }
        return __builtin_clzll(a ^ b);
    };
    for (int i = 0; i < n - 1; i++) {
        int d = (delta(i, i + 1) - delta(i, i - 1) >= 0) ? 1 : -1;
        int dmin = delta(i, i - d);
        int lmax = 128;
        while (delta(i, i + lmax * d) > dmin) lmax *= 4;
        int l = 0;
        for (unsigned t = lmax; t >= 1; t /= 2)
            if (delta(i, i + (l + (int)t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta(i, j);
        int s = 0;
        for (int t = (l + 1) / 2; t >= 1; t = (t == 1 ? 0 : (t + 1) / 2)) {
            int ns = s + t;
            if (ns < l && delta(i, i + ns * d) > dnode) s = ns;
        }
        int gamma = i + s * d + std::min(d, 0);
        unsigned g = (unsigned)(i + n);
        if (std::min(i, j) == gamma) { c.left[g] = gamma; c.parent[gamma] = g; }
        else { c.left[g] = n + gamma; c.parent[n + gamma] = g; }
        if (std::max(i, j) == gamma + 1) { c.right[g] = gamma + 1; c.parent[gamma + 1] = g; }
        else { c.right[g] = n + gamma + 1; c.parent[n + gamma + 1] = g; }
    }
    unsigned node = 0;
    while (c.parent[node] != INV) node = c.parent[node];
    c.root = node;
    for (int l = 0; l < n; l++) { c.leaf_count[l] = 1; c.subtree[l] = 1; }
}

// LBVHBuilder::assembleBVH, serial refit (collision/LBVHBuilder.cpp:410-453)
static void refit(Ctx& c, unsigned n) {
    unsigned nn = 2 * n - 1;
    c.nbounds.assign((size_t)nn * 6, 0);
    std::vector<uint8_t> visited(nn, 0);
    for (unsigned l = 0; l < n; l++) {
        const double* b = &c.aabb[(size_t)c.sorted[l] * 6];
        for (int k = 0; k < 6; k++) c.nbounds[(size_t)l * 6 + k] = b[k];
        unsigned node = c.parent[l];
        while (node != UINT32_MAX) {
            if (visited[node]++ == 0) break;
            unsigned a = c.left[node], bb = c.right[node];
            for (int k = 0; k < 3; k++) {
                c.nbounds[(size_t)node * 6 + k] = dmin_(c.nbounds[(size_t)a * 6 + k], c.nbounds[(size_t)bb * 6 + k]);
                c.nbounds[(size_t)node * 6 + 3 + k] = dmax_(c.nbounds[(size_t)a * 6 + 3 + k], c.nbounds[(size_t)bb * 6 + 3 + k]);
            }
            c.subtree[node] = c.subtree[a] + c.subtree[bb];
            node = c.parent[node];
        }
    }
}

// LBVHTraversal::traverseSelfIterative (collision/LBVHTraversal.hpp:30-88)
static void traverse(Ctx& c) {
    c.pairs.clear();
    std::vector<std::pair<unsigned, unsigned>> st;
    st.push_back({c.root, c.root});
    auto ov = [&](unsigned a, unsigned b) {
        const double* A = &c.nbounds[(size_t)a * 6];
        const double* B = &c.nbounds[(size_t)b * 6];
        return A[0] <= B[3] && A[1] <= B[4] && A[2] <= B[5] && A[3] >= B[0] && A[4] >= B[1] && A[5] >= B[2];
    };
    while (!st.empty()) {
        auto [a, b] = st.back();
        st.pop_back();
        if (!ov(a, b)) continue;
        bool la = c.leaf_count[a] > 0, lb = c.leaf_count[b] > 0;
        if (la && lb) { if (a < b) c.pairs.push_back({a, b}); continue; }
        if (a == b) {
            unsigned l = c.left[a], r = c.right[a];
            st.push_back({l, l}); st.push_back({r, r}); st.push_back({l, r});
            continue;
        }
        if (la || (!lb && c.subtree[b] > c.subtree[a])) {
            st.push_back({a, c.left[b]}); st.push_back({a, c.right[b]});
        } else {
            st.push_back({c.left[a], b}); st.push_back({c.right[a], b});
        }
    }
    std::sort(c.pairs.begin(), c.pairs.end());
}

// ------------------------------------------------ narrow phase
// SDF::evaluate / SDF::gradient for spheres (collision/SDF.hpp:46-107)
static inline double sdf_sphere(double r, V3 p) { return norm(p) - r; }
static inline V3 sdf_sphere_grad(V3 p) {
    double d = norm(p);
    return d > 1e-8 ? p / d : V3(1, 0, 0);
}

// Algorithm::goldenSectionSearch (common/Algorithm.hpp:252-294): minimises f
// over the segment [lo, hi] (a time interval or a segment in space); the
// search stops when the bracket is 1e-3 wide.
static inline double gss_width(double x) { return std::fabs(x); }
static inline double gss_width(V3 x) { return norm(x); }
static inline double gss_lerp(double a, double b, double s) { return (1 - s) * a + s * b; }
static inline V3 gss_lerp(V3 a, V3 b, double s) { return (1 - s) * a + s * b; }
template <typename T, typename F>
static T gss(T lo, T hi, F&& f) {
    const double phi = 1.61803398875, r = 1 / phi, sg = 1 - r, tol = 1e-3;
    double a0 = 0, a1 = sg, a2 = r, a3 = 1;
    T t0 = lo, t1 = gss_lerp(lo, hi, a1), t2 = gss_lerp(lo, hi, a2), t3 = hi;
    double f0 = f(t0), f1 = f(t1), f2 = f(t2), f3 = f(t3);
    while (gss_width(t3 - t0) > tol) {
        if (std::min(f0, f1) < std::min(f2, f3)) {
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
static inline V3 barycentric(V3 p, V3 a, V3 b, V3 c) {
    V3 v0 = b - a, v1 = c - a, v2 = p - a;
    double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    double den = d00 * d11 - d01 * d01;
    double v = (d11 * d20 - d01 * d21) / den;
    double w = (d00 * d21 - d01 * d20) / den;
    return V3(1 - v - w, v, w);
}

// rotation of v by the inverse of q (Eigen's inverse: conjugate / |q|^2)
static inline V3 qrot_inv(Q4 q, V3 v) {
    double n2 = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    Q4 i{q.w / n2, -q.x / n2, -q.y / n2, -q.z / n2};
    return qrot(i, v);
}

// CollisionDetector::_triangleSDF_CCD (collision/CollisionDetector.cpp:689-876):
// alternating temporal and spatial golden-section searches for the first
// contact of a moving triangle with a moving sphere over [0, dt].
static bool tri_sphere_ccd(const Ctx& c, const Prim& T, const Prim& S, V3& normal, V3& barys, V3& cp_local) {
    const unsigned rb = S.idx[0];
    const double rad = S.radius, dt = c.dt;
    const V3 xr = c.x[rb], vr = c.v[rb], wr = c.w[c.rot[rb]];
    const Q4 qr = c.q[c.rot[rb]];
    auto rb_pos = [&](double t) { return xr + t * vr; };
    auto rb_rot = [&](double t) { return qmul(qr, exp_s3(t * wr)); };
    auto to_local = [&](V3 xg, double t) { return qrot_inv(rb_rot(t), xg - rb_pos(t)); };
    auto body_vel = [&](V3 xg, double t) { return vr + cross(qrot(rb_rot(t), wr), xg - rb_pos(t)); };
    auto rel_vel = [&](V3 xg, V3 vg, double t) { return qrot_inv(rb_rot(t), vg - body_vel(xg, t)); };
    const V3 p1 = c.x[T.idx[0]], p2 = c.x[T.idx[1]], p3 = c.x[T.idx[2]];
    const V3 v1 = c.v[T.idx[0]], v2 = c.v[T.idx[1]], v3 = c.v[T.idx[2]];
    auto first_eval = [&](V3 pk, V3 vk) { return dot(rel_vel(pk, vk, 0), sdf_sphere_grad(to_local(pk, 0))); };
    const double e1 = first_eval(p1, v1), e2 = first_eval(p2, v2), e3 = first_eval(p3, v3);
    double t_start = 0, t_end = dt, t = 0, u, v, w;
    if (e1 < e2 && e1 < e3) { u = 1; v = 0; w = 0; }
    else if (e2 < e1 && e2 < e3) { u = 0; v = 1; w = 0; }
    else { u = 0; v = 0; w = 1; }
    auto interp = [&](double t_) { return u * (p1 + t_ * v1) + v * (p2 + t_ * v2) + w * (p3 + t_ * v3); };
    auto sd_time = [&](double t_) { return sdf_sphere(rad, to_local(interp(t_), t_)); };
    auto ud_time = [&](double t_) { return std::fabs(sd_time(t_)); };
    auto sd_point = [&](V3 xl) { return sdf_sphere(rad, xl); };
    double sd = 0;
    V3 grad, x_ti;
    for (int it = 0; it < 16; it++) {
        const double t_old = t;
        V3 xg = interp(t), vg = u * v1 + v * v2 + w * v3;
        x_ti = to_local(xg, t);
        V3 v_ti = rel_vel(xg, vg, t);
        sd = sdf_sphere(rad, x_ti);
        if (sd <= 0) {
            t_end = std::min(t, t_end);
            t = gss(t_start, t, ud_time);
        } else {
            double vdg = dot(v_ti, sdf_sphere_grad(x_ti));
            if (vdg > 0) t = gss(t_start, t, sd_time);
            else t = gss(t, t_end, sd_time);
        }
        xg = interp(t);
        x_ti = to_local(xg, t);
        sd = sdf_sphere(rad, x_ti);
        grad = sdf_sphere_grad(x_ti);
        if (sd <= 0) t_end = std::min(t, t_end);
        V3 l1 = to_local(p1 + t * v1, t), l2 = to_local(p2 + t * v2, t), l3 = to_local(p3 + t * v3, t);
        double s1 = dot(l1, grad), s2 = dot(l2, grad), s3 = dot(l3, grad);
        V3 sv = (s1 < s2 && s1 < s3) ? l1 : ((s2 < s1 && s2 < s3) ? l2 : l3);
        V3 x_new = gss(x_ti, sv, sd_point);
        V3 b = barycentric(x_new, l1, l2, l3);
        u = b.x; v = b.y; w = b.z;
        if (std::fabs(t_old - t) < 1e-6 && norm(x_new - x_ti) < 1e-6) break;
    }
    barys = V3(u, v, w);
    cp_local = x_ti - sd * grad;
    normal = qrot(rb_rot(t), grad);
    return sd < c.margin;
}

// DetectedCollision::generateKey (collision/DetectedCollision.hpp:43-66)
static inline uint64_t collision_key(unsigned type, unsigned a, unsigned b, unsigned code) {
    if (a > b) std::swap(a, b);
    uint64_t k = type & 31u;
    k = (k << 26) | (a & 0x3FFFFFFu);
    k = (k << 26) | (b & 0x3FFFFFFu);
    return (k << 7) | (code & 127u);
}

// Math::closestPoint_PointTriangle (common/Math.hpp:446-500), Ericson's regions
static V3 closest_point_triangle(V3 p, V3 a, V3 b, V3 c) {
    V3 ab = b - a, ac = c - a, ap = p - a;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return a;
    V3 bp = p - b;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return b;
    V3 cp = p - c;
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return c;
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return a + (d1 / (d1 - d3)) * ab;
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return a + (d2 / (d2 - d6)) * ac;
    double va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
    double den = 1.0 / (va + vb + vc);
    double v = vb * den, w = vc * den;
    return a + v * ab + w * ac;
}

static inline double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }   // std::clamp

// Math::closestPoint_SegmentSegment (common/Math.hpp:508-560), Ericson's
// ClosestPtSegmentSegment: s on (p1, q1), t on (p2, q2)
static void closest_segment_segment(V3 p1, V3 q1, V3 p2, V3 q2, double& s, double& t) {
    V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    const double EPS = 1e-8;
    if (a <= EPS && e <= EPS) { s = t = 0.0; return; }
    if (a <= EPS) {
        s = 0.0;
        t = clamp01(f / e);
    } else {
        double cc = dot(d1, r);
        if (e <= EPS) {
            t = 0.0;
            s = clamp01(-cc / a);
        } else {
            double b = dot(d1, d2);
            double den = a * e - b * b;
            s = den != 0.0 ? clamp01((b * f - cc * e) / den) : 0.0;
            t = (b * s + f) / e;
            if (t < 0.0) { t = 0.0; s = clamp01(-cc / a); }
            else if (t > 1.0) { t = 1.0; s = clamp01((b - cc) / a); }
        }
    }
}

// Math::pointInTriangle (common/Math.hpp:562-591)
static bool point_in_triangle(V3 p, V3 a, V3 b, V3 c) {
    V3 v0 = b - a, v1 = c - a, v2 = p - a;
    double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    double den = d00 * d11 - d01 * d01;
    if (std::fabs(den) < 1e-12) return false;
    double v = (d11 * d20 - d01 * d21) / den;
    double w = (d00 * d21 - d01 * d20) / den;
    double u = 1.0 - v - w;
    const double EPS = 1e-8;
    return u >= -EPS && v >= -EPS && w >= -EPS;
}

// Math::closestPoint_SegmentTriangle (common/Math.hpp:593-681): the segment's
// crossing of the triangle, else the closest of the three edge tests and the
// two end points.  The edge test measures its distance to (1-s) q0 + s q1,
// the edge point at the SEGMENT's parameter, as the reference does.
static void closest_segment_triangle(V3 p0, V3 p1, V3 a, V3 b, V3 c, double& s_out, V3& bary, double& dist) {
    const double EPS = 1e-8;
    V3 dir = p1 - p0;
    V3 nrm = cross(b - a, c - a);
    s_out = 0.0;
    bary = V3(1, 0, 0);
    dist = std::numeric_limits<double>::max();
    if (sqnorm(nrm) > EPS) {
        double den = dot(nrm, dir);
        if (std::fabs(den) > EPS) {
            double s = dot(nrm, a - p0) / den;
            if (s >= 0.0 && s <= 1.0) {
                V3 p = p0 + s * dir;
                if (point_in_triangle(p, a, b, c)) {
                    s_out = s;
                    bary = barycentric(p, a, b, c);
                    dist = 0.0;
                    return;
                }
            }
        }
    }
    auto edge = [&](V3 q0, V3 q1, int i0, int i1) {
        double s, t;
        closest_segment_segment(p0, p1, q0, q1, s, t);
        V3 cp = (1 - s) * p0 + s * p1;
        V3 cq = (1 - s) * q0 + s * q1;
        double d2 = sqnorm(cp - cq);
        if (d2 < dist * dist) {
            s_out = s;
            bary = V3(0, 0, 0);
            bary[i0] = 1 - t;
            bary[i1] = t;
            dist = std::sqrt(d2);
        }
    };
    edge(a, b, 0, 1);
    edge(a, c, 0, 2);
    edge(b, c, 1, 2);
    V3 c0 = closest_point_triangle(p0, a, b, c);
    double d0 = sqnorm(p0 - c0);
    if (d0 < dist * dist) { s_out = 0.0; bary = barycentric(c0, a, b, c); dist = std::sqrt(d0); }
    V3 c1 = closest_point_triangle(p1, a, b, c);
    double d1 = sqnorm(p1 - c1);
    if (d1 < dist * dist) { s_out = 1.0; bary = barycentric(c1, a, b, c); dist = std::sqrt(d1); }
}

// CollisionDetector::_triangleRod (collision/CollisionDetector.cpp:601-666):
// contact when the centreline's distance to the triangle is below radius +
// margin; the normal points from the centreline point to the triangle point,
// the rod point is radius * normal in the frame interpolated at s.
static bool tri_rod_contact(const Ctx& c, const Prim& T, const Prim& R, V3& normal, V3& barys, double& s,
                            V3& cp_local) {
    V3 v1 = c.x[T.idx[0]], v2 = c.x[T.idx[1]], v3 = c.x[T.idx[2]];
    V3 s1 = c.x[R.idx[0]], s2 = c.x[R.idx[1]];
    double dist;
    closest_segment_triangle(s1, s2, v1, v2, v3, s, barys, dist);
    if (!(dist < R.radius + c.margin)) return false;
    V3 cl = (1 - s) * s1 + s * s2;
    V3 ct = barys.x * v1 + barys.y * v2 + barys.z * v3;
    V3 d = ct - cl;
    double m = norm(d);
    normal = m > 1e-8 ? d / m : V3(1, 0, 0);
    Q4 q1 = c.q[c.rot[R.idx[0]]], q2 = c.q[c.rot[R.idx[1]]];
    Q4 qm = plus_s3(q1, s * minus_s3(q2, q1));
    cp_local = qrot_inv(qm, R.radius * normal);
    return true;
}

// CollisionDetector::_narrowPhaseCollisionDetection + _processPotentialCollision
// (collision/CollisionDetector.cpp:132-215) for the pairs this engine
// supports: same-object primitives sharing a vertex are skipped,
// triangle-triangle and rod-rod are no-ops, triangle-sphere runs the CCD
// (DetectedCollisionType::TriangleRigid = 2).  Detections are kept in
// ascending key order, as _handleDetectedCollisions sorts them.
static void narrow_phase(Ctx& c) {
    c.detected.clear();
    for (auto [la, lb] : c.pairs) {
        unsigned a = c.sorted[la], b = c.sorted[lb];
        const Prim& A = c.prims[a];
        const Prim& B = c.prims[b];
        if (A.object_id == B.object_id) {
            bool share = false;
            for (int i = 0; i < A.np; i++)
                for (int j = 0; j < B.np; j++) share |= A.idx[i] == B.idx[j];
            if (share) continue;
        }
        unsigned ia = a, ib = b;
        if (c.prims[ia].type > c.prims[ib].type) std::swap(ia, ib);
        const Prim& P = c.prims[ia];
        const Prim& Q = c.prims[ib];
        // sphere-rod has no case and sphere-sphere throws (CollisionDetector.cpp:180-213,678-687)
        if (Q.type == 2 && P.type != 0) throw std::runtime_error("Unsupported collision!");
        if (P.type == 0 && Q.type == 2) {
            Ctx::Detected d;
            if (tri_sphere_ccd(c, P, Q, d.normal, d.barys, d.cp_local)) {
                d.key = collision_key(2, ia, ib, 0);
                d.type = 2;
                d.tri[0] = P.idx[0]; d.tri[1] = P.idx[1]; d.tri[2] = P.idx[2];
                d.rb = Q.idx[0];
                c.detected.push_back(d);
            }
        } else if (P.type == 0 && Q.type == 1) {
            Ctx::Detected d;
            if (tri_rod_contact(c, P, Q, d.normal, d.barys, d.s, d.cp_local)) {
                d.key = collision_key(3, ia, ib, 0);   // DetectedCollisionType::TriangleRod
                d.type = 3;
                d.tri[0] = P.idx[0]; d.tri[1] = P.idx[1]; d.tri[2] = P.idx[2];
                d.rod[0] = Q.idx[0]; d.rod[1] = Q.idx[1];
                c.detected.push_back(d);
            }
        }
    }
    std::stable_sort(c.detected.begin(), c.detected.end(),
                     [](const Ctx::Detected& x, const Ctx::Detected& y) { return x.key < y.key; });
}

// ------------------------------------------------ dynamic contact energies
static constexpr unsigned DIRTY_SENTINEL = 0xFFFFFFFFu;   // ColorList::SENTINEL

// Eigen's MatrixBase::unitOrthogonal for a 3-vector (Eigen 3.3+, the
// third-party library of the reference; the published behaviour: a unit
// vector orthogonal to v, built from (x, y) unless both are negligible next
// to z at dummy precision 1e-12, then from (y, z)).
static V3 unit_orthogonal(V3 v) {
    const double prec = 1e-12;
    auto negligible = [&](double a, double b) { return std::fabs(a) <= std::fabs(b) * prec; };
    if (!negligible(v.x, v.z) || !negligible(v.y, v.z)) {
        double inv = 1.0 / std::sqrt(v.x * v.x + v.y * v.y);
        return V3(-v.y * inv, v.x * inv, 0.0);
    }
    double inv = 1.0 / std::sqrt(v.y * v.y + v.z * v.z);
    return V3(0.0, -v.z * inv, v.y * inv);
}

// Math::completeOrthonormalBasisGivenNormal (common/Math.hpp:323-327)
static void normal_basis(V3 n, V3& t, V3& b) {
    t = unit_orthogonal(n);
    b = cross(n, t);
}

// CollisionConstraintEnergySolver::updateCollisionFrame
// (energy/collision/CollisionConstraintEnergySolver.hpp:17-53): the tangent is
// carried over by projection, the friction multipliers keep the force
static void update_frame(Contact& e, V3 nn) {
    V3 f = e.lam_t * e.t + e.lam_b * e.b;
    V3 tp = e.t - dot(e.t, nn) * nn;
    double m = norm(tp);
    if (m > 1e-8) {
        e.t = tp / m;
        e.b = cross(nn, e.t);
    } else {
        normal_basis(nn, e.t, e.b);
    }
    e.n = nn;
    e.lam_t = dot(f, e.t);
    e.lam_b = dot(f, e.b);
}

// ColorList::markParticleDirty (common/ColorList.hpp:365-378)
static void mark_dirty(Ctx& c, unsigned p) {
    if (c.last_dirty[p] != 0) {
        c.last_dirty[p] = 0;
        c.touched_frame.push_back(p);
        c.dirty.push_back(p);
    }
}

// CollisionDetector::_addCollision, TriangleRigid case (collision/CollisionDetector.cpp:336-378)
static void add_contact(Ctx& c, Ctx::Detected& d) {
    double mn = std::min({c.m[d.tri[0]], c.m[d.tri[1]], c.m[d.tri[2]], c.m[d.rb]});
    double ks = mn / (c.dt * c.dt);
    V3 t, b;
    normal_basis(d.normal, t, b);
    unsigned slot = c.trc_pool.alloc();
    if (slot >= c.trc.size()) c.trc.resize(slot + 1);
    TriRigid& e = c.trc[slot];
    e = TriRigid{};
    // CollisionConstraintEnergyPool::addEnergy (energy/collision/CollisionConstraintEnergyPool.hpp:48-69)
    e.lam_n = e.lam_t = e.lam_b = 0;
    e.k_start = e.k_n = e.k_t = e.k_b = ks;
    e.cn_prev = 0;
    e.mu_s = 0.4; e.mu_k = 0.2;
    e.use_static = false; e.unclamped = false;
    e.p[0] = d.tri[0]; e.p[1] = d.tri[1]; e.p[2] = d.tri[2]; e.p[3] = d.rb;
    e.n = d.normal; e.t = t; e.b = b;
    e.barys = d.barys;
    e.cp_local = d.cp_local;
    d.e_idx = slot;
    for (int k = 0; k < 3; k++) mark_dirty(c, d.tri[k]);
    mark_dirty(c, d.rb);
}

// CollisionDetector::_addCollision, TriangleRod case (collision/CollisionDetector.cpp:379-418)
static void add_rod_contact(Ctx& c, Ctx::Detected& d) {
    double mn = std::min({c.m[d.tri[0]], c.m[d.tri[1]], c.m[d.tri[2]], c.m[d.rod[0]], c.m[d.rod[1]]});
    double ks = mn / (c.dt * c.dt);
    V3 t, b;
    normal_basis(d.normal, t, b);
    unsigned slot = c.trd_pool.alloc();
    if (slot >= c.trd.size()) c.trd.resize(slot + 1);
    TriRod& e = c.trd[slot];
    e = TriRod{};
    e.lam_n = e.lam_t = e.lam_b = 0;
    e.k_start = e.k_n = e.k_t = e.k_b = ks;
    e.cn_prev = 0;
    e.mu_s = 0.4; e.mu_k = 0.2;
    e.use_static = false; e.unclamped = false;
    for (int k = 0; k < 3; k++) e.p[k] = d.tri[k];
    e.p[3] = d.rod[0]; e.p[4] = d.rod[1];
    e.n = d.normal; e.t = t; e.b = b;
    e.barys = d.barys;
    e.s = d.s;
    e.cp_local = d.cp_local;
    d.e_idx = slot;
    for (int k = 0; k < 3; k++) mark_dirty(c, d.tri[k]);
    mark_dirty(c, d.rod[0]);
    mark_dirty(c, d.rod[1]);
}

// CollisionDetector::_updateCollision (collision/CollisionDetector.cpp:460-491)
static void update_contact(Ctx& c, const Ctx::Detected& d) {
    if (d.type == 2) {
        TriRigid& e = c.trc[d.e_idx];
        e.cp_local = d.cp_local;
        e.barys = d.barys;
        update_frame(e, d.normal);
    } else {
        TriRod& e = c.trd[d.e_idx];
        e.s = d.s;
        e.cp_local = d.cp_local;
        e.barys = d.barys;
        update_frame(e, d.normal);
    }
}

static void add_any(Ctx& c, Ctx::Detected& d) {
    if (d.type == 2) add_contact(c, d);
    else add_rod_contact(c, d);
}
// CollisionDetector::_removeCollision (collision/CollisionDetector.cpp:421-458)
static void remove_any(Ctx& c, const Ctx::Detected& d) {
    if (d.type == 2) c.trc_pool.free(d.e_idx);
    else c.trd_pool.free(d.e_idx);
}

// CollisionDetector::_handleDetectedCollisions (collision/CollisionDetector.cpp:265-318):
// merge of this stage's detections with the last stage's, both in ascending
// key order.  Collision primitives are never removed here, so the generation
// check of equal keys always passes.
static void handle_detections(Ctx& c) {
    auto& cur = c.contacts;
    auto& prev = c.prev_contacts;
    size_t i = 0, j = 0;
    while (i < cur.size() && j < prev.size()) {
        if (cur[i].key < prev[j].key) {
            add_any(c, cur[i++]);
        } else if (cur[i].key > prev[j].key) {
            remove_any(c, prev[j++]);
        } else {
            cur[i].e_idx = prev[j].e_idx;
            update_contact(c, cur[i]);
            i++;
            j++;
        }
    }
    for (; i < cur.size(); i++) add_any(c, cur[i]);
    for (; j < prev.size(); j++) remove_any(c, prev[j]);
}

// DynamicParticleAdjacency::buildAdjacency (common/DynamicParticleAdjacency.hpp:33-118):
// per particle its contact entries, triangle-rigid then triangle-rod, each in
// slot order; neighbours with repeats
static void build_dynamic_adjacency(Ctx& c) {
    const unsigned n = c.np();
    c.dyn_off.assign(n + 1, 0);
    c.dnb_off.assign(n + 1, 0);
    auto count = [&](const unsigned* ps, int np_) {
        for (int k = 0; k < np_; k++) { c.dyn_off[ps[k] + 1]++; c.dnb_off[ps[k] + 1] += np_ - 1; }
    };
    for (unsigned s = 0; s < c.trc_pool.size(); s++)
        if (c.trc_pool.active[s]) count(c.trc[s].p, 4);
    for (unsigned s = 0; s < c.trd_pool.size(); s++)
        if (c.trd_pool.active[s]) count(c.trd[s].p, 5);
    for (unsigned p = 0; p < n; p++) { c.dyn_off[p + 1] += c.dyn_off[p]; c.dnb_off[p + 1] += c.dnb_off[p]; }
    c.dyn_ent.assign(c.dyn_off[n], DynEnt{0, 0u, (uint16_t)0});
    c.dnb.assign(c.dnb_off[n], 0);
    std::vector<unsigned> ec(c.dyn_off.begin(), c.dyn_off.end() - 1), nc(c.dnb_off.begin(), c.dnb_off.end() - 1);
    auto scatter = [&](uint8_t type, unsigned slot, const unsigned* ps, int np_) {
        for (int k = 0; k < np_; k++) {
            unsigned p = ps[k];
            c.dyn_ent[ec[p]++] = DynEnt{type, slot, (uint16_t)k};
            for (int k2 = 0; k2 < np_; k2++)
                if (k2 != k) c.dnb[nc[p]++] = ps[k2];
        }
    };
    for (unsigned s = 0; s < c.trc_pool.size(); s++)
        if (c.trc_pool.active[s]) scatter(DYN_TRI_RIGID, s, c.trc[s].p, 4);
    for (unsigned s = 0; s < c.trd_pool.size(); s++)
        if (c.trd_pool.active[s]) scatter(DYN_TRI_ROD, s, c.trd[s].p, 5);
}

// ForEachNeighbor (common/ColorList.hpp:41-60): static, then dynamic neighbours
template <typename F>
static void for_each_neighbor(const Ctx& c, unsigned p, F&& f) {
    for (unsigned k = c.p_off[p]; k < c.p_off[p + 1]; k++) f(c.p_nbr[k]);
    if (!c.dnb_off.empty())
        for (unsigned k = c.dnb_off[p]; k < c.dnb_off[p + 1]; k++) f(c.dnb[k]);
}

// ColorList::finalizeConflicts (common/ColorList.hpp:476-522)
static void finalize_conflicts(Ctx& c) {
    for (unsigned p : c.dirty)
        for_each_neighbor(c, p, [&](unsigned q) {
            if (c.color[q] == c.color[p]) {
                if (!c.conflicted[p]) { c.conflicted[p] = 1; c.touched_conflicted.push_back(p); }
                if (!c.conflicted[q]) { c.conflicted[q] = 1; c.touched_conflicted.push_back(q); }
            }
        });
    std::vector<unsigned> cnt(c.num_colors, 0);
    for (unsigned p : c.touched_conflicted) cnt[c.color[p]]++;
    c.conf_off.assign(c.num_colors + 1, 0);
    for (unsigned k = 0; k < c.num_colors; k++) c.conf_off[k + 1] = c.conf_off[k] + cnt[k];
    c.conf_list.assign(c.conf_off.back(), 0);
    std::vector<unsigned> cur(c.conf_off.begin(), c.conf_off.end() - 1);
    for (unsigned p : c.touched_conflicted) c.conf_list[cur[c.color[p]]++] = p;
}

// ColorList::incrementalRecoloring (common/ColorList.hpp:381-474): at most six
// rounds; a dirty particle with a same-colored neighbour of lower index takes
// the first color unused by its neighbours (256 colors at most); a changed
// color makes every neighbour dirty for the next round.  Particles still dirty
// after the last round stay dirty for the next stage, and they and their
// same-colored neighbours are marked conflicted.
static void incremental_recoloring(Ctx& c) {
    const unsigned MAX_ROUNDS = c.recolor_rounds;
    for (unsigned p : c.touched_conflicted) c.conflicted[p] = 0;
    c.touched_conflicted.clear();
    unsigned iter = 0;
    while (!c.dirty.empty() && iter < MAX_ROUNDS) {
        for (unsigned p : c.dirty) {
            uint64_t bits[4] = {0, 0, 0, 0};
            bool must = false;
            for_each_neighbor(c, p, [&](unsigned q) {
                unsigned cq = c.color[q];
                if (cq >= 256) throw std::runtime_error("Ran out of colors!");
                bits[cq / 64] |= 1ull << (cq % 64);
                if (cq == c.color[p] && q < p) must = true;
            });
            if (must) {
                unsigned cand = UINT32_MAX;
                for (unsigned w = 0; w < 4 && cand == UINT32_MAX; w++)
                    if (~bits[w]) cand = w * 64 + (unsigned)__builtin_ctzll(~bits[w]);
                if (cand == UINT32_MAX) throw std::runtime_error("Ran out of colors!");
                c.cand_color[p] = cand;
                if (cand >= c.num_colors) c.num_colors++;
            } else {
                c.cand_color[p] = c.color[p];
            }
        }
        c.next_dirty.clear();
        for (unsigned p : c.dirty) {
            if (c.cand_color[p] == c.color[p]) continue;
            c.color[p] = c.cand_color[p];
            for_each_neighbor(c, p, [&](unsigned q) {
                if (c.last_dirty[q] != iter + 1) {
                    c.last_dirty[q] = iter + 1;
                    c.touched_frame.push_back(q);
                    c.next_dirty.push_back(q);
                }
            });
        }
        c.dirty.swap(c.next_dirty);
        iter++;
    }
    if (!c.dirty.empty()) {
        finalize_conflicts(c);
    } else {
        c.conf_off.assign(c.num_colors + 1, 0);
        c.conf_list.clear();
    }
    rebuild_work_list(c);
    for (unsigned p : c.touched_frame) c.last_dirty[p] = DIRTY_SENTINEL;
    c.touched_frame.clear();
    for (unsigned p : c.dirty) c.last_dirty[p] = 0;
}

// LBVHBuilder::buildBVH + broad phase (collision/LBVHBuilder.cpp:13-25,
// collision/CollisionDetector.cpp:24-55).  Narrow phase: triangle-triangle and
// rod-rod are no-ops in the reference (CollisionDetector.cpp:589-599,668-676);
// sphere-sphere and sphere-rod throw there (CollisionDetector.cpp:180-213,678-687).
// `manage` adds the contact handling of detectCollisionsAndRecolor_Parallel
// (CollisionDetector.cpp:57-128): merge into the contact pool, dynamic
// adjacency, incremental recoloring.  Without it the stage only detects.
static void collision_stage(Ctx& c, bool manage) {
    unsigned n = (unsigned)c.prims.size();
    if (n == 0) { c.pairs.clear(); return; }
    c.aabb.assign((size_t)n * 6, 0);
    double smin[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(), std::numeric_limits<double>::max()};
    double smax[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest()};
    std::vector<double> cen((size_t)n * 3);
    for (unsigned p = 0; p < n; p++) {
        double* b = &c.aabb[(size_t)p * 6];
        spec_bounds(c, c.prims[p], b);
        for (int i = 0; i < 3; i++) {
            cen[(size_t)p * 3 + i] = (b[i] + b[3 + i]) * 0.5;
            smin[i] = dmin_(smin[i], b[i]);
            smax[i] = dmax_(smax[i], b[3 + i]);
        }
    }
    double ext[3];
    for (int i = 0; i < 3; i++) ext[i] = dmax_(smax[i] - smin[i], 1e-6);
    c.morton.assign(n, 0);
    for (unsigned p = 0; p < n; p++) {
        double nc[3];
        for (int i = 0; i < 3; i++) nc[i] = (cen[(size_t)p * 3 + i] - smin[i]) / ext[i];
        c.morton[p] = morton64(nc[0], nc[1], nc[2]);
    }
    // Algorithm::radixSort: stable LSD, 8 passes of 8 bits (common/Algorithm.hpp:22-56)
    c.sorted.resize(n);
    std::iota(c.sorted.begin(), c.sorted.end(), 0u);
    std::vector<unsigned> tmp(n);
    for (int sh = 0; sh < 64; sh += 8) {
        size_t cnt[256] = {};
        for (unsigned i : c.sorted) cnt[(c.morton[i] >> sh) & 255]++;
        size_t s = 0;
        for (int b = 0; b < 256; b++) { size_t t = cnt[b]; cnt[b] = s; s += t; }
        for (unsigned i : c.sorted) tmp[cnt[(c.morton[i] >> sh) & 255]++] = i;
        c.sorted.swap(tmp);
    }
    construct_tree(c, n);
    refit(c, n);
    traverse(c);
    narrow_phase(c);
    if (!manage) return;
    c.prev_contacts.swap(c.contacts);
    c.contacts = c.detected;
    handle_detections(c);
    build_dynamic_adjacency(c);
    incremental_recoloring(c);
}

}  // namespace orc

// =================================================================== C API
using namespace orc;

static thread_local std::string g_err;

#define ORC_TRY(body) try { body; return 0; } catch (const std::exception& ex) { g_err = ex.what(); return 2; }

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

void* orc_create(void) { return new Ctx(); }
void orc_destroy(void* h) { delete (Ctx*)h; }

void orc_set_params(void* h, double dt, double g, double margin) {
    Ctx& c = *(Ctx*)h; c.dt = dt; c.g = g; c.margin = margin;
}
void orc_set_solver(void* h, unsigned iters, double rho, double tol, unsigned max_iters) {
    Ctx& c = *(Ctx*)h; c.iters = iters; c.rho = rho; c.tol = tol; c.max_iters = max_iters;
}
void orc_set_threads(void* h, int n) {
    Ctx& c = *(Ctx*)h;
    c.nthreads = n < 1 ? 1 : n;
    c.pool.start(c.nthreads);
}

// Scenes are disjoint components; DSATUR over disjoint components colors each
// component exactly as a separate context would, so no bookkeeping is needed.
void orc_begin_scene(void* h) { ((Ctx*)h)->num_scenes++; }

// ParticlePool::addParticle (common/ParticlePool.hpp:217-240)
unsigned orc_particles_add(void* h, unsigned n, const double* pos, const double* mass) {
    Ctx& c = *(Ctx*)h;
    unsigned first = c.np();
    bool first_scene = c.x.empty();
    for (unsigned i = 0; i < n; i++) {
        V3 p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        c.x.push_back(p); c.xb.push_back(p); c.y.push_back(p); c.xp.push_back(p); c.xl.push_back(p); c.xll.push_back(p);
        c.v.push_back(V3()); c.vp.push_back(V3());
        c.m.push_back(mass[i]); c.fixed.push_back(0); c.rot.push_back(UINT32_MAX);
        c.scene_of.push_back(first_scene ? 0 : c.num_scenes - 1);
    }
    return first;
}
// ParticlePool::addOrientedParticle (common/ParticlePool.hpp:257-263)
unsigned orc_particles_add_oriented(void* h, unsigned n, const double* pos, const double* quat,
                                    const double* mass, const double* inertia) {
    Ctx& c = *(Ctx*)h;
    unsigned first = orc_particles_add(h, n, pos, mass);
    for (unsigned i = 0; i < n; i++) {
        Q4 q{quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]};
        c.rot[first + i] = (unsigned)c.q.size();
        c.q.push_back(q); c.qb.push_back(q); c.qy.push_back(q); c.qp.push_back(q); c.ql.push_back(q); c.qll.push_back(q);
        c.w.push_back(V3()); c.wp.push_back(V3());
        c.I.push_back(V3(inertia[3 * i], inertia[3 * i + 1], inertia[3 * i + 2]));
    }
    return first;
}
void orc_set_fixed(void* h, unsigned n, const unsigned* idx, const uint8_t* f) {
    Ctx& c = *(Ctx*)h; for (unsigned i = 0; i < n; i++) c.fixed[idx[i]] = f[i];
}
void orc_set_velocities(void* h, unsigned first, unsigned n, const double* v, const double* vp) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < n; i++) {
        c.v[first + i] = V3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
        const double* s = vp ? vp : v;
        c.vp[first + i] = V3(s[3 * i], s[3 * i + 1], s[3 * i + 2]);
    }
}
void orc_set_positions_raw(void* h, unsigned first, unsigned n, const double* x) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < n; i++) c.x[first + i] = V3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
}
void orc_set_rotations_raw(void* h, unsigned first, unsigned n, const double* q) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < n; i++) c.q[c.rot[first + i]] = Q4{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
}
void orc_set_angular_velocities(void* h, unsigned first, unsigned n, const double* w) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < n; i++)
        if (c.oriented(first + i)) c.w[c.rot[first + i]] = V3(w[3 * i], w[3 * i + 1], w[3 * i + 2]);
}
void orc_get_positions(void* h, double* out) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < c.np(); i++) { out[3 * i] = c.x[i].x; out[3 * i + 1] = c.x[i].y; out[3 * i + 2] = c.x[i].z; }
}
void orc_get_velocities(void* h, double* out) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < c.np(); i++) { out[3 * i] = c.v[i].x; out[3 * i + 1] = c.v[i].y; out[3 * i + 2] = c.v[i].z; }
}
void orc_get_rotations(void* h, double* out) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < c.np(); i++) {
        Q4 q = c.oriented(i) ? c.q[c.rot[i]] : Q4();
        out[4 * i] = q.w; out[4 * i + 1] = q.x; out[4 * i + 2] = q.y; out[4 * i + 3] = q.z;
    }
}
void orc_get_angular_velocities(void* h, double* out) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < c.np(); i++) {
        V3 w = c.oriented(i) ? c.w[c.rot[i]] : V3();
        out[3 * i] = w.x; out[3 * i + 1] = w.y; out[3 * i + 2] = w.z;
    }
}
unsigned orc_num_particles(void* h) { return ((Ctx*)h)->np(); }

unsigned orc_neo_hookean_add(void* h, unsigned n, const unsigned* idx, const double* lam, const double* mu,
                             const double* kd, const double* Q, const double* V) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.nh.size();
    for (unsigned i = 0; i < n; i++) {
        NH e;
        for (int k = 0; k < 4; k++) e.idx[k] = idx[4 * i + k];
        e.lambda = lam[i]; e.mu = mu[i]; e.kd = kd[i]; e.V = V[i];
        for (int r = 0; r < 3; r++) for (int s = 0; s < 3; s++) e.Q.a[r][s] = Q[9 * i + 3 * r + s];
        c.nh.push_back(e);
    }
    return first;
}
unsigned orc_cosserat_rod_add(void* h, unsigned n, const unsigned* idx, const double* K, const double* L,
                              const double* kappa) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.rods.size();
    for (unsigned i = 0; i < n; i++) {
        Rod e;
        e.idx[0] = idx[2 * i]; e.idx[1] = idx[2 * i + 1];
        for (int k = 0; k < 6; k++) e.K[k] = K[6 * i + k];
        e.L = L[i];
        e.kappa0 = V3(kappa[3 * i], kappa[3 * i + 1], kappa[3 * i + 2]);
        c.rods.push_back(e);
    }
    return first;
}
// CollisionConstraintEnergyPool::addEnergy (energy/collision/CollisionConstraintEnergyPool.hpp:48-69)
static void init_contact(Contact& e, double ks, double ms, double mk) {
    e.lam_n = e.lam_t = e.lam_b = 0;
    e.k_start = e.k_n = e.k_t = e.k_b = ks;
    e.cn_prev = 0; e.mu_s = ms; e.mu_k = mk; e.use_static = false; e.unclamped = false;
}
unsigned orc_ground_add(void* h, unsigned n, const unsigned* p, const double* ks, const double* ms, const double* mk) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.ground.size();
    for (unsigned i = 0; i < n; i++) {
        Ground e; init_contact(e, ks[i], ms[i], mk[i]); e.p = p[i]; e.cp_x = e.cp_z = 0;
        c.ground.push_back(e);
    }
    return first;
}
unsigned orc_rigid_ground_add(void* h, unsigned n, const unsigned* p, const uint8_t* shape, const double* radius,
                              const double* cpl, const double* ks, const double* ms, const double* mk) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.rground.size();
    for (unsigned i = 0; i < n; i++) {
        RGround e; init_contact(e, ks[i], ms[i], mk[i]);
        e.p = p[i]; e.shape = shape[i]; e.radius = radius[i];
        e.cp_local = V3(cpl[3 * i], cpl[3 * i + 1], cpl[3 * i + 2]);
        e.cp_ground = V3();
        e.n = V3(0, 1, 0); e.t = V3(1, 0, 0); e.b = V3(0, 0, 1);
        c.rground.push_back(e);
    }
    return first;
}
unsigned orc_joint_add(void* h, unsigned n, const unsigned* p, const double* po, const double* ro,
                       const double* rp, const double* rq) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.joints.size();
    for (unsigned i = 0; i < n; i++) {
        Joint e;
        e.p = p[i];
        for (int k = 0; k < 6; k++) { e.k[k] = c.joint_k_start; e.lam[k] = 0; e.cprev[k] = 0; }
        e.pos_off = V3(po[3 * i], po[3 * i + 1], po[3 * i + 2]);
        e.rot_off = Q4{ro[4 * i], ro[4 * i + 1], ro[4 * i + 2], ro[4 * i + 3]};
        e.ref_p = V3(rp[3 * i], rp[3 * i + 1], rp[3 * i + 2]);
        e.ref_q = Q4{rq[4 * i], rq[4 * i + 1], rq[4 * i + 2], rq[4 * i + 3]};
        c.joints.push_back(e);
    }
    return first;
}
unsigned orc_add_triangles(void* h, unsigned n, const unsigned* idx, unsigned obj) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.prims.size();
    for (unsigned i = 0; i < n; i++) c.prims.push_back(Prim{0, {idx[3 * i], idx[3 * i + 1], idx[3 * i + 2]}, 3, obj, 0});
    return first;
}
unsigned orc_add_rod_segments(void* h, unsigned n, const unsigned* idx, double radius, unsigned obj) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.prims.size();
    for (unsigned i = 0; i < n; i++) c.prims.push_back(Prim{1, {idx[2 * i], idx[2 * i + 1], 0}, 2, obj, radius});
    return first;
}
unsigned orc_add_spheres(void* h, unsigned n, const unsigned* p, const double* r, const unsigned* obj) {
    Ctx& c = *(Ctx*)h;
    unsigned first = (unsigned)c.prims.size();
    for (unsigned i = 0; i < n; i++) c.prims.push_back(Prim{2, {p[i], 0, 0}, 1, obj[i], r[i]});
    return first;
}

// 0 = heap DSATUR, 1 = verbatim O(V^2) DSATUR
int orc_finalize(void* h, int reference_dsatur) {
    Ctx& c = *(Ctx*)h;
    ORC_TRY({
        for (const Prim& pr : c.prims)
            if (pr.type == 1 && (!c.oriented(pr.idx[0]) || !c.oriented(pr.idx[1])))
                throw std::runtime_error("rod segment primitive on a positional particle");
        build_adjacency(c);
        if (reference_dsatur) dsatur_reference(c); else dsatur_fast(c);
        if (c.num_colors > 256) throw std::runtime_error("Ran out of colors!");
        rebuild_work_list(c);
        const unsigned n = c.np();
        c.last_dirty.assign(n, DIRTY_SENTINEL);
        c.cand_color.assign(n, 0);
        c.conflicted.assign(n, 0);
        c.buffered.assign(n, V3());
        c.conf_off.assign(c.num_colors + 1, 0);
        c.finalized = true;
    });
}

int orc_step(void* h, unsigned n) {
    Ctx& c = *(Ctx*)h;
    if (!c.finalized) { g_err = "finalize first"; return 8; }
    ORC_TRY({ for (unsigned s = 0; s < n; s++) time_step(c); });
}

// Wall time (seconds) of n steps, the CPU-baseline measurement.
double orc_time_steps(void* h, unsigned n) {
    Ctx& c = *(Ctx*)h;
    auto t0 = std::chrono::steady_clock::now();
    for (unsigned s = 0; s < n; s++) time_step(c);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

int orc_collision_stage(void* h) { ORC_TRY(collision_stage(*(Ctx*)h, false)); }
void orc_after_time_step(void* h) { after_time_step(*(Ctx*)h); }

void orc_get_coloring(void* h, unsigned* colors, unsigned* num_colors) {
    Ctx& c = *(Ctx*)h;
    for (unsigned i = 0; i < c.np(); i++) colors[i] = c.color[i];
    *num_colors = c.num_colors;
}
unsigned orc_num_entries(void* h) { return (unsigned)((Ctx*)h)->entries.size(); }
void orc_get_adjacency(void* h, unsigned* e_off, uint8_t* type, unsigned* idx, uint16_t* local,
                       unsigned* p_off, unsigned* p_nbr) {
    Ctx& c = *(Ctx*)h;
    if (e_off) std::copy(c.e_off.begin(), c.e_off.end(), e_off);
    for (size_t k = 0; k < c.entries.size(); k++) {
        if (type) type[k] = c.entries[k].type;
        if (idx) idx[k] = c.entries[k].idx;
        if (local) local[k] = c.entries[k].local;
    }
    if (p_off) std::copy(c.p_off.begin(), c.p_off.end(), p_off);
    if (p_nbr) std::copy(c.p_nbr.begin(), c.p_nbr.end(), p_nbr);
}
unsigned orc_num_neighbors(void* h) { return (unsigned)((Ctx*)h)->p_nbr.size(); }

unsigned orc_num_pairs(void* h) { return (unsigned)((Ctx*)h)->pairs.size(); }
// contacts of the last collision stage: per contact key, tri[3], rigid,
// normal[3], barys[3], cp_local[3] (ascending key)
unsigned orc_get_contacts(void* h, uint64_t* keys, unsigned* idx4, double* vec9) {
    Ctx& c = *(Ctx*)h;
    std::vector<Ctx::Detected> sph;
    for (const auto& d : c.detected)
        if (d.type == 2) sph.push_back(d);
    for (size_t k = 0; k < sph.size(); k++) {
        const auto& d = sph[k];
        if (keys) keys[k] = d.key;
        if (idx4) { idx4[4 * k] = d.tri[0]; idx4[4 * k + 1] = d.tri[1]; idx4[4 * k + 2] = d.tri[2]; idx4[4 * k + 3] = d.rb; }
        if (vec9) {
            for (int i = 0; i < 3; i++) {
                vec9[9 * k + i] = d.normal[i];
                vec9[9 * k + 3 + i] = d.barys[i];
                vec9[9 * k + 6 + i] = d.cp_local[i];
            }
        }
    }
    return (unsigned)sph.size();
}

// triangle-rod contacts of the last collision stage: key, tri[3] + rod[2],
// normal[3], barys[3], cp_local[3], s (ascending key)
unsigned orc_get_rod_contacts(void* h, uint64_t* keys, unsigned* idx5, double* vec10) {
    Ctx& c = *(Ctx*)h;
    unsigned k = 0;
    for (const auto& d : c.detected) {
        if (d.type != 3) continue;
        if (keys) keys[k] = d.key;
        if (idx5) {
            for (int i = 0; i < 3; i++) idx5[5 * k + i] = d.tri[i];
            idx5[5 * k + 3] = d.rod[0];
            idx5[5 * k + 4] = d.rod[1];
        }
        if (vec10) {
            for (int i = 0; i < 3; i++) {
                vec10[10 * k + i] = d.normal[i];
                vec10[10 * k + 3 + i] = d.barys[i];
                vec10[10 * k + 6 + i] = d.cp_local[i];
            }
            vec10[10 * k + 9] = d.s;
        }
        k++;
    }
    return k;
}

// Dynamic contact state: [0] live triangle-rigid contacts, [1] their pool
// size (highest slot + 1), [2] colors, [3] conflicted particles, [4]
// particles still dirty, [5] dynamic adjacency entries, [6] live
// triangle-rod contacts, [7] their pool size
void orc_dynamic_info(void* h, unsigned* out) {
    Ctx& c = *(Ctx*)h;
    out[0] = c.trc_pool.count;
    out[1] = c.trc_pool.size();
    out[2] = c.num_colors;
    out[3] = (unsigned)c.touched_conflicted.size();
    out[4] = (unsigned)c.dirty.size();
    out[5] = (unsigned)c.dyn_ent.size();
    out[6] = c.trd_pool.count;
    out[7] = c.trd_pool.size();
}

// Triangle-rod pool slots [0, pool size): particles (5 per slot), active flag,
// and 25 doubles per slot: n, t, b, barys, cp_local, s, k_start, k_n, k_t,
// k_b, lam_n, lam_t, lam_b, C_n_prev, use_static + 2 unclamped
void orc_get_trd(void* h, unsigned* p5, uint8_t* active, double* data) {
    Ctx& c = *(Ctx*)h;
    for (size_t s = 0; s < c.trd_pool.size(); s++) {
        const TriRod& e = c.trd[s];
        if (p5) for (int k = 0; k < 5; k++) p5[5 * s + k] = e.p[k];
        if (active) active[s] = c.trd_pool.active[s];
        if (data) {
            double* d = data + 25 * s;
            const V3 v[5] = {e.n, e.t, e.b, e.barys, e.cp_local};
            for (int i = 0; i < 5; i++) for (int j = 0; j < 3; j++) d[3 * i + j] = v[i][j];
            d[15] = e.s;
            d[16] = e.k_start; d[17] = e.k_n; d[18] = e.k_t; d[19] = e.k_b;
            d[20] = e.lam_n; d[21] = e.lam_t; d[22] = e.lam_b; d[23] = e.cn_prev;
            d[24] = (e.use_static ? 1 : 0) + (e.unclamped ? 2 : 0);
        }
    }
}

// Contact pool slots [0, pool size): particles (4 per slot), active flag, and
// 24 doubles per slot: n, t, b, barys, cp_local, k_start, k_n, k_t, k_b,
// lam_n, lam_t, lam_b, C_n_prev, use_static + 2 unclamped
void orc_get_trc(void* h, unsigned* p4, uint8_t* active, double* data) {
    Ctx& c = *(Ctx*)h;
    for (size_t s = 0; s < c.trc_pool.size(); s++) {
        const TriRigid& e = c.trc[s];
        if (p4) for (int k = 0; k < 4; k++) p4[4 * s + k] = e.p[k];
        if (active) active[s] = c.trc_pool.active[s];
        if (data) {
            double* d = data + 24 * s;
            const V3 v[5] = {e.n, e.t, e.b, e.barys, e.cp_local};
            for (int i = 0; i < 5; i++) for (int j = 0; j < 3; j++) d[3 * i + j] = v[i][j];
            d[15] = e.k_start; d[16] = e.k_n; d[17] = e.k_t; d[18] = e.k_b;
            d[19] = e.lam_n; d[20] = e.lam_t; d[21] = e.lam_b; d[22] = e.cn_prev;
            d[23] = (e.use_static ? 1 : 0) + (e.unclamped ? 2 : 0);
        }
    }
}

// test hook: the recoloring's round limit (6 in the reference)
void orc_set_recolor_rounds(void* h, unsigned rounds) { ((Ctx*)h)->recolor_rounds = rounds; }

// per-particle conflict flags of the last recoloring
void orc_get_conflicted(void* h, uint8_t* out) {
    Ctx& c = *(Ctx*)h;
    for (unsigned p = 0; p < c.np(); p++) out[p] = c.conflicted.empty() ? 0 : c.conflicted[p];
}
void orc_get_lbvh(void* h, uint64_t* morton, unsigned* sorted, unsigned* left, unsigned* right, unsigned* parent,
                  unsigned* subtree, double* bounds, unsigned* root, unsigned* pairs) {
    Ctx& c = *(Ctx*)h;
    unsigned n = (unsigned)c.prims.size();
    if (morton) std::copy(c.morton.begin(), c.morton.end(), morton);
    if (sorted) std::copy(c.sorted.begin(), c.sorted.end(), sorted);
    if (n == 0) return;
    if (left) std::copy(c.left.begin(), c.left.end(), left);
    if (right) std::copy(c.right.begin(), c.right.end(), right);
    if (parent) std::copy(c.parent.begin(), c.parent.end(), parent);
    if (subtree) std::copy(c.subtree.begin(), c.subtree.end(), subtree);
    if (bounds) std::copy(c.nbounds.begin(), c.nbounds.end(), bounds);
    if (root) *root = c.root;
    if (pairs) for (size_t k = 0; k < c.pairs.size(); k++) { pairs[2 * k] = c.pairs[k].first; pairs[2 * k + 1] = c.pairs[k].second; }
}

// Karras tree + refit + traversal on caller-provided codes and boxes
// (the inputs of test/test_lbvh.cpp:31-70 and :168-301).
int orc_lbvh_from_codes(void* h, unsigned n, const uint64_t* codes, const double* boxes) {
    Ctx& c = *(Ctx*)h;
    if (n == 0) { c.pairs.clear(); return 0; }
    ORC_TRY({
        c.prims.assign(n, Prim{0, {0, 0, 0}, 0, 0, 0});
        c.morton.assign(codes, codes + n);
        c.aabb.assign((size_t)n * 6, 0);
        if (boxes) std::copy(boxes, boxes + (size_t)n * 6, c.aabb.begin());
        c.sorted.resize(n);
        std::iota(c.sorted.begin(), c.sorted.end(), 0u);
        std::stable_sort(c.sorted.begin(), c.sorted.end(), [&](unsigned a, unsigned b) { return c.morton[a] < c.morton[b]; });
        construct_tree(c, n);
        refit(c, n);
        traverse(c);
    });
}

int orc_debug_block(void* h, unsigned p, double* G, double* H, int* dof) {
    Ctx& c = *(Ctx*)h;
    if (c.oriented(p)) {
        double HH[6][6], GG[6];
        accumulate_block<6>(c, p, HH, GG);
        for (int i = 0; i < 6; i++) { G[i] = GG[i]; for (int j = 0; j < 6; j++) H[6 * i + j] = HH[i][j]; }
        *dof = 6;
    } else {
        double HH[3][3], GG[3];
        accumulate_block<3>(c, p, HH, GG);
        for (int i = 0; i < 3; i++) { G[i] = GG[i]; for (int j = 0; j < 3; j++) H[3 * i + j] = HH[i][j]; }
        *dof = 3;
    }
    return 0;
}

// Per-element energies (NeoHookeanEnergySolver::energy, CosseratRodEnergySolver::energy,
// HardConstraintEnergySolver::energy) for the finite-difference checks.
double orc_energy(void* h, int type, unsigned slot) {
    Ctx& c = *(Ctx*)h;
    switch (type) {
        case NEO_HOOKEAN: return nh_energy(c, c.nh[slot], c.dt);
        case COSSERAT_ROD: return rod_energy(c, c.rods[slot]);
        case JOINT: return joint_energy(c, c.joints[slot]);
    }
    return 0;
}
// Single-element accumulate for the finite-difference checks (no adjacency needed).
void orc_element_accumulate(void* h, int type, unsigned slot, unsigned local, double* G, double* H) {
    Ctx& c = *(Ctx*)h;
    if (type == NEO_HOOKEAN) {
        double HH[3][3] = {}, GG[3] = {};
        nh_accumulate(c, c.nh[slot], local, HH, GG, c.dt);
        for (int i = 0; i < 3; i++) { G[i] = GG[i]; for (int j = 0; j < 3; j++) H[3 * i + j] = HH[i][j]; }
    } else {
        double HH[6][6] = {}, GG[6] = {};
        if (type == COSSERAT_ROD) rod_accumulate(c, c.rods[slot], local, HH, GG);
        else if (type == JOINT) joint_accumulate(c, c.joints[slot], HH, GG);
        for (int i = 0; i < 6; i++) { G[i] = GG[i]; for (int j = 0; j < 6; j++) H[6 * i + j] = HH[i][j]; }
    }
}

double orc_residual(void* h) { return residual(*(Ctx*)h); }
double orc_last_residual(void* h) { return ((Ctx*)h)->last_residual; }
unsigned long long orc_iterations(void* h) { return ((Ctx*)h)->iterations; }
// iterations each scene ran in the last run-to-tolerance step
unsigned orc_scene_iterations(void* h, unsigned* out) {
    Ctx& c = *(Ctx*)h;
    for (size_t s = 0; s < c.scene_iters.size(); s++) out[s] = c.scene_iters[s];
    return (unsigned)c.scene_iters.size();
}

// Math::Exp_s3 / Log_S3 / QuaternionFromXYZEulerAngles for test inputs
void orc_exp_s3(const double* v, double* q) {
    Q4 r = exp_s3(V3(v[0], v[1], v[2])); q[0] = r.w; q[1] = r.x; q[2] = r.y; q[3] = r.z;
}
void orc_quat_from_xyz_euler(const double* e, double* q) {  // common/Math.hpp:298-318
    double x = e[0] * M_PI / 180.0, y = e[1] * M_PI / 180.0, z = e[2] * M_PI / 180.0;
    Q4 qx{std::cos(x * 0.5), std::sin(x * 0.5), 0, 0};
    Q4 qy{std::cos(y * 0.5), 0, std::sin(y * 0.5), 0};
    Q4 qz{std::cos(z * 0.5), 0, 0, std::sin(z * 0.5)};
    Q4 r = qmul(qmul(qz, qy), qx);
    q[0] = r.w; q[1] = r.x; q[2] = r.y; q[3] = r.z;
}
void orc_plus_s3(const double* q, const double* v, double* out) {
    Q4 r = plus_s3(Q4{q[0], q[1], q[2], q[3]}, V3(v[0], v[1], v[2]));
    out[0] = r.w; out[1] = r.x; out[2] = r.y; out[3] = r.z;
}

}  // extern "C"
