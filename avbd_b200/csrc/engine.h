// engine.h -- host-side context of the engine and the launch wrappers each
// .cu file exports.  Everything here is internal; the public surface is
// include/avbd.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "../../include/avbd.h"

namespace avbd {

// ------------------------------------------------------------ device data

// One NeoHookean incidence (tet, local vertex) of a solved vertex, stored in
// the order the color phases stream them.  The tet is restated relative to the
// solved vertex i: F = sum_k (x_ok - x_i) (x) d_k over the three other
// vertices o_k, where d_k are the rows of D = [Q; -1^T Q] belonging to them
// (NeoHookeanEnergySolver::computeF, energy/elastic/NeoHookeanEnergySolver.hpp:96-109).
// The solved vertex's own row is -(d_1 + d_2 + d_3).
template <typename R> struct IncRec;
template <> struct alignas(16) IncRec<float> {
    uint32_t o[3];
    uint32_t tet;
    float d[9];
    float vlam, vmu, mol;  // V*lambda, V*mu, mu/lambda
};
template <> struct alignas(16) IncRec<double> {
    uint32_t o[3];
    uint32_t tet;
    double d[9];
    double vlam, vmu, mol;
};
static_assert(sizeof(IncRec<float>) == 64, "FP32 incidence record must be 64 B");
static_assert(sizeof(IncRec<double>) == 112, "FP64 incidence record must be 112 B");

enum VertexFlags : uint8_t { VF_FIXED = 1, VF_ORIENTED = 2, VF_GROUND = 4 };
enum GroundFlags : uint8_t { GF_USE_STATIC = 1, GF_UNCLAMPED = 2 };

// One dynamic contact pool on the device, by slot (see DevState::cp).
template <typename R>
struct ContactPoolDev {
    using V4 = typename Vec4Of<R>::T;
    unsigned cap = 0;                // slots allocated
    uint4* p = nullptr;              // internal vertex ids: triangle x3, rigid body / first rod node
    uint32_t* p5 = nullptr;          // second rod node (triangle-rod pool)
    V4* n = nullptr;                 // contact frame: normal (w: s along the segment, triangle-rod),
    V4* t = nullptr;                 //   tangent,
    V4* b = nullptr;                 //   binormal
    V4* bar = nullptr;               // barycentrics of the triangle point, mu_s in w
    V4* cpl = nullptr;               // contact point in the body (or interpolated rod) frame, mu_k in w
    V4* k = nullptr;                 // k_n, k_t, k_b, k_start
    V4* lam = nullptr;               // lam_n, lam_t, lam_b, C_n_prev
    uint8_t* flag = nullptr;         // ContactFlags
};
enum ContactPoolType { POOL_TRI_RIGID = 0, POOL_TRI_ROD = 1 };

// Device arrays of one precision.  All per-vertex arrays use the internal
// (color-major) vertex order.
template <typename R>
struct DevState {
    using V4 = typename Vec4Of<R>::T;
    unsigned n = 0;
    // xl, xll: the Chebyshev history, two buffers by iteration parity.
    // Iteration k reads o_(k-2) from buffer k&1 (xl even, xll odd) and writes
    // its accelerated iterate o_k there; both hold the step's start position
    // before iteration 0.
    V4 *x = nullptr, *y = nullptr, *xp = nullptr, *xl = nullptr, *xll = nullptr, *v = nullptr, *vp = nullptr;
    uint8_t* flags = nullptr;
    IncRec<R>* inc = nullptr;
    IncRec<float>* inc32 = nullptr;   // FP32 records of the mixed mode (double state)
    uint32_t* inc_begin = nullptr;
    // per-tet data (damping path only)
    unsigned ntets = 0;
    uint4* tet_idx = nullptr;
    V4* tet_q = nullptr;   // 3 rows per tet
    V4* tet_e = nullptr;   // E_prev (00,11,22,01) (02,12,V*kd,0) per tet
    // per-vertex ground contact (GroundCollisionEnergyInfo)
    V4* gk = nullptr;      // k_n, k_t, k_b, k_start
    V4* glam = nullptr;    // lam_n, lam_t, lam_b, C_n_prev
    V4* gcp = nullptr;     // cp_x, cp_z, mu_s, mu_k
    uint8_t* gflag = nullptr;
    int* err = nullptr;    // device-side status (AVBD_ERR_*), 0 when healthy

    // ---- oriented particles (RotationPool, common/ParticlePool.hpp:7-68).
    // rot[p] is the rotation slot of internal vertex p (UINT32_MAX if positional);
    // quaternions are stored (w, x, y, z) in the x, y, z, w fields.
    unsigned no = 0;
    uint32_t* rot = nullptr;
    V4 *q = nullptr, *qy = nullptr, *qp = nullptr, *ql = nullptr, *qll = nullptr;
    V4 *w = nullptr, *wp = nullptr, *Iv = nullptr;
    // Cosserat rods: per oriented vertex a CSR of (rod << 1 | local)
    unsigned nrods = 0;
    uint32_t* rod_begin = nullptr;   // n + 1
    uint32_t* rod_inc = nullptr;
    uint2* rod_idx = nullptr;        // internal vertex ids of the two nodes
    V4* rod_K = nullptr;             // (K0..K3), (K4, K5, rest length, 0) per rod
    V4* rod_k0 = nullptr;            // precurvature
    // rigid-body ground contact, one per rotation slot
    V4* rgk = nullptr;               // k_n, k_t, k_b, k_start
    V4* rglam = nullptr;             // lam_n, lam_t, lam_b, C_n_prev
    V4* rgcp = nullptr;              // cp_ground.x, cp_ground.z, mu_s, mu_k
    V4* rgloc = nullptr;             // cp_rb_local xyz, shape radius
    // one-sided fixed joint, one per rotation slot (6 rows)
    V4* jk = nullptr;                // k rows 0-3, 4-5 (2 per slot)
    V4* jlam = nullptr;              // lambda rows (2 per slot)
    V4* jcp = nullptr;               // C_prev rows (2 per slot)
    V4* jpo = nullptr;               // position offset
    V4* jro = nullptr;               // rotation offset (quaternion)
    V4* jrp = nullptr;               // reference position
    V4* jrq = nullptr;               // reference rotation (quaternion)
    uint8_t* oflag = nullptr;        // per rotation slot, OrientedFlags

    // ---- dynamic contacts: cp[0] triangle-rigid (TriangleRigidCollisionEnergyPool),
    // cp[1] triangle-rod (TriangleRodCollisionEnergyPool), by pool slot; the
    // host manages the pools between steps (contacts.cu)
    ContactPoolDev<R> cp[2];
    // dynamic adjacency per internal vertex, entries (slot << 4 | pool << 3 |
    // local), by pool then slot; null when the context has no dynamic contacts
    uint32_t* dyn_begin = nullptr;   // n + 1
    uint32_t* dyn_ent = nullptr;
    uint8_t* dyn_skip = nullptr;     // 1: has contacts or a new color, solved from its color's list, not its slab
    uint8_t* conflicted = nullptr;   // 1: intra-color conflict, the update is buffered
    V4* buffered = nullptr;          // buffered positions of conflicted vertices
};

enum OrientedFlags : uint8_t {
    OF_RGROUND = 1, OF_RG_USE_STATIC = 2, OF_RG_UNCLAMPED = 4, OF_RG_ROUND = 8, OF_JOINT = 16
};
enum ContactFlags : uint8_t { CF_ACTIVE = 1, CF_USE_STATIC = 2, CF_UNCLAMPED = 4 };

// Per-scene run-to-tolerance state passed to the solve, Chebyshev and residual
// kernels.  Null pointers disable the corresponding behaviour.
struct MlpDevice;  // learned warm-start weights on the device (mlp.cu)
struct DynHost;    // host side of the dynamic contacts (contacts.cu)

struct SceneTol {
    const uint32_t* scene = nullptr;  // scene of each internal vertex
    const uint8_t* active = nullptr;  // solve / update only vertices of these scenes
    const uint8_t* cand = nullptr;    // exact residual only for these scenes
    double* r2 = nullptr;             // per-scene sum of in-sweep block residuals^2
    double* ex = nullptr;             // per-scene sum of exact block residuals^2
    const double* omega = nullptr;    // Chebyshev weight of this iteration in device memory
                                      // (device-driven iteration loop), else the launch argument
    const uint32_t* it = nullptr;     // index of this iteration in device memory, likewise
};

// Scalar arguments of a step.
struct StepConsts {
    double dt;
    double g;            // magnitude of gravity along -y
    double kappa_max;    // condition threshold of the FP64 block fallback
};

// ---------------------------------------------------------- host staging

struct HostNH { unsigned idx[4]; double lambda, mu, kd, Q[9], V; };
struct HostGround { unsigned p; double k_start, mu_s, mu_k; };
struct HostRod { unsigned idx[2]; double K[6], L, kappa[3]; };
struct HostRGround { unsigned p; uint8_t shape; double radius, cp[3], k_start, mu_s, mu_k; };
struct HostJoint { unsigned p; double po[3], ro[4], rp[3], rq[4]; };
struct HostPrim { uint8_t type; unsigned idx[3]; unsigned object_id; double radius; };

// ------------------------------------------------------------ LBVH state
struct LbvhState {
    unsigned n = 0;                 // primitives
    uint8_t* type = nullptr;
    uint4* pidx = nullptr;          // particle indices (internal order) of each primitive
    double* radius = nullptr;
    double* aabb = nullptr;         // 6 per primitive
    uint64_t* morton = nullptr;
    uint64_t* keys_tmp = nullptr;
    uint32_t* sorted = nullptr;
    uint32_t* sorted_tmp = nullptr;
    uint32_t* hist = nullptr;       // radix histograms
    uint32_t* left = nullptr;
    uint32_t* right = nullptr;
    uint32_t* parent = nullptr;
    uint32_t* subtree = nullptr;
    uint32_t* visited = nullptr;
    double* nbounds = nullptr;      // 6 per node
    double* scene_box = nullptr;    // 6 doubles (+ scratch)
    uint32_t* root = nullptr;
    uint2* pairs = nullptr;
    uint2* range = nullptr;         // leaf range [lo, hi] of each internal node
    uint32_t* pair_count = nullptr;
    unsigned pair_capacity = 0;
    double* xd = nullptr;           // FP64 copies of positions / velocities
    double* vd = nullptr;
    unsigned hist_blocks = 0;
    uint32_t* obj = nullptr;        // object id of each primitive
    // narrow-phase detections, allocated when triangles meet spheres or rod segments
    unsigned contact_capacity = 0;
    uint64_t* contact_key = nullptr;  // DetectedCollision key: type 2 triangle-sphere, 3 triangle-rod
    uint4* contact_idx = nullptr;   // triangle's three vertices, sphere particle / first rod node (internal order)
    uint32_t* contact_idx5 = nullptr;  // second rod node
    double* contact_vec = nullptr;  // 10 per contact: normal, barycentrics, contact point in the body
                                    // (or interpolated rod) frame, s along the segment
    uint32_t* contact_count = nullptr;
};

}  // namespace avbd

// The context behind the opaque avbd_ctx handle.
struct avbd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    avbd_params params{1e-3, 60, 9.81, 33, 1e-3};
    avbd_solver_params solver{1, 0.5, 0.0, 0, AVBD_PRECISION_FP32};
    double kappa_max = 1e4;

    // capacities (SimulationContext(particles, oriented, energies, prims, sdf))
    unsigned cap_particles, cap_oriented, cap_energies, cap_prims, cap_sdf;
    unsigned debug_pair_capacity = 0;   // 0: max(1024, 64 primitives) candidate pairs

    // host staging in the reference's FP64 layout (external order)
    std::vector<double> x, v, vp, mass;
    std::vector<uint8_t> fixed;
    std::vector<unsigned> rot;          // rotation slot or UINT32_MAX
    std::vector<double> q, inertia;     // 4 / 3 per oriented particle
    std::vector<unsigned> scene_begin{0};
    std::vector<avbd::HostNH> nh;
    std::vector<avbd::HostGround> ground;
    std::vector<avbd::HostRod> rods;
    std::vector<avbd::HostRGround> rground;
    std::vector<avbd::HostJoint> joints;
    std::vector<avbd::HostPrim> prims;

    // set-up products
    bool finalized = false;
    bool damping = false;
    std::vector<unsigned> color;        // external order
    unsigned num_colors = 0;
    std::vector<unsigned> perm;         // internal -> external
    std::vector<unsigned> inv;          // external -> internal
    std::vector<unsigned> color_begin;  // internal offset of each color slab
    std::vector<unsigned> color_solve;  // vertices of the slab that run the 3-DOF solve
    std::vector<unsigned> color_orient; // oriented non-fixed vertices after them (6-DOF solve)
    std::vector<double> color_bytes;    // algorithmic bytes of each color's solve launch
    std::vector<double> color_scene_bytes;  // [color][scene]: each scene's part of it
    unsigned max_color_solve = 0;

    avbd::DevState<float> f;
    avbd::DevState<double> d;
    avbd::LbvhState lbvh;
    double* d_residual = nullptr;       // FP64 reduction scratch
    double* d_h2d = nullptr;            // FP64 staging for host uploads/downloads
    size_t h2d_cap = 0;
    unsigned long long* d_counters = nullptr;  // [0] fp64 fallbacks
    uint32_t* d_perm = nullptr;         // internal -> external
    uint32_t* d_inv = nullptr;          // external -> internal
    int* d_error = nullptr;             // device-side status
    unsigned long long launches_per_step = 0;
    // per-scene run-to-tolerance state (num_scenes entries, scene ids per vertex)
    unsigned num_scenes = 1;
    uint32_t* d_scene = nullptr;
    uint8_t* d_scene_active = nullptr;
    uint8_t* d_scene_cand = nullptr;
    double* d_scene_r2 = nullptr;
    double* d_scene_ex = nullptr;
    double* d_scene_rin = nullptr;      // in-sweep residual of each scene's last iteration
    double* d_scene_mg2 = nullptr;
    uint32_t* d_scene_iters = nullptr;
    int* d_tol_count = nullptr;
    // device-driven iteration loop of run-to-tolerance steps (one CUDA graph
    // with a conditional while node): iteration index, Chebyshev weight of the
    // current iteration and the weights of iterations 0..omega_tab_n-1
    uint32_t* d_tol_it = nullptr;
    double* d_tol_omega = nullptr;
    double* d_omega_tab = nullptr;
    unsigned omega_tab_n = 0;
    double omega_tab_rho = -1;          // the rho the table was computed for
    // one iteration (sweep, Chebyshev, index advance) of a fixed-iteration
    // step with dynamic contacts, recorded after the step's host contact
    // management and replayed solver_iters times; updated in place while
    // the iteration's launch sequence keeps its shape
    cudaGraphExec_t dyn_graph = nullptr;
    // (first internal vertex, count, scene) pieces of at most solve_chunk
    // vertices of each scene's solved vertices in each color slab, color by
    // color (offsets solve_range_off): the sweeps and the residual pass of
    // run-to-tolerance steps launch one block per piece
    uint4* d_solve_ranges = nullptr;
    std::vector<unsigned> solve_range_off;
    uint32_t* d_solve_range_off = nullptr;  // device copy of solve_range_off
    unsigned solve_chunk = 512;
    // persistent sweep (default; AVBD_PERSISTENT=0 turns it off): all colors
    // of an iteration in one cooperative launch with grid barriers;
    // [ticket, arrivals, generation]
    bool persistent = true;
    uint32_t* d_sweep_sync = nullptr;
    unsigned num_sms = 0;
    int sweep_blocks_per_sm = 0;        // 0: not queried yet, -1: the kernel cannot run
    unsigned long long host_iterations = 0;  // scene-iterations of fixed-iteration steps

    // CUDA graph of one full step: fixed iterations, or (graph_tol) the
    // run-to-tolerance step whose iteration loop is a conditional while node
    cudaGraphExec_t graph = nullptr;
    bool graph_dirty = true;
    bool graph_tol = false;
    bool use_graph = true;
    int lanes = 8;                      // threads per vertex in the tet solve
    int block = 256;

    // learned warm start (mlp.cu): 0 off, 1 record features/targets, 2 apply
    int ws_mode = 0;
    avbd::MlpDevice* ws_mlp = nullptr;
    void* d_ws_feat = nullptr;          // BF16 [n][32]
    void* d_ws_x0 = nullptr;            // warm-start positions of the last step (state type)
    float* d_ws_target = nullptr;       // FP32 [n][4]: (x_end - x0) / s of the last step
    const float* ws_prev_arg = nullptr; // previous-correction rows for the features launch in flight
    float ws_kappa = 0.5f;              // relative error assumed by the acceptance test
    bool ws_recorded = false;
    double* d_ws_guess = nullptr;       // caller's initial guess of the next step (external order, FP64)
    bool ws_guess_pending = false;

    // dynamic triangle-rigid contacts: pool, recoloring and per-color lists,
    // managed on the host every step (contacts.cu); null without sphere primitives
    avbd::DynHost* dyn = nullptr;

    avbd_stats stats{};
    std::vector<void*> allocations;
};

namespace avbd {

// ---- learned warm start (mlp.cu)
int mlp_device_upload(MlpDevice** m, int device, const float* params, cudaStream_t st);
void mlp_device_free(MlpDevice* m);
int mlp_device_error(const MlpDevice* m, cudaStream_t st);
// x0 += scale * MLP(features) for every internal vertex that is neither fixed nor oriented
template <typename P>
int mlp_apply_state(const MlpDevice& m, const void* feat, unsigned n, typename Vec4Of<P>::T* x,
                    typename Vec4Of<P>::T* xl, typename Vec4Of<P>::T* xll, const uint8_t* flags, double scale,
                    float kappa, unsigned long long* applied, cudaStream_t st);
template <typename R>
void launch_features(avbd_ctx* c, DevState<R>& s, const StepConsts& k, void* feat, const float* prev,
                     cudaStream_t st);
template <typename R>
void launch_ws_save(avbd_ctx* c, DevState<R>& s, void* x0, cudaStream_t st);
template <typename R>
void launch_ws_target(avbd_ctx* c, DevState<R>& s, const void* x0, double inv_s, float* t, cudaStream_t st);

// ---- dynamic triangle-rigid contacts (contacts.cu)
// set-up after the static coloring: keeps the static adjacency and colors
int dyn_create(avbd_ctx* c, const std::vector<unsigned>& p_off, const std::vector<unsigned>& p_nbr,
               std::string& err);
void dyn_destroy(avbd_ctx* c);
// contact handling of the collision stage: merge of the narrow phase's
// detections into the pool, dynamic adjacency, incremental recoloring, then
// the contacts' step-start hook (run before the inertial prediction)
template <typename R>
int dyn_manage(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st);
// the solve of one color: static slabs (less recolored vertices), recolored
// vertices of this color, commit of the color's conflicted vertices
template <typename R>
void dyn_solve_color(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned color, cudaStream_t st,
                     const SceneTol& T);
template <typename R>
void launch_contact_after_iter(avbd_ctx* c, DevState<R>& s, cudaStream_t st, const SceneTol& T);
unsigned dyn_num_colors(const avbd_ctx* c);
// the positional vertices solved from lists (all colors), for the residual pass
void dyn_positional_list(const avbd_ctx* c, const uint32_t** list, unsigned* count);
int dyn_coloring(const avbd_ctx* c, unsigned* colors);

// ---- solve kernels (solve.cu)
template <typename R>
void launch_begin_step(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st);
template <typename R>
void launch_tet_eprev(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st);
// list: when given, the count vertices of list (internal ids) instead of the
// slab [begin, begin + count)
// ranges: when given, (first vertex, count, scene) pieces of the slab, one block each
template <typename R>
void launch_solve_color(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned begin, unsigned count,
                        cudaStream_t st, const SceneTol& T = SceneTol(), const uint32_t* list = nullptr,
                        const uint4* ranges = nullptr, unsigned nranges = 0);
// the whole sweep of a run-to-tolerance iteration as one cooperative launch
// (persistent contexts); false when the context does not qualify
template <typename R>
bool launch_sweep_persistent(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st, const SceneTol& T);
// poll limit of the persistent sweep's grid barriers (avbd_debug_set_wait_limit)
int solve_set_wait_limit(unsigned polls);
// poll limit of the recoloring's grid barriers (avbd_debug_set_wait_limit)
int contacts_set_wait_limit(unsigned polls);
template <typename R>
void launch_chebyshev_dual(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double omega, unsigned it, cudaStream_t st,
                           const SceneTol& T = SceneTol());
template <typename R>
void launch_velocity(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st);
template <typename R>
void launch_residual(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double* out2, cudaStream_t st,
                     const SceneTol& T = SceneTol());
// ---- oriented particles (rods.cu); rod solve modes: 0 solve, 1 residual, 2 debug
template <typename R>
void launch_begin_step_rot(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st);
template <typename R>
void launch_solve_rod(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned begin, unsigned count,
                      cudaStream_t st, const SceneTol& T, int mode, double* out, const uint32_t* list = nullptr);
template <typename R>
void launch_chebyshev_rot(avbd_ctx* c, DevState<R>& s, const StepConsts& k, double omega, unsigned it, cudaStream_t st,
                          const SceneTol& T = SceneTol());
template <typename R>
void launch_velocity_rot(avbd_ctx* c, DevState<R>& s, const StepConsts& k, cudaStream_t st);
template <typename R>
void launch_store_rot(const DevState<R>& s, int which, double* dst, const uint32_t* inv_map, unsigned n,
                      cudaStream_t st);
// per-scene tolerance bookkeeping kernels
void launch_tol_init(avbd_ctx* c, cudaStream_t st);
void launch_tol_decide_a(avbd_ctx* c, double tol, cudaStream_t st);
void launch_tol_decide_b(avbd_ctx* c, double tol, unsigned max_it, cudaStream_t st);
void launch_tol_loop_next(avbd_ctx* c, cudaGraphConditionalHandle h, unsigned max_it, unsigned body_launches,
                          cudaStream_t st);
// iteration index / Chebyshev weight in device memory for the one-iteration
// graph of fixed-iteration steps: set to iteration 0, advanced by one
void launch_iter_set(avbd_ctx* c, cudaStream_t st);
void launch_iter_next(avbd_ctx* c, unsigned n, cudaStream_t st);
template <typename R>
void launch_debug_block(avbd_ctx* c, DevState<R>& s, const StepConsts& k, unsigned p, double* out, cudaStream_t st);
template <typename R>
void launch_load_positions(DevState<R>& s, const double* src, const uint32_t* inv_map, unsigned first, unsigned n,
                           int mode, cudaStream_t st);
template <typename R>
void launch_store_vec(const DevState<R>& s, int which, double* dst, const uint32_t* perm, unsigned n, cudaStream_t st);

// ---- coloring (coloring.cu): exact DSATUR, one CTA per scene
int gpu_dsatur(const std::vector<unsigned>& p_off, const std::vector<unsigned>& p_nbr,
               const std::vector<unsigned>& scene_begin, std::vector<unsigned>& color, unsigned& num_colors,
               cudaStream_t st, std::string& err);

// ---- LBVH (lbvh.cu)
int lbvh_allocate(avbd_ctx* c, std::string& err);
template <typename R>
void lbvh_stage(avbd_ctx* c, DevState<R>& s, cudaStream_t st);
// narrow phase over the broad phase's pairs (narrow.cu)
template <typename R>
void launch_narrow(avbd_ctx* c, DevState<R>& s, cudaStream_t st);

// counts launches for the stats
void count_launch(avbd_ctx* c, unsigned k = 1);
// records the message returned by avbd_last_error_string and returns code
int set_error(int code, const std::string& msg);

}  // namespace avbd
