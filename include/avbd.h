/*
 * avbd.h -- C-ABI of the B200-native Augmented Vertex Block Descent engine.
 *
 * This is the drop-in boundary for the per-step solve of smtobin/avbd.  Every
 * entry point below replaces one piece of that project's C++ step API; the
 * replaced interface is cited as reference-path:line next to each declaration.
 * The signatures use only plain pointers, sizes and PODs: positions, velocities
 * and energy parameters cross the boundary in the reference's own FP64 layout
 * (a std::vector<Vec3r> is `double[3*n]`, a Quaternion is `double[4]` in
 * (w, x, y, z) order, a Mat3r is `double[9]` row-major).
 *
 * Conventions
 *  - Every function returns an int status (AVBD_OK == 0).  No C++ exception
 *    crosses this boundary; avbd_last_error_string() describes the last
 *    failure on the calling thread.
 *  - A context is used by one host thread at a time (calls on one context are
 *    not re-entrant).  Contexts are independent: there is no process-wide
 *    state, unlike the reference's static WorkerThreadContext::NUM_THREADS
 *    (common/WorkerThreadContext.hpp:15).
 *  - "Slots" are indices into the corresponding pool, exactly like the value
 *    returned by the reference's TombstonePool::allocSlot
 *    (common/TombstonePool.hpp:58-65).  Bulk adds return the first slot; the
 *    n slots are consecutive.
 */
#ifndef AVBD_H
#define AVBD_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AVBD_API __attribute__((visibility("default")))
#else
#define AVBD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define AVBD_OK                   0
#define AVBD_ERR_INVALID_ARG      1  /* bad pointer / index / size                         */
#define AVBD_ERR_CAPACITY         2  /* pool overflow (TombstonePool.hpp:61-65)            */
#define AVBD_ERR_COLORS           3  /* more than 256 colors (ColorList.hpp:36)            */
#define AVBD_ERR_UNSUPPORTED_PAIR 4  /* sphere-rod / sphere-sphere (CollisionDetector.cpp:211,686) */
#define AVBD_ERR_NAN              5  /* non-finite state detected after a step             */
#define AVBD_ERR_BARRIER_TIMEOUT  6  /* a bounded device-side wait gave up                 */
#define AVBD_ERR_CUDA             7  /* CUDA runtime failure                               */
#define AVBD_ERR_STATE            8  /* call out of order (e.g. step before finalize)      */
#define AVBD_ERR_UNSUPPORTED      9  /* configuration this engine does not implement       */
#define AVBD_ERR_NO_DEVICE       10  /* no CUDA device visible                             */

/* Shape types, values of Collision::CollisionGeometryType
 * (collision/CollisionGeometryType.hpp:16-27). */
#define AVBD_SHAPE_TRIANGLE     0
#define AVBD_SHAPE_ROD_SEGMENT  1
#define AVBD_SHAPE_SPHERE       2

/* Arithmetic of the solve.
 *  FP32:  FP32 state, element records, accumulation and updates; FP64 block
 *         inverse on ill-conditioned blocks; FP64 residual reduction.  Its
 *         residual floor grows with stiffness (FP32 position quantisation and
 *         gradient cancellation), so it suits fixed-iteration stepping.
 *  FP64:  every kernel in double precision (parity/debug path).
 *  MIXED: FP64 state and gradient, FP32 element records and Hessian: the same
 *         HBM record traffic as FP32 with an FP64-accurate residual; the mode
 *         for run-to-tolerance stepping of stiff scenes. */
#define AVBD_PRECISION_FP32 0
#define AVBD_PRECISION_FP64 1
#define AVBD_PRECISION_MIXED 2

typedef struct avbd_ctx avbd_ctx;

/* Sim::SimulationParams (simulation/SimulationParams.hpp:9-16). */
typedef struct avbd_params {
    double dt;
    double end_time;
    double g_accel;
    double viewer_refresh_time_ms;
    double collision_margin;
} avbd_params;

/* Arguments of VBDSolver(ctx, solver_iters, iter_acceleration)
 * (simulation/VBDSolver.hpp:37-42) plus the engine's own options.
 * residual_tolerance == 0 keeps the reference behaviour: exactly solver_iters
 * iterations per step.  residual_tolerance > 0 iterates until the residual
 * R <= residual_tolerance (checked after every full sweep) or max_iters. */
typedef struct avbd_solver_params {
    unsigned solver_iters;
    double   iter_acceleration;
    double   residual_tolerance;
    unsigned max_iters;
    int      precision;
} avbd_solver_params;

/* Execution statistics of the last avbd_step call. */
typedef struct avbd_stats {
    unsigned long long kernel_launches;   /* kernels launched by the engine   */
    unsigned long long iterations;        /* solver iterations executed       */
    unsigned long long fp64_fallbacks;    /* blocks solved in FP64            */
    unsigned long long candidate_pairs;   /* broad-phase pairs of last step   */
    double   last_residual;               /* run-to-tolerance steps: largest final
                                             residual R over the last step's scenes
                                             (exact where the stopping iteration
                                             evaluated it, else a capped scene's
                                             in-sweep R); 0 in fixed-iteration mode */
    unsigned num_colors;
    unsigned num_scenes;
    unsigned long long capped_scene_steps; /* run-to-tolerance scene-steps that
                                              stopped at max_iters unconverged */
    unsigned long long warmstart_applied;  /* vertex-steps whose learned correction
                                              passed the acceptance test */
} avbd_stats;

/* ------------------------------------------------------------- lifetime */

/* Sim::SimulationContext(particles, oriented, energies, prims, sdf)
 * (simulation/SimulationContext.hpp:46-59).  Binds the context to CUDA device
 * `device` and creates its stream. */
AVBD_API int avbd_create(avbd_ctx** out, int device,
                unsigned particles_capacity, unsigned oriented_capacity,
                unsigned energies_capacity, unsigned primitives_capacity,
                unsigned sdf_capacity);
AVBD_API int avbd_destroy(avbd_ctx* ctx);

/* Replaces the context's stream with a caller-owned one (not destroyed by the
 * engine).  Pass NULL to go back to the engine's own stream. */
AVBD_API int avbd_set_stream(avbd_ctx* ctx, void* cuda_stream);

/* SimulationContext::params (simulation/SimulationContext.hpp:39). */
AVBD_API int avbd_set_params(avbd_ctx* ctx, const avbd_params* params);
/* VBDSolver(ctx, solver_iters, iter_acceleration) (simulation/VBDSolver.hpp:37-42). */
AVBD_API int avbd_set_solver(avbd_ctx* ctx, const avbd_solver_params* solver);

/* Starts a new independent scene: particles added after this call form scene
 * k+1.  Scenes never share energies; they are colored independently and
 * advance together in one launch per color phase.  A context that never calls
 * this holds one scene. */
AVBD_API int avbd_begin_scene(avbd_ctx* ctx, unsigned* scene_index);

/* ------------------------------------------------------------ particles */

/* ParticlePool::addParticle(position, mass) x n (common/ParticlePool.hpp:217-240). */
AVBD_API int avbd_particles_add(avbd_ctx* ctx, unsigned n, const double* positions,
                       const double* masses, unsigned* first_slot);
/* ParticlePool::addOrientedParticle(position, rotation, mass, inertia) x n
 * (common/ParticlePool.hpp:257-263).  rotations are (w,x,y,z). */
AVBD_API int avbd_particles_add_oriented(avbd_ctx* ctx, unsigned n, const double* positions,
                                const double* rotations, const double* masses,
                                const double* rotational_inertias, unsigned* first_slot);
/* ParticlePool::fixed[idx] = flag (common/ParticlePool.hpp:87). */
AVBD_API int avbd_particles_set_fixed(avbd_ctx* ctx, unsigned n, const unsigned* slots,
                             const uint8_t* fixed);

/* State transfer for n consecutive particles starting at `first`.
 * set_positions also resets previous/inertial/last-iterate positions like
 * ParticlePool::addParticle; set_state only overwrites positions and
 * velocities (the per-step drop-in upload). */
AVBD_API int avbd_set_positions(avbd_ctx* ctx, unsigned first, unsigned n, const double* positions);
AVBD_API int avbd_set_velocities(avbd_ctx* ctx, unsigned first, unsigned n,
                        const double* velocities, const double* previous_velocities);
AVBD_API int avbd_set_state(avbd_ctx* ctx, const double* positions, const double* velocities);
AVBD_API int avbd_get_positions(avbd_ctx* ctx, unsigned first, unsigned n, double* positions);
AVBD_API int avbd_get_velocities(avbd_ctx* ctx, unsigned first, unsigned n, double* velocities);
AVBD_API int avbd_get_rotations(avbd_ctx* ctx, unsigned first, unsigned n, double* rotations);
AVBD_API int avbd_get_angular_velocities(avbd_ctx* ctx, unsigned first, unsigned n, double* w);
AVBD_API int avbd_num_particles(avbd_ctx* ctx, unsigned* n);

/* -------------------------------------------------------------- energies */

/* NeoHookeanEnergyPool::addEnergy(indices, lambda, mu, kd, Q, rest_volume) x n
 * (energy/elastic/NeoHookeanEnergyPool.hpp:40-67).  Q is row-major 3x3. */
AVBD_API int avbd_neo_hookean_add(avbd_ctx* ctx, unsigned n, const unsigned* indices4,
                         const double* lambda, const double* mu, const double* kd,
                         const double* Q9, const double* rest_volume, unsigned* first_slot);

/* CosseratRodEnergyPool::addEnergy(indices, stiffness, rest_length, precurvature) x n
 * (energy/elastic/CosseratRodEnergyPool.hpp:36-51). */
AVBD_API int avbd_cosserat_rod_add(avbd_ctx* ctx, unsigned n, const unsigned* indices2,
                          const double* stiffness6, const double* rest_length,
                          const double* precurvature3, unsigned* first_slot);

/* GroundCollisionEnergyPool::addEnergy(particle_index, k_start, mu_s, mu_k) x n
 * (energy/collision/GroundCollisionEnergyPool.hpp:32-43). */
AVBD_API int avbd_ground_collision_add(avbd_ctx* ctx, unsigned n, const unsigned* particle_index,
                              const double* k_start, const double* mu_s, const double* mu_k,
                              unsigned* first_slot);

/* RigidBodyGroundCollisionEnergyPool::addEnergy(particle_index, shape_params,
 * cp_rb_local, k_start, mu_s, mu_k) x n
 * (energy/collision/RigidBodyGroundCollisionEnergyPool.hpp:36-58).
 * shape_type is AVBD_SHAPE_SPHERE or AVBD_SHAPE_ROD_SEGMENT; shape_radius is
 * CollisionShapeParams::sphere.radius / rod.radius. */
AVBD_API int avbd_rigid_body_ground_collision_add(avbd_ctx* ctx, unsigned n,
                                         const unsigned* particle_index,
                                         const uint8_t* shape_type, const double* shape_radius,
                                         const double* cp_rb_local3, const double* k_start,
                                         const double* mu_s, const double* mu_k,
                                         unsigned* first_slot);

/* OneSidedFixedJointEnergyPool::addEnergy(particle_index, pos_offset, rot_offset,
 * ref_position, ref_rotation) x n (energy/joint/OneSidedFixedJointEnergyPool.hpp:36-55).
 * k_start = 1e4 on all six rows (OneSidedFixedJointEnergyPool.hpp:27). */
AVBD_API int avbd_one_sided_fixed_joint_add(avbd_ctx* ctx, unsigned n, const unsigned* particle_index,
                                   const double* position_offset3, const double* rotation_offset4,
                                   const double* ref_position3, const double* ref_rotation4,
                                   unsigned* first_slot);

/* --------------------------------------------------- collision primitives */

/* CollisionPrimitivePool::addObject(TetMeshObject) surface triangles
 * (collision/CollisionPrimitivePool.cpp:36-50): one Triangle per face. */
AVBD_API int avbd_collision_add_triangles(avbd_ctx* ctx, unsigned n, const unsigned* indices3,
                                 unsigned object_id, unsigned* first_slot);
/* CollisionPrimitivePool::addObject(Rod): one RodSegment per element. */
AVBD_API int avbd_collision_add_rod_segments(avbd_ctx* ctx, unsigned n, const unsigned* indices2,
                                    double radius, unsigned object_id, unsigned* first_slot);
/* CollisionPrimitivePool::addObject(RigidSphere). */
AVBD_API int avbd_collision_add_spheres(avbd_ctx* ctx, unsigned n, const unsigned* particle_index,
                               const double* radius, const unsigned* object_id,
                               unsigned* first_slot);

/* ------------------------------------------------------------ set-up/step */

/* StaticParticleAdjacency::buildAdjacency + DynamicParticleAdjacency::buildAdjacency
 * + ColorList::buildInitialColorList (simulation/Simulation.cpp:86-89):
 * builds the per-vertex energy CSR, exact DSATUR coloring on the GPU (one CTA
 * per scene) and an empty conflict CSR, and uploads everything to HBM. */
AVBD_API int avbd_finalize(avbd_ctx* ctx);

/* SimulationExecutor::timeStep() (simulation/SimulationExecutor.hpp:107-115):
 * collision stage (LBVH build + self traversal) then VBDSolver::solve_Parallel
 * (simulation/VBDSolver.hpp:48-103), n_steps times, stream-ordered. */
AVBD_API int avbd_step(avbd_ctx* ctx, unsigned n_steps);
/* Waits for the context's stream. */
AVBD_API int avbd_synchronize(avbd_ctx* ctx);

/* Runs only the collision stage (LBVH build + candidate pairs) on the current
 * state, without advancing time. */
AVBD_API int avbd_collision_stage(avbd_ctx* ctx);

AVBD_API int avbd_get_stats(avbd_ctx* ctx, avbd_stats* stats);

/* -------------------------------------------------------- parity queries */

/* ColorList::color / num_colors (common/ColorList.hpp:66-67). */
AVBD_API int avbd_get_coloring(avbd_ctx* ctx, unsigned* colors, unsigned* num_colors);

/* LBVH of the last collision stage: CollisionPrimitivePool::morton_code and
 * sorted_order (collision/CollisionPrimitivePool.hpp:57-60) and the SoA nodes
 * of Collision::LBVH (collision/LBVH.hpp:17-85).  Arrays sized n (primitives)
 * and 2n-1 (nodes); bounds6 is min_x,min_y,min_z,max_x,max_y,max_z per node.
 * Any output pointer may be NULL. */
AVBD_API int avbd_get_lbvh(avbd_ctx* ctx, unsigned* num_primitives, uint64_t* morton,
                  unsigned* sorted_order, unsigned* left, unsigned* right,
                  unsigned* parent, unsigned* subtree_size, double* bounds6,
                  unsigned* root);
/* Candidate leaf pairs (a<b, sorted-leaf indices) of LBVHTraversal
 * (collision/LBVHTraversal.hpp:30-88), sorted lexicographically. */
AVBD_API int avbd_get_candidate_pairs(avbd_ctx* ctx, unsigned capacity, unsigned* pairs2,
                             unsigned* count);

/* Triangle-sphere contacts found by the last collision stage's narrow phase
 * (CollisionDetector::_triangleSphere / _triangleSDF_CCD,
 * collision/CollisionDetector.cpp:504-540,689-876), in ascending key order
 * (DetectedCollision::generateKey, collision/DetectedCollision.hpp:43-66).
 * Per contact: keys[k]; idx4 = the triangle's three particle slots and the
 * sphere's particle slot; vec9 = contact normal (world), barycentrics of the
 * contact point on the triangle, contact point on the sphere in its body
 * frame.  Up to `capacity` contacts are written (pointers may be NULL);
 * *count receives the number found.  Inside avbd_step these detections
 * become the triangle-rigid contact energies below. */
AVBD_API int avbd_get_contacts(avbd_ctx* ctx, unsigned capacity, uint64_t* keys, unsigned* idx4, double* vec9,
                               unsigned* count);

/* Triangle-rod-segment contacts found by the last collision stage's narrow
 * phase (CollisionDetector::_triangleRod, collision/CollisionDetector.cpp:
 * 601-666, with Math::closestPoint_SegmentTriangle, common/Math.hpp:593-681),
 * in ascending key order.  Per contact: keys[k]; idx5 = the triangle's three
 * particle slots and the segment's two nodes; vec10 = contact normal (world,
 * centreline to triangle), barycentrics on the triangle, contact point in
 * the rod frame interpolated at s, and s along the segment.  Up to
 * `capacity` contacts are written (pointers may be NULL); *count receives
 * the number found. */
AVBD_API int avbd_get_rod_contacts(avbd_ctx* ctx, unsigned capacity, uint64_t* keys, unsigned* idx5,
                                   double* vec10, unsigned* count);

/* Dynamic contact state after the last step's collision stage (contexts
 * with triangles and spheres or rod segments; zeros otherwise): out[0] live
 * triangle-rigid contacts, out[1] their pool size (highest slot + 1,
 * TombstonePool::totalSize, common/TombstonePool.hpp:53), out[2] colors after
 * the incremental recoloring (ColorList::incrementalRecoloring,
 * common/ColorList.hpp:381-474), out[3] conflicted particles
 * (ColorList::finalizeConflicts, :476-522), out[4] particles left dirty for
 * the next stage, out[5] dynamic adjacency entries
 * (DynamicParticleAdjacency::buildAdjacency,
 * common/DynamicParticleAdjacency.hpp:33-118), out[6] live triangle-rod
 * contacts, out[7] their pool size. */
AVBD_API int avbd_dynamic_info(avbd_ctx* ctx, unsigned out[8]);

/* The triangle-rigid contact pool (TriangleRigidCollisionEnergyPool,
 * energy/collision/TriangleRigidCollisionEnergyPool.hpp:10-78) by slot, slots
 * [0, min(capacity, pool size)): p4 = the triangle's three particle slots and
 * the rigid body's; active[s] = 1 for a live slot; data24 = per slot the
 * normal, tangent, binormal, barycentrics, contact point in the body frame
 * (3 each), k_start, k_n, k_t, k_b, lambda_n, lambda_t, lambda_b, C_n_prev,
 * and flags (1 static friction, 2 unclamped friction) as a double.  Values
 * as of the device state when called.  Pointers may be NULL; *size receives
 * the pool size. */
AVBD_API int avbd_get_contact_pool(avbd_ctx* ctx, unsigned capacity, unsigned* p4, uint8_t* active, double* data24,
                                   unsigned* size);

/* The triangle-rod contact pool (TriangleRodCollisionEnergyPool,
 * energy/collision/TriangleRodCollisionEnergyPool.hpp:9-86) by slot, as
 * avbd_get_contact_pool: p5 = the triangle's three particle slots and the
 * segment's two nodes; data25 = normal, tangent, binormal, barycentrics,
 * contact point in the interpolated rod frame (3 each), s, k_start, k_n, k_t,
 * k_b, lambda_n, lambda_t, lambda_b, C_n_prev, flags. */
AVBD_API int avbd_get_rod_contact_pool(avbd_ctx* ctx, unsigned capacity, unsigned* p5, uint8_t* active,
                                       double* data25, unsigned* size);

/* Test hook: the round limit of the incremental recoloring (6 in the
 * reference, ColorList.hpp:384).  Fewer rounds leave more particles
 * conflicted, which exercises the conflict buffering of the solve
 * (VBDSolver.hpp:82-87,108-119,474-509). */
AVBD_API int avbd_debug_set_recolor_rounds(avbd_ctx* ctx, unsigned rounds);

/* Test hook (before avbd_finalize): the capacity of the broad-phase
 * candidate-pair buffer, max(1024, 64 x primitives) unless set (0 restores
 * that).  The reference's pair list grows without bound
 * (CollisionDetector.cpp:100-129); here a step whose traversal finds more
 * pairs than the buffer holds fails with AVBD_ERR_CAPACITY instead of losing
 * collisions.  A small capacity lets a test reach that path. */
AVBD_API int avbd_debug_set_pair_capacity(avbd_ctx* ctx, unsigned capacity);

/* Block gradient and Hessian of particle p at the current state: the
 * grad/hess accumulated by VBDSolver::_solveParticle<DOF>
 * (simulation/VBDSolver.hpp:293-447).  G is 3 or 6 doubles, H is 9 or 36
 * (row-major); *dof receives 3 or 6. */
AVBD_API int avbd_debug_block(avbd_ctx* ctx, unsigned p, double* G, double* H, int* dof);

/* Residual R of the current iterate (sqrt(sum_v |m/h^2 (x-y) + g_v|^2) /
 * sqrt(sum_v |m g|^2)), FP64 reduction on the device. */
AVBD_API int avbd_residual(avbd_ctx* ctx, double* residual);

/* Run-to-tolerance steps: the iterations each scene ran in the last step
 * (num_scenes entries, scene order of avbd_begin_scene).  The reference has
 * no tolerance mode; its counterpart is the fixed solver_iters of every
 * step (simulation/VBDSolver.hpp:64). */
AVBD_API int avbd_get_scene_iterations(avbd_ctx* ctx, unsigned* iterations);

/* No counterpart in the reference.  Morton codes and the stable sorted order
 * of an LBVH build for caller-provided primitive boxes, allocating nothing:
 * for callers that must not allocate device memory while they run (a loop
 * being recorded into a CUDA graph, a real-time loop on a fixed memory
 * budget, an application whose device memory belongs to another framework's
 * allocator).  Scratch lives in file-scope device arrays sized for
 * AVBD_NOALLOC_MAX_PRIMITIVES primitives (about 6 MiB, resident on every GPU
 * that loads the library until exit); larger n returns AVBD_ERR_CAPACITY.
 * aabb6 (n x {min xyz, max xyz} doubles), morton (n codes, one per primitive)
 * and sorted_order (n indices) are device pointers owned by the caller;
 * stream is a cudaStream_t (NULL: the default stream).  Results equal the
 * codes and sorted order of avbd_get_lbvh for the same boxes.  Every call
 * shares the scratch; calls that overlap on the GPU race.  The first call on
 * a device resolves the scratch addresses and should come before any stream
 * capture.  Each CUDA call it makes is checked on its own: a CUDA error left
 * pending by earlier work is not consumed, and AVBD_ERR_CUDA means one of
 * this call's own launches or copies failed. */
#define AVBD_NOALLOC_MAX_PRIMITIVES 262144u
AVBD_API int avbd_lbvh_morton_sort_noalloc(const double* aabb6, unsigned n, uint64_t* morton,
                                           unsigned* sorted_order, void* stream);

/* Measurement entry point (no counterpart in the reference): runs `iterations`
 * further solver iterations on the current state without the CUDA graph,
 * bracketing every per-color vertex-solve launch with CUDA events on the
 * context's stream.  Returns the summed kernel time, the algorithmic bytes
 * those launches had to move (per solved vertex: x read + y read + x write,
 * its two incidence offsets and flags, contact state when present, and one
 * incidence record per incident tet) and the number of launches. */
AVBD_API int avbd_profile_solve(avbd_ctx* ctx, unsigned iterations, double* solve_ms, double* solve_bytes,
                                unsigned* launches);

/* Measurement entry point (no counterpart in the reference): advances one
 * run-to-tolerance step with exactly the launches a timed step uses (the
 * per-scene pieces of each color slab, scenes that have converged gated
 * out), driven from the host, with CUDA events around every color's
 * vertex-solve launch.  Returns their summed time, the algorithmic bytes of
 * the scenes still iterating when each launch started (per solved vertex as
 * for avbd_profile_solve), the launches and the iterations the step ran.
 * Contexts with dynamic contacts are refused (AVBD_ERR_STATE). */
AVBD_API int avbd_profile_step(avbd_ctx* ctx, double* solve_ms, double* solve_bytes, unsigned* launches,
                               unsigned* iterations);

/* ------------------------------------------------ learned warm start
 * No counterpart in the reference (it has no learned component).  A
 * per-vertex MLP 27 -> 128 -> 128 -> 128 -> 3 with SiLU, BF16 weights and
 * activations, FP32 accumulation (tcgen05.mma), predicts the correction of
 * the inertial initial guess of every solved tet vertex at the start of a
 * step: x0 <- x0 + s * f(features), s = g h^2.  Parameters travel as one FP32
 * array of AVBD_MLP_NPARAMS values, PyTorch Linear layout ([out][in],
 * row-major) with padded shapes:
 *   W1 [128][32]  at 0        (inputs 27..31 are zero padding)
 *   b1 [128]      at 4096
 *   W2 [128][128] at 4224,    b2 [128] at 20608
 *   W3 [128][128] at 20736,   b3 [128] at 37120
 *   W4 [16][128]  at 37248    (outputs 3..15 are zero padding)
 *   b4 [16]       at 39296
 * Feature rows are 32 BF16 values (27 used, the layout is listed with
 * avbd_warmstart_sample); target rows are 4 FP32 values (3 used). */
#define AVBD_MLP_IN 27
#define AVBD_MLP_IN_PAD 32
#define AVBD_MLP_HIDDEN 128
#define AVBD_MLP_OUT 3
#define AVBD_MLP_OUT_PAD 16
#define AVBD_MLP_NPARAMS 39312u

/* D = A B^T on the tensor cores: A [M x K] and B [N x K] row-major BF16 device
 * arrays (lda, ldb in elements, multiples of 8; K a multiple of 16), C [M x N]
 * FP32 (ldc in elements).  accumulate != 0 adds to C.  stream: cudaStream_t. */
AVBD_API int avbd_gemm_bf16(const void* A, unsigned lda, const void* B, unsigned ldb, float* C, unsigned ldc,
                            unsigned M, unsigned N, unsigned K, int accumulate, void* stream);

/* Inference of the MLP on n feature rows (device, BF16 [n][32]) into out
 * (device, FP32 [n][16], columns 3..15 are the zero padding). */
typedef struct avbd_mlp avbd_mlp;
AVBD_API int avbd_mlp_create(avbd_mlp** out, int device, const float* params);
AVBD_API int avbd_mlp_forward(avbd_mlp* m, const void* features, unsigned n, float* out, void* stream);
AVBD_API int avbd_mlp_destroy(avbd_mlp* m);

/* Debug hook with no counterpart in the reference: the number of polls a
 * bounded wait may take on `device` before it gives up
 * (AVBD_DEFAULT_WAIT_POLLS unless changed; 0 gives up at once): the
 * tensor-core barrier waits of the MLP and GEMM kernels, and the grid-barrier
 * waits of the persistent sweep (unless AVBD_PERSISTENT=0 is in the
 * environment when a context is created, each run-to-tolerance sweep of a
 * tetrahedral context runs as one cooperative launch whose blocks meet at a
 * grid barrier between colors), and of the dynamic contacts' recoloring
 * (its rounds run as one cooperative launch per step).  A wait that gives up
 * sets AVBD_ERR_BARRIER_TIMEOUT, which the launching call (avbd_step for the
 * sweep and the recoloring) returns; every result of that launch is then
 * invalid.  The MLP kernels still wait, bounded, for the MMAs they issued
 * before they free their tensor memory, and every block of the sweep or the
 * recoloring leaves the kernel, so the context stays usable.  Tests lower the limit to make the wait run out
 * without any fault. */
#define AVBD_DEFAULT_WAIT_POLLS (1u << 22)
AVBD_API int avbd_debug_set_wait_limit(int device, unsigned polls);

/* Training: mini-batches of `batch` rows (a multiple of 128) of device
 * features (BF16 [batch][32]) and targets (FP32 [batch][4]: 3 outputs and
 * the row's loss weight w); loss = mean over rows and outputs of
 * w (y - t)^2; Adam (beta1 0.9, beta2 0.999, eps 1e-8)
 * on FP32 master weights.  avbd_mlp_trainer_grad evaluates the loss and the
 * gradient (host FP32 [AVBD_MLP_NPARAMS]) without updating. */
typedef struct avbd_mlp_trainer avbd_mlp_trainer;
AVBD_API int avbd_mlp_trainer_create(avbd_mlp_trainer** out, int device, unsigned batch, const float* params);
AVBD_API int avbd_mlp_trainer_step(avbd_mlp_trainer* t, const void* features, const float* targets, float lr,
                                   float* loss);
AVBD_API int avbd_mlp_trainer_grad(avbd_mlp_trainer* t, const void* features, const float* targets, float* loss,
                                   float* grad);
AVBD_API int avbd_mlp_trainer_get_params(avbd_mlp_trainer* t, float* params);
AVBD_API int avbd_mlp_trainer_destroy(avbd_mlp_trainer* t);

/* Warm start of a context (after avbd_finalize; tet vertices only):
 *   mode 0  off (the adaptive inertial guess of VBDSolver.hpp:208-248);
 *   mode 1  record: every step stores the features of each solved tet vertex
 *           at the inertial guess x0 and, after the step, the target
 *           (x_end - x0) / s, for avbd_warmstart_sample;
 *   mode 2  apply: x0 <- x0 + s * y, y = MLP(features), before the
 *           iterations, for each vertex whose correction passes an
 *           acceptance test: the block residual at x0 (L1 of features 12-14,
 *           units of m g) must exceed 1e-4 and the residual the correction's
 *           error would add, kappa * sum_a (1 + H_aa h^2/m) |y_a| with
 *           kappa = 0.5 (the environment variable AVBD_WS_KAPPA overrides it
 *           when the mode is set).  Other vertices keep the inertial guess;
 *           avbd_stats.warmstart_applied counts the accepted ones.
 * params (mode 2): AVBD_MLP_NPARAMS floats, with any input normalisation
 * folded into W1/b1 and the output scale folded into W4/b4. */
AVBD_API int avbd_set_warmstart(avbd_ctx* ctx, int mode, const float* params);

/* Features and targets of the last recorded step, one row per solved tet
 * vertex (*rows of them, internal order), into caller device buffers
 * (features BF16 [rows][32], targets FP32 [rows][4]; either may be NULL to
 * query *rows).  Feature layout, displacements in units of s = g h^2:
 *   0-2   x0 - y                      (inertial guess minus inertial target)
 *   3-5   v h                         (last step's displacement)
 *   6-8   previous step's (x_end - x0) / s  (0 on the first step)
 *   9-11  (mean over incident tets of the other vertices' v - v) h
 *   12-14 block RHS h^2 / m = -(x0 - y) - grad E(x0) h^2 / m
 *   15-17 block Newton step A^-1 RHS  (A = m/h^2 I + H(x0))
 *   18-20 log(1 + diag H(x0) h^2 / m)
 *   21    mean mu/lambda of the incident tets
 *   22    log10(m) + 3
 *   23    tanh(x0_y / 10),  26 tanh(y_y)   (height above the ground)
 *   24    ground normal multiplier lambda_n h^2 / (m s)
 *   25    incident tet count / 24 */
AVBD_API int avbd_warmstart_sample(avbd_ctx* ctx, void* features, float* targets, unsigned* rows);

/* No counterpart in the reference: the initial guess x0 of the next step's
 * iterations for every solved positional particle, supplied by the caller
 * (positions: particles x 3 doubles, the order of avbd_particles_add),
 * replacing the adaptive inertial initialisation (VBDSolver.hpp:208-248)
 * once; the inertial prediction y itself is unchanged.  For an external
 * predictor, and for bounding what any displacement warm start can save:
 * given the step's converged positions, the iterations still needed are a
 * floor for every predictor of them.  NULL cancels a pending guess. */
AVBD_API int avbd_set_initial_guess(avbd_ctx* ctx, const double* positions);

AVBD_API const char* avbd_last_error_string(void);
AVBD_API const char* avbd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* AVBD_H */
