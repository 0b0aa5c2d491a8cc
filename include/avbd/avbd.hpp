// avbd.hpp -- header-only C++ facade over the C-ABI of avbd.h, with the
// class and method names of smtobin/avbd's step API so that reference code
// ports line by line:
//
//   Sim::SimulationContext ctx(particles, oriented, energies, prims, sdf);
//   unsigned p = ctx.particles.addParticle({x, y, z}, mass);
//   ctx.energies.neo_hookean.addEnergy({a, b, c, d}, lambda, mu, kd, Q, V);
//   ctx.energies.ground_collision.addEnergy(p, k_start, 0.4, 0.2);
//   ctx.params.dt = 1.0 / 60;
//   Sim::SimulationExecutor exec(&ctx, solver_iters, iter_acceleration, 0);
//   exec.timeStep();                      // collision stage + AVBD solve on the GPU
//
// Objects mirror simulation/SimulationContext.hpp:18-60,
// energy/EnergyRegistry.hpp:17-173, simulation/VBDSolver.hpp:37-103 and
// simulation/SimulationExecutor.hpp:65-115.  Errors throw avbd::Error (the
// reference throws std::runtime_error for the same conditions).
#pragma once

#include <array>
#include <stdexcept>
#include <string>
#include <vector>

#include "../avbd.h"

namespace avbd {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != AVBD_OK) throw Error(rc, avbd_last_error_string());
}

using Vec3 = std::array<double, 3>;
using Quat = std::array<double, 4>;  // (w, x, y, z)
using Mat3 = std::array<double, 9>;  // row-major

}  // namespace avbd

namespace Sim {

class SimulationContext;

// ParticlePool (common/ParticlePool.hpp:76-285)
class ParticlePool {
  public:
    explicit ParticlePool(avbd_ctx* c) : c_(c) {}
    unsigned addParticle(const avbd::Vec3& position, double mass) {
        unsigned slot = 0;
        avbd::check(avbd_particles_add(c_, 1, position.data(), &mass, &slot));
        return slot;
    }
    unsigned addOrientedParticle(const avbd::Vec3& position, const avbd::Quat& rotation, double mass,
                                 const avbd::Vec3& rotational_inertia) {
        unsigned slot = 0;
        avbd::check(avbd_particles_add_oriented(c_, 1, position.data(), rotation.data(), &mass,
                                                rotational_inertia.data(), &slot));
        return slot;
    }
    void setFixed(unsigned p, bool fixed) {
        uint8_t f = fixed ? 1 : 0;
        avbd::check(avbd_particles_set_fixed(c_, 1, &p, &f));
    }
    unsigned totalSize() const {
        unsigned n = 0;
        avbd::check(avbd_num_particles(c_, &n));
        return n;
    }
    // std::vector<Vec3r> layout: 3 doubles per particle
    void positions(std::vector<double>& out) const {
        out.resize(3ull * totalSize());
        avbd::check(avbd_get_positions(c_, 0, totalSize(), out.data()));
    }
    void velocities(std::vector<double>& out) const {
        out.resize(3ull * totalSize());
        avbd::check(avbd_get_velocities(c_, 0, totalSize(), out.data()));
    }

  private:
    avbd_ctx* c_;
};

}  // namespace Sim

namespace Energy {

// NeoHookeanEnergyPool::addEnergy (energy/elastic/NeoHookeanEnergyPool.hpp:40-67)
struct NeoHookeanEnergyPool {
    avbd_ctx* c;
    unsigned addEnergy(const std::array<unsigned, 4>& indices, double lambda, double mu, double kd,
                       const avbd::Mat3& Q, double rest_volume) {
        unsigned slot = 0;
        avbd::check(avbd_neo_hookean_add(c, 1, indices.data(), &lambda, &mu, &kd, Q.data(), &rest_volume, &slot));
        return slot;
    }
};

// CosseratRodEnergyPool::addEnergy (energy/elastic/CosseratRodEnergyPool.hpp:36-51)
struct CosseratRodEnergyPool {
    avbd_ctx* c;
    unsigned addEnergy(const std::array<unsigned, 2>& indices, const std::array<double, 6>& stiffness,
                       double rest_length, const avbd::Vec3& precurvature) {
        unsigned slot = 0;
        avbd::check(avbd_cosserat_rod_add(c, 1, indices.data(), stiffness.data(), &rest_length, precurvature.data(),
                                          &slot));
        return slot;
    }
};

// GroundCollisionEnergyPool::addEnergy (energy/collision/GroundCollisionEnergyPool.hpp:32-43)
struct GroundCollisionEnergyPool {
    avbd_ctx* c;
    unsigned addEnergy(unsigned particle_index, double k_start, double mu_s, double mu_k) {
        unsigned slot = 0;
        avbd::check(avbd_ground_collision_add(c, 1, &particle_index, &k_start, &mu_s, &mu_k, &slot));
        return slot;
    }
};

// RigidBodyGroundCollisionEnergyPool::addEnergy
// (energy/collision/RigidBodyGroundCollisionEnergyPool.hpp:36-58)
struct RigidBodyGroundCollisionEnergyPool {
    avbd_ctx* c;
    unsigned addEnergy(unsigned particle_index, uint8_t shape_type, double shape_radius,
                       const avbd::Vec3& cp_rb_local, double k_start, double mu_s, double mu_k) {
        unsigned slot = 0;
        avbd::check(avbd_rigid_body_ground_collision_add(c, 1, &particle_index, &shape_type, &shape_radius,
                                                         cp_rb_local.data(), &k_start, &mu_s, &mu_k, &slot));
        return slot;
    }
};

// OneSidedFixedJointEnergyPool::addEnergy (energy/joint/OneSidedFixedJointEnergyPool.hpp:36-55)
struct OneSidedFixedJointEnergyPool {
    avbd_ctx* c;
    unsigned addEnergy(unsigned particle_index, const avbd::Vec3& pos_offset, const avbd::Quat& rot_offset,
                       const avbd::Vec3& ref_position, const avbd::Quat& ref_rotation) {
        unsigned slot = 0;
        avbd::check(avbd_one_sided_fixed_joint_add(c, 1, &particle_index, pos_offset.data(), rot_offset.data(),
                                                   ref_position.data(), ref_rotation.data(), &slot));
        return slot;
    }
};

// Energy::EnergyRegistry (energy/EnergyRegistry.hpp:17-37)
struct EnergyRegistry {
    NeoHookeanEnergyPool neo_hookean;
    CosseratRodEnergyPool cosserat_rod;
    GroundCollisionEnergyPool ground_collision;
    RigidBodyGroundCollisionEnergyPool rigid_body_ground_collision;
    OneSidedFixedJointEnergyPool one_sided_fixed_joint;
    explicit EnergyRegistry(avbd_ctx* c)
        : neo_hookean{c}, cosserat_rod{c}, ground_collision{c}, rigid_body_ground_collision{c},
          one_sided_fixed_joint{c} {}
};

}  // namespace Energy

namespace Sim {

// Sim::SimulationParams (simulation/SimulationParams.hpp:9-16)
struct SimulationParams {
    double dt = 1e-3, end_time = 60, g_accel = 9.81, viewer_refresh_time_ms = 33, collision_margin = 1e-3;
};

// Sim::SimulationContext (simulation/SimulationContext.hpp:18-60): owns one
// engine context on a CUDA device.
class SimulationContext {
  public:
    SimulationContext(unsigned particles_capacity, unsigned oriented_particles_capacity, unsigned energies_capacity,
                      unsigned collision_primitive_capacity, unsigned collision_sdf_capacity, int device = 0)
        : c_(create(device, particles_capacity, oriented_particles_capacity, energies_capacity,
                    collision_primitive_capacity, collision_sdf_capacity)),
          particles(c_),
          energies(c_) {}
    ~SimulationContext() { avbd_destroy(c_); }
    SimulationContext(const SimulationContext&) = delete;
    SimulationContext& operator=(const SimulationContext&) = delete;

    avbd_ctx* handle() const { return c_; }

  private:
    static avbd_ctx* create(int device, unsigned p, unsigned o, unsigned e, unsigned pr, unsigned sdf) {
        avbd_ctx* c = nullptr;
        avbd::check(avbd_create(&c, device, p, o, e, pr, sdf));
        return c;
    }
    avbd_ctx* c_;

  public:
    ParticlePool particles;
    Energy::EnergyRegistry energies;
    SimulationParams params;
};

// Sim::VBDSolver (simulation/VBDSolver.hpp:37-103).  solve_Parallel() runs one
// full step (collision stage + solve) on the context's stream.
class VBDSolver {
  public:
    VBDSolver(SimulationContext* ctx, unsigned solver_iters, double iter_acceleration)
        : ctx_(ctx), iters_(solver_iters), rho_(iter_acceleration) {}
    void setTolerance(double residual_tolerance, unsigned max_iters) {
        tol_ = residual_tolerance;
        max_iters_ = max_iters;
        ready_ = false;
    }
    void setPrecision(int precision) {
        precision_ = precision;
        ready_ = false;
    }
    void solve_Parallel() {
        if (!ready_) setup();
        avbd::check(avbd_step(ctx_->handle(), 1));
    }

  private:
    void setup() {
        avbd_params p{ctx_->params.dt, ctx_->params.end_time, ctx_->params.g_accel,
                      ctx_->params.viewer_refresh_time_ms, ctx_->params.collision_margin};
        avbd::check(avbd_set_params(ctx_->handle(), &p));
        avbd_solver_params s{iters_, rho_, tol_, max_iters_, precision_};
        avbd::check(avbd_set_solver(ctx_->handle(), &s));
        avbd::check(avbd_finalize(ctx_->handle()));
        ready_ = true;
    }
    SimulationContext* ctx_;
    unsigned iters_;
    double rho_;
    double tol_ = 0;
    unsigned max_iters_ = 0;
    int precision_ = AVBD_PRECISION_FP32;
    bool ready_ = false;
};

// Sim::SimulationExecutor (simulation/SimulationExecutor.hpp:65-115).
// num_threads is accepted for signature compatibility; the work runs on the GPU.
class SimulationExecutor {
  public:
    SimulationExecutor(SimulationContext* ctx, unsigned solver_iters, double iter_acceleration, unsigned num_threads)
        : solver_(ctx, solver_iters, iter_acceleration) {
        (void)num_threads;
    }
    VBDSolver& solver() { return solver_; }
    void timeStep() { solver_.solve_Parallel(); }

  private:
    VBDSolver solver_;
};

}  // namespace Sim
