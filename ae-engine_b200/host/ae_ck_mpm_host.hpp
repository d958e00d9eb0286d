// ae_ck_mpm_host.hpp -- C++ mirror of the reference's CK-MPM solver API
// (ae_compute::ck_mpm, ae_compute/src/ck_mpm.rs), running on the CUDA library.
//
// Same names and argument meaning as the Rust module: CkMpmConfig with its defaults, CkMpmParticle
// with CkMpmParticle::new, CkMpmSolver with new / add_particle / step / kinetic_energy /
// average_velocity / average_volume_ratio and the kernel functions weight / weight_grad.  The
// particles live in the solver's host vector, as in the reference; step() hands them to the
// library (include/ae_mpm.h, ae_mpm_ck_step), which copies them to the GPU, steps them and copies
// them back.  grid_a and grid_b are allocated as the reference allocates them, but the device keeps
// its own grid and does not write these back (the reference reads them nowhere outside step).
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "ae_mpm.h"
#include "ae_mpm_host.hpp"

namespace ae_compute {

struct Vec3 {  // glam::Vec3
  float x = 0.0f, y = 0.0f, z = 0.0f;
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

struct Mat3 {  // glam::Mat3: three columns
  Vec3 x_axis, y_axis, z_axis;
  static Mat3 zero() { return Mat3{}; }
  static Mat3 identity() { return Mat3{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}; }
  float determinant() const {  // z_axis . (x_axis cross y_axis), as glam computes it
    const Vec3 c{x_axis.y * y_axis.z - y_axis.y * x_axis.z, x_axis.z * y_axis.x - y_axis.z * x_axis.x,
                 x_axis.x * y_axis.y - y_axis.x * x_axis.y};
    return z_axis.x * c.x + z_axis.y * c.y + z_axis.z * c.z;
  }
  bool operator==(const Mat3& o) const {
    const float* a = &x_axis.x;
    const float* b = &o.x_axis.x;
    for (int i = 0; i < 9; ++i)
      if (a[i] != b[i]) return false;
    return true;
  }
};

// ck_mpm.rs:41-77
struct CkMpmConfig {
  float dt = 1.0f / 240.0f;
  float grid_h = 0.05f;
  size_t grid_n = 32;
  Vec3 gravity{0.0f, -9.81f, 0.0f};
  float youngs_modulus = 1e5f;
  float poissons_ratio = 0.3f;
  float density = 1000.0f;
  Vec3 bounds_min{-1.0f, -1.0f, -1.0f};
  Vec3 bounds_max{1.0f, 1.0f, 1.0f};
  float restitution = 0.3f;
  bool dual_grid = true;
};

// ck_mpm.rs:84-108; laid out as the library's ae_mpm_ck_particle
struct CkMpmParticle {
  Vec3 position;
  Vec3 velocity;
  Mat3 affine;
  Mat3 deformation;
  float rest_volume = 0.0f;
  float mass = 0.0f;

  static CkMpmParticle new_(Vec3 position, float mass, float rest_volume) {
    CkMpmParticle p;
    p.position = position;
    p.affine = Mat3::zero();
    p.deformation = Mat3::identity();
    p.rest_volume = rest_volume;
    p.mass = mass;
    return p;
  }
};
static_assert(sizeof(CkMpmParticle) == sizeof(ae_mpm_ck_particle) && std::is_standard_layout<CkMpmParticle>::value,
              "CkMpmParticle must have the library's record layout");

// ck_mpm.rs:114-120
struct GridNode {
  Vec3 velocity;
  float mass = 0.0f;
  Vec3 force;
};

// ck_mpm.rs:126-508
class CkMpmSolver {
 public:
  CkMpmConfig config;
  std::vector<CkMpmParticle> particles;
  std::vector<GridNode> grid_a, grid_b;
  // add node sums in particle order, as the reference does (bitwise reproducible, slower)
  bool deterministic = false;

  explicit CkMpmSolver(const CkMpmConfig& c) : config(c) {
    const size_t n = c.grid_n + 2;
    grid_a.resize(n * n * n);
    grid_b.resize(n * n * n);
  }
  static CkMpmSolver new_(const CkMpmConfig& c) { return CkMpmSolver(c); }

  size_t add_particle(const CkMpmParticle& p) {
    particles.push_back(p);
    return particles.size() - 1;
  }

  // CkMpmSolver::step (:187-480) on the GPU
  void step() { step_n(1); }
  // `steps` calls of step() in one library call: the particles stay on the GPU in between
  void step_n(uint32_t steps) {
    if (particles.empty()) return;
    const ae_mpm_ck_config c = to_c();
    auto* recs = reinterpret_cast<ae_mpm_ck_particle*>(particles.data());
    ae_particle::check(deterministic
                           ? ae_mpm_ck_step_deterministic(ae_particle::gpu_context(), recs, particles.size(), &c, steps)
                           : ae_mpm_ck_step(ae_particle::gpu_context(), recs, particles.size(), &c, steps));
  }

  // :484-503
  float kinetic_energy() const { return stats().kinetic_energy; }
  Vec3 average_velocity() const {
    const ae_mpm_ck_stats s = stats();
    return Vec3{s.average_velocity[0], s.average_velocity[1], s.average_velocity[2]};
  }
  float average_volume_ratio() const { return stats().average_volume_ratio; }

  // :163-185, evaluated by the device code the step uses
  static float weight(float x, float h) { return weights(x, h)[0]; }
  static float weight_grad(float x, float h) { return weights(x, h)[1]; }

 private:
  ae_mpm_ck_config to_c() const {
    ae_mpm_ck_config c{};
    c.dt = config.dt;
    c.grid_h = config.grid_h;
    c.grid_n = uint32_t(config.grid_n);
    for (int a = 0; a < 3; ++a) {
      c.gravity[a] = config.gravity[a];
      c.bounds_min[a] = config.bounds_min[a];
      c.bounds_max[a] = config.bounds_max[a];
    }
    c.youngs_modulus = config.youngs_modulus;
    c.poissons_ratio = config.poissons_ratio;
    c.density = config.density;
    c.restitution = config.restitution;
    c.dual_grid = config.dual_grid ? 1 : 0;
    return c;
  }
  ae_mpm_ck_stats stats() const {
    ae_mpm_ck_stats s{};
    ae_particle::check(ae_mpm_ck_stats_compute(ae_particle::gpu_context(),
                                               reinterpret_cast<const ae_mpm_ck_particle*>(particles.data()),
                                               particles.size(), &s));
    return s;
  }
  static std::array<float, 2> weights(float x, float h) {
    float w = 0.0f, dw = 0.0f;
    ae_particle::check(ae_mpm_ck_weights(ae_particle::gpu_context(), &x, 1, h, &w, &dw));
    return {w, dw};
  }
};

}  // namespace ae_compute
