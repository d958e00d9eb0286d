// ae_mpm_host.hpp -- C++ mirror of the reference's Rust MPM API, running on the CUDA library.
//
// Mirrors ae_particle::mpm_solver (ae_particle/src/mpm_solver.rs), ae_particle::constitutive
// (ae_particle/src/constitutive.rs) and the MPM fields of ae_particle::mpss::MpssBuffer
// (ae_particle/src/mpss.rs:105-445): same names, same argument meaning.  Where the Rust code
// panics (empty material table, index out of range) these functions throw std::runtime_error
// carrying the library's message.  The substep itself runs on the GPU through include/ae_mpm.h;
// this header only packs arguments, exactly as a Rust FFI crate would.
#pragma once
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "ae_mpm.h"

namespace ae_particle {

// constitutive.rs:12-27
enum class ConstitutiveModel : int32_t {
  NeoHookean = AE_MPM_NEO_HOOKEAN,
  DruckerPrager = AE_MPM_DRUCKER_PRAGER,
  VonMises = AE_MPM_VON_MISES,
  NewtonianFluid = AE_MPM_NEWTONIAN_FLUID,
  Corotated = AE_MPM_COROTATED,
  FixedCorotated = AE_MPM_FIXED_COROTATED,
  Rigid = AE_MPM_RIGID,
};

// constitutive.rs:31-82
struct MaterialParams {
  float young_modulus = 1e6f;
  float poisson_ratio = 0.3f;
  float yield_stress = 1e4f;
  float hardening = 0.01f;
  float density = 1000.0f;
  float friction_angle = 35.0f;
  float cohesion = 0.0f;
  float clamped_nu() const { return std::fmin(std::fmax(poisson_ratio, -0.999f), 0.4999f); }
  float lambda() const {
    float nu = clamped_nu();
    return young_modulus * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
  }
  float mu() const { return young_modulus / (2.0f * (1.0f + clamped_nu())); }
  float bulk_modulus() const { return young_modulus / (3.0f * (1.0f - 2.0f * clamped_nu())); }
};

// mpm_solver.rs:46-70
struct MpmConfig {
  float grid_dx = 1.6f;
  std::array<size_t, 3> grid_size{{16, 16, 16}};
  size_t substeps = 1;
  std::array<float, 3> gravity{{0.0f, -9.81f, 0.0f}};
  float damping = 0.995f;
  bool enable_plasticity = true;
  bool enable_contact = true;
  bool use_sparse_grid = true;
};

// mpm_solver.rs:73-176.  The node arrays live on the device during a step; `mass` and `vel`
// are filled by download_from_device() on request.
struct Grid {
  std::vector<float> mass;
  std::vector<std::array<float, 3>> vel;
  std::vector<std::array<float, 3>> force;
  size_t nx = 0, ny = 0, nz = 0;
  float dx = 1.0f, inv_dx = 1.0f;
  std::array<float, 3> origin{{0.0f, 0.0f, 0.0f}};

  static Grid create(size_t nx, size_t ny, size_t nz, float dx) {
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.dx = dx;
    g.inv_dx = 1.0f / dx;
    g.mass.assign(nx * ny * nz, 0.0f);
    g.vel.assign(nx * ny * nz, {{0.0f, 0.0f, 0.0f}});
    g.force.assign(nx * ny * nz, {{0.0f, 0.0f, 0.0f}});
    return g;
  }
  void reset() {
    std::fill(mass.begin(), mass.end(), 0.0f);
    std::fill(vel.begin(), vel.end(), std::array<float, 3>{{0.0f, 0.0f, 0.0f}});
    std::fill(force.begin(), force.end(), std::array<float, 3>{{0.0f, 0.0f, 0.0f}});
  }
  size_t index(size_t i, size_t j, size_t k) const { return i + j * nx + k * nx * ny; }
  // mpm_solver.rs:161-175
  void pos_to_grid(const std::array<float, 3>& pos, size_t out_g[3], float fx[3]) const {
    for (int a = 0; a < 3; ++a) {
      float q = (pos[a] - origin[a]) * inv_dx - 0.5f;
      long g = long(std::floor(q));
      fx[a] = q - float(g);
      out_g[a] = size_t(g < 0 ? 0 : g);
    }
  }
};

// The MPM-relevant part of MpssBuffer (mpss.rs:105-213, 431-445).
struct MpssBuffer {
  size_t capacity = 0, count = 0;
  std::vector<std::array<float, 3>> pos, vel;
  std::vector<std::array<float, 9>> strain;
  std::vector<float> jacobian;
  std::vector<std::array<float, 9>> c;
  std::vector<float> mass;
  std::vector<uint16_t> material_idx;
  std::vector<float> lifetime, age;
  std::vector<bool> active;
  std::vector<size_t> free_list;

  explicit MpssBuffer(size_t cap)
      : capacity(cap), pos(cap, {{0, 0, 0}}), vel(cap, {{0, 0, 0}}), strain(cap, {{0, 0, 0, 0, 0, 0, 0, 0, 0}}),
        jacobian(cap, 1.0f), c(cap, {{0, 0, 0, 0, 0, 0, 0, 0, 0}}), mass(cap, 1.0f), material_idx(cap, 0),
        lifetime(cap, std::numeric_limits<float>::max()), age(cap, 0.0f), active(cap, false) {}

  void reset_slot(size_t i) {
    pos[i] = {{0, 0, 0}};
    vel[i] = {{0, 0, 0}};
    strain[i] = {{1, 0, 0, 0, 1, 0, 0, 0, 1}};
    jacobian[i] = 1.0f;
    c[i] = {{0, 0, 0, 0, 0, 0, 0, 0, 0}};
    mass[i] = 1.0f;
    material_idx[i] = 0;
    lifetime[i] = std::numeric_limits<float>::max();
    age[i] = 0.0f;
  }
  // mpss.rs:189-204; returns capacity when full (Rust: None)
  size_t spawn() {
    size_t idx;
    if (!free_list.empty()) {
      idx = free_list.back();
      free_list.pop_back();
    } else if (count < capacity) {
      idx = count;
    } else {
      return capacity;
    }
    reset_slot(idx);
    active[idx] = true;
    ++count;
    return idx;
  }
  void kill(size_t idx) {
    if (idx < capacity && active[idx]) {
      active[idx] = false;
      free_list.push_back(idx);
      --count;
    }
  }
  std::vector<size_t> update_lifetimes(float dt) {  // mpss.rs:431-445
    std::vector<size_t> expired;
    for (size_t i = 0; i < count; ++i)
      if (active[i]) {
        age[i] += dt;
        if (age[i] >= lifetime[i]) expired.push_back(i);
      }
    for (size_t i : expired) kill(i);
    return expired;
  }
  ae_mpm_particles view() {
    ae_mpm_particles v;
    v.pos = pos[0].data();
    v.vel = vel[0].data();
    v.strain = strain[0].data();
    v.jacobian = jacobian.data();
    v.c = c[0].data();
    v.mass = mass.data();
    v.material_idx = material_idx.data();
    return v;
  }
};

// Process-wide library context on device 0 (the Rust crate keeps the same in a OnceLock).
inline ae_mpm_ctx* gpu_context() {
  static std::once_flag once;
  static ae_mpm_ctx* ctx = nullptr;
  std::call_once(once, [] {
    if (ae_mpm_ctx_create(0, &ctx) != AE_MPM_OK) ctx = nullptr;
  });
  if (!ctx) throw std::runtime_error("ae_mpm: no usable CUDA device");
  return ctx;
}

inline void check(int rc) {
  if (rc != AE_MPM_OK) throw std::runtime_error(std::string("ae_mpm: ") + ae_mpm_last_error(gpu_context()));
}

inline ae_mpm_config to_c(const MpmConfig& c) {
  ae_mpm_config o{};
  o.grid_dx = c.grid_dx;
  for (int a = 0; a < 3; ++a) {
    o.grid_size[a] = c.grid_size[a];
    o.gravity[a] = c.gravity[a];
  }
  o.substeps = c.substeps;
  o.damping = c.damping;
  o.enable_plasticity = c.enable_plasticity;
  o.enable_contact = c.enable_contact;
  o.use_sparse_grid = c.use_sparse_grid;
  return o;
}

inline ae_mpm_grid to_c(const Grid& g) {
  ae_mpm_grid o{};
  o.nx = g.nx;
  o.ny = g.ny;
  o.nz = g.nz;
  o.dx = g.dx;
  for (int a = 0; a < 3; ++a) o.origin[a] = g.origin[a];
  return o;
}

// mpm_solver.rs:1063-1084
inline void mpm_step_parallel_with_grid(MpssBuffer& buffer, Grid& grid, const MpmConfig& config,
                                        const std::vector<MaterialParams>& material_table,
                                        const std::vector<ConstitutiveModel>& model_table, float total_dt,
                                        const std::vector<size_t>& particle_indices) {
  if (particle_indices.empty()) return;
  if (material_table.empty()) throw std::runtime_error("index out of bounds: the len is 0 but the index is 0");
  std::vector<ae_mpm_material> mats(material_table.size());
  for (size_t k = 0; k < mats.size(); ++k) {
    const MaterialParams& m = material_table[k];
    mats[k] = ae_mpm_material{m.young_modulus, m.poisson_ratio, m.yield_stress, m.hardening, m.density,
                              m.friction_angle, m.cohesion, AE_MPM_NEO_HOOKEAN, 0, 0, 0, 0};
  }
  std::vector<int32_t> models(model_table.size());
  for (size_t k = 0; k < models.size(); ++k) models[k] = int32_t(model_table[k]);
  std::vector<uint64_t> idx(particle_indices.begin(), particle_indices.end());
  ae_mpm_particles v = buffer.view();
  ae_mpm_grid g = to_c(grid);
  ae_mpm_config c = to_c(config);
  check(ae_mpm_step_parallel_with_grid(gpu_context(), &v, buffer.capacity, &g, &c, mats.data(), uint32_t(mats.size()),
                                       models.data(), uint32_t(models.size()), total_dt, idx.data(), idx.size()));
  buffer.update_lifetimes(total_dt);
}

// indices of the particles `mpm_substep` visits: 0..count with the active check (mpm_solver.rs:189-193)
inline std::vector<size_t> active_indices(const MpssBuffer& b) {
  std::vector<size_t> idx;
  for (size_t i = 0; i < b.count; ++i)
    if (b.active[i]) idx.push_back(i);
  return idx;
}

// mpm_solver.rs:493-509 (reusable grid; the substep has the serial path's rules)
inline void mpm_step_with_grid(MpssBuffer& buffer, Grid& grid, const MpmConfig& config,
                               const std::vector<MaterialParams>& material_table,
                               const std::vector<ConstitutiveModel>& model_table, float total_dt) {
  std::vector<size_t> idx = active_indices(buffer);
  if (idx.empty()) {
    buffer.update_lifetimes(total_dt);
    return;
  }
  MpssBuffer& b = buffer;
  if (material_table.empty()) throw std::runtime_error("index out of bounds: the len is 0 but the index is 0");
  std::vector<ae_mpm_material> mats(material_table.size());
  for (size_t k = 0; k < mats.size(); ++k) {
    const MaterialParams& m = material_table[k];
    mats[k] = ae_mpm_material{m.young_modulus, m.poisson_ratio, m.yield_stress, m.hardening, m.density,
                              m.friction_angle, m.cohesion, AE_MPM_NEO_HOOKEAN, 0, 0, 0, 0};
  }
  std::vector<int32_t> models(model_table.size());
  for (size_t k = 0; k < models.size(); ++k) models[k] = int32_t(model_table[k]);
  std::vector<uint64_t> id64(idx.begin(), idx.end());
  ae_mpm_particles v = b.view();
  ae_mpm_grid g = to_c(grid);
  ae_mpm_config c = to_c(config);
  check(ae_mpm_step_parallel_with_grid(gpu_context(), &v, b.capacity, &g, &c, mats.data(), uint32_t(mats.size()),
                                       models.data(), uint32_t(models.size()), total_dt, id64.data(), id64.size()));
  buffer.update_lifetimes(total_dt);
}

// mpm_solver.rs:470-490 (allocates a grid from the config)
inline void mpm_step(MpssBuffer& buffer, const MpmConfig& config, const std::vector<MaterialParams>& material_table,
                     const std::vector<ConstitutiveModel>& model_table, float total_dt) {
  Grid grid = Grid::create(config.grid_size[0], config.grid_size[1], config.grid_size[2], config.grid_dx);
  mpm_step_with_grid(buffer, grid, config, material_table, model_table, total_dt);
}

// mpm_solver.rs:1337-1351
inline void mpm_step_velocity_only_parallel(MpssBuffer& buffer, Grid& grid, const MpmConfig& config, float total_dt,
                                            const std::vector<size_t>& particle_indices) {
  if (particle_indices.empty()) return;
  std::vector<uint64_t> idx(particle_indices.begin(), particle_indices.end());
  ae_mpm_particles v = buffer.view();
  ae_mpm_grid g = to_c(grid);
  ae_mpm_config c = to_c(config);
  check(ae_mpm_step_velocity_only_parallel(gpu_context(), &v, buffer.capacity, &g, &c, total_dt, idx.data(), idx.size()));
}

// mpm_solver.rs:1575-1588 (host-side: a reduction over the caller's buffer)
inline float estimate_cfl(const MpssBuffer& buffer, float dx) {
  float max_v = 0.0f;
  for (size_t i = 0; i < buffer.capacity; ++i)
    if (buffer.active[i]) {
      const auto& v = buffer.vel[i];
      max_v = std::fmax(max_v, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
  if (max_v < 1e-6f) return 0.016f;
  return std::fmin(dx * 0.3f / max_v, 0.016f);
}

// Copies the device grid of the last step into grid.mass / grid.vel (reference index order).
inline void download_grid(Grid& grid) {
  std::vector<float> v(3 * grid.nx * grid.ny * grid.nz);
  check(ae_mpm_grid_download(gpu_context(), grid.mass.data(), v.data(), grid.mass.size()));
  for (size_t i = 0; i < grid.vel.size(); ++i) grid.vel[i] = {{v[3 * i], v[3 * i + 1], v[3 * i + 2]}};
}

}  // namespace ae_particle
