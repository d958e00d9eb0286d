// test_host_mirror.cpp -- the reference's own mpm_solver unit tests, re-run on the GPU through
// the C++ mirror of its API (ae-engine_b200/host/ae_mpm_host.hpp -> include/ae_mpm.h).
//
//   test_sandpile_static_angle   ae_particle/src/mpm_solver.rs:1611-1657
//   test_water_pressure          ae_particle/src/mpm_solver.rs:1659-1711
//   test_steel_rigid_fall        ae_particle/src/mpm_solver.rs:1713-1745
// plus the engine's near-field call shape (ae_engine/src/managers/simulation.rs:573-581) with an
// index list, the velocity-only mid-field call (:598-607), and the panic paths.
// Prints one line per test and exits non-zero if any failed.
#include <cmath>
#include <cstdio>
#include <functional>
#include <string>

#include "ae_mpm_host.hpp"

using namespace ae_particle;

static int failures = 0;

static void run(const char* name, const std::function<std::string()>& f) {
  std::string msg;
  try {
    msg = f();
  } catch (const std::exception& e) {
    msg = std::string("exception: ") + e.what();
  }
  if (msg.empty()) {
    std::printf("PASS %s\n", name);
  } else {
    std::printf("FAIL %s: %s\n", name, msg.c_str());
    ++failures;
  }
  std::fflush(stdout);
}

int main() {
  run("test_sandpile_static_angle", [] {
    MpssBuffer buf(1000);
    MpmConfig config;
    config.substeps = 8;
    MaterialParams sand{1.0e4f, 0.2f, 1.0e3f, 0.005f, 1600.0f, 35.0f, 0.0f};
    std::vector<MaterialParams> materials{sand};
    std::vector<ConstitutiveModel> models{ConstitutiveModel::DruckerPrager};
    for (int x = 0; x < 10; ++x)
      for (int y = 0; y < 10; ++y)
        for (int z = 0; z < 10; ++z) {
          size_t idx = buf.spawn();
          buf.pos[idx] = {{x * 0.05f, y * 0.05f + 0.5f, z * 0.05f}};
          buf.mass[idx] = 0.001f;
          buf.material_idx[idx] = 0;
        }
    for (int f = 0; f < 60; ++f) mpm_step(buf, config, materials, models, 0.016f);
    for (size_t i = 0; i < buf.capacity; ++i)
      if (buf.active[i] && !(buf.pos[i][1] >= 0.0f))
        return "particle " + std::to_string(i) + " penetrated floor: y=" + std::to_string(buf.pos[i][1]);
    return std::string();
  });

  run("test_water_pressure", [] {
    MpssBuffer buf(300);
    MpmConfig config;
    config.grid_dx = 0.05f;
    config.grid_size = {{32, 32, 32}};
    config.substeps = 8;
    MaterialParams water{1.0e3f, 0.499f, 0.0f, 0.0f, 1000.0f, 0.0f, 0.0f};
    std::vector<MaterialParams> materials{water};
    std::vector<ConstitutiveModel> models{ConstitutiveModel::NewtonianFluid};
    for (int y = 0; y < 10; ++y)
      for (int x = 0; x < 5; ++x)
        for (int z = 0; z < 5; ++z) {
          size_t idx = buf.spawn();
          buf.pos[idx] = {{x * 0.05f, y * 0.05f + 0.1f, z * 0.05f}};
          buf.mass[idx] = 0.001f;
          buf.material_idx[idx] = 0;
          buf.jacobian[idx] = 0.95f;
        }
    mpm_step(buf, config, materials, models, 0.016f);
    for (size_t i = 0; i < buf.capacity; ++i)
      if (buf.active[i]) {
        float j = buf.jacobian[i];
        if (!std::isfinite(j)) return "J is NaN/inf at " + std::to_string(i);
        if (!(j > 0.0f && j < 100.0f)) return "J exploded at " + std::to_string(i) + ": " + std::to_string(j);
      }
    return std::string();
  });

  run("test_steel_rigid_fall", [] {
    MpssBuffer buf(100);
    MpmConfig config;
    config.grid_dx = 0.02f;
    config.grid_size = {{32, 32, 32}};
    config.substeps = 8;
    MaterialParams steel{1.0e5f, 0.3f, 1.0e4f, 0.01f, 7850.0f, 0.0f, 0.0f};
    std::vector<MaterialParams> materials{steel};
    std::vector<ConstitutiveModel> models{ConstitutiveModel::VonMises};
    size_t idx = buf.spawn();
    buf.pos[idx] = {{0.2f, 0.5f, 0.2f}};
    buf.mass[idx] = 0.01f;
    float y0 = buf.pos[idx][1];
    for (int f = 0; f < 30; ++f) mpm_step(buf, config, materials, models, 0.016f);
    float y1 = buf.pos[idx][1];
    if (!(y1 < y0)) return "steel didn't fall: " + std::to_string(y0) + " -> " + std::to_string(y1);
    if (!(y1 >= 0.0f)) return "steel penetrated floor: " + std::to_string(y1);
    return std::string();
  });

  // engine call shape: 64^3 grid at dx 1.6 around a moving-window origin, the engine's 4-entry
  // material/model tables (simulation.rs:251-294), near-field index list, lifetimes updated
  run("engine_near_field_call", [] {
    MpssBuffer buf(4096);
    MpmConfig cfg;
    cfg.grid_size = {{64, 64, 64}};
    Grid grid = Grid::create(64, 64, 64, 1.6f);
    grid.origin = {{-51.2f, 0.0f, -51.2f}};
    std::vector<MaterialParams> mats{{1.0e6f, 0.3f, 1.0e4f, 0.01f, 1000.0f, 35.0f, 0.0f},
                                     {2.0e6f, 0.45f, 0.0f, 0.0f, 1000.0f, 0.0f, 0.0f},
                                     {5.0e7f, 0.3f, 0.0f, 0.0f, 1600.0f, 35.0f, 0.0f},
                                     {2.0e11f, 0.3f, 2.5e8f, 0.01f, 7850.0f, 0.0f, 0.0f}};
    std::vector<ConstitutiveModel> models{ConstitutiveModel::NeoHookean, ConstitutiveModel::NewtonianFluid,
                                          ConstitutiveModel::DruckerPrager, ConstitutiveModel::VonMises};
    std::vector<size_t> near;
    for (int i = 0; i < 3000; ++i) {
      size_t idx = buf.spawn();
      buf.pos[idx] = {{-5.0f + 0.37f * (i % 27), 2.0f + 0.41f * ((i / 27) % 11), -4.0f + 0.29f * (i / 297)}};
      buf.mass[idx] = 1.0f;
      buf.material_idx[idx] = uint16_t(i % 5);  // index 4 exercises the material_table[0] fallback
      buf.lifetime[idx] = (i % 7 == 0) ? 0.01f : 1e9f;
      if (i % 3 != 0) near.push_back(idx);
    }
    size_t before = buf.count;
    for (int f = 0; f < 5; ++f) mpm_step_parallel_with_grid(buf, grid, cfg, mats, models, 1.0f / 60.0f, near);
    for (size_t i : near)
      for (int a = 0; a < 3; ++a)
        if (!std::isfinite(buf.pos[i][a])) return std::string("non-finite position at ") + std::to_string(i);
    if (buf.count >= before) return std::string("update_lifetimes expired nothing");
    download_grid(grid);
    double m = 0;
    for (float x : grid.mass) m += x;
    if (!(m > 0.0)) return std::string("grid mass after the step is zero");
    return std::string();
  });

  run("velocity_only_mid_field", [] {
    MpssBuffer buf(2000);
    MpmConfig cfg;
    Grid grid = Grid::create(16, 16, 16, 25.0f);
    std::vector<size_t> mid;
    for (int i = 0; i < 2000; ++i) {
      size_t idx = buf.spawn();
      buf.pos[idx] = {{50.0f + (i % 20) * 7.0f, 120.0f + (i / 20 % 10) * 5.0f, 60.0f + (i / 200) * 9.0f}};
      mid.push_back(idx);
    }
    mpm_step_velocity_only_parallel(buf, grid, cfg, 12.0f / 60.0f, mid);
    for (size_t i : mid)
      if (!(buf.vel[i][1] < 0.0f)) return "mid-field particle did not start falling: " + std::to_string(i);
    return std::string();
  });

  run("empty_material_table_panics", [] {
    MpssBuffer buf(4);
    size_t i = buf.spawn();
    buf.pos[i] = {{0.5f, 0.5f, 0.5f}};
    Grid grid = Grid::create(8, 8, 8, 0.25f);
    try {
      mpm_step_parallel_with_grid(buf, grid, MpmConfig{}, {}, {}, 0.016f, {i});
    } catch (const std::runtime_error&) {
      return std::string();
    }
    return std::string("no panic on an empty material table");
  });

  run("empty_index_list_is_a_no_op", [] {
    MpssBuffer buf(4);
    size_t i = buf.spawn();
    buf.pos[i] = {{0.5f, 0.5f, 0.5f}};
    buf.lifetime[i] = 0.001f;
    Grid grid = Grid::create(8, 8, 8, 0.25f);
    mpm_step_parallel_with_grid(buf, grid, MpmConfig{}, {}, {}, 0.016f, {});
    if (buf.count != 1) return std::string("lifetimes were updated on an empty call");
    return std::string();
  });

  std::printf("%s\n", failures ? "SOME HOST-MIRROR TESTS FAILED" : "ALL HOST-MIRROR TESTS PASSED");
  return failures ? 1 : 0;
}
