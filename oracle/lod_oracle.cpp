// lod_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the engine tick's particle passes around the MPM substep, from
// ae_engine/src/managers/simulation.rs:
//   * LOD classification (near / mid / far by distance to the player, near capped to the closest
//     max_near_particles, the rest moved to mid)            simulation.rs:495-532
//   * far-field update (gravity on y, nearest-cell blend toward the coarse temperature field)
//                                                          simulation.rs:612-679
//   * coarse temperature field update (mass-weighted injection from the near particles,
//     relaxation, one 6-neighbour FTCS diffusion step)       simulation.rs:877-966
//   * MpssBuffer housekeeping after the substep (ae_engine/src/lib.rs:347-358): reflecting world
//     bounds, temperature clamp, material phase transitions   ae_particle/src/mpss.rs:449-548
// Only tests/ and bench.py's CPU baseline load it, as the checker; the library never does.
//
// Rounding follows Rust's f32 semantics: this file is built with -ffp-contract=off (Rust never
// fuses a*b+c), `f32 as isize` truncates toward zero (NaN -> 0, saturating), and f32::max/min
// return the other argument when one is NaN, like fmaxf/fminf.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

namespace {

int64_t as_isize(float v) {  // Rust `f32 as isize`
  if (v != v) return 0;
  if (v >= 9.2233720368547758e18f) return INT64_MAX;
  if (v <= -9.2233720368547758e18f) return INT64_MIN;
  return static_cast<int64_t>(v);
}

// nearest coarse cell of a position, or -1 when outside [0, n)^3 (simulation.rs:632-647, 894-904)
int64_t coarse_cell(const float* p, const float* origin, float dx, bool by_division, uint64_t n) {
  int64_t g[3];
  for (int a = 0; a < 3; ++a) {
    // the far-field pass divides by dx (:633-635); the injection multiplies by 1/dx (:894-896)
    const float q = by_division ? (p[a] - origin[a]) / dx : (p[a] - origin[a]) * (1.0f / dx);
    g[a] = as_isize(q);
  }
  for (int a = 0; a < 3; ++a)
    if (g[a] < 0 || uint64_t(g[a]) >= n) return -1;
  return g[0] + g[1] * int64_t(n) + g[2] * int64_t(n * n);
}

}  // namespace

extern "C" {

// simulation.rs:495-532.  near_out holds the kept near particles in the order select_nth leaves
// them (the reference defines the set, not the order); mid_out the mid particles in index order
// followed by the culled near ones; far_out index order.  active may be null (all active).
void oracle_lod_classify(const float* pos, const uint8_t* active, uint64_t count, const float* player, float near_dist,
                         float mid_dist, uint64_t max_near, uint32_t* near_out, uint64_t* n_near, uint32_t* mid_out,
                         uint64_t* n_mid, uint32_t* far_out, uint64_t* n_far) {
  const float near2 = near_dist * near_dist, mid2 = mid_dist * mid_dist;
  std::vector<std::pair<uint32_t, float>> nearv;
  std::vector<uint32_t> midv, farv;
  for (uint64_t i = 0; i < count; ++i) {
    if (active && !active[i]) continue;
    const float dx = pos[3 * i] - player[0], dy = pos[3 * i + 1] - player[1], dz = pos[3 * i + 2] - player[2];
    const float d2 = dx * dx + dy * dy + dz * dz;
    if (d2 < near2)
      nearv.emplace_back(uint32_t(i), d2);
    else if (d2 < mid2)
      midv.push_back(uint32_t(i));
    else
      farv.push_back(uint32_t(i));
  }
  if (nearv.size() > max_near) {
    std::nth_element(nearv.begin(), nearv.begin() + std::ptrdiff_t(max_near), nearv.end(),
                     [](const std::pair<uint32_t, float>& a, const std::pair<uint32_t, float>& b) {
                       return a.second < b.second;
                     });
    for (size_t k = max_near; k < nearv.size(); ++k) midv.push_back(nearv[k].first);
    nearv.resize(max_near);
  }
  for (size_t k = 0; k < nearv.size(); ++k) near_out[k] = nearv[k].first;
  std::copy(midv.begin(), midv.end(), mid_out);
  std::copy(farv.begin(), farv.end(), far_out);
  *n_near = nearv.size();
  *n_mid = midv.size();
  *n_far = farv.size();
}

// simulation.rs:612-679 (the parallel and serial branches do the same per particle).
void oracle_far_field_update(float* pos, float* vel, float* temperature, const uint32_t* far_idx, uint64_t n_far,
                             const float* coarse, uint64_t coarse_n, float coarse_dx, const float* origin, float far_dt) {
  for (uint64_t k = 0; k < n_far; ++k) {
    const uint64_t i = far_idx[k];
    vel[3 * i + 1] -= 9.81f * far_dt;
    pos[3 * i + 1] += vel[3 * i + 1] * far_dt;
    const int64_t gid = coarse_cell(pos + 3 * i, origin, coarse_dx, true, coarse_n);
    if (gid >= 0) {
      const float field_t = coarse[gid];
      temperature[i] += (field_t - temperature[i]) * 0.02f * far_dt;
    }
  }
}

// simulation.rs:877-966.  coarse is n^3 cells, x fastest; updated in place.
void oracle_coarse_field_update(const float* pos, const float* mass, const float* temperature, const uint8_t* active,
                                const uint32_t* near_idx, uint64_t n_near, float* coarse, uint64_t n, float dx,
                                const float* origin, float dt) {
  const uint64_t cells = n * n * n;
  std::vector<float> tacc(cells, 0.0f), macc(cells, 0.0f);
  for (uint64_t k = 0; k < n_near; ++k) {
    const uint64_t i = near_idx[k];
    if (active && !active[i]) continue;
    const int64_t gid = coarse_cell(pos + 3 * i, origin, dx, false, n);
    if (gid < 0) continue;
    const float m = std::fmax(mass[i], 1e-6f);
    tacc[gid] += temperature[i] * m;
    macc[gid] += m;
  }
  const float inject_rate = 0.1f;
  const float blend = std::fmin(inject_rate * dt, 1.0f);
  for (uint64_t c = 0; c < cells; ++c)
    if (macc[c] > 1e-6f) {
      const float particle_temp = tacc[c] / macc[c];
      coarse[c] += (particle_temp - coarse[c]) * blend;
    }
  const float alpha = 10.0f;
  const float coef = std::fmin(alpha * dt / (dx * dx), 0.16f);
  std::vector<float> next(coarse, coarse + cells);
  const uint64_t nn = n * n;
  for (uint64_t k = 0; k < n; ++k)
    for (uint64_t j = 0; j < n; ++j)
      for (uint64_t i = 0; i < n; ++i) {
        const uint64_t gid = i + j * n + k * nn;
        float lap = 0.0f;
        int count = 0;
        if (i > 0) lap += coarse[gid - 1], ++count;
        if (i + 1 < n) lap += coarse[gid + 1], ++count;
        if (j > 0) lap += coarse[gid - n], ++count;
        if (j + 1 < n) lap += coarse[gid + n], ++count;
        if (k > 0) lap += coarse[gid - nn], ++count;
        if (k + 1 < n) lap += coarse[gid + nn], ++count;
        if (count > 0) {
          const float avg = lap / float(count);
          next[gid] += coef * (avg - coarse[gid]) * float(count);
        }
      }
  std::copy(next.begin(), next.end(), coarse);
}

// MpssPhase (mpss.rs:67-75): Solid 0, Liquid 1, Gas 2, Plasma 3, Granular 4, Crystal 5, Amorphous 6.
// One hop of the transition table of apply_phase_transitions (mpss.rs:401-416, 512-524): the arms
// in order, a failing guard falling through to the next arm.
static uint8_t phase_hop(uint16_t m, uint8_t cur, float t) {
  if (m == 1 && cur == 0 && t >= 273.0f) return 1;
  if (m == 1 && cur == 1 && t >= 373.0f) return 2;
  if (m == 1 && cur == 2 && t < 373.0f) return 1;
  if (m == 1 && cur == 1 && t < 273.0f) return 0;
  if (m == 3 && cur == 0 && t >= 1811.0f) return 1;
  if (m == 3 && cur == 1 && t >= 3134.0f) return 2;
  if (m == 3 && cur == 2 && t < 3134.0f) return 1;
  if (m == 3 && cur == 1 && t < 1811.0f) return 0;
  if (m == 0 && cur == 0 && t >= 500.0f) return 2;
  if (m == 2 && cur == 0 && t >= 1923.0f) return 2;
  return cur;
}

// The three passes ae_engine/src/lib.rs:347-358 runs after update_fields_and_particles, as their
// serial forms (mpss.rs:344-430; the _par forms do the same per particle).  passes: 1 boundary,
// 2 temperature clamp, 4 phase transitions, applied in that order.  Returns the transition count.
uint32_t oracle_mpss_housekeeping(float* pos, float* vel, float* temperature, uint8_t* phase, const uint16_t* material,
                                  const uint8_t* active, uint64_t count, const float* bmin, const float* bmax,
                                  float min_temp, float max_temp, uint32_t passes) {
  if (passes & 1u)
    for (uint64_t i = 0; i < count; ++i) {
      if (active && !active[i]) continue;
      for (int d = 0; d < 3; ++d) {
        float& p = pos[3 * i + d];
        float& v = vel[3 * i + d];
        if (p < bmin[d]) {
          p = bmin[d];
          if (v < 0.0f) v = -v * 0.5f;
        } else if (p > bmax[d]) {
          p = bmax[d];
          if (v > 0.0f) v = -v * 0.5f;
        }
      }
    }
  if (passes & 2u)
    for (uint64_t i = 0; i < count; ++i) {
      if (active && !active[i]) continue;
      if (temperature[i] > max_temp)
        temperature[i] = max_temp;
      else if (temperature[i] < min_temp)
        temperature[i] = min_temp;
    }
  uint32_t transitions = 0;
  if (passes & 4u)
    for (uint64_t i = 0; i < count; ++i) {
      if (active && !active[i]) continue;
      uint8_t cur = phase[i];
      for (int hop = 0; hop < 3; ++hop) {
        const uint8_t next = phase_hop(material[i], cur, temperature[i]);
        if (next == cur) break;
        cur = next;
      }
      if (cur != phase[i]) {
        phase[i] = cur;
        ++transitions;
      }
    }
  return transitions;
}

}  // extern "C"
