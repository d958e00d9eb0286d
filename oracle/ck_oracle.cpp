// ck_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's CK-MPM solver, CkMpmSolver::step
// (ae_compute/src/ck_mpm.rs:187-480): compact C^2 kernel w(x) = (1 - (x/h)^2)^3 / h on the 2 nodes
// per axis around a particle (nodes at (i + 1/2) h, i = floor(x/h) + {0, 1}), APIC transfer,
// neo-Hookean forces, guarded grid and particle updates.  Only tests/ and bench.py's CPU baseline
// load it, as the checker.
//
// Kept as the reference has it: `dual_grid` is read nowhere (grid_b is never written); the
// velocity gradient scales the APIC matrix by D^-1 = 4/h^2 a second time (:438).
// Rounding follows Rust's f32 semantics: built with -ffp-contract=off, glam's operation order
// for Mat3 x Vec3 (x_axis*v.x + y_axis*v.y + z_axis*v.z), determinant (z . (x cross y)) and
// inverse (columns y cross z, z cross x, x cross y, transposed, times 1/det), and f32::ln as
// the C library's logf.
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct V3 {
  float x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
float length(V3 a) { return std::sqrt(dot(a, a)); }
bool finite(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

struct M3 {  // glam Mat3: three columns
  V3 c[3];
};
V3 mul(const M3& m, V3 v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }
M3 mul(const M3& a, const M3& b) { return {{mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2])}}; }
M3 add(const M3& a, const M3& b) { return {{a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]}}; }
M3 sub(const M3& a, const M3& b) { return {{a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]}}; }
M3 scale(const M3& a, float s) { return {{a.c[0] * s, a.c[1] * s, a.c[2] * s}}; }
M3 transpose(const M3& m) {
  return {{{m.c[0].x, m.c[1].x, m.c[2].x}, {m.c[0].y, m.c[1].y, m.c[2].y}, {m.c[0].z, m.c[1].z, m.c[2].z}}};
}
float det(const M3& m) { return dot(m.c[2], cross(m.c[0], m.c[1])); }
M3 inverse(const M3& m) {
  const V3 t0 = cross(m.c[1], m.c[2]), t1 = cross(m.c[2], m.c[0]), t2 = cross(m.c[0], m.c[1]);
  const float d = dot(m.c[2], t2);
  const float inv = 1.0f / d;
  return scale(transpose(M3{{t0, t1, t2}}), inv);
}
const M3 kIdentity{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};

float weight(float x, float h) {  // ck_mpm.rs:163-176
  const float r = std::fabs(x) / h;
  if (r >= 1.0f) return 0.0f;
  const float a = 1.0f - r * r;
  return a * a * a / h;  // powi(3): a * a * a
}
float weight_grad(float x, float h) {  // :178-185
  const float r = std::fabs(x) / h;
  if (r >= 1.0f) return 0.0f;
  const float a = 1.0f - r * r;
  return -6.0f * x * (a * a) / (h * h * h);
}

// Rust `f32 as i32`: truncation, NaN -> 0, saturating.  The stencil offsets are then added in
// 64 bits: where Rust's i32 add wraps past i32::MAX the node is out of range either way.
int32_t as_i32(float v) {
  if (v != v) return 0;
  if (v >= 2147483648.0f) return INT32_MAX;
  if (v <= -2147483904.0f) return INT32_MIN;
  return static_cast<int32_t>(v);
}

}  // namespace

extern "C" {

// CkMpmConfig (ck_mpm.rs:41-59) and CkMpmParticle (:84-95) in the library's C layout
struct OracleCkConfig {
  float dt, grid_h;
  uint32_t grid_n;
  float gravity[3];
  float youngs_modulus, poissons_ratio, density;
  float bounds_min[3], bounds_max[3];
  float restitution;
  uint8_t dual_grid, pad[3];
};
struct OracleCkParticle {
  float position[3], velocity[3], affine[9], deformation[9], rest_volume, mass;
};

// correctly_rounded_ln: take f32::ln as the correctly rounded logarithm (the double-precision
// log rounded to f32) instead of the C library's logf.  Only a checker for the device's
// deterministic mode uses it, to isolate the one operation where the device and the reference's
// libm may differ; the reference's semantics are correctly_rounded_ln = 0.
void oracle_ck_step_ln(OracleCkParticle* ps, uint64_t n, const OracleCkConfig* cfg, uint32_t steps,
                       int correctly_rounded_ln) {
  const float h = cfg->grid_h, dt = cfg->dt;
  const int32_t gn = int32_t(cfg->grid_n);
  const uint64_t np = uint64_t(gn) + 2;
  std::vector<V3> gvel(np * np * np), gforce(np * np * np);
  std::vector<float> gmass(np * np * np);
  auto gidx = [np](int64_t i, int64_t j, int64_t k) { return uint64_t(i) + np * (uint64_t(j) + np * uint64_t(k)); };
  auto load = [](const float* a) { return M3{{{a[0], a[1], a[2]}, {a[3], a[4], a[5]}, {a[6], a[7], a[8]}}}; };
  auto store = [](const M3& m, float* a) {
    for (int c = 0; c < 3; ++c) {
      a[3 * c] = m.c[c].x;
      a[3 * c + 1] = m.c[c].y;
      a[3 * c + 2] = m.c[c].z;
    }
  };
  const V3 g{cfg->gravity[0], cfg->gravity[1], cfg->gravity[2]};
  const float bmin[3] = {cfg->bounds_min[0], cfg->bounds_min[1], cfg->bounds_min[2]};
  const float bmax[3] = {cfg->bounds_max[0], cfg->bounds_max[1], cfg->bounds_max[2]};
  for (uint32_t s = 0; s < steps && n > 0; ++s) {
    std::fill(gvel.begin(), gvel.end(), V3{0, 0, 0});
    std::fill(gforce.begin(), gforce.end(), V3{0, 0, 0});
    std::fill(gmass.begin(), gmass.end(), 0.0f);
    // 2. P2G (:200-242)
    for (uint64_t q = 0; q < n; ++q) {
      const OracleCkParticle& p = ps[q];
      const V3 pos{p.position[0], p.position[1], p.position[2]};
      const V3 vel{p.velocity[0], p.velocity[1], p.velocity[2]};
      const M3 B = load(p.affine);
      const int32_t cx = as_i32(std::floor(pos.x / h)), cy = as_i32(std::floor(pos.y / h)),
                    cz = as_i32(std::floor(pos.z / h));
      for (int dk = 0; dk <= 1; ++dk)
        for (int dj = 0; dj <= 1; ++dj)
          for (int di = 0; di <= 1; ++di) {
            const int64_t i = int64_t(cx) + di, j = int64_t(cy) + dj, k = int64_t(cz) + dk;
            if (i < 0 || j < 0 || k < 0 || i >= gn || j >= gn || k >= gn) continue;
            const V3 node{(float(i) + 0.5f) * h, (float(j) + 0.5f) * h, (float(k) + 0.5f) * h};
            const V3 diff = node - pos;
            const float wx = weight(diff.x, h), wy = weight(diff.y, h);
            const float w = wx * wy * weight(diff.z, h);
            const uint64_t id = gidx(i, j, k);
            gmass[id] += w * p.mass;
            const V3 vg = vel + mul(B, diff);
            gvel[id] = gvel[id] + vg * (w * p.mass);
          }
    }
    // 3. momentum -> velocity (:245-251)
    for (uint64_t id = 0; id < gvel.size(); ++id) gvel[id] = gmass[id] > 1e-10f ? gvel[id] / gmass[id] : V3{0, 0, 0};
    // 4. forces (:253-320)
    const float mu = cfg->youngs_modulus / (2.0f * (1.0f + cfg->poissons_ratio));
    const float lambda = cfg->youngs_modulus * cfg->poissons_ratio /
                         ((1.0f + cfg->poissons_ratio) * (1.0f - 2.0f * cfg->poissons_ratio));
    for (uint64_t q = 0; q < n; ++q) {
      const OracleCkParticle& p = ps[q];
      const V3 pos{p.position[0], p.position[1], p.position[2]};
      const int32_t cx = as_i32(std::floor(pos.x / h)), cy = as_i32(std::floor(pos.y / h)),
                    cz = as_i32(std::floor(pos.z / h));
      const M3 F = load(p.deformation);
      const float fdet = std::fmax(det(F), 1e-10f);
      const M3 fit = inverse(transpose(F));
      const float ln_j = correctly_rounded_ln ? float(std::log(double(fdet))) : std::log(fdet);
      const M3 P = add(scale(sub(F, fit), mu), scale(fit, lambda * ln_j));
      const float coeff = -p.rest_volume;
      for (int dk = 0; dk <= 1; ++dk)
        for (int dj = 0; dj <= 1; ++dj)
          for (int di = 0; di <= 1; ++di) {
            const int64_t i = int64_t(cx) + di, j = int64_t(cy) + dj, k = int64_t(cz) + dk;
            if (i < 0 || j < 0 || k < 0 || i >= gn || j >= gn || k >= gn) continue;
            const V3 node{(float(i) + 0.5f) * h, (float(j) + 0.5f) * h, (float(k) + 0.5f) * h};
            const V3 diff = node - pos;
            const V3 grad{weight_grad(diff.x, h) * weight(diff.y, h) * weight(diff.z, h),
                          weight(diff.x, h) * weight_grad(diff.y, h) * weight(diff.z, h),
                          weight(diff.x, h) * weight(diff.y, h) * weight_grad(diff.z, h)};
            const V3 force = mul(P, grad) * coeff;
            const float fl = length(force);
            const V3 fc = fl > 1e4f ? force * (1e4f / fl) : force;
            const uint64_t id = gidx(i, j, k);
            gforce[id] = gforce[id] + fc;
          }
    }
    // 5. grid velocity update (:323-339)
    for (uint64_t id = 0; id < gvel.size(); ++id) {
      if (!(gmass[id] > 1e-10f)) continue;
      const V3 acc = gforce[id] / gmass[id] + g;
      V3 nv = gvel[id] + acc * dt;
      if (!finite(nv)) nv = V3{0, 0, 0};
      const float vl = length(nv);
      if (vl > 50.0f) nv = nv * (50.0f / vl);
      gvel[id] = nv;
    }
    // 6. grid boundaries (:341-363)
    for (int32_t k = 0; k < gn; ++k)
      for (int32_t j = 0; j < gn; ++j)
        for (int32_t i = 0; i < gn; ++i) {
          const uint64_t id = gidx(i, j, k);
          if (gmass[id] < 1e-10f) continue;
          const float node[3] = {(float(i) + 0.5f) * h, (float(j) + 0.5f) * h, (float(k) + 0.5f) * h};
          float* v = &gvel[id].x;
          for (int a = 0; a < 3; ++a) {
            if (node[a] < bmin[a] && v[a] < 0.0f)
              v[a] *= -cfg->restitution;
            else if (node[a] > bmax[a] && v[a] > 0.0f)
              v[a] *= -cfg->restitution;
          }
        }
    // 7-8. G2P, F, position (:365-459)
    const float d_inv = 4.0f / (h * h);
    for (uint64_t q = 0; q < n; ++q) {
      OracleCkParticle& p = ps[q];
      const V3 pos{p.position[0], p.position[1], p.position[2]};
      const int32_t cx = as_i32(std::floor(pos.x / h)), cy = as_i32(std::floor(pos.y / h)),
                    cz = as_i32(std::floor(pos.z / h));
      V3 nv{0, 0, 0};
      M3 nb{{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}};
      for (int dk = 0; dk <= 1; ++dk)
        for (int dj = 0; dj <= 1; ++dj)
          for (int di = 0; di <= 1; ++di) {
            const int64_t i = int64_t(cx) + di, j = int64_t(cy) + dj, k = int64_t(cz) + dk;
            if (i < 0 || j < 0 || k < 0 || i >= gn || j >= gn || k >= gn) continue;
            const V3 node{(float(i) + 0.5f) * h, (float(j) + 0.5f) * h, (float(k) + 0.5f) * h};
            const V3 diff = node - pos;
            const float w = weight(diff.x, h) * weight(diff.y, h) * weight(diff.z, h);
            const V3 vn = gvel[gidx(i, j, k)];
            nv = nv + vn * w;
            const M3 outer{{vn * (diff.x * d_inv), vn * (diff.y * d_inv), vn * (diff.z * d_inv)}};
            nb = add(nb, scale(outer, w));
          }
      if (!finite(nv)) nv = V3{0, 0, 0};
      const float vl = length(nv);
      if (vl > 50.0f) nv = nv * (50.0f / vl);
      p.velocity[0] = nv.x;
      p.velocity[1] = nv.y;
      p.velocity[2] = nv.z;
      store(nb, p.affine);
      const M3 gv = scale(nb, d_inv);
      auto abs_len = [](V3 c) { return length(V3{std::fabs(c.x), std::fabs(c.y), std::fabs(c.z)}); };
      const float gnorm = std::fmax(std::fmax(abs_len(gv.c[0]), abs_len(gv.c[1])), abs_len(gv.c[2]));
      const float gs = gnorm > 100.0f ? 100.0f / gnorm : 1.0f;
      const M3 fnew = mul(add(kIdentity, scale(scale(gv, gs), dt)), load(p.deformation));
      const float fd = det(fnew);
      if (std::isfinite(fd) && std::fabs(fd) > 1e-10f && std::fabs(fd) < 100.0f) store(fnew, p.deformation);
      const V3 np_ = pos + nv * dt;
      if (finite(np_)) {
        p.position[0] = np_.x;
        p.position[1] = np_.y;
        p.position[2] = np_.z;
      }
    }
    // 9. particle bounds (:462-478)
    for (uint64_t q = 0; q < n; ++q) {
      OracleCkParticle& p = ps[q];
      for (int a = 0; a < 3; ++a) {
        if (p.position[a] < bmin[a]) {
          p.position[a] = bmin[a];
          if (p.velocity[a] < 0.0f) p.velocity[a] = -p.velocity[a] * cfg->restitution;
        } else if (p.position[a] > bmax[a]) {
          p.position[a] = bmax[a];
          if (p.velocity[a] > 0.0f) p.velocity[a] = -p.velocity[a] * cfg->restitution;
        }
      }
    }
  }
}

void oracle_ck_step(OracleCkParticle* ps, uint64_t n, const OracleCkConfig* cfg, uint32_t steps) {
  oracle_ck_step_ln(ps, n, cfg, steps, 0);
}

// CkMpmSolver::weight / weight_grad (:163-185), for known-answer tests
float oracle_ck_weight(float x, float h) { return weight(x, h); }
float oracle_ck_weight_grad(float x, float h) { return weight_grad(x, h); }

}  // extern "C"
