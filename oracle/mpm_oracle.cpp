// mpm_oracle.cpp -- CPU oracle for the MPM substep.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, in C++17, the CPU algorithms of AE-ENGINE's MPM path so that the CUDA
// library can be checked against them.  It is linked only by tests/, by __graft_entry__.smoke()
// and by bench.py's CPU-baseline leg; the product library (libae_mpm.so) never calls it.
//
// What it restates (file:line in the reference project):
//   * ae_particle/src/mpm_solver.rs:442-464     b_spline / b_spline_deriv
//   * ae_particle/src/mpm_solver.rs:812-1054    mpm_substep_serial_active (reference mode)
//   * ae_particle/src/mpm_solver.rs:1088-1326   mpm_substep_parallel_with_indices (threads with
//                                               thread-local grids merged in order, as rayon
//                                               fold/reduce does at :1108-1193)
//   * ae_particle/src/mpm_solver.rs:112-139     Grid::update_parallel
//   * ae_particle/src/mpm_solver.rs:1063-1084   mpm_step_parallel_with_grid (50 000 switch)
//   * ae_particle/src/mpm_solver.rs:1337-1572   velocity-only substep
//   * ae_particle/src/constitutive.rs:55-82, 234-617   MaterialParams and the 7 stress models
//   * ae_compute/src/mpm_compute.rs:137-164, 244-459   MLS stencil (nodes at i*dx,
//                                               base = floor(x/dx - 0.5)), fluid J update
//   * ae_physics/src/mpm.rs:429-454, 565-639    neo-Hookean P and the snow singular-value clamp
// Physics mode fixes the reference inconsistencies that the tests document (force sign,
// partition of unity, C scale) and adds Stomakhin hardening; the deviations are listed beside
// each function.
//
// Parity of this restatement with the Rust reference is unpinned by execution (cargo is not
// available to run the reference); it is pinned against the reference's own known-answer and
// property tests, which tests/test_oracle.py re-runs against this file.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../include/ae_mpm.h"

namespace {

// ------------------------------------------------------------------------------------------
// Kernels: quadratic B-spline (ae_particle/src/mpm_solver.rs:442-464,
// ae_compute/src/mpm_compute.rs:137-164).  The two files agree on value and derivative.
// ------------------------------------------------------------------------------------------
template <class T>
T b_spline(T x) {
  T ax = std::fabs(x);
  if (ax < T(0.5)) return T(0.75) - ax * ax;
  if (ax < T(1.5)) {
    T t = T(1.5) - ax;
    return T(0.5) * t * t;
  }
  return T(0);
}

template <class T>
T b_spline_deriv(T x) {
  T ax = std::fabs(x);
  if (ax < T(0.5)) return T(-2) * x;
  if (ax < T(1.5)) return -(T(1.5) - ax) * (std::signbit(x) ? T(-1) : T(1));
  return T(0);
}

// ------------------------------------------------------------------------------------------
// Material constants, MaterialParams::{mu, lambda, bulk_modulus} (constitutive.rs:55-82),
// evaluated in f32 like the reference.
// ------------------------------------------------------------------------------------------
struct Lame {
  float mu, lambda, bulk;
};

Lame lame_of(const ae_mpm_material& m) {
  float nu = std::min(std::max(m.poisson_ratio, -0.999f), 0.4999f);
  Lame l;
  l.lambda = m.young_modulus * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
  l.mu = m.young_modulus / (2.0f * (1.0f + nu));
  l.bulk = m.young_modulus / (3.0f * (1.0f - 2.0f * nu));
  return l;
}

// ------------------------------------------------------------------------------------------
// 3x3 helpers (row-major, as constitutive.rs:254-282)
// ------------------------------------------------------------------------------------------
template <class T>
void mat_mul(const T* a, const T* b, T* o) {
  T r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] + a[i * 3 + 2] * b[2 * 3 + j];
  std::memcpy(o, r, sizeof(r));
}
template <class T>
void transpose(const T* m, T* o) {
  T r[9] = {m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]};
  std::memcpy(o, r, sizeof(r));
}
template <class T>
T det3(const T* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
template <class T>
void identity3(T* m) {
  for (int i = 0; i < 9; ++i) m[i] = (i % 4 == 0) ? T(1) : T(0);
}

// inv_transpose (constitutive.rs:306-324)
template <class T>
void inv_transpose(const T* m, T* o) {
  T det = det3(m);
  if (std::fabs(det) < T(1e-15)) {
    identity3(o);
    return;
  }
  T inv_det = T(1) / det;
  T r[9] = {(m[4] * m[8] - m[5] * m[7]) * inv_det,  -(m[1] * m[8] - m[2] * m[7]) * inv_det,
            (m[1] * m[5] - m[2] * m[4]) * inv_det,  -(m[3] * m[8] - m[5] * m[6]) * inv_det,
            (m[0] * m[8] - m[2] * m[6]) * inv_det,  -(m[0] * m[5] - m[2] * m[3]) * inv_det,
            (m[3] * m[7] - m[4] * m[6]) * inv_det,  -(m[0] * m[7] - m[1] * m[6]) * inv_det,
            (m[0] * m[4] - m[1] * m[3]) * inv_det};
  std::memcpy(o, r, sizeof(r));
}

// polar_decomp by Newton iteration R <- (R + R^-T)/2, 8 iterations (constitutive.rs:284-304)
template <class T>
void polar_decomp(const T* F, T* R, T* S) {
  T r[9];
  std::memcpy(r, F, sizeof(r));
  for (int it = 0; it < 8; ++it) {
    T rit[9], nr[9];
    inv_transpose(r, rit);
    T diff = 0;
    for (int i = 0; i < 9; ++i) {
      nr[i] = T(0.5) * (r[i] + rit[i]);
      diff += std::fabs(nr[i] - r[i]);
    }
    std::memcpy(r, nr, sizeof(r));
    if (diff < T(1e-10)) break;
  }
  T rt[9];
  transpose(r, rt);
  std::memcpy(R, r, sizeof(r));
  mat_mul(rt, F, S);
}

// ------------------------------------------------------------------------------------------
// Reference Cauchy stress (constitutive.rs:234-617).  The plastic return (new F) is computed
// for completeness but the reference substep discards it (mpm_solver.rs:843-844).
// ------------------------------------------------------------------------------------------
template <class T>
bool compute_stress(int model, const ae_mpm_material& p, const T* F, T J, T* stress, T* newF) {
  const Lame l = lame_of(p);
  const T mu = l.mu, lambda = l.lambda;
  std::memcpy(newF, F, 9 * sizeof(T));
  switch (model) {
    case AE_MPM_RIGID:  // rigid_stress returns the identity as stress (constitutive.rs:370-373)
      identity3(stress);
      return false;
    case AE_MPM_COROTATED: {  // constitutive.rs:395-415
      T R[9], S[9];
      polar_decomp(F, R, S);
      for (int i = 0; i < 9; ++i) stress[i] = T(2) * mu * (F[i] - R[i]);
      for (int i : {0, 4, 8}) stress[i] += lambda * (J - T(1));
      return false;
    }
    case AE_MPM_FIXED_COROTATED: {  // constitutive.rs:417-441
      T R[9], S[9], Rt[9], d[9], dRt[9];
      polar_decomp(F, R, S);
      transpose(R, Rt);
      for (int i = 0; i < 9; ++i) d[i] = F[i] - R[i];
      mat_mul(d, Rt, dRt);
      for (int i = 0; i < 9; ++i) stress[i] = T(2) * mu * dRt[i];
      for (int i : {0, 4, 8}) stress[i] += lambda * (J - T(1)) * J;
      return false;
    }
    case AE_MPM_DRUCKER_PRAGER:
    case AE_MPM_VON_MISES: {  // constitutive.rs:443-530 and 532-601
      T R[9], S[9];
      polar_decomp(F, R, S);
      T eps[9] = {S[0] - T(1), S[1], S[2], S[3], S[4] - T(1), S[5], S[6], S[7], S[8] - T(1)};
      T tr = eps[0] + eps[4] + eps[8];
      T tr3 = tr / T(3);
      T dev[9];
      std::memcpy(dev, eps, sizeof(dev));
      dev[0] -= tr3;
      dev[4] -= tr3;
      dev[8] -= tr3;
      T sdev[9];
      for (int i = 0; i < 9; ++i) sdev[i] = T(2) * mu * dev[i];
      T s_norm = std::sqrt(T(0.5) * (sdev[0] * sdev[0] + sdev[4] * sdev[4] + sdev[8] * sdev[8] +
                                     T(2) * (sdev[1] * sdev[1] + sdev[2] * sdev[2] + sdev[3] * sdev[3] +
                                             sdev[5] * sdev[5] + sdev[6] * sdev[6] + sdev[7] * sdev[7])));
      T pressure = -lambda * tr;
      bool plastic = false;
      T scale = T(1);
      if (model == AE_MPM_DRUCKER_PRAGER) {
        // friction_angle.to_radians(): times the degree-to-radian constant pi / 180 rounded to T
        T phi = T(p.friction_angle) * (T(3.14159265358979323846) / T(180));
        T sphi = std::sin(phi), cphi = std::cos(phi), s3 = std::sqrt(T(3));
        T alpha = (T(2) * sphi) / (s3 * (T(3) - sphi));
        T k = (T(6) * T(p.cohesion) * cphi) / (s3 * (T(3) - sphi));
        T yield = s_norm + alpha * pressure - k;
        if (yield > T(0)) {
          scale = std::max(k - alpha * pressure, T(0)) / std::max(s_norm, T(1e-10));
          plastic = true;
        }
      } else {
        T thr = T(p.yield_stress) / std::sqrt(T(3));
        if (s_norm > thr) {
          scale = thr / s_norm;
          plastic = true;
        }
      }
      if (plastic) {
        T ns[9];
        for (int i = 0; i < 9; ++i) {
          T id = (i % 4 == 0) ? T(1) : T(0);
          ns[i] = id + scale * (S[i] - id);
        }
        for (int i : {0, 4, 8}) ns[i] += (T(1) - scale) * tr3;
        mat_mul(R, ns, newF);
        for (int i = 0; i < 9; ++i) sdev[i] *= scale;
      }
      std::memcpy(stress, sdev, sizeof(sdev));
      for (int i : {0, 4, 8}) stress[i] -= pressure;
      return plastic;
    }
    case AE_MPM_NEWTONIAN_FLUID: {  // constitutive.rs:603-617
      T k = T(l.bulk);
      T sd = k * (J - T(1));
      for (int i = 0; i < 9; ++i) stress[i] = T(0);
      stress[0] = stress[4] = stress[8] = sd;
      return false;
    }
    case AE_MPM_NEO_HOOKEAN:
    default: {  // constitutive.rs:375-393
      T Ft[9], b[9];
      transpose(F, Ft);
      mat_mul(F, Ft, b);
      T p_term = (J > T(0)) ? lambda * std::log(J) / J : T(0);
      T scale = mu / std::max(J, T(1e-10));
      for (int i = 0; i < 9; ++i) {
        T dev = (i % 4 == 0) ? b[i] - T(1) + p_term / scale : b[i];
        stress[i] = scale * dev;
      }
      return false;
    }
  }
}

// ------------------------------------------------------------------------------------------
// 3x3 SVD used by the snow clamp.  The reference (ae_physics/src/mpm.rs:824-951) diagonalises
// F^T F by cyclic Jacobi rotations in Q32.32 and forms U = F V / sigma with a determinant fix.
// The same construction in floating point: cyclic Jacobi on A = F^T F with the stable rotation
// of Golub & Van Loan (Matrix Computations, sec. 8.5), eigenpairs sorted descending, U by
// Gram-Schmidt on F V and u2 = u0 x u1 so U and V are rotations; the last singular value
// carries the sign of det F.  The CUDA kernel implements the identical steps.
// ------------------------------------------------------------------------------------------
template <class T>
struct SvdEps;
template <>
struct SvdEps<float> {
  static constexpr float off_tol = 2.3e-13f;  // (4 eps_f32)^2, relative to the squared diagonal
};
template <>
struct SvdEps<double> {
  static constexpr double off_tol = 7.9e-31;  // (4 eps_f64)^2
};

template <class T>
void svd3(const T* F, T* U, T* s, T* V) {
  T a[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i * 3 + j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] + F[2 * 3 + i] * F[2 * 3 + j];
  T v[9];
  identity3(v);
  for (int sweep = 0; sweep < 8; ++sweep) {
    T off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
    T dia = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
    if (off <= SvdEps<T>::off_tol * dia) break;
    const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
    for (int r = 0; r < 3; ++r) {
      int p = P[r], q = Q[r];
      T apq = a[p * 3 + q];
      if (apq == T(0)) continue;
      T app = a[p * 3 + p], aqq = a[q * 3 + q];
      T tau = (aqq - app) / (T(2) * apq);
      T t = (tau >= T(0) ? T(1) : T(-1)) / (std::fabs(tau) + std::sqrt(T(1) + tau * tau));
      T c = T(1) / std::sqrt(T(1) + t * t);
      T sn = t * c;
      int o = 3 - p - q;  // the remaining index
      T aop = a[o * 3 + p], aoq = a[o * 3 + q];
      T nop = c * aop - sn * aoq, noq = sn * aop + c * aoq;
      a[p * 3 + p] = app - t * apq;
      a[q * 3 + q] = aqq + t * apq;
      a[p * 3 + q] = a[q * 3 + p] = T(0);
      a[o * 3 + p] = a[p * 3 + o] = nop;
      a[o * 3 + q] = a[q * 3 + o] = noq;
      for (int k = 0; k < 3; ++k) {
        T vp = v[k * 3 + p], vq = v[k * 3 + q];
        v[k * 3 + p] = c * vp - sn * vq;
        v[k * 3 + q] = sn * vp + c * vq;
      }
    }
  }
  // sort eigenpairs descending; every swap negates one column to keep det V = +1
  T lam[3] = {a[0], a[4], a[8]};
  auto swapcol = [&](int i, int j) {
    std::swap(lam[i], lam[j]);
    for (int k = 0; k < 3; ++k) {
      T t = v[k * 3 + i];
      v[k * 3 + i] = v[k * 3 + j];
      v[k * 3 + j] = -t;
    }
  };
  if (lam[0] < lam[1]) swapcol(0, 1);
  if (lam[0] < lam[2]) swapcol(0, 2);
  if (lam[1] < lam[2]) swapcol(1, 2);
  // columns of F V
  T fv[9];
  mat_mul(F, v, fv);
  T u0[3] = {fv[0], fv[3], fv[6]}, u1[3] = {fv[1], fv[4], fv[7]}, f2[3] = {fv[2], fv[5], fv[8]};
  T n0 = std::sqrt(u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]);
  if (n0 > T(0)) {
    for (T& x : u0) x /= n0;
  } else {
    u0[0] = T(1);
    u0[1] = u0[2] = T(0);
  }
  T d01 = u0[0] * u1[0] + u0[1] * u1[1] + u0[2] * u1[2];
  for (int k = 0; k < 3; ++k) u1[k] -= d01 * u0[k];
  T n1 = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  if (n1 > T(0)) {
    for (T& x : u1) x /= n1;
  } else {  // any unit vector orthogonal to u0
    T e[3] = {T(0), T(0), T(0)};
    int m = (std::fabs(u0[0]) < std::fabs(u0[1])) ? 0 : 1;
    if (std::fabs(u0[2]) < std::fabs(u0[m])) m = 2;
    e[m] = T(1);
    T d = u0[m];
    for (int k = 0; k < 3; ++k) u1[k] = e[k] - d * u0[k];
    T nn = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    for (T& x : u1) x /= nn;
  }
  T u2[3] = {u0[1] * u1[2] - u0[2] * u1[1], u0[2] * u1[0] - u0[0] * u1[2], u0[0] * u1[1] - u0[1] * u1[0]};
  s[0] = n0;
  s[1] = u1[0] * fv[1] + u1[1] * fv[4] + u1[2] * fv[7];
  s[2] = u2[0] * f2[0] + u2[1] * f2[1] + u2[2] * f2[2];
  for (int k = 0; k < 3; ++k) {
    U[k * 3 + 0] = u0[k];
    U[k * 3 + 1] = u1[k];
    U[k * 3 + 2] = u2[k];
  }
  std::memcpy(V, v, sizeof(v));
}

// Relative gap below which two FP32 singular values count as near-degenerate: sqrt(eps_f32),
// the gap at which FP32 singular vectors keep only half their digits.
constexpr double kSvdGapTol = 3.5e-4;

// Whether the symmetric matrix [[a d e] [d b f] [e f c]] is positive definite (Sylvester's
// criterion: every leading principal minor is positive).
template <class T>
bool sym3_positive_definite(T a, T b, T c, T d, T e, T f) {
  T m2 = a * b - d * d;
  T m3 = a * (b * c - f * f) - d * (d * c - f * e) + e * (d * f - b * e);
  return a > T(0) && m2 > T(0) && m3 > T(0);
}

// True when every singular value of F lies strictly inside (lo, hi) and det F > 0, so the snow
// clamp of ae_physics/src/mpm.rs:565-606 is the identity map and its SVD can be skipped: the
// eigenvalues of F^T F (the squared singular values) lie in (lo^2, hi^2) exactly when
// F^T F - lo^2 I and hi^2 I - F^T F are positive definite.  Exact up to rounding in the minors.
template <class T>
bool clamp_is_identity(const T* F, T lo, T hi) {
  T m[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = i; j < 3; ++j) m[i][j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] + F[2 * 3 + i] * F[2 * 3 + j];
  T lo2 = lo * lo, hi2 = hi * hi;
  return sym3_positive_definite(m[0][0] - lo2, m[1][1] - lo2, m[2][2] - lo2, m[0][1], m[0][2], m[1][2]) &&
         sym3_positive_definite(hi2 - m[0][0], hi2 - m[1][1], hi2 - m[2][2], -m[0][1], -m[0][2], -m[1][2]) &&
         det3(F) > T(0);
}

// FP32 SVD, redone in FP64 when a near-degenerate pair of singular values straddles a clamp
// threshold (the one case where the clamped result depends on the individual singular vectors).
template <class T>
bool svd3_with_fallback(const T* F, T* U, T* s, T* V, bool allow_fallback, T lo, T hi) {
  svd3(F, U, s, V);
  if (!allow_fallback || sizeof(T) == sizeof(double)) return false;
  T smax = std::max(std::fabs(s[0]), T(1e-30));
  bool need = false;
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (std::fabs(s[i] - s[j]) < T(kSvdGapTol) * smax && ((s[i] < lo) != (s[j] < lo) || (s[i] > hi) != (s[j] > hi)))
        need = true;
  if (!need) return false;
  double Fd[9], Ud[9], sd[3], Vd[9];
  for (int i = 0; i < 9; ++i) Fd[i] = double(F[i]);
  svd3(Fd, Ud, sd, Vd);
  for (int i = 0; i < 9; ++i) {
    U[i] = T(Ud[i]);
    V[i] = T(Vd[i]);
  }
  for (int i = 0; i < 3; ++i) s[i] = T(sd[i]);
  return true;
}

// ------------------------------------------------------------------------------------------
// Reference-mode grid (ae_particle/src/mpm_solver.rs:73-176): dense mass, momentum, force.
// ------------------------------------------------------------------------------------------
template <class T>
struct RefGrid {
  size_t nx, ny, nz;
  T dx, inv_dx;
  T origin[3];
  std::vector<T> mass, vel, force;  // vel/force: 3 per node
  RefGrid(size_t x, size_t y, size_t z, T d, const float* o)
      : nx(x), ny(y), nz(z), dx(d), inv_dx(T(1) / d), mass(x * y * z, T(0)), vel(3 * x * y * z, T(0)), force(3 * x * y * z, T(0)) {
    for (int k = 0; k < 3; ++k) origin[k] = o ? T(o[k]) : T(0);
  }
  void reset() {
    std::fill(mass.begin(), mass.end(), T(0));
    std::fill(vel.begin(), vel.end(), T(0));
    std::fill(force.begin(), force.end(), T(0));
  }
  void merge(const RefGrid& o) {  // Grid::merge (mpm_solver.rs:142-155)
    for (size_t i = 0; i < mass.size(); ++i) mass[i] += o.mass[i];
    for (size_t i = 0; i < vel.size(); ++i) vel[i] += o.vel[i];
    for (size_t i = 0; i < force.size(); ++i) force[i] += o.force[i];
  }
  // Grid::update_parallel (mpm_solver.rs:112-139)
  void update(const T* grav, T dt) {
    size_t n = nx * ny * nz;
    for (size_t gid = 0; gid < n; ++gid) {
      T m = mass[gid];
      if (m > T(1e-12)) {
        T* v = &vel[3 * gid];
        const T* f = &force[3 * gid];
        v[0] /= m;
        v[1] /= m;
        v[2] /= m;
        v[0] += (grav[0] + f[0] / m) * dt;
        v[1] += (grav[1] + f[1] / m) * dt;
        v[2] += (grav[2] + f[2] / m) * dt;
        size_t j = (gid % (nx * ny)) / nx;
        if (j == 0) {
          v[1] = std::max(v[1], T(0));
          v[0] *= T(0.9);
          v[2] *= T(0.9);
        }
      }
    }
  }
};

template <class T>
struct Buf {  // the MpssBuffer fields one substep touches
  T *pos, *vel, *F, *J, *C;
  const T* mass;
  const uint16_t* mat;
};

struct MatTable {  // material_table / model_table lookups with the reference's fallbacks
  std::vector<ae_mpm_material> params;
  std::vector<int32_t> models;
  const ae_mpm_material& param(size_t i) const { return i < params.size() ? params[i] : params[0]; }
  int32_t model(size_t i) const { return i < models.size() ? models[i] : AE_MPM_NEO_HOOKEAN; }
};

template <class T>
void cell_of(const RefGrid<T>& g, const T* pos, long* gi, T* fx) {
  for (int a = 0; a < 3; ++a) {
    T q = (pos[a] - g.origin[a]) * g.inv_dx - T(0.5);
    long b = long(std::floor(q));
    fx[a] = q - T(b);
    gi[a] = std::max(b, 0L);
  }
}

// P2G of one particle into grid g (mpm_solver.rs:831-903; parallel copy :1108-1193)
template <class T>
void ref_p2g_particle(RefGrid<T>& g, const Buf<T>& b, const MatTable& mt, size_t i) {
  const T* pos = &b.pos[3 * i];
  const T* vel = &b.vel[3 * i];
  const T* c = &b.C[9 * i];
  T mass = b.mass[i];
  size_t mi = b.mat[i];
  const ae_mpm_material& params = mt.param(mi);
  T stress[9], nf[9];
  compute_stress<T>(mt.model(mi), params, &b.F[9 * i], b.J[i], stress, nf);
  T vol = mass / T(params.density);
  T sv[9];
  for (int k = 0; k < 9; ++k) sv[k] = vol * stress[k];
  long gi[3];
  T fx[3];
  cell_of(g, pos, gi, fx);
  for (int dk = 0; dk < 3; ++dk)
    for (int dj = 0; dj < 3; ++dj)
      for (int di = 0; di < 3; ++di) {
        T wx = b_spline(T(di) - fx[0]), wy = b_spline(T(dj) - fx[1]), wz = b_spline(T(dk) - fx[2]);
        T w = wx * wy * wz;
        if (w < T(1e-10)) continue;
        size_t x = gi[0] + di, y = gi[1] + dj, z = gi[2] + dk;
        if (x >= g.nx || y >= g.ny || z >= g.nz) continue;
        size_t gid = x + y * g.nx + z * g.nx * g.ny;
        T dxg = (T(x) + T(0.5)) * g.dx + g.origin[0] - pos[0];
        T dyg = (T(y) + T(0.5)) * g.dx + g.origin[1] - pos[1];
        T dzg = (T(z) + T(0.5)) * g.dx + g.origin[2] - pos[2];
        T vx = vel[0] + c[0] * dxg + c[1] * dyg + c[2] * dzg;
        T vy = vel[1] + c[3] * dxg + c[4] * dyg + c[5] * dzg;
        T vz = vel[2] + c[6] * dxg + c[7] * dyg + c[8] * dzg;
        g.mass[gid] += w * mass;
        g.vel[3 * gid + 0] += w * mass * vx;
        g.vel[3 * gid + 1] += w * mass * vy;
        g.vel[3 * gid + 2] += w * mass * vz;
        T dwx = b_spline_deriv(T(di) - fx[0]) * g.inv_dx;
        T dwy = b_spline_deriv(T(dj) - fx[1]) * g.inv_dx;
        T dwz = b_spline_deriv(T(dk) - fx[2]) * g.inv_dx;
        g.force[3 * gid + 0] += sv[0] * dwx + sv[1] * dwy + sv[2] * dwz;
        g.force[3 * gid + 1] += sv[3] * dwx + sv[4] * dwy + sv[5] * dwz;
        g.force[3 * gid + 2] += sv[6] * dwx + sv[7] * dwy + sv[8] * dwz;
      }
}

// G2P of one particle (mpm_solver.rs:914-1053; parallel copy :1206-1325).  wall_origin selects
// the parallel path's origin-relative x/z walls (:1290-1297) over the serial path's (:998-1015).
template <class T>
void ref_g2p_particle(const RefGrid<T>& g, const Buf<T>& b, size_t i, T dt, T damping, bool wall_origin) {
  T pos[3] = {b.pos[3 * i], b.pos[3 * i + 1], b.pos[3 * i + 2]};
  long gi[3];
  T fx[3];
  cell_of(g, pos, gi, fx);
  T nv[3] = {0, 0, 0}, nc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, gv_[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int dk = 0; dk < 3; ++dk)
    for (int dj = 0; dj < 3; ++dj)
      for (int di = 0; di < 3; ++di) {
        T wx = b_spline(T(di) - fx[0]), wy = b_spline(T(dj) - fx[1]), wz = b_spline(T(dk) - fx[2]);
        T w = wx * wy * wz;
        if (w < T(1e-10)) continue;
        size_t x = gi[0] + di, y = gi[1] + dj, z = gi[2] + dk;
        if (x >= g.nx || y >= g.ny || z >= g.nz) continue;
        size_t gid = x + y * g.nx + z * g.nx * g.ny;
        if (g.mass[gid] < T(1e-12)) continue;
        const T* gv = &g.vel[3 * gid];
        nv[0] += w * gv[0];
        nv[1] += w * gv[1];
        nv[2] += w * gv[2];
        T dxg = (T(x) + T(0.5)) * g.dx + g.origin[0] - pos[0];
        T dyg = (T(y) + T(0.5)) * g.dx + g.origin[1] - pos[1];
        T dzg = (T(z) + T(0.5)) * g.dx + g.origin[2] - pos[2];
        T scale = T(4) * g.inv_dx * g.inv_dx * w;
        T d3[3] = {dxg, dyg, dzg};
        for (int r = 0; r < 3; ++r)
          for (int cc = 0; cc < 3; ++cc) nc[r * 3 + cc] += scale * gv[r] * d3[cc];
        T dw[3] = {b_spline_deriv(T(di) - fx[0]) * g.inv_dx, b_spline_deriv(T(dj) - fx[1]) * g.inv_dx,
                   b_spline_deriv(T(dk) - fx[2]) * g.inv_dx};
        for (int r = 0; r < 3; ++r)
          for (int cc = 0; cc < 3; ++cc) gv_[r * 3 + cc] -= w * gv[r] * dw[cc];
      }
  for (T v : nv)
    if (!std::isfinite(v)) {
      nv[0] = nv[1] = nv[2] = T(0);
      for (T& x : nc) x = T(0);
      break;
    }
  for (T& v : nv) v = std::min(std::max(v, T(-50)), T(50));
  T np[3] = {pos[0] + nv[0] * dt, pos[1] + nv[1] * dt, pos[2] + nv[2] * dt};
  for (T v : np)
    if (!std::isfinite(v)) {
      np[0] = T(6);
      np[1] = T(5);
      np[2] = T(6);
      nv[0] = nv[1] = nv[2] = T(0);
      break;
    }
  if (np[1] < T(0)) {
    np[1] = T(0);
    nv[1] = std::max(nv[1], T(0)) * T(0.5);
  }
  T gmx = T(g.nx - 1) * g.dx, gmz = T(g.nz - 1) * g.dx;
  T lox = wall_origin ? g.origin[0] : T(0), loz = wall_origin ? g.origin[2] : T(0);
  if (np[0] < lox) {
    np[0] = lox;
    nv[0] = std::max(nv[0], T(0)) * T(0.5);
  } else if (np[0] > gmx + lox) {
    np[0] = gmx + lox;
    nv[0] = std::min(nv[0], T(0)) * T(0.5);
  }
  if (np[2] < loz) {
    np[2] = loz;
    nv[2] = std::max(nv[2], T(0)) * T(0.5);
  } else if (np[2] > gmz + loz) {
    np[2] = gmz + loz;
    nv[2] = std::min(nv[2], T(0)) * T(0.5);
  }
  const T* f = &b.F[9 * i];
  T nf[9];
  for (int r = 0; r < 3; ++r)
    for (int cc = 0; cc < 3; ++cc) {
      T sum = 0;
      for (int k = 0; k < 3; ++k) {
        T kr = (r == k) ? T(1) : T(0);
        sum += (kr + gv_[r * 3 + k] * dt) * f[k * 3 + cc];
      }
      nf[r * 3 + cc] = sum;
    }
  bool valid = true;
  for (T v : nf)
    if (!std::isfinite(v) || std::fabs(v) > T(1e3)) {
      valid = false;
      break;
    }
  T fj;
  if (valid) {
    T j = det3(nf);
    fj = std::min(std::max(j, T(0.1)), T(10));
  } else {
    identity3(nf);
    fj = T(1);
  }
  for (int k = 0; k < 3; ++k) b.vel[3 * i + k] = nv[k] * damping;
  std::memcpy(&b.C[9 * i], nc, sizeof(nc));
  for (int k = 0; k < 3; ++k) b.pos[3 * i + k] = np[k];
  std::memcpy(&b.F[9 * i], nf, sizeof(nf));
  b.J[i] = fj;
}

template <class F>
void parallel_for(size_t n, int threads, F&& f) {
  if (threads <= 1 || n < 2) {
    for (size_t i = 0; i < n; ++i) f(i, 0);
    return;
  }
  std::vector<std::thread> th;
  size_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    size_t lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([=, &f] {
      for (size_t i = lo; i < hi; ++i) f(i, t);
    });
  }
  for (auto& x : th) x.join();
}

// One reference substep over `idx` (serial: mpm_substep_serial_active; threads > 1: the
// fold/reduce parallel path with one thread-local grid per thread merged in thread order).
template <class T>
void ref_substep(RefGrid<T>& g, const Buf<T>& b, const MatTable& mt, const uint64_t* idx, size_t n, T dt,
                 const T* grav, T damping, bool wall_origin, int threads) {
  g.reset();
  if (threads <= 1) {
    for (size_t k = 0; k < n; ++k) ref_p2g_particle(g, b, mt, idx[k]);
  } else {
    std::vector<RefGrid<T>> locals;
    float o[3] = {float(g.origin[0]), float(g.origin[1]), float(g.origin[2])};
    int used = int(std::min<size_t>(threads, n));
    for (int t = 0; t < used; ++t) locals.emplace_back(g.nx, g.ny, g.nz, g.dx, o);
    for (auto& l : locals)
      for (int a = 0; a < 3; ++a) l.origin[a] = g.origin[a];
    parallel_for(n, used, [&](size_t k, int t) { ref_p2g_particle(locals[t], b, mt, idx[k]); });
    for (auto& l : locals) g.merge(l);
  }
  g.update(grav, dt);
  parallel_for(n, threads, [&](size_t k, int) { ref_g2p_particle(g, b, idx[k], dt, damping, wall_origin); });
}

// mpm_substep_velocity_only (mpm_solver.rs:1353-1572)
template <class T>
void velonly_substep(RefGrid<T>& g, const Buf<T>& b, const uint64_t* idx, size_t n, T dt, const T* grav, T damping,
                     int threads) {
  g.reset();
  for (size_t k = 0; k < n; ++k) {  // serial P2G (:1377-1449)
    size_t i = idx[k];
    const T* pos = &b.pos[3 * i];
    const T* vel = &b.vel[3 * i];
    T m = b.mass[i];
    long gi[3];
    T fx[3];
    cell_of(g, pos, gi, fx);
    T wx[3], wy[3], wz[3];
    for (int a = 0; a < 3; ++a) {
      wx[a] = b_spline(T(a) - fx[0]);
      wy[a] = b_spline(T(a) - fx[1]);
      wz[a] = b_spline(T(a) - fx[2]);
    }
    for (int dk = 0; dk < 3; ++dk) {
      if (wz[dk] < T(1e-10)) continue;
      size_t z = gi[2] + dk;
      if (z >= g.nz) continue;
      for (int dj = 0; dj < 3; ++dj) {
        if (wy[dj] < T(1e-10)) continue;
        size_t y = gi[1] + dj;
        if (y >= g.ny) continue;
        T wyz = wy[dj] * wz[dk];
        for (int di = 0; di < 3; ++di) {
          T w = wx[di] * wyz;
          if (w < T(1e-10)) continue;
          size_t x = gi[0] + di;
          if (x >= g.nx) continue;
          size_t gid = x + y * g.nx + z * g.nx * g.ny;
          g.mass[gid] += w * m;
          g.vel[3 * gid + 0] += w * m * vel[0];
          g.vel[3 * gid + 1] += w * m * vel[1];
          g.vel[3 * gid + 2] += w * m * vel[2];
        }
      }
    }
  }
  g.update(grav, dt);
  T gmx = T(g.nx - 1) * g.dx, gmz = T(g.nz - 1) * g.dx;
  parallel_for(n, threads, [&](size_t k, int) {  // parallel G2P (:1465-1571)
    size_t i = idx[k];
    T pos[3] = {b.pos[3 * i], b.pos[3 * i + 1], b.pos[3 * i + 2]};
    long gi[3];
    T fx[3];
    cell_of(g, pos, gi, fx);
    T wx[3], wy[3], wz[3];
    for (int a = 0; a < 3; ++a) {
      wx[a] = b_spline(T(a) - fx[0]);
      wy[a] = b_spline(T(a) - fx[1]);
      wz[a] = b_spline(T(a) - fx[2]);
    }
    T nv[3] = {0, 0, 0};
    for (int dk = 0; dk < 3; ++dk) {
      if (wz[dk] < T(1e-10)) continue;
      size_t z = gi[2] + dk;
      if (z >= g.nz) continue;
      for (int dj = 0; dj < 3; ++dj) {
        if (wy[dj] < T(1e-10)) continue;
        size_t y = gi[1] + dj;
        if (y >= g.ny) continue;
        T wyz = wy[dj] * wz[dk];
        for (int di = 0; di < 3; ++di) {
          T w = wx[di] * wyz;
          if (w < T(1e-10)) continue;
          size_t x = gi[0] + di;
          if (x >= g.nx) continue;
          size_t gid = x + y * g.nx + z * g.nx * g.ny;
          if (g.mass[gid] < T(1e-12)) continue;
          nv[0] += w * g.vel[3 * gid + 0];
          nv[1] += w * g.vel[3 * gid + 1];
          nv[2] += w * g.vel[3 * gid + 2];
        }
      }
    }
    for (T v : nv)
      if (!std::isfinite(v)) {
        nv[0] = nv[1] = nv[2] = T(0);
        break;
      }
    for (T& v : nv) v = std::min(std::max(v, T(-50)), T(50));
    T np[3] = {pos[0] + nv[0] * dt, pos[1] + nv[1] * dt, pos[2] + nv[2] * dt};
    for (T v : np)
      if (!std::isfinite(v)) {
        np[0] = pos[0];
        np[1] = pos[1];
        np[2] = pos[2];
        nv[0] = nv[1] = nv[2] = T(0);
        break;
      }
    if (np[1] < T(0)) {
      np[1] = T(0);
      nv[1] = std::max(nv[1], T(0)) * T(0.5);
    }
    // lower walls at 0, upper walls offset by origin, exactly as :1543-1556
    if (np[0] < T(0)) {
      np[0] = T(0);
      nv[0] = std::max(nv[0], T(0)) * T(0.5);
    } else if (np[0] > gmx + g.origin[0]) {
      np[0] = gmx + g.origin[0];
      nv[0] = std::min(nv[0], T(0)) * T(0.5);
    }
    if (np[2] < T(0)) {
      np[2] = T(0);
      nv[2] = std::max(nv[2], T(0)) * T(0.5);
    } else if (np[2] > gmz + g.origin[2]) {
      np[2] = gmz + g.origin[2];
      nv[2] = std::min(nv[2], T(0)) * T(0.5);
    }
    for (int a = 0; a < 3; ++a) {
      b.vel[3 * i + a] = nv[a] * damping;
      b.pos[3 * i + a] = np[a];
    }
  });
}

// ------------------------------------------------------------------------------------------
// Physics mode (MLS-MPM).  Stencil and fluid J update of ae_compute/src/mpm_compute.rs:244-459
// (nodes at origin + i*dx, base = floor(x/dx - 0.5), fx in [0.5, 1.5)); the affine form of
// Hu et al. 2018 with the physically correct stress sign (the ae_compute force is sign-flipped,
// mpm_compute.rs:328-335) and C scaled by 4/dx^2 (mpm_compute.rs:418 divides by 4 dx^2 instead).
// ------------------------------------------------------------------------------------------
struct PhysMat {
  int model;
  float mu, lambda, bulk, rho, theta_c, theta_s, xi;
};

PhysMat phys_of(const ae_mpm_material& m) {
  Lame l = lame_of(m);
  PhysMat p;
  p.model = m.model;
  p.mu = l.mu;
  p.lambda = l.lambda;
  p.bulk = m.bulk_modulus > 0.0f ? m.bulk_modulus : l.bulk;
  p.rho = m.density;
  p.theta_c = m.theta_c;
  p.theta_s = m.theta_s;
  p.xi = m.hardening_xi;
  return p;
}

template <class T>
struct PhysGrid {
  size_t n[3];
  std::vector<T> m, p;  // mass and momentum (3 per node)
  PhysGrid(const uint32_t* nn) : m(size_t(nn[0]) * nn[1] * nn[2], T(0)), p(3 * size_t(nn[0]) * nn[1] * nn[2], T(0)) {
    for (int a = 0; a < 3; ++a) n[a] = nn[a];
  }
  void reset() {
    std::fill(m.begin(), m.end(), T(0));
    std::fill(p.begin(), p.end(), T(0));
  }
};

template <class T>
struct Stencil {
  long base[3];
  T w[3][3];   // w[axis][a]
  T dp[3][3];  // dpos[axis][a] = (a - fx) * dx
};

template <class T>
Stencil<T> phys_stencil(const T* x, const T* origin, T dx, T inv_dx) {
  Stencil<T> s;
  for (int a = 0; a < 3; ++a) {
    T X = (x[a] - origin[a]) * inv_dx;
    long b = long(std::floor(X - T(0.5)));
    T fx = X - T(b);
    s.base[a] = b;
    T t0 = T(1.5) - fx, t1 = fx - T(1), t2 = fx - T(0.5);
    s.w[a][0] = T(0.5) * t0 * t0;
    s.w[a][1] = T(0.75) - t1 * t1;
    s.w[a][2] = T(0.5) * t2 * t2;
    for (int k = 0; k < 3; ++k) s.dp[a][k] = (T(k) - fx) * dx;
  }
  return s;
}

// Kirchhoff stress of a physics-mode material at state (F, Jslot)
template <class T>
void phys_tau(const PhysMat& pm, const T* F, T jslot, T* tau) {
  for (int i = 0; i < 9; ++i) tau[i] = T(0);
  if (pm.model == AE_MPM_PHYS_FLUID) {  // tau = K (J - 1) I (mpm_compute.rs:287-291 times J)
    T s = T(pm.bulk) * (jslot - T(1));
    tau[0] = tau[4] = tau[8] = s;
    return;
  }
  T mu = T(pm.mu), la = T(pm.lambda);
  if (pm.model == AE_MPM_PHYS_SNOW) {  // Stomakhin et al. 2013 hardening, capped to [0.1, 5]
    T h = std::exp(T(pm.xi) * (T(1) - jslot));
    h = std::min(std::max(h, T(0.1)), T(5));
    mu *= h;
    la *= h;
  }
  // neo-Hookean Kirchhoff stress P F^T = mu (F F^T - I) + lambda ln(Jc) I, with
  // Jc = clamp(det F, 0.01, 100) (ae_physics/src/mpm.rs:443-452)
  T J = det3(F);
  T Jc = std::min(std::max(J, T(0.01)), T(100));
  T lnJ = std::log(Jc);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      T bb = F[r * 3 + 0] * F[c * 3 + 0] + F[r * 3 + 1] * F[c * 3 + 1] + F[r * 3 + 2] * F[c * 3 + 2];
      tau[r * 3 + c] = mu * (bb - (r == c ? T(1) : T(0))) + (r == c ? la * lnJ : T(0));
    }
}

template <class T>
struct PhysStats {
  uint64_t fallbacks = 0, clamps = 0, nans = 0;
};

template <class T>
void phys_p2g_particle(PhysGrid<T>& g, const Buf<T>& b, const std::vector<PhysMat>& mats, size_t i, T dt, T dx,
                       T inv_dx, const T* origin) {
  const T* x = &b.pos[3 * i];
  const T* v = &b.vel[3 * i];
  const T* C = &b.C[9 * i];
  T m = b.mass[i];
  size_t mi = b.mat[i];
  const PhysMat& pm = mats[mi < mats.size() ? mi : 0];
  T tau[9];
  phys_tau(pm, &b.F[9 * i], b.J[i], tau);
  T vol0 = m / T(pm.rho);
  T kst = T(4) * dt * vol0 * inv_dx * inv_dx;
  T A[9];
  for (int k = 0; k < 9; ++k) A[k] = m * C[k] - kst * tau[k];
  Stencil<T> s = phys_stencil(x, origin, dx, inv_dx);
  for (int c = 0; c < 3; ++c)
    for (int bb = 0; bb < 3; ++bb)
      for (int a = 0; a < 3; ++a) {
        long X = s.base[0] + a, Y = s.base[1] + bb, Z = s.base[2] + c;
        if (X < 0 || Y < 0 || Z < 0 || size_t(X) >= g.n[0] || size_t(Y) >= g.n[1] || size_t(Z) >= g.n[2]) continue;
        T w = s.w[0][a] * s.w[1][bb] * s.w[2][c];
        T d0 = s.dp[0][a], d1 = s.dp[1][bb], d2 = s.dp[2][c];
        size_t gid = size_t(X) + g.n[0] * (size_t(Y) + g.n[1] * size_t(Z));
        g.m[gid] += w * m;
        for (int r = 0; r < 3; ++r) g.p[3 * gid + r] += w * (m * v[r] + A[r * 3 + 0] * d0 + A[r * 3 + 1] * d1 + A[r * 3 + 2] * d2);
      }
}

template <class T>
void phys_grid_update(PhysGrid<T>& g, const ae_mpm_scene_desc& sc, T dt, int threads) {
  size_t N = g.n[0] * g.n[1] * g.n[2];
  long mg = sc.wall_margin;
  parallel_for(N, threads, [&](size_t gid, int) {
    T m = g.m[gid];
    T* p = &g.p[3 * gid];
    if (!(m > T(0))) {
      p[0] = p[1] = p[2] = T(0);
      return;
    }
    T v[3] = {p[0] / m, p[1] / m, p[2] / m};
    for (int a = 0; a < 3; ++a) v[a] += dt * T(sc.gravity[a]);
    long idx[3] = {long(gid % g.n[0]), long((gid / g.n[0]) % g.n[1]), long(gid / (g.n[0] * g.n[1]))};
    if (sc.wall_mode == AE_MPM_WALL_STICKY) {
      bool wall = false;
      for (int a = 0; a < 3; ++a) wall = wall || idx[a] < mg || idx[a] >= long(g.n[a]) - mg;
      if (wall) v[0] = v[1] = v[2] = T(0);
    } else {
      for (int a = 0; a < 3; ++a) {
        if (idx[a] < mg && v[a] < T(0)) v[a] = -v[a] * T(sc.restitution);
        if (idx[a] >= long(g.n[a]) - mg && v[a] > T(0)) v[a] = -v[a] * T(sc.restitution);
      }
    }
    p[0] = v[0];
    p[1] = v[1];
    p[2] = v[2];
  });
}

template <class T>
void phys_g2p_particle(const PhysGrid<T>& g, const Buf<T>& b, const std::vector<PhysMat>& mats, size_t i, T dt, T dx,
                       T inv_dx, const T* origin, bool fallback, PhysStats<T>& st) {
  T* x = &b.pos[3 * i];
  Stencil<T> s = phys_stencil(x, origin, dx, inv_dx);
  T v[3] = {0, 0, 0}, B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int c = 0; c < 3; ++c)
    for (int bb = 0; bb < 3; ++bb)
      for (int a = 0; a < 3; ++a) {
        long X = s.base[0] + a, Y = s.base[1] + bb, Z = s.base[2] + c;
        if (X < 0 || Y < 0 || Z < 0 || size_t(X) >= g.n[0] || size_t(Y) >= g.n[1] || size_t(Z) >= g.n[2]) continue;
        T w = s.w[0][a] * s.w[1][bb] * s.w[2][c];
        size_t gid = size_t(X) + g.n[0] * (size_t(Y) + g.n[1] * size_t(Z));
        const T* gv = &g.p[3 * gid];
        T d[3] = {s.dp[0][a], s.dp[1][bb], s.dp[2][c]};
        for (int r = 0; r < 3; ++r) {
          v[r] += w * gv[r];
          for (int k = 0; k < 3; ++k) B[r * 3 + k] += w * gv[r] * d[k];
        }
      }
  T C[9];
  T cs = T(4) * inv_dx * inv_dx;
  for (int k = 0; k < 9; ++k) C[k] = cs * B[k];
  // advect, then keep the particle where its whole stencil is inside the grid
  bool clamped = false, nan = false;
  for (int a = 0; a < 3; ++a) {
    T nx = x[a] + dt * v[a];
    if (!std::isfinite(nx)) nan = true;
    T lo = origin[a] + dx, hi = origin[a] + T(g.n[a] - 2) * dx;
    T cx = std::fmin(std::fmax(nx, lo), hi);
    if (cx != nx) clamped = true;
    x[a] = cx;
  }
  if (nan) st.nans++;
  if (clamped) st.clamps++;
  for (int a = 0; a < 3; ++a) b.vel[3 * i + a] = v[a];
  std::memcpy(&b.C[9 * i], C, sizeof(C));
  size_t mi = b.mat[i];
  const PhysMat& pm = mats[mi < mats.size() ? mi : 0];
  T* F = &b.F[9 * i];
  if (pm.model == AE_MPM_PHYS_FLUID) {  // J-only (mpm_compute.rs:453-457)
    T J = b.J[i] * (T(1) + dt * (C[0] + C[4] + C[8]));
    b.J[i] = std::max(J, T(0.01));
    return;
  }
  T G[9];
  for (int k = 0; k < 9; ++k) G[k] = ((k % 4 == 0) ? T(1) : T(0)) + dt * C[k];
  T nF[9];
  mat_mul(G, F, nF);
  if (pm.model == AE_MPM_PHYS_SNOW) {  // ae_physics/src/mpm.rs:565-606 with J_p bookkeeping
    T lo = T(1) - T(pm.theta_c), hi = T(1) + T(pm.theta_s);
    if (clamp_is_identity(nF, lo, hi)) {  // elastic: F_E and J_p unchanged
      std::memcpy(F, nF, sizeof(nF));
      return;
    }
    T U[9], sg[3], V[9];
    if (svd3_with_fallback(nF, U, sg, V, fallback, lo, hi)) st.fallbacks++;
    T sc[3];
    for (int k = 0; k < 3; ++k) sc[k] = std::min(std::max(sg[k], lo), hi);
    b.J[i] = b.J[i] * ((sg[0] * sg[1] * sg[2]) / (sc[0] * sc[1] * sc[2]));
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) nF[r * 3 + c] = U[r * 3 + 0] * sc[0] * V[c * 3 + 0] + U[r * 3 + 1] * sc[1] * V[c * 3 + 1] + U[r * 3 + 2] * sc[2] * V[c * 3 + 2];
  } else {
    b.J[i] = det3(nF);
  }
  std::memcpy(F, nF, sizeof(nF));
}

template <class T>
PhysStats<T> phys_substep(PhysGrid<T>& g, const Buf<T>& b, const std::vector<PhysMat>& mats, size_t n,
                          const ae_mpm_scene_desc& sc, bool fallback, int threads) {
  T dt = T(sc.dt), dx = T(sc.dx), inv_dx = T(1) / dx;
  T origin[3] = {T(sc.origin[0]), T(sc.origin[1]), T(sc.origin[2])};
  g.reset();
  if (threads <= 1) {
    for (size_t i = 0; i < n; ++i) phys_p2g_particle(g, b, mats, i, dt, dx, inv_dx, origin);
  } else {
    int used = int(std::min<size_t>(threads, std::max<size_t>(n, 1)));
    std::vector<PhysGrid<T>> locals;
    for (int t = 0; t < used; ++t) {
      uint32_t nn[3] = {uint32_t(g.n[0]), uint32_t(g.n[1]), uint32_t(g.n[2])};
      locals.emplace_back(nn);
    }
    parallel_for(n, used, [&](size_t i, int t) { phys_p2g_particle(locals[t], b, mats, i, dt, dx, inv_dx, origin); });
    for (auto& l : locals) {
      for (size_t k = 0; k < g.m.size(); ++k) g.m[k] += l.m[k];
      for (size_t k = 0; k < g.p.size(); ++k) g.p[k] += l.p[k];
    }
  }
  phys_grid_update(g, sc, dt, threads);
  std::vector<PhysStats<T>> per(std::max(threads, 1));
  parallel_for(n, threads, [&](size_t i, int t) { phys_g2p_particle(g, b, mats, i, dt, dx, inv_dx, origin, fallback, per[t]); });
  PhysStats<T> tot;
  for (auto& p : per) {
    tot.fallbacks += p.fallbacks;
    tot.clamps += p.clamps;
    tot.nans += p.nans;
  }
  return tot;
}

template <class T, class P>
Buf<T> buf_of(P* p) {
  Buf<T> b;
  b.pos = p->pos;
  b.vel = p->vel;
  b.F = p->strain;
  b.J = p->jacobian;
  b.C = p->c;
  b.mass = p->mass;
  b.mat = p->material_idx;
  return b;
}

template <class T, class P>
int run_scene(const ae_mpm_scene_desc* sc, P* p, uint64_t n, uint32_t substeps, int threads, int svd_fallback,
              uint64_t* counters) {
  if (!sc || !p || sc->n_materials == 0 || !sc->materials) return AE_MPM_EINVAL;
  Buf<T> b = buf_of<T>(p);
  uint64_t cnt[3] = {0, 0, 0};
  if (sc->mode == AE_MPM_MODE_PHYSICS) {
    std::vector<PhysMat> mats;
    for (uint32_t k = 0; k < sc->n_materials; ++k) mats.push_back(phys_of(sc->materials[k]));
    PhysGrid<T> g(sc->n);
    for (uint32_t s = 0; s < substeps; ++s) {
      PhysStats<T> st = phys_substep(g, b, mats, n, *sc, svd_fallback != 0, threads);
      cnt[0] += st.fallbacks;
      cnt[1] += st.clamps;
      cnt[2] += st.nans;
    }
  } else {
    RefGrid<T> g(sc->n[0], sc->n[1], sc->n[2], T(sc->dx), sc->origin);
    MatTable mt;
    for (uint32_t k = 0; k < sc->n_materials; ++k) {
      mt.params.push_back(sc->materials[k]);
      mt.models.push_back(sc->materials[k].model);
    }
    std::vector<uint64_t> idx(n);
    for (uint64_t i = 0; i < n; ++i) idx[i] = i;
    T grav[3] = {T(sc->gravity[0]), T(sc->gravity[1]), T(sc->gravity[2])};
    for (uint32_t s = 0; s < substeps; ++s) {
      if (sc->mode == AE_MPM_MODE_VELOCITY_ONLY)
        velonly_substep(g, b, idx.data(), n, T(sc->dt), grav, T(sc->damping), threads);
      else
        ref_substep(g, b, mt, idx.data(), n, T(sc->dt), grav, T(sc->damping), sc->wall_origin != 0, threads);
    }
  }
  if (counters)
    for (int k = 0; k < 3; ++k) counters[k] = cnt[k];
  return AE_MPM_OK;
}

template <class T, class P>
void totals_of(const P* p, uint64_t n, double* out) {
  double m = 0, px = 0, py = 0, pz = 0, ke = 0;
  for (uint64_t i = 0; i < n; ++i) {
    double mi = double(p->mass[i]);
    double vx = double(p->vel[3 * i]), vy = double(p->vel[3 * i + 1]), vz = double(p->vel[3 * i + 2]);
    m += mi;
    px += mi * vx;
    py += mi * vy;
    pz += mi * vz;
    ke += 0.5 * mi * (vx * vx + vy * vy + vz * vz);
  }
  out[0] = m;
  out[1] = px;
  out[2] = py;
  out[3] = pz;
  out[4] = ke;
}

MatTable table_of(const ae_mpm_material* mats, uint32_t nm, const int32_t* models, uint32_t nmod) {
  MatTable mt;
  for (uint32_t k = 0; k < nm; ++k) mt.params.push_back(mats[k]);
  for (uint32_t k = 0; k < nmod; ++k) mt.models.push_back(models[k]);
  return mt;
}

}  // namespace

// ==========================================================================================
// C entry points (ctypes)
// ==========================================================================================
extern "C" {

float oracle_b_spline(float x) { return b_spline(x); }
float oracle_b_spline_deriv(float x) { return b_spline_deriv(x); }
// quadratic_weight / quadratic_weight_grad (ae_compute/src/mpm_compute.rs:137-164)
float oracle_quadratic_weight(float d) { return b_spline(d); }
float oracle_quadratic_weight_grad(float d) { return b_spline_deriv(d); }

void oracle_material_lame(const ae_mpm_material* m, float out[3]) {
  Lame l = lame_of(*m);
  out[0] = l.mu;
  out[1] = l.lambda;
  out[2] = l.bulk;
}

int oracle_compute_stress(int32_t model, const ae_mpm_material* params, const float F[9], float J, float stress[9],
                          float new_F[9]) {
  return compute_stress<float>(model, *params, F, J, stress, new_F) ? 1 : 0;
}

void oracle_polar_decomp(const float F[9], float R[9], float S[9]) { polar_decomp<float>(F, R, S); }

// lo/hi: the clamp interval deciding whether a near-degenerate pair needs the FP64 redo
int oracle_svd3_f32(const float F[9], float U[9], float s[3], float V[9], int32_t allow_fallback, float lo, float hi) {
  return svd3_with_fallback<float>(F, U, s, V, allow_fallback != 0, lo, hi) ? 1 : 0;
}
int oracle_clamp_is_identity_f32(const float F[9], float lo, float hi) { return clamp_is_identity<float>(F, lo, hi) ? 1 : 0; }
void oracle_svd3_f64(const double F[9], double U[9], double s[3], double V[9]) { svd3<double>(F, U, s, V); }

void oracle_phys_tau_f64(const ae_mpm_material* m, const double F[9], double jslot, double tau[9]) {
  phys_tau<double>(phys_of(*m), F, jslot, tau);
}

// Run `substeps` substeps of one scene over particles 0..n-1 (all modes).  threads > 1 uses the
// thread-local-grid fold/merge pattern of mpm_substep_parallel_with_indices.
int oracle_run_f32(const ae_mpm_scene_desc* scene, ae_mpm_particles* p, uint64_t n, uint32_t substeps, int32_t threads,
                   int32_t svd_fallback, uint64_t counters[3]) {
  return run_scene<float>(scene, p, n, substeps, threads, svd_fallback, counters);
}
int oracle_run_f64(const ae_mpm_scene_desc* scene, ae_mpm_particles_f64* p, uint64_t n, uint32_t substeps,
                   int32_t threads, int32_t svd_fallback, uint64_t counters[3]) {
  return run_scene<double>(scene, p, n, substeps, threads, svd_fallback, counters);
}

void oracle_totals_f32(const ae_mpm_particles* p, uint64_t n, double out[5]) { totals_of<float>(p, n, out); }
void oracle_totals_f64(const ae_mpm_particles_f64* p, uint64_t n, double out[5]) { totals_of<double>(p, n, out); }

int oracle_mpm_step_parallel_with_grid_export(const ae_mpm_particles* buffer, uint64_t capacity,
                                              const ae_mpm_grid* grid, const ae_mpm_config* config,
                                              const ae_mpm_material* material_table, uint32_t n_materials,
                                              const int32_t* model_table, uint32_t n_models, float total_dt,
                                              const uint64_t* particle_indices, uint64_t n_indices, int32_t threads,
                                              float* grid_mass, float* grid_vel);

// mpm_step_parallel_with_grid (ae_particle/src/mpm_solver.rs:1063-1084) on the caller's buffer,
// minus update_lifetimes.  threads > 1 runs the >= 50 000 branch's fold/reduce with that many
// thread-local grids.
int oracle_mpm_step_parallel_with_grid(const ae_mpm_particles* buffer, uint64_t capacity, const ae_mpm_grid* grid,
                                       const ae_mpm_config* config, const ae_mpm_material* material_table,
                                       uint32_t n_materials, const int32_t* model_table, uint32_t n_models,
                                       float total_dt, const uint64_t* particle_indices, uint64_t n_indices,
                                       int32_t threads) {
  return oracle_mpm_step_parallel_with_grid_export(buffer, capacity, grid, config, material_table, n_materials,
                                                   model_table, n_models, total_dt, particle_indices, n_indices,
                                                   threads, nullptr, nullptr);
}

// The same call, and afterwards the Grid the reference leaves behind (mpm_solver.rs:73-86): the
// node mass and velocity (after Grid::update_parallel of the last substep) in the reference's
// dense index order i + j*nx + k*nx*ny, when grid_mass / grid_vel are given.  Nodes at or below
// the 1e-12 mass threshold keep the momentum the update leaves in `vel` (mpm_solver.rs:116).
int oracle_mpm_step_parallel_with_grid_export(const ae_mpm_particles* buffer, uint64_t capacity,
                                              const ae_mpm_grid* grid, const ae_mpm_config* config,
                                              const ae_mpm_material* material_table, uint32_t n_materials,
                                              const int32_t* model_table, uint32_t n_models, float total_dt,
                                              const uint64_t* particle_indices, uint64_t n_indices, int32_t threads,
                                              float* grid_mass, float* grid_vel) {
  if (n_indices == 0) return AE_MPM_OK;
  if (n_materials == 0 || !config || config->substeps == 0) return AE_MPM_EINVAL;
  for (uint64_t k = 0; k < n_indices; ++k)
    if (particle_indices[k] >= capacity) return AE_MPM_EINVAL;
  Buf<float> b = buf_of<float>(buffer);
  MatTable mt = table_of(material_table, n_materials, model_table, n_models);
  RefGrid<float> g(grid->nx, grid->ny, grid->nz, grid->dx, grid->origin);
  float sub_dt = total_dt / float(config->substeps);
  for (uint64_t s = 0; s < config->substeps; ++s) {
    bool parallel = n_indices >= 50000;
    ref_substep(g, b, mt, particle_indices, n_indices, sub_dt, config->gravity, config->damping, parallel,
                parallel ? std::max(threads, 1) : 1);
  }
  if (grid_mass) std::copy(g.mass.begin(), g.mass.end(), grid_mass);
  if (grid_vel) std::copy(g.vel.begin(), g.vel.end(), grid_vel);
  return AE_MPM_OK;
}

// mpm_step_velocity_only_parallel (ae_particle/src/mpm_solver.rs:1337-1351)
int oracle_mpm_step_velocity_only_parallel(const ae_mpm_particles* buffer, uint64_t capacity, const ae_mpm_grid* grid,
                                           const ae_mpm_config* config, float total_dt,
                                           const uint64_t* particle_indices, uint64_t n_indices, int32_t threads) {
  if (n_indices == 0) return AE_MPM_OK;
  if (!config || config->substeps == 0) return AE_MPM_EINVAL;
  for (uint64_t k = 0; k < n_indices; ++k)
    if (particle_indices[k] >= capacity) return AE_MPM_EINVAL;
  Buf<float> b = buf_of<float>(buffer);
  RefGrid<float> g(grid->nx, grid->ny, grid->nz, grid->dx, grid->origin);
  float sub_dt = total_dt / float(config->substeps);
  for (uint64_t s = 0; s < config->substeps; ++s)
    velonly_substep(g, b, particle_indices, n_indices, sub_dt, config->gravity, config->damping, threads);
  return AE_MPM_OK;
}

}  // extern "C"
