// mpm_math.cuh -- per-particle arithmetic of the MPM substep, templated on the scalar type
// (float for production runs, double for the FP64 error-reference runs of the same kernels).
//
// Formula sources (reference project paths):
//   b_spline / b_spline_deriv          ae_particle/src/mpm_solver.rs:442-464
//   MaterialParams::{mu,lambda,bulk}   ae_particle/src/constitutive.rs:55-82
//   reference Cauchy stress models     ae_particle/src/constitutive.rs:234-617
//   polar decomposition (Newton)       ae_particle/src/constitutive.rs:284-324
//   neo-Hookean Kirchhoff stress       ae_physics/src/mpm.rs:429-454
//   snow singular-value clamp          ae_physics/src/mpm.rs:565-606 (SVD of F^T F by Jacobi, :824-951)
//   J-only fluid                        ae_compute/src/mpm_compute.rs:287-291, 453-457
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define AE_HD __host__ __device__ __forceinline__

namespace aemp {

// ---------------------------------------------------------------- scalar helpers
template <class T>
AE_HD T t_abs(T x) { return x < T(0) ? -x : x; }
AE_HD float t_sqrt(float x) { return sqrtf(x); }
AE_HD double t_sqrt(double x) { return sqrt(x); }
AE_HD float t_log(float x) { return logf(x); }
AE_HD double t_log(double x) { return log(x); }
AE_HD float t_exp(float x) { return expf(x); }
AE_HD double t_exp(double x) { return exp(x); }
AE_HD float t_floor(float x) { return floorf(x); }
AE_HD double t_floor(double x) { return floor(x); }
AE_HD float t_sin(float x) { return sinf(x); }
AE_HD double t_sin(double x) { return sin(x); }
AE_HD float t_cos(float x) { return cosf(x); }
AE_HD double t_cos(double x) { return cos(x); }
template <class T>
AE_HD T t_min(T a, T b) { return a < b ? a : b; }
template <class T>
AE_HD T t_max(T a, T b) { return a > b ? a : b; }
template <class T>
AE_HD T t_clamp(T x, T lo, T hi) { return t_min(t_max(x, lo), hi); }
AE_HD bool t_finite(float x) { return isfinite(x); }
AE_HD bool t_finite(double x) { return isfinite(x); }
// fmin/fmax return the non-NaN operand, so a NaN position is pulled back onto the domain
AE_HD float t_fclamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
AE_HD double t_fclamp(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }
// a + b * c with the product and the sum each rounded, as the reference's Rust computes it (Rust
// never contracts to a fused multiply-add); used where the result feeds a branch that exact ties
// reach, e.g. a wall test on x + v dt after an earlier clamp left x at exactly v dt
__device__ __forceinline__ float t_add_mul_rn(float a, float b, float c) { return __fadd_rn(a, __fmul_rn(b, c)); }
__device__ __forceinline__ double t_add_mul_rn(double a, double b, double c) { return __dadd_rn(a, __dmul_rn(b, c)); }

// ---------------------------------------------------------------- quadratic B-spline
template <class T>
AE_HD T b_spline(T x) {
  T ax = t_abs(x);
  if (ax < T(0.5)) return T(0.75) - ax * ax;
  if (ax < T(1.5)) {
    T t = T(1.5) - ax;
    return T(0.5) * t * t;
  }
  return T(0);
}
template <class T>
AE_HD T b_spline_deriv(T x) {
  T ax = t_abs(x);
  if (ax < T(0.5)) return T(-2) * x;
  if (ax < T(1.5)) return -(T(1.5) - ax) * (signbit(x) ? T(-1) : T(1));
  return T(0);
}

// ---------------------------------------------------------------- 3x3 row-major
template <class T>
struct M3 {
  T m[9];
};
template <class T>
AE_HD void mm3(const T* a, const T* b, T* o) {
  T r[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] + a[i * 3 + 2] * b[2 * 3 + j];
#pragma unroll
  for (int i = 0; i < 9; ++i) o[i] = r[i];
}
template <class T>
AE_HD T det3(const T* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
template <class T>
AE_HD void ident3(T* m) {
#pragma unroll
  for (int i = 0; i < 9; ++i) m[i] = (i % 4 == 0) ? T(1) : T(0);
}
template <class T>
AE_HD void inv_transpose3(const T* m, T* o) {  // constitutive.rs:306-324
  T det = det3(m);
  if (t_abs(det) < T(1e-15)) {
    ident3(o);
    return;
  }
  T id = T(1) / det;
  T r[9] = {(m[4] * m[8] - m[5] * m[7]) * id,  -(m[1] * m[8] - m[2] * m[7]) * id, (m[1] * m[5] - m[2] * m[4]) * id,
            -(m[3] * m[8] - m[5] * m[6]) * id, (m[0] * m[8] - m[2] * m[6]) * id,  -(m[0] * m[5] - m[2] * m[3]) * id,
            (m[3] * m[7] - m[4] * m[6]) * id,  -(m[0] * m[7] - m[1] * m[6]) * id, (m[0] * m[4] - m[1] * m[3]) * id};
#pragma unroll
  for (int i = 0; i < 9; ++i) o[i] = r[i];
}
// R <- (R + R^-T)/2 for 8 iterations, early exit when the l1 change is below 1e-10; S = R^T F
template <class T>
AE_HD void polar_decomp3(const T* F, T* R, T* S) {
  T r[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = F[i];
  for (int it = 0; it < 8; ++it) {
    T rit[9];
    inv_transpose3(r, rit);
    T diff = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      T nr = T(0.5) * (r[i] + rit[i]);
      diff += t_abs(nr - r[i]);
      r[i] = nr;
    }
    if (diff < T(1e-10)) break;
  }
  T rt[9] = {r[0], r[3], r[6], r[1], r[4], r[7], r[2], r[5], r[8]};
#pragma unroll
  for (int i = 0; i < 9; ++i) R[i] = r[i];
  mm3(rt, F, S);
}

// ---------------------------------------------------------------- material constants
// Device copy of one material: the reference's MaterialParams plus f32-evaluated derived
// constants (MaterialParams::{mu,lambda,bulk_modulus} clamp nu to [-0.999, 0.4999]).
struct MatDev {
  int32_t model;
  float mu, lambda, bulk, rho;
  float yield_stress, friction_angle, cohesion;
  float theta_c, theta_s, xi;
  float pad;
};

// ---------------------------------------------------------------- reference Cauchy stress
enum { kNeoHookean = 0, kDruckerPrager = 1, kVonMises = 2, kNewtonianFluid = 3, kCorotated = 4, kFixedCorotated = 5,
       kRigid = 6, kPhysJelly = 16, kPhysSnow = 17, kPhysFluid = 18 };

template <class T>
AE_HD void ref_stress(const MatDev& p, const T* F, T J, T* st) {
  const T mu = T(p.mu), lambda = T(p.lambda);
  switch (p.model) {
    case kRigid:
      ident3(st);
      return;
    case kCorotated: {
      T R[9], S[9];
      polar_decomp3(F, R, S);
#pragma unroll
      for (int i = 0; i < 9; ++i) st[i] = T(2) * mu * (F[i] - R[i]);
      st[0] += lambda * (J - T(1));
      st[4] += lambda * (J - T(1));
      st[8] += lambda * (J - T(1));
      return;
    }
    case kFixedCorotated: {
      T R[9], S[9], d[9];
      polar_decomp3(F, R, S);
      T Rt[9] = {R[0], R[3], R[6], R[1], R[4], R[7], R[2], R[5], R[8]};
#pragma unroll
      for (int i = 0; i < 9; ++i) d[i] = F[i] - R[i];
      T dRt[9];
      mm3(d, Rt, dRt);
#pragma unroll
      for (int i = 0; i < 9; ++i) st[i] = T(2) * mu * dRt[i];
      T add = lambda * (J - T(1)) * J;
      st[0] += add;
      st[4] += add;
      st[8] += add;
      return;
    }
    case kDruckerPrager:
    case kVonMises: {
      T R[9], S[9];
      polar_decomp3(F, R, S);
      T e[9] = {S[0] - T(1), S[1], S[2], S[3], S[4] - T(1), S[5], S[6], S[7], S[8] - T(1)};
      T tr = e[0] + e[4] + e[8];
      T tr3 = tr / T(3);
      e[0] -= tr3;
      e[4] -= tr3;
      e[8] -= tr3;
      T sd[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) sd[i] = T(2) * mu * e[i];
      T sn = t_sqrt(T(0.5) * (sd[0] * sd[0] + sd[4] * sd[4] + sd[8] * sd[8] +
                              T(2) * (sd[1] * sd[1] + sd[2] * sd[2] + sd[3] * sd[3] + sd[5] * sd[5] + sd[6] * sd[6] + sd[7] * sd[7])));
      T pressure = -lambda * tr;
      T scale = T(1);
      bool plastic = false;
      if (p.model == kDruckerPrager) {
        // friction_angle.to_radians(): times the degree-to-radian constant pi / 180 rounded to T
        T phi = T(p.friction_angle) * (T(3.14159265358979323846) / T(180));
        T sphi = t_sin(phi), cphi = t_cos(phi), s3 = t_sqrt(T(3));
        T alpha = (T(2) * sphi) / (s3 * (T(3) - sphi));
        T k = (T(6) * T(p.cohesion) * cphi) / (s3 * (T(3) - sphi));
        if (sn + alpha * pressure - k > T(0)) {
          scale = t_max(k - alpha * pressure, T(0)) / t_max(sn, T(1e-10));
          plastic = true;
        }
      } else {
        T thr = T(p.yield_stress) / t_sqrt(T(3));
        if (sn > thr) {
          scale = thr / sn;
          plastic = true;
        }
      }
      if (plastic) {
#pragma unroll
        for (int i = 0; i < 9; ++i) sd[i] *= scale;
      }
#pragma unroll
      for (int i = 0; i < 9; ++i) st[i] = sd[i];
      st[0] -= pressure;
      st[4] -= pressure;
      st[8] -= pressure;
      return;
    }
    case kNewtonianFluid: {
      T s = T(p.bulk) * (J - T(1));
#pragma unroll
      for (int i = 0; i < 9; ++i) st[i] = T(0);
      st[0] = st[4] = st[8] = s;
      return;
    }
    default: {  // neo-Hookean, constitutive.rs:375-393
      T b[9];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) b[r * 3 + c] = F[r * 3 + 0] * F[c * 3 + 0] + F[r * 3 + 1] * F[c * 3 + 1] + F[r * 3 + 2] * F[c * 3 + 2];
      T p_term = (J > T(0)) ? lambda * t_log(J) / J : T(0);
      T scale = mu / t_max(J, T(1e-10));
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        T dev = (i % 4 == 0) ? b[i] - T(1) + p_term / scale : b[i];
        st[i] = scale * dev;
      }
      return;
    }
  }
}

// ---------------------------------------------------------------- physics-mode Kirchhoff stress
template <class T>
AE_HD void phys_tau(const MatDev& p, const T* F, T jslot, T* tau) {
  if (p.model == kPhysFluid) {
    T s = T(p.bulk) * (jslot - T(1));
#pragma unroll
    for (int i = 0; i < 9; ++i) tau[i] = T(0);
    tau[0] = tau[4] = tau[8] = s;
    return;
  }
  T mu = T(p.mu), la = T(p.lambda);
  if (p.model == kPhysSnow) {
    T h = t_clamp(t_exp(T(p.xi) * (T(1) - jslot)), T(0.1), T(5));
    mu *= h;
    la *= h;
  }
  T J = det3(F);
  T lnJ = t_log(t_clamp(J, T(0.01), T(100)));
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T bb = F[r * 3 + 0] * F[c * 3 + 0] + F[r * 3 + 1] * F[c * 3 + 1] + F[r * 3 + 2] * F[c * 3 + 2];
      tau[r * 3 + c] = mu * (bb - (r == c ? T(1) : T(0))) + (r == c ? la * lnJ : T(0));
    }
}

// ---------------------------------------------------------------- 3x3 SVD
// Cyclic Jacobi on A = F^T F (rotation of Golub & Van Loan, sec. 8.5), eigenpairs sorted
// descending (each swap negates a column so det V stays +1), U by Gram-Schmidt on F V with
// u2 = u0 x u1; the third singular value is signed.  Same steps as the CPU oracle.
template <class T>
struct SvdTol;
template <>
struct SvdTol<float> {
  static constexpr float off = 2.3e-13f;
};
template <>
struct SvdTol<double> {
  static constexpr double off = 7.9e-31;
};

// Quotient and reciprocal square root for the rotation angles.  FP32 on the device uses the
// hardware approximations (MUFU reciprocal, 2 ulp reciprocal square root): a rotation only has to
// shrink the off-diagonal entry, the next sweep removes what it leaves, and c^2 + s^2 = 1 holds to
// a few ulp, so U, V stay orthogonal to FP32 accuracy.  FP64 and the host keep IEEE operations.
AE_HD float rot_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdividef(a, b);
#else
  return a / b;
#endif
}
AE_HD double rot_div(double a, double b) { return a / b; }
AE_HD float rot_rsqrt(float x) {
#ifdef __CUDA_ARCH__
  return rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}
AE_HD double rot_rsqrt(double x) { return 1.0 / sqrt(x); }

template <class T>
AE_HD void jacobi_rot(T* a, T* v, int p, int q) {
  T apq = a[p * 3 + q];
  if (apq == T(0)) return;
  T app = a[p * 3 + p], aqq = a[q * 3 + q];
  const T dq = aqq - app;
  T tau = dq == T(0) ? T(0) : rot_div(dq, T(2) * apq);  // 0 * rcp(tiny) would be NaN
  // |tau| + sqrt(1 + tau^2) overflows to +inf for huge tau: t is then 0 (no rotation needed)
  T t = rot_div(tau >= T(0) ? T(1) : T(-1), t_abs(tau) + t_sqrt(T(1) + tau * tau));
  T c = rot_rsqrt(T(1) + t * t);  // 1 + t^2 in [1, 2]
  T sn = t * c;
  int o = 3 - p - q;
  T aop = a[o * 3 + p], aoq = a[o * 3 + q];
  T nop = c * aop - sn * aoq, noq = sn * aop + c * aoq;
  a[p * 3 + p] = app - t * apq;
  a[q * 3 + q] = aqq + t * apq;
  a[p * 3 + q] = a[q * 3 + p] = T(0);
  a[o * 3 + p] = a[p * 3 + o] = nop;
  a[o * 3 + q] = a[q * 3 + o] = noq;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    T vp = v[k * 3 + p], vq = v[k * 3 + q];
    v[k * 3 + p] = c * vp - sn * vq;
    v[k * 3 + q] = sn * vp + c * vq;
  }
}

template <class T>
AE_HD void svd3(const T* F, T* U, T* s, T* V) {
  T a[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a[i * 3 + j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] + F[2 * 3 + i] * F[2 * 3 + j];
  T v[9];
  ident3(v);
  for (int sweep = 0; sweep < 8; ++sweep) {
    T off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
    T dia = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
    if (off <= SvdTol<T>::off * dia) break;
    jacobi_rot(a, v, 0, 1);
    jacobi_rot(a, v, 0, 2);
    jacobi_rot(a, v, 1, 2);
  }
  T lam[3] = {a[0], a[4], a[8]};
#define AE_SWAPCOL(i, j)                 \
  {                                      \
    T tl = lam[i];                       \
    lam[i] = lam[j];                     \
    lam[j] = tl;                         \
    for (int k = 0; k < 3; ++k) {        \
      T tv = v[k * 3 + i];               \
      v[k * 3 + i] = v[k * 3 + j];       \
      v[k * 3 + j] = -tv;                \
    }                                    \
  }
  if (lam[0] < lam[1]) AE_SWAPCOL(0, 1);
  if (lam[0] < lam[2]) AE_SWAPCOL(0, 2);
  if (lam[1] < lam[2]) AE_SWAPCOL(1, 2);
#undef AE_SWAPCOL
  T fv[9];
  mm3(F, v, fv);
  T u0[3] = {fv[0], fv[3], fv[6]}, u1[3] = {fv[1], fv[4], fv[7]};
  T n0 = t_sqrt(u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]);
  if (n0 > T(0)) {
    u0[0] /= n0;
    u0[1] /= n0;
    u0[2] /= n0;
  } else {
    u0[0] = T(1);
    u0[1] = u0[2] = T(0);
  }
  T d01 = u0[0] * u1[0] + u0[1] * u1[1] + u0[2] * u1[2];
#pragma unroll
  for (int k = 0; k < 3; ++k) u1[k] -= d01 * u0[k];
  T n1 = t_sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  if (n1 > T(0)) {
    u1[0] /= n1;
    u1[1] /= n1;
    u1[2] /= n1;
  } else {
    int m = (t_abs(u0[0]) < t_abs(u0[1])) ? 0 : 1;
    if (t_abs(u0[2]) < t_abs(u0[m])) m = 2;
    T d = u0[m];
#pragma unroll
    for (int k = 0; k < 3; ++k) u1[k] = ((k == m) ? T(1) : T(0)) - d * u0[k];
    T nn = t_sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    u1[0] /= nn;
    u1[1] /= nn;
    u1[2] /= nn;
  }
  T u2[3] = {u0[1] * u1[2] - u0[2] * u1[1], u0[2] * u1[0] - u0[0] * u1[2], u0[0] * u1[1] - u0[1] * u1[0]};
  s[0] = n0;
  s[1] = u1[0] * fv[1] + u1[1] * fv[4] + u1[2] * fv[7];
  s[2] = u2[0] * fv[2] + u2[1] * fv[5] + u2[2] * fv[8];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    U[k * 3 + 0] = u0[k];
    U[k * 3 + 1] = u1[k];
    U[k * 3 + 2] = u2[k];
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) V[i] = v[i];
}

// relative gap below which two FP32 singular values count as near-degenerate (sqrt(eps_f32))
constexpr double kSvdGapTol = 3.5e-4;

// Whether the symmetric matrix [[a d e] [d b f] [e f c]] is positive definite: its leading
// principal minors are all positive (Sylvester's criterion).
template <class T>
AE_HD bool sym3_positive_definite(T a, T b, T c, T d, T e, T f) {
  const T m2 = a * b - d * d;
  const T m3 = a * (b * c - f * f) - d * (d * c - f * e) + e * (d * f - b * e);
  return a > T(0) && m2 > T(0) && m3 > T(0);
}

// Every singular value of F strictly inside (lo, hi) and det F > 0, so the snow clamp is the
// identity map and needs no SVD.  The squared singular values are the eigenvalues of M = F^T F,
// so the test is that M - lo^2 I and hi^2 I - M are both positive definite.  It is exact up to
// rounding in the minors: F whose singular values come within rounding of lo or hi may go either
// way, and those are clamped by at most that rounding.
template <class T>
AE_HD bool clamp_is_identity(const T* F, T lo, T hi) {
  T m[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j) m[i][j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] + F[2 * 3 + i] * F[2 * 3 + j];
  const T lo2 = lo * lo, hi2 = hi * hi;
  return sym3_positive_definite(m[0][0] - lo2, m[1][1] - lo2, m[2][2] - lo2, m[0][1], m[0][2], m[1][2]) &&
         sym3_positive_definite(hi2 - m[0][0], hi2 - m[1][1], hi2 - m[2][2], -m[0][1], -m[0][2], -m[1][2]) &&
         det3(F) > T(0);
}

// FP32 SVD, redone in FP64 when a near-degenerate pair straddles a clamp threshold
template <class T>
AE_HD bool svd3_fallback(const T* F, T* U, T* s, T* V, bool allow, T lo, T hi) {
  svd3(F, U, s, V);
  if (!allow || sizeof(T) == sizeof(double)) return false;
  T smax = t_max(t_abs(s[0]), T(1e-30));
  bool need = false;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i + 1; j < 3; ++j)
      if (t_abs(s[i] - s[j]) < T(kSvdGapTol) * smax && ((s[i] < lo) != (s[j] < lo) || (s[i] > hi) != (s[j] > hi)))
        need = true;
  if (!need) return false;
  double Fd[9], Ud[9], sd[3], Vd[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) Fd[i] = double(F[i]);
  svd3(Fd, Ud, sd, Vd);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    U[i] = T(Ud[i]);
    V[i] = T(Vd[i]);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) s[i] = T(sd[i]);
  return true;
}

}  // namespace aemp
