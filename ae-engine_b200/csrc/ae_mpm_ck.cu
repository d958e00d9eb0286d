// ae_mpm_ck.cu -- CK-MPM (compact-kernel MPM), the reference's CkMpmSolver::step
// (ae_compute/src/ck_mpm.rs:187-480), on B200.
//
// One reference step is four serial passes: P2G (mass and APIC momentum, :200-242), forces
// (neo-Hookean first Piola stress through the kernel gradient, :253-320), the grid update
// (momentum to velocity, gravity and force, NaN guard, speed cap, boundary reflection, :245-363)
// and G2P (velocity, affine matrix, deformation gradient, position, particle bounds, :365-478).
// Here:
//   * the force pass is fused into P2G: both depend on the particle state alone, so one read of a
//     particle scatters mass, momentum and force into two 16-byte accumulators per node;
//   * G2P of step s and P2G of step s+1 are one kernel (ck_particles_kernel<true, true>): each
//     particle record is read and written once per step;
//   * P2G flags the 4x4x4 node blocks it touches with plain stores (nothing waits on them); a
//     sweep compacts the flags into a list, and the grid update visits only the listed blocks,
//     leaving their accumulators zeroed for the next step.
// Particle records (26 floats, ae_mpm_ck_particle) move between HBM and shared memory with
// coalesced 16-byte loads and stores; nodes accumulate through 16-byte vector atomics
// (red.global.add.v4.f32) into a block-major grid that stays resident in L2.
//
// Rounding: this file is compiled with --fmad=false, IEEE division and square root, and every
// expression keeps the operand order of the reference's f32 / glam 0.29 arithmetic (Mat3 x Vec3
// as x_axis*v.x + y_axis*v.y + z_axis*v.z; determinant z . (x cross y); inverse from the three
// cross products times 1/det), so each particle's contribution to a node, and each particle's
// update from given node velocities, equal the reference's bit for bit.  Two things differ: node
// sums accumulate in atomic order rather than particle order, and f32::ln is the double-precision
// logarithm rounded to f32 (the correctly rounded value; the C library's logf returns it for all
// but rare arguments).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ae_mpm_ck.cuh"

namespace aemp {
namespace {

constexpr int kCkThreads = 256;     // particles per CTA
constexpr int kRecFloats = 26;      // ae_mpm_ck_particle
constexpr int kGridThreads = 256;   // 4 node blocks per CTA in the grid update

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(V3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ bool finite3(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

struct M3 {  // three columns, as glam's Mat3
  V3 c0, c1, c2;
};
__device__ __forceinline__ V3 mulv(const M3& m, V3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
__device__ __forceinline__ M3 mulm(const M3& a, const M3& b) { return {mulv(a, b.c0), mulv(a, b.c1), mulv(a, b.c2)}; }
__device__ __forceinline__ M3 addm(const M3& a, const M3& b) { return {a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2}; }
__device__ __forceinline__ M3 subm(const M3& a, const M3& b) { return {a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2}; }
__device__ __forceinline__ M3 scalem(const M3& a, float s) { return {a.c0 * s, a.c1 * s, a.c2 * s}; }
__device__ __forceinline__ M3 transposem(const M3& m) {
  return {{m.c0.x, m.c1.x, m.c2.x}, {m.c0.y, m.c1.y, m.c2.y}, {m.c0.z, m.c1.z, m.c2.z}};
}
__device__ __forceinline__ float detm(const M3& m) { return dot3(m.c2, cross3(m.c0, m.c1)); }
__device__ __forceinline__ M3 inversem(const M3& m) {
  const V3 t0 = cross3(m.c1, m.c2), t1 = cross3(m.c2, m.c0), t2 = cross3(m.c0, m.c1);
  const float inv = 1.0f / dot3(m.c2, t2);
  return transposem(M3{t0 * inv, t1 * inv, t2 * inv});
}
__device__ __forceinline__ float col_abs_len(V3 c) { return len3(V3{fabsf(c.x), fabsf(c.y), fabsf(c.z)}); }

// The grid spacing and, when h = 2^k with |k| <= 40, its exact reciprocals 2^-k and 2^-3k.  Then
// x / h and x / (h h h) equal x * 2^-k and x * 2^-3k bit for bit: both round the same real
// number (subnormal results included), and the products cost one instruction instead of an IEEE
// division sequence.  POW2 selects that form; otherwise the divisions are written as such.
struct Spacing {
  float h, inv_h, inv_h3;
};
template <bool POW2>
__device__ __forceinline__ float div_h(float x, const Spacing& sp) {
  return POW2 ? x * sp.inv_h : x / sp.h;
}
template <bool POW2>
__device__ __forceinline__ float div_h3(float x, const Spacing& sp) {
  return POW2 ? x * sp.inv_h3 : x / (sp.h * sp.h * sp.h);
}

// CkMpmSolver::weight (:163-176): (1 - r^2)^3 / h for r = |x| / h < 1
template <bool POW2 = false>
__device__ __forceinline__ float ck_weight(float x, const Spacing& sp) {
  const float r = div_h<POW2>(fabsf(x), sp);
  if (r >= 1.0f) return 0.0f;
  const float a = 1.0f - r * r;
  return div_h<POW2>(a * a * a, sp);
}
// CkMpmSolver::weight_grad (:178-185): -6 x (1 - r^2)^2 / h^3
template <bool POW2 = false>
__device__ __forceinline__ float ck_weight_grad(float x, const Spacing& sp) {
  const float r = div_h<POW2>(fabsf(x), sp);
  if (r >= 1.0f) return 0.0f;
  const float a = 1.0f - r * r;
  return div_h3<POW2>(-6.0f * x * (a * a), sp);
}

// Rust `f32 as i32`: truncation toward zero, NaN -> 0, saturating at the i32 range
__device__ __forceinline__ int as_i32(float v) {
  if (v != v) return 0;
  if (v >= 2147483648.0f) return 2147483647;
  if (v <= -2147483648.0f) return -2147483647 - 1;
  return static_cast<int>(v);
}

struct CkArgs {
  float* rec;          // n records of 26 floats
  uint64_t n;
  float4* acc;         // [node][2]
  const float4* vel;   // [node]
  uint32_t* flags;     // [block] touched by the last P2G
  uint32_t* list;      // touched blocks, compacted
  uint32_t* count;
  uint32_t* next_count;  // the counter the next step's compaction appends to
  int gn, nb;
  Spacing sp;
  float h, dt, youngs, poisson, restitution;
  float g[3], bmin[3], bmax[3];
  int aligned16;
};

// block-major node index: 4x4x4 node blocks, x fastest inside and across blocks
__device__ __forceinline__ uint32_t node_index(int i, int j, int k, int nb) {
  const uint32_t b = (uint32_t(k >> 2) * uint32_t(nb) + uint32_t(j >> 2)) * uint32_t(nb) + uint32_t(i >> 2);
  return b * 64u + uint32_t((k & 3) * 16 + (j & 3) * 4 + (i & 3));
}

// The 2 nodes per axis around a particle (i = floor(x / h) + {0, 1}, node at (i + 1/2) h):
// whether each exists, its offset from the particle and its kernel weight and gradient.
// `zero`: the node's weight and gradient on this axis are exactly 0 (r >= 1).  For a particle at a
// finite position its contributions through such a node are then +-0, and the reference's sums
// start at +0 and only ever hold +0 or a nonzero value, so skipping them leaves every sum's bits
// unchanged.  (A non-finite position skips nothing: 0 times its NaN weights is NaN.)
struct Stencil {
  int i[3][2];
  bool ok[3][2], zero[3][2];
  float diff[3][2], w[3][2], gw[3][2];
};

template <bool POW2>
__device__ __forceinline__ void make_stencil(Stencil& st, V3 pos, const Spacing& sp, int gn, bool grads) {
  const float p[3] = {pos.x, pos.y, pos.z};
  const float h = sp.h;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int c = as_i32(floorf(div_h<POW2>(p[a], sp)));
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int i = int(uint32_t(c) + uint32_t(d));  // i32 add, wrapping like the reference's release build
      st.i[a][d] = i;
      st.ok[a][d] = i >= 0 && i < gn;
      const float df = (float(i) + 0.5f) * h - p[a];
      st.diff[a][d] = df;
      st.w[a][d] = ck_weight<POW2>(df, sp);
      st.gw[a][d] = grads ? ck_weight_grad<POW2>(df, sp) : 0.0f;
      st.zero[a][d] = st.w[a][d] == 0.0f && st.gw[a][d] == 0.0f;
    }
  }
  const bool fin = isfinite(pos.x) && isfinite(pos.y) && isfinite(pos.z);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int d = 0; d < 2; ++d) st.zero[a][d] = st.zero[a][d] && fin;
}

// whether node (di, dj, dk) of the stencil exists and can contribute
__device__ __forceinline__ bool live(const Stencil& st, int di, int dj, int dk) {
  return st.ok[0][di] && st.ok[1][dj] && st.ok[2][dk] && !(st.zero[0][di] || st.zero[1][dj] || st.zero[2][dk]);
}

// |v| > cap, with the square root taken only when it can decide: below (0.995 cap)^2 the rounded
// root is below the cap too.  Returns the rounded length in *len when computed.
__device__ __forceinline__ bool above(V3 v, float cap2_safe, float cap, float* len) {
  const float d2 = dot3(v, v);
  if (!(d2 > cap2_safe)) return false;  // also false for NaN, where the root is NaN and compares false
  *len = sqrtf(d2);
  return *len > cap;
}

// a plain store: the flag is only ever set here and cleared by the compaction, so no read or
// atomic is needed, and no thread waits for it
__device__ __forceinline__ void mark_block(const CkArgs& a, uint32_t b, uint32_t& last) {
  if (b == last) return;
  last = b;
  a.flags[b] = 1u;
}

// The first Piola stress of the force pass (:262-268): P = mu (F - F^-T) + lambda ln(max(det F, 1e-10)) F^-T
__device__ __forceinline__ M3 piola_stress(const CkArgs& a, const M3& F) {
  const float mu = a.youngs / (2.0f * (1.0f + a.poisson));
  const float lambda = a.youngs * a.poisson / ((1.0f + a.poisson) * (1.0f - 2.0f * a.poisson));
  const float fdet = fmaxf(detm(F), 1e-10f);
  const M3 fit = inversem(transposem(F));
  const float ln_j = float(log(double(fdet)));
  return addm(scalem(subm(F, fit), mu), scalem(fit, lambda * ln_j));
}

// One particle's contribution to one node (:221-240 and :276-318): wm = w m to the mass, (v + B d) wm
// to the momentum, -V0 P grad w (clamped to |f| <= 1e4) to the force.  Both the atomic scatter and
// the deterministic node gather call this, so their contributions are the same bits.
__device__ __forceinline__ void node_contribution(float wx, float wy, float wz, float gx, float gy, float gz, V3 diff,
                                                  V3 vel, const M3& B, const M3& P, float mass, float coeff, float& wm,
                                                  V3& mom, V3& force) {
  wm = wx * wy * wz * mass;
  const V3 vg = vel + mulv(B, diff);
  mom = vg * wm;
  const V3 grad{gx * wy * wz, wx * gy * wz, wx * wy * gz};
  force = mulv(P, grad) * coeff;
  float fl;
  if (above(force, 9.9e7f, 1e4f, &fl)) force = force * (1e4f / fl);
}

// P2G (:200-242) and the force pass (:253-320) of one particle
template <bool POW2>
__device__ __forceinline__ void scatter(const CkArgs& a, V3 pos, V3 vel, const M3& B, const M3& F, float rest_volume,
                                        float mass) {
  Stencil st;
  make_stencil<POW2>(st, pos, a.sp, a.gn, true);
  const M3 P = piola_stress(a, F);
  const float coeff = -rest_volume;
  uint32_t last = 0xffffffffu;
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        if (!live(st, di, dj, dk)) continue;
        const V3 diff{st.diff[0][di], st.diff[1][dj], st.diff[2][dk]};
        float wm;
        V3 mom, force;
        node_contribution(st.w[0][di], st.w[1][dj], st.w[2][dk], st.gw[0][di], st.gw[1][dj], st.gw[2][dk], diff, vel, B,
                          P, mass, coeff, wm, mom, force);
        const uint32_t node = node_index(st.i[0][di], st.i[1][dj], st.i[2][dk], a.nb);
        atomicAdd(a.acc + 2 * node, make_float4(mom.x, mom.y, mom.z, wm));
        atomicAdd(a.acc + 2 * node + 1, make_float4(force.x, force.y, force.z, 0.0f));
        mark_block(a, node >> 6, last);
      }
}

// particle bounds, one axis (:462-478)
__device__ __forceinline__ void clamp_axis(float& p, float& v, float lo, float hi, float restitution) {
  if (p < lo) {
    p = lo;
    if (v < 0.0f) v = -v * restitution;
  } else if (p > hi) {
    p = hi;
    if (v > 0.0f) v = -v * restitution;
  }
}

// grid boundary, one axis (:341-363)
__device__ __forceinline__ void reflect_axis(float& v, float node_pos, float lo, float hi, float restitution) {
  if (node_pos < lo && v < 0.0f)
    v *= -restitution;
  else if (node_pos > hi && v > 0.0f)
    v *= -restitution;
}

// G2P (:365-459) and the particle bounds (:462-478) of one particle
template <bool POW2>
__device__ __forceinline__ void gather_update(const CkArgs& a, V3& pos, V3& vel, M3& B, M3& F) {
  const float h = a.h, dt = a.dt;
  Stencil st;
  make_stencil<POW2>(st, pos, a.sp, a.gn, false);
  const float d_inv = 4.0f / (h * h);
  // all eight node loads first, so their latencies overlap
  float4 vnode[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int di = q & 1, dj = (q >> 1) & 1, dk = q >> 2;
    vnode[q] = live(st, di, dj, dk) ? __ldg(a.vel + node_index(st.i[0][di], st.i[1][dj], st.i[2][dk], a.nb))
                                    : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  V3 nv{0.0f, 0.0f, 0.0f};
  M3 nb{{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        if (!live(st, di, dj, dk)) continue;
        const float w = st.w[0][di] * st.w[1][dj] * st.w[2][dk];
        const float4 v4 = vnode[(dk << 2) | (dj << 1) | di];
        const V3 vn{v4.x, v4.y, v4.z};
        nv = nv + vn * w;
        const M3 outer{vn * (st.diff[0][di] * d_inv), vn * (st.diff[1][dj] * d_inv), vn * (st.diff[2][dk] * d_inv)};
        nb = addm(nb, scalem(outer, w));
      }
  if (!finite3(nv)) nv = V3{0.0f, 0.0f, 0.0f};
  float vl;
  if (above(nv, 2475.0f, 50.0f, &vl)) nv = nv * (50.0f / vl);
  vel = nv;
  B = nb;
  const M3 gv = scalem(nb, d_inv);
  // column norms of |grad v|: the roots only when one of them can exceed 100
  float gs = 1.0f;
  const float c0 = dot3(gv.c0, gv.c0), c1 = dot3(gv.c1, gv.c1), c2 = dot3(gv.c2, gv.c2);
  if (!(c0 <= 9900.0f && c1 <= 9900.0f && c2 <= 9900.0f)) {
    const float gnorm = fmaxf(fmaxf(col_abs_len(gv.c0), col_abs_len(gv.c1)), col_abs_len(gv.c2));
    gs = gnorm > 100.0f ? 100.0f / gnorm : 1.0f;
  }
  const M3 ident{{1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}};
  const M3 fnew = mulm(addm(ident, scalem(scalem(gv, gs), dt)), F);
  const float fd = detm(fnew);
  if (isfinite(fd) && fabsf(fd) > 1e-10f && fabsf(fd) < 100.0f) F = fnew;
  const V3 np = pos + nv * dt;
  if (finite3(np)) pos = np;
  clamp_axis(pos.x, vel.x, a.bmin[0], a.bmax[0], a.restitution);
  clamp_axis(pos.y, vel.y, a.bmin[1], a.bmax[1], a.restitution);
  clamp_axis(pos.z, vel.z, a.bmin[2], a.bmax[2], a.restitution);
}

// One CTA = 256 consecutive particles.  G2P: gather from a.vel and update the record in place.
// P2G: scatter the (updated) particle into a.acc for the next grid update.
template <bool G2P, bool P2G, bool POW2>
__global__ void __launch_bounds__(kCkThreads, 3) ck_particles_kernel(CkArgs a) {
  __shared__ __align__(16) float srec[kCkThreads * kRecFloats];
  const uint64_t base = uint64_t(blockIdx.x) * kCkThreads;
  const uint64_t rem = a.n - base;
  const int cnt = rem < uint64_t(kCkThreads) ? int(rem) : kCkThreads;
  const int nf = cnt * kRecFloats;
  float* g = a.rec + base * kRecFloats;
  const int t = threadIdx.x;
  if (a.aligned16) {
    const float4* g4 = reinterpret_cast<const float4*>(g);
    float4* s4 = reinterpret_cast<float4*>(srec);
    for (int q = t; q < nf / 4; q += kCkThreads) s4[q] = __ldcs(g4 + q);
    for (int q = (nf / 4) * 4 + t; q < nf; q += kCkThreads) srec[q] = g[q];
  } else {
    for (int q = t; q < nf; q += kCkThreads) srec[q] = g[q];
  }
  __syncthreads();
  if (t < cnt) {
    float* r = srec + t * kRecFloats;
    V3 pos{r[0], r[1], r[2]}, vel{r[3], r[4], r[5]};
    M3 B{{r[6], r[7], r[8]}, {r[9], r[10], r[11]}, {r[12], r[13], r[14]}};
    M3 F{{r[15], r[16], r[17]}, {r[18], r[19], r[20]}, {r[21], r[22], r[23]}};
    const float rest_volume = r[24], mass = r[25];
    if (G2P) {
      gather_update<POW2>(a, pos, vel, B, F);
      r[0] = pos.x, r[1] = pos.y, r[2] = pos.z;
      r[3] = vel.x, r[4] = vel.y, r[5] = vel.z;
      r[6] = B.c0.x, r[7] = B.c0.y, r[8] = B.c0.z, r[9] = B.c1.x, r[10] = B.c1.y, r[11] = B.c1.z;
      r[12] = B.c2.x, r[13] = B.c2.y, r[14] = B.c2.z;
      r[15] = F.c0.x, r[16] = F.c0.y, r[17] = F.c0.z, r[18] = F.c1.x, r[19] = F.c1.y, r[20] = F.c1.z;
      r[21] = F.c2.x, r[22] = F.c2.y, r[23] = F.c2.z;
    }
    if (P2G) scatter<POW2>(a, pos, vel, B, F, rest_volume, mass);
  }
  if (G2P) {
    __syncthreads();
    if (a.aligned16) {
      float4* g4 = reinterpret_cast<float4*>(g);
      const float4* s4 = reinterpret_cast<const float4*>(srec);
      for (int q = t; q < nf / 4; q += kCkThreads) __stcs(g4 + q, s4[q]);
      for (int q = (nf / 4) * 4 + t; q < nf; q += kCkThreads) g[q] = srec[q];
    } else {
      for (int q = t; q < nf; q += kCkThreads) g[q] = srec[q];
    }
  }
}

// Compaction of the block flags P2G set: one warp ballot per 32 flags, one atomic per warp to
// reserve list space.  Clears the flags it reads, and zeroes the counter the next step uses.
__global__ void __launch_bounds__(256) ck_compact_kernel(uint32_t* flags, uint64_t blocks, uint32_t* list,
                                                         uint32_t* count, uint32_t* next_count) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *next_count = 0u;
  const int lane = threadIdx.x & 31;
  for (uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; b - lane < blocks;
       b += uint64_t(gridDim.x) * blockDim.x) {
    const bool touched = b < blocks && flags[b] != 0u;
    const unsigned m = __ballot_sync(0xffffffffu, touched);
    if (!m) continue;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(count, uint32_t(__popc(m)));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (touched) {
      list[base + __popc(m & ((1u << lane) - 1u))] = uint32_t(b);
      flags[b] = 0u;
    }
  }
}

// Grid update (:245-251, :323-363) over the touched node blocks a.list[0..*a.count): velocity
// from momentum, gravity and force, NaN guard, speed cap 50, reflection at the bounds.  Leaves
// the accumulators zeroed.  Each 64-thread group takes kGridU listed blocks per iteration and
// issues all their accumulator loads before using any, so the list is not walked one
// latency-bound load after another.
constexpr int kGridU = 4;

__device__ __forceinline__ void grid_node(const CkArgs& a, uint32_t b, int local, float4 a0, float4 a1, float4* vel) {
  const uint32_t node = b * 64u + uint32_t(local);
  const float m = a0.w;
  V3 nv{0.0f, 0.0f, 0.0f};
  if (m > 1e-10f) {
    const V3 v{a0.x / m, a0.y / m, a0.z / m};
    const V3 acc{a1.x / m + a.g[0], a1.y / m + a.g[1], a1.z / m + a.g[2]};
    nv = v + acc * a.dt;
    if (!finite3(nv)) nv = V3{0.0f, 0.0f, 0.0f};
    float vl;
    if (above(nv, 2475.0f, 50.0f, &vl)) nv = nv * (50.0f / vl);
    const uint32_t nb = uint32_t(a.nb);
    const int i = int((b % nb) * 4u + uint32_t(local & 3)), j = int(((b / nb) % nb) * 4u + uint32_t((local >> 2) & 3)),
              k = int((b / (nb * nb)) * 4u + uint32_t(local >> 4));
    const float h = a.h;
    reflect_axis(nv.x, (float(i) + 0.5f) * h, a.bmin[0], a.bmax[0], a.restitution);
    reflect_axis(nv.y, (float(j) + 0.5f) * h, a.bmin[1], a.bmax[1], a.restitution);
    reflect_axis(nv.z, (float(k) + 0.5f) * h, a.bmin[2], a.bmax[2], a.restitution);
  }
  vel[node] = make_float4(nv.x, nv.y, nv.z, 0.0f);
}

__global__ void __launch_bounds__(kGridThreads) ck_grid_kernel(CkArgs a, float4* vel) {
  // written by the compaction, unchanged here: through the read-only cache, once per SM
  const uint32_t count = __ldg(a.count);
  const int local = threadIdx.x & 63;
  const uint32_t groups = gridDim.x * (kGridThreads / 64);
  for (uint32_t t0 = (blockIdx.x * (kGridThreads / 64) + (threadIdx.x >> 6)) * kGridU; t0 < count;
       t0 += groups * kGridU) {
    uint32_t b[kGridU];
    float4 a0[kGridU], a1[kGridU];
#pragma unroll
    for (int u = 0; u < kGridU; ++u) b[u] = t0 + u < count ? a.list[t0 + u] : 0xffffffffu;
#pragma unroll
    for (int u = 0; u < kGridU; ++u)
      if (b[u] != 0xffffffffu) {
        const uint32_t node = b[u] * 64u + uint32_t(local);
        a0[u] = a.acc[2 * node];
        a1[u] = a.acc[2 * node + 1];
      }
#pragma unroll
    for (int u = 0; u < kGridU; ++u)
      if (b[u] != 0xffffffffu) {
        const uint32_t node = b[u] * 64u + uint32_t(local);
        a.acc[2 * node] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        a.acc[2 * node + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        grid_node(a, b[u], local, a0[u], a1[u], vel);
      }
  }
}

// ------------------------------------------------------------------ deterministic mode
// P2G as a gather in particle order: particles are sorted (stably) by base cell, every touched node
// merges the particle lists of the 8 cells whose stencils reach it by particle index, and adds the
// contributions in that order, which is the order of the reference's serial loops (:201, :262).
// Each contribution is the atomic scatter's (node_contribution), so node sums, and with them the
// whole step, equal the reference's bit for bit except where ln(det F) differs.
//
// Cell key of a particle with base cell c = floor(x / h) (per axis): ((cz+1)(gn+1) + cy+1)(gn+1)
// + cx+1 when -1 <= c <= gn-1 on every axis (the particle has a node in the grid), else the dead
// key (gn+1)^3, which sorts last and belongs to no cell.

template <bool POW2>
__global__ void __launch_bounds__(256) ck_det_prep_kernel(CkArgs a, uint32_t* keys, float* stress) {
  const uint32_t g1 = uint32_t(a.gn) + 1u;
  for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < a.n; q += uint64_t(gridDim.x) * blockDim.x) {
    const float* r = a.rec + q * kRecFloats;
    const V3 pos{r[0], r[1], r[2]};
    const M3 F{{r[15], r[16], r[17]}, {r[18], r[19], r[20]}, {r[21], r[22], r[23]}};
    Stencil st;
    make_stencil<POW2>(st, pos, a.sp, a.gn, true);
    uint32_t last = 0xffffffffu;
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di)
          if (live(st, di, dj, dk)) mark_block(a, node_index(st.i[0][di], st.i[1][dj], st.i[2][dk], a.nb) >> 6, last);
    bool in = true;
    uint32_t kc[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const int c = st.i[ax][0];
      in = in && c >= -1 && c <= a.gn - 1;
      kc[ax] = uint32_t(c + 1);
    }
    keys[q] = in ? (kc[2] * g1 + kc[1]) * g1 + kc[0] : g1 * g1 * g1;
    const M3 P = piola_stress(a, F);
    float* o = stress + 9 * q;
    o[0] = P.c0.x, o[1] = P.c0.y, o[2] = P.c0.z, o[3] = P.c1.x, o[4] = P.c1.y, o[5] = P.c1.z;
    o[6] = P.c2.x, o[7] = P.c2.y, o[8] = P.c2.z;
  }
}

// [begin, end) of every cell's run in the sorted order (set), or back to empty (clear)
template <bool SET>
__global__ void __launch_bounds__(256) ck_det_ranges_kernel(const uint32_t* skeys, uint64_t n, uint32_t dead,
                                                            uint2* range) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t k = skeys[i];
    if (k == dead) continue;
    const bool first = i == 0 || skeys[i - 1] != k;
    if (SET) {
      if (first) range[k].x = uint32_t(i);
      if (i + 1 == n || skeys[i + 1] != k) range[k].y = uint32_t(i + 1);
    } else if (first) {
      range[k] = make_uint2(0u, 0u);
    }
  }
}

// Every node of the listed blocks: the in-order merge of its 8 cells' particles, accumulated the
// way the reference accumulates; nodes outside the grid (padding blocks) get zeros.
template <bool POW2>
__global__ void __launch_bounds__(256) ck_det_nodes_kernel(CkArgs a, const uint32_t* perm, const uint2* range,
                                                           const float* stress) {
  const uint32_t count = __ldg(a.count);
  const int local = threadIdx.x & 63;
  const uint32_t nb = uint32_t(a.nb), g1 = uint32_t(a.gn) + 1u;
  const float h = a.h;
  for (uint32_t item = blockIdx.x * (kGridThreads / 64) + (threadIdx.x >> 6); item < count;
       item += gridDim.x * (kGridThreads / 64)) {
    const uint32_t b = a.list[item];
    const int i = int((b % nb) * 4u + uint32_t(local & 3)), j = int(((b / nb) % nb) * 4u + uint32_t((local >> 2) & 3)),
              k = int((b / (nb * nb)) * 4u + uint32_t(local >> 4));
    float m = 0.0f;
    V3 mom_sum{0.0f, 0.0f, 0.0f}, force_sum{0.0f, 0.0f, 0.0f};
    if (i < a.gn && j < a.gn && k < a.gn) {
      uint32_t head[8], end[8], cur[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t key = (uint32_t(k - (q >> 2) + 1) * g1 + uint32_t(j - ((q >> 1) & 1) + 1)) * g1 +
                             uint32_t(i - (q & 1) + 1);
        const uint2 r = range[key];
        head[q] = r.x;
        end[q] = r.y;
        cur[q] = r.x < r.y ? perm[r.x] : 0xffffffffu;
      }
      const V3 node{(float(i) + 0.5f) * h, (float(j) + 0.5f) * h, (float(k) + 0.5f) * h};
      for (;;) {
        uint32_t p = 0xffffffffu;
#pragma unroll
        for (int q = 0; q < 8; ++q) p = cur[q] < p ? cur[q] : p;
        if (p == 0xffffffffu) break;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (cur[q] == p) {  // particle indices are unique: exactly one list holds p
            ++head[q];
            cur[q] = head[q] < end[q] ? perm[head[q]] : 0xffffffffu;
          }
        const float* r = a.rec + uint64_t(p) * kRecFloats;
        const V3 pos{r[0], r[1], r[2]};
        const V3 diff = node - pos;
        const float wx = ck_weight<POW2>(diff.x, a.sp), wy = ck_weight<POW2>(diff.y, a.sp),
                    wz = ck_weight<POW2>(diff.z, a.sp);
        const float gx = ck_weight_grad<POW2>(diff.x, a.sp), gy = ck_weight_grad<POW2>(diff.y, a.sp),
                    gz = ck_weight_grad<POW2>(diff.z, a.sp);
        const bool fin = isfinite(pos.x) && isfinite(pos.y) && isfinite(pos.z);
        if (fin && ((wx == 0.0f && gx == 0.0f) || (wy == 0.0f && gy == 0.0f) || (wz == 0.0f && gz == 0.0f))) continue;
        const V3 vel{r[3], r[4], r[5]};
        const M3 B{{r[6], r[7], r[8]}, {r[9], r[10], r[11]}, {r[12], r[13], r[14]}};
        const float* ps = stress + 9 * uint64_t(p);
        const M3 P{{ps[0], ps[1], ps[2]}, {ps[3], ps[4], ps[5]}, {ps[6], ps[7], ps[8]}};
        float wm;
        V3 mom, force;
        node_contribution(wx, wy, wz, gx, gy, gz, diff, vel, B, P, r[25], -r[24], wm, mom, force);
        m = m + wm;
        mom_sum = mom_sum + mom;
        force_sum = force_sum + force;
      }
    }
    const uint32_t node_id = b * 64u + uint32_t(local);
    a.acc[2 * node_id] = make_float4(mom_sum.x, mom_sum.y, mom_sum.z, m);
    a.acc[2 * node_id + 1] = make_float4(force_sum.x, force_sum.y, force_sum.z, 0.0f);
  }
}

// kinetic_energy, average_velocity, average_volume_ratio (:484-503), summed in double
__global__ void __launch_bounds__(256) ck_stats_kernel(const float* rec, uint64_t n, double* sums) {
  double s[5] = {0, 0, 0, 0, 0};
  for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += uint64_t(gridDim.x) * blockDim.x) {
    const float* r = rec + q * kRecFloats;
    const V3 v{r[3], r[4], r[5]};
    const M3 F{{r[15], r[16], r[17]}, {r[18], r[19], r[20]}, {r[21], r[22], r[23]}};
    s[0] += double(0.5f * r[25] * dot3(v, v));
    s[1] += double(v.x);
    s[2] += double(v.y);
    s[3] += double(v.z);
    s[4] += double(detm(F));
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double x = s[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sums + k, x);
  }
}

__global__ void ck_weights_kernel(const float* x, uint64_t n, Spacing sp, float* w, float* dw) {
  for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += uint64_t(gridDim.x) * blockDim.x) {
    w[q] = ck_weight(x[q], sp);
    dw[q] = ck_weight_grad(x[q], sp);
  }
}

}  // namespace

CkWork::~CkWork() {
  cudaFree(det_keys_);
  cudaFree(det_stress_);
  cudaFree(det_range_);
  sort_scratch_free(det_sort_);
  cudaFree(acc_);
  cudaFree(vel_);
  cudaFree(flags_);
  cudaFree(lists_);
  cudaFree(counts_);
  cudaFree(sums_);
}

cudaError_t CkWork::ensure(uint32_t grid_n) {
  if (!counts_) {
    cudaError_t e = cudaMalloc(&counts_, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&sums_, 5 * sizeof(double));
    if (e != cudaSuccess) return e;
  }
  if (grid_n == gn_) return cudaSuccess;
  cudaFree(acc_);
  cudaFree(vel_);
  cudaFree(flags_);
  cudaFree(lists_);
  acc_ = nullptr, vel_ = nullptr, flags_ = nullptr, lists_ = nullptr;
  gn_ = 0xffffffffu;
  clean_ = false;
  const uint64_t nb = grid_n ? (uint64_t(grid_n) + 3) / 4 : 1;
  const uint64_t blocks = nb * nb * nb;
  cudaError_t e = cudaMalloc(&acc_, blocks * 64 * 2 * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&vel_, blocks * 64 * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&flags_, blocks * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&lists_, blocks * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  gn_ = grid_n;
  blocks_ = blocks;
  return cudaSuccess;
}

namespace {
// Kernel arguments for a call over grid buffers laid out for cfg.grid_n.  Sets *pow2 when the
// divisions by h can be exact reciprocal multiplications.
CkArgs make_args(float4* acc, float4* vel, uint32_t* flags, uint32_t* lists, ae_mpm_ck_particle* particles, uint64_t n,
                 const ae_mpm_ck_config& cfg, bool* pow2) {
  CkArgs a{};
  a.rec = reinterpret_cast<float*>(particles);
  a.n = n;
  a.acc = acc;
  a.vel = vel;
  a.flags = flags;
  a.list = lists;
  a.gn = int(cfg.grid_n);
  a.nb = int(cfg.grid_n ? (cfg.grid_n + 3) / 4 : 1);
  a.h = cfg.grid_h, a.dt = cfg.dt, a.youngs = cfg.youngs_modulus, a.poisson = cfg.poissons_ratio;
  a.sp = Spacing{cfg.grid_h, 0.0f, 0.0f};
  int e2 = 0;
  *pow2 = std::isfinite(cfg.grid_h) && cfg.grid_h > 0.0f && std::frexp(cfg.grid_h, &e2) == 0.5f && e2 - 1 >= -40 &&
          e2 - 1 <= 40;
  if (*pow2) a.sp.inv_h = std::ldexp(1.0f, 1 - e2), a.sp.inv_h3 = std::ldexp(1.0f, 3 * (1 - e2));
  a.restitution = cfg.restitution;
  for (int k = 0; k < 3; ++k) a.g[k] = cfg.gravity[k], a.bmin[k] = cfg.bounds_min[k], a.bmax[k] = cfg.bounds_max[k];
  a.aligned16 = (reinterpret_cast<uintptr_t>(particles) & 15u) == 0;
  return a;
}
}  // namespace

cudaError_t CkWork::begin_call(uint32_t grid_n, cudaStream_t s) {
  cudaError_t e = ensure(grid_n);
  if (e != cudaSuccess) return e;
  if (!clean_) {
    e = cudaMemsetAsync(acc_, 0, blocks_ * 64 * 2 * sizeof(float4), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(flags_, 0, blocks_ * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    clean_ = true;
  }
  return cudaMemsetAsync(counts_, 0, 2 * sizeof(uint32_t), s);
}

cudaError_t CkWork::step(ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config& cfg, uint32_t steps,
                         cudaStream_t s, double* kernel_ms) {
  launches_ = 0;
  if (n == 0 || steps == 0) return cudaSuccess;
  cudaError_t e = begin_call(cfg.grid_n, s);
  if (e != cudaSuccess) return e;
  bool pow2 = false;
  CkArgs a = make_args(acc_, vel_, flags_, lists_, particles, n, cfg, &pow2);
  const unsigned pgrid = unsigned((n + kCkThreads - 1) / kCkThreads);
  const unsigned ggrid = unsigned(std::min<uint64_t>(148 * 4, (blocks_ + 4 * kGridU - 1) / (4 * kGridU)));
  const unsigned cgrid = unsigned(std::min<uint64_t>(148 * 8, (blocks_ + 255) / 256));
  // optional per-launch events: [2 k] before and [2 k + 1] after launch k
  const uint32_t n_launch = 1 + 3 * steps;
  std::vector<cudaEvent_t> ev(kernel_ms ? 2 * n_launch : 0);
  for (auto& x : ev)
    if (e == cudaSuccess) e = cudaEventCreate(&x);
  if (e != cudaSuccess) {
    for (auto x : ev)
      if (x) cudaEventDestroy(x);
    return e;
  }
  std::vector<uint8_t> is_particle_launch;
  uint32_t launches = 0;
  auto before = [&] {
    if (kernel_ms) cudaEventRecord(ev[2 * launches], s);
  };
  auto after = [&](bool particles) {
    if (kernel_ms) {
      cudaEventRecord(ev[2 * launches + 1], s);
      is_particle_launch.push_back(particles);
    }
    ++launches;
  };
  a.list = lists_;
  before();
  if (pow2)
    ck_particles_kernel<false, true, true><<<pgrid, kCkThreads, 0, s>>>(a);
  else
    ck_particles_kernel<false, true, false><<<pgrid, kCkThreads, 0, s>>>(a);
  after(true);
  for (uint32_t st = 0; st < steps; ++st) {
    // counters alternate by step: this step's compaction appends to one and zeroes the other
    a.count = counts_ + (st & 1);
    a.next_count = counts_ + ((st + 1) & 1);
    before();
    ck_compact_kernel<<<cgrid, 256, 0, s>>>(flags_, blocks_, lists_, a.count, a.next_count);
    after(false);
    before();
    ck_grid_kernel<<<ggrid, kGridThreads, 0, s>>>(a, vel_);
    after(false);
    before();
    if (st + 1 < steps && pow2)
      ck_particles_kernel<true, true, true><<<pgrid, kCkThreads, 0, s>>>(a);
    else if (st + 1 < steps)
      ck_particles_kernel<true, true, false><<<pgrid, kCkThreads, 0, s>>>(a);
    else if (pow2)
      ck_particles_kernel<true, false, true><<<pgrid, kCkThreads, 0, s>>>(a);
    else
      ck_particles_kernel<true, false, false><<<pgrid, kCkThreads, 0, s>>>(a);
    after(true);
  }
  e = cudaGetLastError();
  if (kernel_ms) {
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    kernel_ms[0] = kernel_ms[1] = 0.0;
    for (uint32_t k = 0; k < n_launch && e == cudaSuccess; ++k) {
      float ms = 0.0f;
      e = cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
      kernel_ms[is_particle_launch[k] ? 0 : 1] += ms;
    }
    for (auto x : ev) cudaEventDestroy(x);
  }
  if (e != cudaSuccess) clean_ = false;
  launches_ = launches;
  return e;
}

cudaError_t CkWork::ensure_det(uint64_t n, uint32_t grid_n) {
  const uint64_t g1 = uint64_t(grid_n) + 1, cells = g1 * g1 * g1;
  cudaError_t e = cudaSuccess;
  if (n > det_cap_) {
    cudaFree(det_keys_);
    cudaFree(det_stress_);
    det_keys_ = nullptr, det_stress_ = nullptr, det_cap_ = 0;
    sort_scratch_free(det_sort_);
    e = cudaMalloc(&det_keys_, n * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&det_stress_, 9 * n * sizeof(float));
    if (e == cudaSuccess) e = sort_scratch_alloc(det_sort_, n);
    if (e != cudaSuccess) return e;
    det_cap_ = n;
  }
  if (cells != det_cells_) {
    cudaFree(det_range_);
    det_range_ = nullptr, det_cells_ = 0;
    e = cudaMalloc(&det_range_, cells * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMemset(det_range_, 0, cells * sizeof(uint2));  // every cell empty
    if (e != cudaSuccess) return e;
    det_cells_ = cells;
  }
  return cudaSuccess;
}

cudaError_t CkWork::step_deterministic(ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config& cfg,
                                       uint32_t steps, cudaStream_t s) {
  launches_ = 0;
  if (n == 0 || steps == 0) return cudaSuccess;
  cudaError_t e = begin_call(cfg.grid_n, s);
  if (e == cudaSuccess) e = ensure_det(n, cfg.grid_n);
  if (e != cudaSuccess) return e;
  bool pow2 = false;
  CkArgs a = make_args(acc_, vel_, flags_, lists_, particles, n, cfg, &pow2);
  const uint32_t g1 = cfg.grid_n + 1u, dead = g1 * g1 * g1;
  int key_bits = 1;
  while (key_bits < 32 && (dead >> key_bits) != 0u) ++key_bits;
  const unsigned pgrid = unsigned((n + kCkThreads - 1) / kCkThreads);
  const unsigned sgrid = unsigned(std::min<uint64_t>(148 * 8, (n + 255) / 256));
  const unsigned ngrid = unsigned(std::min<uint64_t>(148 * 8, (blocks_ + 3) / 4));
  const unsigned ggrid = unsigned(std::min<uint64_t>(148 * 4, (blocks_ + 4 * kGridU - 1) / (4 * kGridU)));
  const unsigned cgrid = unsigned(std::min<uint64_t>(148 * 8, (blocks_ + 255) / 256));
  uint32_t launches = 0;
  for (uint32_t st = 0; st < steps; ++st) {
    a.count = counts_ + (st & 1);
    a.next_count = counts_ + ((st + 1) & 1);
    if (pow2)
      ck_det_prep_kernel<true><<<sgrid, 256, 0, s>>>(a, det_keys_, det_stress_);
    else
      ck_det_prep_kernel<false><<<sgrid, 256, 0, s>>>(a, det_keys_, det_stress_);
    const uint32_t *skeys = nullptr, *perm = nullptr;
    launches += 1 + uint32_t(radix_sort_pairs(det_keys_, n, key_bits, det_sort_, s, &skeys, &perm));
    ck_det_ranges_kernel<true><<<sgrid, 256, 0, s>>>(skeys, n, dead, det_range_);
    ck_compact_kernel<<<cgrid, 256, 0, s>>>(flags_, blocks_, lists_, a.count, a.next_count);
    if (pow2)
      ck_det_nodes_kernel<true><<<ngrid, kGridThreads, 0, s>>>(a, perm, det_range_, det_stress_);
    else
      ck_det_nodes_kernel<false><<<ngrid, kGridThreads, 0, s>>>(a, perm, det_range_, det_stress_);
    ck_grid_kernel<<<ggrid, kGridThreads, 0, s>>>(a, vel_);
    ck_det_ranges_kernel<false><<<sgrid, 256, 0, s>>>(skeys, n, dead, det_range_);
    if (pow2)
      ck_particles_kernel<true, false, true><<<pgrid, kCkThreads, 0, s>>>(a);
    else
      ck_particles_kernel<true, false, false><<<pgrid, kCkThreads, 0, s>>>(a);
    launches += 6;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) clean_ = false;
  launches_ = launches;
  return e;
}

cudaError_t CkWork::stats(const ae_mpm_ck_particle* particles, uint64_t n, ae_mpm_ck_stats* out, cudaStream_t s) {
  cudaError_t e = ensure(gn_ == 0xffffffffu ? 0u : gn_);
  if (e != cudaSuccess) return e;
  double h[5] = {0, 0, 0, 0, 0};
  if (n) {
    e = cudaMemsetAsync(sums_, 0, 5 * sizeof(double), s);
    if (e != cudaSuccess) return e;
    const unsigned grid = unsigned(std::min<uint64_t>(148 * 4, (n + 255) / 256));
    ck_stats_kernel<<<grid, 256, 0, s>>>(reinterpret_cast<const float*>(particles), n, sums_);
    e = cudaMemcpyAsync(h, sums_, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
  }
  out->kinetic_energy = float(h[0]);
  const float fn = float(n);
  for (int k = 0; k < 3; ++k) out->average_velocity[k] = n ? float(h[1 + k]) / fn : 0.0f;
  out->average_volume_ratio = n ? float(h[4]) / fn : 1.0f;
  return cudaSuccess;
}

cudaError_t CkWork::weights(const float* x, uint64_t n, float h, float* w, float* dw, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned grid = unsigned(std::min<uint64_t>(148 * 4, (n + 255) / 256));
  ck_weights_kernel<<<grid, 256, 0, s>>>(x, n, Spacing{h, 0.0f, 0.0f}, w, dw);
  return cudaGetLastError();
}

}  // namespace aemp
