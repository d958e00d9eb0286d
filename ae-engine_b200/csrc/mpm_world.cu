// mpm_world.cu -- the MPM substep on sm_100a: kernels and the world driver.
//
// Substep (every scene of a world at once):
//   sort     radix sort of cell keys -> perm (sorted position -> storage slot)
//   P2G      one block per chunk of sorted particles; the chunk's stencil bounding box is a
//            shared-memory tile with halo that absorbs all same-cell contributions, then is
//            flushed with 16-byte vector atomics (red.global.add.v4.f32) into the grid
//   grid     one pass over the blocks P2G touched: momentum -> velocity, gravity, walls;
//            clears the accumulator and the touched flags for the next substep
//   G2P      one thread per sorted particle: gather, APIC C, F update and material return
//            mapping, written to the other particle buffer in sorted order (the reorder costs
//            nothing extra), plus the next substep's cell key
// Deterministic mode replaces P2G's float atomics with per-cell fixed-order sums and a per-node
// fixed-order gather (no float atomics anywhere), so two runs are bitwise identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>

#include "mpm_world.cuh"

namespace aemp {

// ============================================================================================
// device helpers
// ============================================================================================
template <class T>
struct Bits;
template <>
struct Bits<float> {
  static __device__ __forceinline__ float pack(uint32_t u) { return __uint_as_float(u); }
  static __device__ __forceinline__ uint32_t unpack(float f) { return __float_as_uint(f); }
};
template <>
struct Bits<double> {
  static __device__ __forceinline__ double pack(uint32_t u) { return __longlong_as_double((long long)u); }
  static __device__ __forceinline__ uint32_t unpack(double d) { return uint32_t(__double_as_longlong(d)); }
};

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ld4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 mk4(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
__device__ __forceinline__ double4 mk4(double a, double b, double c, double d) { return make_double4(a, b, c, d); }

__device__ __forceinline__ void atomic_add4(float4* p, float a, float b, float c, float d) {
  atomicAdd(p, make_float4(a, b, c, d));  // one 16-byte vector reduction (sm_90+)
}
__device__ __forceinline__ void atomic_add4(double4* p, double a, double b, double c, double d) {
  atomicAdd(&p->x, a);
  atomicAdd(&p->y, b);
  atomicAdd(&p->z, c);
  atomicAdd(&p->w, d);
}

// asynchronous 16-byte global -> shared copies (cp.async, no registers held while in flight)
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// A work counter that an earlier kernel wrote and that no thread of this kernel changes, read by
// every thread: through the read-only cache, so each SM fetches it once.  (A volatile or L2-only
// load would send every warp of the grid to the same L2 slice before any of them could start.)
__device__ __forceinline__ uint32_t launch_count(const uint32_t* p) { return __ldg(p); }

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <class V4>
__device__ __forceinline__ void cp_async_v4(V4* sdst, const V4* gsrc) {
#pragma unroll
  for (int k = 0; k < int(sizeof(V4) / 16); ++k)
    cp_async16(reinterpret_cast<char*>(sdst) + 16 * k, reinterpret_cast<const char*>(gsrc) + 16 * k);
}

template <class T>
__device__ __forceinline__ int floor_to_int(T v) {
  if (v != v) return 0;  // NaN -> 0, as Rust's `as isize`
  v = t_clamp(v, T(-1.0e9), T(1.0e9));
  return int(t_floor(v));
}

template <class T>
__device__ __forceinline__ uint32_t node_index(const SceneDev<T>& sc, int i, int j, int k) {
  uint32_t b = (uint32_t(k >> 2) * uint32_t(sc.nb[1]) + uint32_t(j >> 2)) * uint32_t(sc.nb[0]) + uint32_t(i >> 2);
  return (sc.blk_off + b) * 64u + ((uint32_t(k & 3) << 4) | (uint32_t(j & 3) << 2) | uint32_t(i & 3));
}

template <class T>
__device__ __forceinline__ T sel3(const T* a, int i) {
  return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]);
}

// cell key of a position: physics mode base clamped into the grid; reference modes base clamped
// at 0 (Grid::pos_to_grid, mpm_solver.rs:161-175) and the dead key when the stencil is off-grid
template <class T>
__device__ __forceinline__ uint32_t cell_key(const SceneDev<T>& sc, int mode, T x, T y, T z) {
  T p[3] = {x, y, z};
  int b[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int g = floor_to_int((p[a] - sc.origin[a]) * sc.inv_dx - T(0.5));
    if (mode == AE_MPM_MODE_PHYSICS) {
      g = min(max(g, 0), sc.n[a] - 1);
    } else {
      g = max(g, 0);
      if (g >= sc.n[a]) return sc.dead_key;
    }
    b[a] = g;
  }
  return node_index(sc, b[0], b[1], b[2]);
}

// The chunk a CTA works on: {scene, first slot, end of the live particles, end of capacity}.
// A world of one scene needs no table (its chunks are consecutive ranges of blockDim.x slots),
// so its CTAs start their particle loads without first waiting for a descriptor load.
template <class T>
__device__ __forceinline__ int4 cta_chunk(const WorldDev<T>& w) {
  if (w.one_scene) {
    const uint64_t lo = uint64_t(w.one_off) + uint64_t(blockIdx.x) * blockDim.x;
    const uint64_t live = lo + blockDim.x < w.one_live_end ? lo + blockDim.x : w.one_live_end;
    const uint64_t cap = lo + blockDim.x < w.one_cap_end ? lo + blockDim.x : w.one_cap_end;
    return make_int4(0, int(lo), int(live > lo ? live : lo), int(cap));
  }
  return w.chunks[blockIdx.x];
}

template <class T>
__device__ __forceinline__ void mark_block(const WorldDev<T>& w, uint32_t gb) {
  volatile uint32_t* f = w.blk_flag + gb;
  if (*f == 0u && atomicExch(w.blk_flag + gb, 1u) == 0u) {
    uint32_t slot = atomicAdd(w.touched_count, 1u);
    w.touched[slot] = gb;
  }
}

template <class T>
__device__ __forceinline__ const MatDev& mat_of(const WorldDev<T>& w, const SceneDev<T>& sc, uint32_t m) {
  return w.mats[sc.mat_off + (m < sc.n_mat ? m : sc.n_mat)];
}

// MLS-MPM affine momentum matrix (Hu et al. 2018): A = m C - k tau(F, J) with
// k = 4 dt V0 / dx^2, V0 = m / rho.  Physics mode stores A in the particle's C slot between
// substeps (G2P computes it while F is in registers), so P2G needs neither F nor the stress;
// pack/unpack convert to and from the caller's C at the boundary.
template <class T>
__device__ __forceinline__ T affine_k(const SceneDev<T>& sc, const MatDev& md, T m) {
  return T(4) * sc.dt * (m / T(md.rho)) * sc.inv_dx * sc.inv_dx;
}
template <class T>
__device__ __forceinline__ void affine_from_c(const SceneDev<T>& sc, const MatDev& md, T m, const T* C, const T* F, T J,
                                              T* A) {
  T tau[9];
  phys_tau(md, F, J, tau);
  const T k = affine_k(sc, md, m);
#pragma unroll
  for (int i = 0; i < 9; ++i) A[i] = m * C[i] - k * tau[i];
}

// ============================================================================================
// per-particle P2G setup
// ============================================================================================
template <class T>
struct P2GPart {
  int g[3];     // stencil base node per axis (nodes g..g+2)
  T w[3][3];    // per-axis weights
  T o[3][3];    // physics: (k - fx) dx;  reference: node position - particle position
  T fx[3];      // physics: position relative to the base node, in cells (in [0.5, 1.5))
  T dw[3][3];   // reference: N'(k - fx) / dx
  T m;
  T v[3];       // physics: m v;  reference/velonly: v
  T A[9];       // physics: m C - 4 dt V0/dx^2 tau;  reference: C
  T sv[9];      // reference: dt * V * sigma
};

template <class T, int MODE>
__device__ __forceinline__ void p2g_setup(const WorldDev<T>& w, const SceneDev<T>& sc, uint32_t src, P2GPart<T>& p) {
  using V4 = typename V4T<T>::type;
  const V4 a0 = ld4(w.in[0] + src);
  const V4 a4 = ld4(w.in[4] + src);
  T x[3] = {a0.x, a0.y, a0.z};
  p.m = a0.w;
  if (MODE == AE_MPM_MODE_VELOCITY_ONLY) {
    p.v[0] = a4.x;
    p.v[1] = a4.y;
    p.v[2] = a4.z;
  } else if (MODE == AE_MPM_MODE_PHYSICS) {
    const V4 a5 = ld4(w.in[5] + src), a6 = ld4(w.in[6] + src);
    const T A[9] = {a4.w, a5.x, a5.y, a5.z, a5.w, a6.x, a6.y, a6.z, a6.w};
#pragma unroll
    for (int k = 0; k < 9; ++k) p.A[k] = A[k];
    p.v[0] = p.m * a4.x;
    p.v[1] = p.m * a4.y;
    p.v[2] = p.m * a4.z;
  } else {
    const V4 a1 = ld4(w.in[1] + src), a2 = ld4(w.in[2] + src), a3 = ld4(w.in[3] + src);
    const V4 a5 = ld4(w.in[5] + src), a6 = ld4(w.in[6] + src);
    T F[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
    T C[9] = {a4.w, a5.x, a5.y, a5.z, a5.w, a6.x, a6.y, a6.z, a6.w};
    T J = a3.y;
    const MatDev& md = mat_of(w, sc, Bits<T>::unpack(a3.z) & 0xffffu);
    {
      T st[9];
      ref_stress(md, F, J, st);
      T vol = p.m / T(md.rho);
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        p.sv[k] = sc.dt * (vol * st[k]);
        p.A[k] = C[k];
      }
      p.v[0] = a4.x;
      p.v[1] = a4.y;
      p.v[2] = a4.z;
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T X = (x[a] - sc.origin[a]) * sc.inv_dx;
    if (MODE == AE_MPM_MODE_PHYSICS) {
      int b = floor_to_int(X - T(0.5));
      T fx = X - T(b);
      p.g[a] = b;
      p.fx[a] = fx;
      T t0 = T(1.5) - fx, t1 = fx - T(1), t2 = fx - T(0.5);
      p.w[a][0] = T(0.5) * t0 * t0;
      p.w[a][1] = T(0.75) - t1 * t1;
      p.w[a][2] = T(0.5) * t2 * t2;
#pragma unroll
      for (int k = 0; k < 3; ++k) p.o[a][k] = (T(k) - fx) * sc.dx;
    } else {
      int gu = floor_to_int(X - T(0.5));
      T fx = X - T(0.5) - T(gu);
      int g = max(gu, 0);
      p.g[a] = g;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        p.w[a][k] = b_spline(T(k) - fx);
        if (MODE == AE_MPM_MODE_REFERENCE) {
          p.dw[a][k] = b_spline_deriv(T(k) - fx) * sc.inv_dx;
          p.o[a][k] = (T(g + k) + T(0.5)) * sc.dx + sc.origin[a] - x[a];
        }
      }
    }
  }
}

// Contribution of a particle to stencil node (a,b,c); returns false when the node is skipped.
template <class T, int MODE>
__device__ __forceinline__ bool p2g_contrib(const SceneDev<T>& sc, const P2GPart<T>& p, int a, int b, int c, T& cm,
                                            T& cx, T& cy, T& cz) {
  int X = p.g[0] + a, Y = p.g[1] + b, Z = p.g[2] + c;
  if (X < 0 || Y < 0 || Z < 0 || X >= sc.n[0] || Y >= sc.n[1] || Z >= sc.n[2]) return false;
  T wx = sel3(p.w[0], a), wy = sel3(p.w[1], b), wz = sel3(p.w[2], c);
  if (MODE == AE_MPM_MODE_PHYSICS) {
    T w = wx * wy * wz;
    T d0 = sel3(p.o[0], a), d1 = sel3(p.o[1], b), d2 = sel3(p.o[2], c);
    cm = w * p.m;
    cx = w * (p.v[0] + p.A[0] * d0 + p.A[1] * d1 + p.A[2] * d2);
    cy = w * (p.v[1] + p.A[3] * d0 + p.A[4] * d1 + p.A[5] * d2);
    cz = w * (p.v[2] + p.A[6] * d0 + p.A[7] * d1 + p.A[8] * d2);
    return true;
  } else if (MODE == AE_MPM_MODE_REFERENCE) {
    T w = wx * wy * wz;
    if (w < T(1e-10)) return false;
    T d0 = sel3(p.o[0], a), d1 = sel3(p.o[1], b), d2 = sel3(p.o[2], c);
    T vx = p.v[0] + p.A[0] * d0 + p.A[1] * d1 + p.A[2] * d2;
    T vy = p.v[1] + p.A[3] * d0 + p.A[4] * d1 + p.A[5] * d2;
    T vz = p.v[2] + p.A[6] * d0 + p.A[7] * d1 + p.A[8] * d2;
    T e0 = sel3(p.dw[0], a), e1 = sel3(p.dw[1], b), e2 = sel3(p.dw[2], c);
    T wm = w * p.m;
    cm = wm;
    cx = wm * vx + (p.sv[0] * e0 + p.sv[1] * e1 + p.sv[2] * e2);
    cy = wm * vy + (p.sv[3] * e0 + p.sv[4] * e1 + p.sv[5] * e2);
    cz = wm * vz + (p.sv[6] * e0 + p.sv[7] * e1 + p.sv[8] * e2);
    return true;
  } else {
    if (wz < T(1e-10) || wy < T(1e-10)) return false;
    T w = wx * (wy * wz);
    if (w < T(1e-10)) return false;
    T wm = w * p.m;
    cm = wm;
    cx = wm * p.v[0];
    cy = wm * p.v[1];
    cz = wm * p.v[2];
    return true;
  }
}

// ============================================================================================
// P2G
// ============================================================================================
enum { kVarTile = 1, kVarWarpAgg = 2, kVarGlobal = 3, kVarLanes = 4 };

template <class T>
__device__ __forceinline__ void shared_add4(typename V4T<T>::type* t, T a, T b, T c, T d) {
  T* q = reinterpret_cast<T*>(t);
  atomicAdd(q + 0, a);
  atomicAdd(q + 1, b);
  atomicAdd(q + 2, c);
  atomicAdd(q + 3, d);
}

template <class T, int MODE, int VAR>
__global__ void __launch_bounds__(512) p2g_kernel(WorldDev<T> w) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  V4* tile = reinterpret_cast<V4*>(smem);
  __shared__ int s_lo[3], s_hi[3];
  const int tid = threadIdx.x, lane = tid & 31;
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  if (tid < 3) {
    s_lo[tid] = INT_MAX;
    s_hi[tid] = INT_MIN;
  }
  __syncthreads();
  const int j = ch.y + tid;
  const bool live = j < ch.z;
  P2GPart<T> p;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  bool has = false;
  if (live) {
    const uint32_t src = w.perm ? w.perm[j] : uint32_t(j);
    p2g_setup<T, MODE>(w, sc, src, p);
    has = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = max(p.g[a], 0);
      hi[a] = min(p.g[a] + 2, sc.n[a] - 1);
      if (lo[a] > hi[a]) has = false;
    }
  }
  // block bounding box of all in-grid stencil nodes
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int l = __reduce_min_sync(0xffffffffu, has ? lo[a] : INT_MAX);
    int h = __reduce_max_sync(0xffffffffu, has ? hi[a] : INT_MIN);
    if (lane == 0 && l != INT_MAX) {
      atomicMin(&s_lo[a], l);
      atomicMax(&s_hi[a], h);
    }
  }
  __syncthreads();
  const int L0 = s_lo[0], L1 = s_lo[1], L2 = s_lo[2];
  const bool any = L0 != INT_MAX;
  const int D0 = any ? s_hi[0] - L0 + 1 : 0, D1 = any ? s_hi[1] - L1 + 1 : 0, D2 = any ? s_hi[2] - L2 + 1 : 0;
  const int vol = D0 * D1 * D2;
  const bool use_tile = VAR != kVarGlobal && any && vol <= w.max_tile_nodes;
  if (!any) return;
  if (use_tile) {
    for (int t = tid; t < vol; t += blockDim.x) tile[t] = mk4(T(0), T(0), T(0), T(0));
    __syncthreads();
    if (VAR == kVarWarpAgg) {
      // lanes of one cell are one run in sorted order: reduce each run with shuffles and let its
      // first lane add the run's sum to the tile
      uint32_t key = has ? uint32_t(((p.g[2] - L2 + 2) * (D1 + 4) + (p.g[1] - L1 + 2)) * (D0 + 4) + (p.g[0] - L0 + 2))
                         : (0x80000000u | uint32_t(lane));
      uint32_t peers = __match_any_sync(0xffffffffu, key);
      int first = __ffs(peers) - 1;
      int cnt = __popc(peers);
      uint32_t run = (cnt == 32) ? 0xffffffffu : (((1u << cnt) - 1u) << first);
      bool contiguous = peers == run;
      int last = first + cnt - 1;
      int gmax = __reduce_max_sync(0xffffffffu, cnt);
      if (__all_sync(0xffffffffu, contiguous)) {
#pragma unroll 1
        for (int o = 0; o < 27; ++o) {
          const int a = o % 3, b = (o / 3) % 3, c = o / 9;
          T cm = T(0), cx = T(0), cy = T(0), cz = T(0);
          bool ok = has && p2g_contrib<T, MODE>(sc, p, a, b, c, cm, cx, cy, cz);
          if (!ok) cm = cx = cy = cz = T(0);
          for (int off = 1; off < gmax; off <<= 1) {
            T tm = __shfl_down_sync(0xffffffffu, cm, off);
            T tx = __shfl_down_sync(0xffffffffu, cx, off);
            T ty = __shfl_down_sync(0xffffffffu, cy, off);
            T tz = __shfl_down_sync(0xffffffffu, cz, off);
            if (lane + off <= last) {
              cm += tm;
              cx += tx;
              cy += ty;
              cz += tz;
            }
          }
          if (has && lane == first) {
            int X = p.g[0] + a, Y = p.g[1] + b, Z = p.g[2] + c;
            if (X >= 0 && Y >= 0 && Z >= 0 && X < sc.n[0] && Y < sc.n[1] && Z < sc.n[2] && cm != T(0))
              shared_add4<T>(tile + ((Z - L2) * D1 + (Y - L1)) * D0 + (X - L0), cm, cx, cy, cz);
          }
        }
      } else if (has) {
        for (int o = 0; o < 27; ++o) {
          const int a = o % 3, b = (o / 3) % 3, c = o / 9;
          T cm, cx, cy, cz;
          if (p2g_contrib<T, MODE>(sc, p, a, b, c, cm, cx, cy, cz))
            shared_add4<T>(tile + ((p.g[2] + c - L2) * D1 + (p.g[1] + b - L1)) * D0 + (p.g[0] + a - L0), cm, cx, cy, cz);
        }
      }
    } else if (has) {
      // lanes of one cell start at different stencil nodes so their shared atomics do not collide
      const int rot = lane % 27;
#pragma unroll 3
      for (int k = 0; k < 27; ++k) {
        int o = k + rot;
        o = (o >= 27) ? o - 27 : o;
        const int a = o % 3, b = (o / 3) % 3, c = o / 9;
        T cm, cx, cy, cz;
        if (p2g_contrib<T, MODE>(sc, p, a, b, c, cm, cx, cy, cz))
          shared_add4<T>(tile + ((p.g[2] + c - L2) * D1 + (p.g[1] + b - L1)) * D0 + (p.g[0] + a - L0), cm, cx, cy, cz);
      }
    }
    __syncthreads();
    for (int t = tid; t < vol; t += blockDim.x) {
      V4 v = tile[t];
      if (v.x != T(0)) {
        int X = L0 + t % D0, Y = L1 + (t / D0) % D1, Z = L2 + t / (D0 * D1);
        atomic_add4(w.acc + node_index(sc, X, Y, Z), v.x, v.y, v.z, v.w);
      }
    }
    const int B0 = L0 >> 2, B1 = L1 >> 2, B2 = L2 >> 2;
    const int E0 = (L0 + D0 - 1) >> 2, E1 = (L1 + D1 - 1) >> 2, E2 = (L2 + D2 - 1) >> 2;
    const int nbx = E0 - B0 + 1, nby = E1 - B1 + 1, nbz = E2 - B2 + 1;
    for (int t = tid; t < nbx * nby * nbz; t += blockDim.x) {
      int bx = B0 + t % nbx, by = B1 + (t / nbx) % nby, bz = B2 + t / (nbx * nby);
      mark_block(w, sc.blk_off + (uint32_t(bz) * sc.nb[1] + by) * sc.nb[0] + bx);
    }
  } else {
    if (VAR != kVarGlobal && tid == 0) atomicAdd(w.err + 4 * ch.x + 3, 1u);
    if (has) {
#pragma unroll 1
      for (int o = 0; o < 27; ++o) {
        const int a = o % 3, b = (o / 3) % 3, c = o / 9;
        T cm, cx, cy, cz;
        if (p2g_contrib<T, MODE>(sc, p, a, b, c, cm, cx, cy, cz))
          atomic_add4(w.acc + node_index(sc, p.g[0] + a, p.g[1] + b, p.g[2] + c), cm, cx, cy, cz);
      }
      for (int t = 0; t < 8; ++t) {
        int bx = (t & 1) ? (hi[0] >> 2) : (lo[0] >> 2);
        int by = (t & 2) ? (hi[1] >> 2) : (lo[1] >> 2);
        int bz = (t & 4) ? (hi[2] >> 2) : (lo[2] >> 2);
        mark_block(w, sc.blk_off + (uint32_t(bz) * sc.nb[1] + by) * sc.nb[0] + bx);
      }
    }
  }
}

// --------------------------------------------------------------------------------------------
// P2G, physics mode, lanes as stencil columns.  Particles are sorted by cell, so a warp's 32
// particles form a few runs of equal cells (about 30 particles per cell in a dense snow block).
// Lanes 0..26 are 3 particle groups x 9 (y,z) columns of the 3x3x3 stencil: lane (G, b + 3c)
// takes particles s0+G, s0+G+3, ... of a run and keeps the sums of nodes (0..2, b, c) of the
// run's cell in 12 registers.  At the end of the run the three groups are summed with shuffles
// and lanes 0..8 add the run's 27 node sums to the grid with 16-byte vector reductions, one per
// node and run instead of one per node and particle.  Warps never wait for one another: each
// stages its own particles and marks the grid blocks its own stencils touch.
//
// Everything that depends on one particle only is computed by the particle's own thread (in
// parallel over particles) and staged particle-major in shared memory:
//   col[q*9 + b + 3c] = (u, wy[b] wz[c])    u = m v + A d, d = node (0,b,c) - particle
//   wxm[q]            = (wx[0], wx[1], wx[2], m)
//   acol[q]           = (dx A[.][0], 0)      node (a+1,b,c) has u + dx A[.][0]
// so a lane's work per particle is 3 shared loads (the 27 column loads are consecutive vectors,
// conflict-free), 3 weight products, 12 FMAs and 6 adds.
// --------------------------------------------------------------------------------------------
constexpr int kLaneVecs = 11;  // shared vectors per particle: 9 columns, x weights + mass, x column

template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) p2g_lanes_kernel(WorldDev<T> w) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nt = blockDim.x;
  V4* col = reinterpret_cast<V4*>(smem);          // col[q * 9 + j]
  V4* wxm = col + 9 * nt;                         // wxm[q]
  V4* acol = wxm + nt;                            // acol[q]
  int4* gk = reinterpret_cast<int4*>(acol + nt);  // gk[q] = (stencil base, cell key)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  const int n0 = sc.n[0], n1 = sc.n[1], n2 = sc.n[2];
  const int j = ch.y + tid;
  const bool live = j < ch.z;
  bool has = false;
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  P2GPart<T> p;
  p.g[0] = p.g[1] = p.g[2] = 0;
  if (live) {
    const uint32_t src = w.perm ? w.perm[j] : uint32_t(j);
    p2g_setup<T, AE_MPM_MODE_PHYSICS>(w, sc, src, p);
    has = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = max(p.g[a], 0);
      hi[a] = min(p.g[a] + 2, sc.n[a] - 1);
      if (lo[a] > hi[a]) has = false;
    }
  }
  // cell key: unique per cell (a stencil with any node in the grid has g in [-2, n-1] per axis)
  const uint32_t key = has ? uint32_t(p.g[0] + 2) + uint32_t(n0 + 2) * (uint32_t(p.g[1] + 2) + uint32_t(n1 + 2) * uint32_t(p.g[2] + 2))
                           : 0xffffffffu;
  // Group equal keys anywhere in the warp (not only adjacent ones: particles that crossed into a
  // neighbouring cell since the last sort rejoin it): groups in order of their first lane, lanes
  // within a group in lane order.  pos is this particle's slot in that grouped order.
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(peers) - 1;
  const uint32_t lead_cnt = lane == leader ? uint32_t(__popc(peers)) : 0u;
  uint32_t incl = lead_cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t lead_off = incl - lead_cnt;
  const int pos = int(__shfl_sync(0xffffffffu, lead_off, leader)) + __popc(peers & ((1u << lane) - 1u));
  uint32_t starts = __reduce_or_sync(0xffffffffu, lane == leader ? (1u << lead_off) : 0u);
  const int q = warp * 32 + pos;
  if (live) {
    const T dx = sc.dx;
    T c0[3], c1[3], c2[3], qv[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      c0[r] = dx * p.A[3 * r + 0];
      c1[r] = dx * p.A[3 * r + 1];
      c2[r] = dx * p.A[3 * r + 2];
      qv[r] = p.v[r] - (c0[r] * p.fx[0] + c1[r] * p.fx[1] + c2[r] * p.fx[2]);
    }
    V4* cq = col + q * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const T ux = qv[0] + T(b) * c1[0] + T(c) * c2[0];
        const T uy = qv[1] + T(b) * c1[1] + T(c) * c2[1];
        const T uz = qv[2] + T(b) * c1[2] + T(c) * c2[2];
        cq[b + 3 * c] = mk4(ux, uy, uz, p.w[1][b] * p.w[2][c]);
      }
    }
    wxm[q] = mk4(p.w[0][0], p.w[0][1], p.w[0][2], p.m);
    acol[q] = mk4(c0[0], c0[1], c0[2], T(0));
  }
  gk[q] = make_int4(p.g[0], p.g[1], p.g[2], int(key));
  __syncwarp();
  // lanes 27..31 mirror the columns of lanes 22..26 (in-bounds reads, results never used)
  const int grp = lane < 27 ? lane / 9 : 2;
  const int jc = lane < 27 ? lane - 9 * grp : lane - 23;
  const int nb = jc % 3, nc = jc / 3;
  const uint32_t nb0u = uint32_t(sc.nb[0]), nb1u = uint32_t(sc.nb[1]);
  const V4* colw = col + warp * 32 * 9 + jc;
  const V4* wxw = wxm + warp * 32;
  const V4* acw = acol + warp * 32;
  while (starts) {
    const int s0 = __ffs(starts) - 1;
    starts &= starts - 1u;
    const int e0 = starts ? __ffs(starts) - 1 : 32;
    const int4 run = gk[warp * 32 + s0];
    if (uint32_t(run.w) == 0xffffffffu) continue;
    const int X = run.x, Y = run.y + nb, Z = run.z + nc;
    T m0 = 0, x0 = 0, y0 = 0, z0 = 0, m1 = 0, x1 = 0, y1 = 0, z1 = 0, m2 = 0, x2 = 0, y2 = 0, z2 = 0;
    if constexpr (sizeof(T) == 4) {  // x and y of each node as one packed pair
      float2 q0 = make_float2(0.f, 0.f), q1 = q0, q2 = q0;
#pragma unroll 2
      for (int i = s0 + grp; i < e0; i += 3) {
        const float4 u = colw[i * 9];
        const float4 r = wxw[i];
        const float4 a = acw[i];
        const float W0 = r.x * u.w, W1 = r.y * u.w, W2 = r.z * u.w;
        const float2 axy = make_float2(a.x, a.y), u0 = make_float2(u.x, u.y);
        const float2 u1 = __fadd2_rn(u0, axy), u2 = __fadd2_rn(u1, axy);
        m0 += W0 * r.w;
        m1 += W1 * r.w;
        m2 += W2 * r.w;
        q0 = __ffma2_rn(make_float2(W0, W0), u0, q0);
        q1 = __ffma2_rn(make_float2(W1, W1), u1, q1);
        q2 = __ffma2_rn(make_float2(W2, W2), u2, q2);
        const float uz1 = u.z + a.z;
        z0 += W0 * u.z;
        z1 += W1 * uz1;
        z2 += W2 * (uz1 + a.z);
      }
      x0 = q0.x, y0 = q0.y, x1 = q1.x, y1 = q1.y, x2 = q2.x, y2 = q2.y;
    } else
#pragma unroll 2
    for (int i = s0 + grp; i < e0; i += 3) {
      const V4 u = colw[i * 9];
      const V4 r = wxw[i];
      const V4 a = acw[i];
      const T W0 = r.x * u.w, W1 = r.y * u.w, W2 = r.z * u.w;
      m0 += W0 * r.w;
      x0 += W0 * u.x;
      y0 += W0 * u.y;
      z0 += W0 * u.z;
      const T ux = u.x + a.x, uy = u.y + a.y, uz = u.z + a.z;
      m1 += W1 * r.w;
      x1 += W1 * ux;
      y1 += W1 * uy;
      z1 += W1 * uz;
      m2 += W2 * r.w;
      x2 += W2 * (ux + a.x);
      y2 += W2 * (uy + a.y);
      z2 += W2 * (uz + a.z);
    }
    if (e0 - s0 > 1) {
      auto groups = [](T v) { return v + __shfl_down_sync(0xffffffffu, v, 9) + __shfl_down_sync(0xffffffffu, v, 18); };
      m0 = groups(m0), x0 = groups(x0), y0 = groups(y0), z0 = groups(z0);
      m1 = groups(m1), x1 = groups(x1), y1 = groups(y1), z1 = groups(z1);
      m2 = groups(m2), x2 = groups(x2), y2 = groups(y2), z2 = groups(z2);
    }
    if (lane < 9 && Y >= 0 && Z >= 0 && Y < n1 && Z < n2) {
      // block-major node index, the (y,z) part once: ((blk_off + (bz nb1 + by) nb0 + bx) << 6) | local
      const uint32_t row = ((sc.blk_off + (uint32_t(Z >> 2) * nb1u + uint32_t(Y >> 2)) * nb0u) << 6) |
                           (uint32_t(Z & 3) << 4) | (uint32_t(Y & 3) << 2);
      auto node = [row](int xa) { return row + ((uint32_t(xa >> 2) << 6) | uint32_t(xa & 3)); };
      if (m0 != T(0) && X >= 0 && X < n0) atomic_add4(w.acc + node(X), m0, x0, y0, z0);
      if (m1 != T(0) && X + 1 >= 0 && X + 1 < n0) atomic_add4(w.acc + node(X + 1), m1, x1, y1, z1);
      if (m2 != T(0) && X + 2 >= 0 && X + 2 < n0) atomic_add4(w.acc + node(X + 2), m2, x2, y2, z2);
    }
  }
  // grid blocks of this warp's stencil bounding box
  int B[3], NB[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int l = __reduce_min_sync(0xffffffffu, has ? lo[a] : INT_MAX);
    const int h = __reduce_max_sync(0xffffffffu, has ? hi[a] : INT_MIN);
    B[a] = l >> 2;
    NB[a] = l == INT_MAX ? 0 : (h >> 2) - (l >> 2) + 1;
  }
  const int nblk = NB[0] * NB[1] * NB[2];
  if (NB[0] <= 4 && NB[1] <= 4 && NB[2] <= 2) {
    const int bx = lane & 3, by = (lane >> 2) & 3, bz = lane >> 4;
    if (bx < NB[0] && by < NB[1] && bz < NB[2])
      mark_block(w, sc.blk_off + (uint32_t(B[2] + bz) * sc.nb[1] + (B[1] + by)) * sc.nb[0] + (B[0] + bx));
  } else {
    for (int t = lane; t < nblk; t += 32) {
      const int bx = B[0] + t % NB[0], by = B[1] + (t / NB[0]) % NB[1], bz = B[2] + t / (NB[0] * NB[1]);
      mark_block(w, sc.blk_off + (uint32_t(bz) * sc.nb[1] + by) * sc.nb[0] + bx);
    }
  }
}

// Column-lane P2G of the velocity-only mode (mpm_substep_velocity_only, mpm_solver.rs:1377-1449):
// per node w m and w m v, w = wx (wy wz), skipping a (y,z) column whose wy or wz is below 1e-10
// and a node whose w is, and nodes past the grid's upper faces.  The structure is
// p2g_lanes_kernel's: the warp groups its particles by cell, stages per particle the nine
// w_y w_z column products, the x weights with the mass and the velocity, and lanes 0..26
// (3 particle groups x 9 columns) sum the three x nodes of their column over each cell's run,
// one vector reduction per node and run.
template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) p2g_lanes_velonly_kernel(WorldDev<T> w) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nt = blockDim.x;
  V4* wxm = reinterpret_cast<V4*>(smem);          // wxm[q] = (wx0, wx1, wx2, m)
  V4* vel = wxm + nt;                             // vel[q] = (vx, vy, vz, -)
  int4* gk = reinterpret_cast<int4*>(vel + nt);   // gk[q] = (stencil base, cell key)
  T* cw = reinterpret_cast<T*>(gk + nt);          // cw[q * 9 + column] = w_y w_z, 0 when skipped
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  const int n0 = sc.n[0], n1 = sc.n[1], n2 = sc.n[2];
  const int j = ch.y + tid;
  const bool live = j < ch.z;
  bool has = false;
  P2GPart<T> p;
  p.g[0] = p.g[1] = p.g[2] = 0;
  if (live) {
    const uint32_t src = w.perm ? w.perm[j] : uint32_t(j);
    p2g_setup<T, AE_MPM_MODE_VELOCITY_ONLY>(w, sc, src, p);
    has = p.g[0] < n0 && p.g[1] < n1 && p.g[2] < n2;  // some stencil node inside the grid (g >= 0)
  }
  const uint32_t key = has ? uint32_t(p.g[0]) + uint32_t(n0) * (uint32_t(p.g[1]) + uint32_t(n1) * uint32_t(p.g[2]))
                           : 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(peers) - 1;
  const uint32_t lead_cnt = lane == leader ? uint32_t(__popc(peers)) : 0u;
  uint32_t incl = lead_cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t lead_off = incl - lead_cnt;
  const int pos = int(__shfl_sync(0xffffffffu, lead_off, leader)) + __popc(peers & ((1u << lane) - 1u));
  uint32_t starts = __reduce_or_sync(0xffffffffu, lane == leader ? (1u << lead_off) : 0u);
  const int q = warp * 32 + pos;
  if (has) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        cw[q * 9 + b + 3 * c] = (p.w[2][c] < T(1e-10) || p.w[1][b] < T(1e-10)) ? T(0) : p.w[1][b] * p.w[2][c];
    wxm[q] = mk4(p.w[0][0], p.w[0][1], p.w[0][2], p.m);
    vel[q] = mk4(p.v[0], p.v[1], p.v[2], T(0));
  }
  gk[q] = make_int4(p.g[0], p.g[1], p.g[2], int(key));
  __syncwarp();
  const int grp = lane < 27 ? lane / 9 : 2;
  const int jc = lane < 27 ? lane - 9 * grp : lane - 23;
  const int nb = jc % 3, nc = jc / 3;
  const T* cww = cw + warp * 32 * 9 + jc;
  const V4* wxw = wxm + warp * 32;
  const V4* vw = vel + warp * 32;
  while (starts) {
    const int s0 = __ffs(starts) - 1;
    starts &= starts - 1u;
    const int e0 = starts ? __ffs(starts) - 1 : 32;
    const int4 run = gk[warp * 32 + s0];
    if (uint32_t(run.w) == 0xffffffffu) continue;
    const int X = run.x, Y = run.y + nb, Z = run.z + nc;
    T m0 = 0, x0 = 0, y0 = 0, z0 = 0, m1 = 0, x1 = 0, y1 = 0, z1 = 0, m2 = 0, x2 = 0, y2 = 0, z2 = 0;
    for (int i = s0 + grp; i < e0; i += 3) {
      const T wyz = cww[i * 9];
      const V4 r = wxw[i];
      const V4 v = vw[i];
      T W0 = r.x * wyz, W1 = r.y * wyz, W2 = r.z * wyz;
      W0 = W0 < T(1e-10) ? T(0) : W0;
      W1 = W1 < T(1e-10) ? T(0) : W1;
      W2 = W2 < T(1e-10) ? T(0) : W2;
      const T a0 = W0 * r.w, a1 = W1 * r.w, a2 = W2 * r.w;  // w m, as the reference forms it
      m0 += a0;
      x0 += a0 * v.x;
      y0 += a0 * v.y;
      z0 += a0 * v.z;
      m1 += a1;
      x1 += a1 * v.x;
      y1 += a1 * v.y;
      z1 += a1 * v.z;
      m2 += a2;
      x2 += a2 * v.x;
      y2 += a2 * v.y;
      z2 += a2 * v.z;
    }
    if (e0 - s0 > 1) {
      auto groups = [](T v) { return v + __shfl_down_sync(0xffffffffu, v, 9) + __shfl_down_sync(0xffffffffu, v, 18); };
      m0 = groups(m0), x0 = groups(x0), y0 = groups(y0), z0 = groups(z0);
      m1 = groups(m1), x1 = groups(x1), y1 = groups(y1), z1 = groups(z1);
      m2 = groups(m2), x2 = groups(x2), y2 = groups(y2), z2 = groups(z2);
    }
    if (lane < 9 && Y < n1 && Z < n2) {
      const uint32_t row = ((sc.blk_off + (uint32_t(Z >> 2) * uint32_t(sc.nb[1]) + uint32_t(Y >> 2)) * uint32_t(sc.nb[0])) << 6) |
                           (uint32_t(Z & 3) << 4) | (uint32_t(Y & 3) << 2);
      auto node = [row](int xa) { return row + ((uint32_t(xa >> 2) << 6) | uint32_t(xa & 3)); };
      if (m0 != T(0) && X < n0) atomic_add4(w.acc + node(X), m0, x0, y0, z0);
      if (m1 != T(0) && X + 1 < n0) atomic_add4(w.acc + node(X + 1), m1, x1, y1, z1);
      if (m2 != T(0) && X + 2 < n0) atomic_add4(w.acc + node(X + 2), m2, x2, y2, z2);
    }
  }
  // grid blocks of this warp's stencil bounding box (inside the grid)
  int B[3], NB[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int l = __reduce_min_sync(0xffffffffu, has ? p.g[a] : INT_MAX);
    const int h = __reduce_max_sync(0xffffffffu, has ? min(p.g[a] + 2, sc.n[a] - 1) : INT_MIN);
    B[a] = l >> 2;
    NB[a] = l == INT_MAX ? 0 : (h >> 2) - (l >> 2) + 1;
  }
  const int nblk = NB[0] * NB[1] * NB[2];
  for (int t = lane; t < nblk; t += 32) {
    const int bx = B[0] + t % NB[0], by = B[1] + (t / NB[0]) % NB[1], bz = B[2] + t / (NB[0] * NB[1]);
    mark_block(w, sc.blk_off + (uint32_t(bz) * uint32_t(sc.nb[1]) + uint32_t(by)) * uint32_t(sc.nb[0]) + uint32_t(bx));
  }
}
// Column-lane P2G of the reference mode (mpm_substep_serial_active / parallel_with_indices P2G,
// mpm_solver.rs:831-903, 1108-1193).  Per node (a,b,c) of a particle: w = (wx wy) wz, skipped below
// 1e-10 (mass, momentum and force alike); momentum w m (v + C d) with d the node minus the particle;
// the force sv . (N'(a), N'(b), N'(c)) / dx, not weighted by w, folded into momentum as dt sv (the
// grid update's v = p/m + g dt then equals the reference's p/m + (g + f/m) dt up to rounding).
// The particle's owner thread stages per (y,z) column u = v + C[.][1] d_y + C[.][2] d_z with wy,
// and f = sv[.][1] N'_y + sv[.][2] N'_z with wz; lanes 0..26 (3 particle groups x 9 columns) add
// the x part of each of their column's three nodes and sum over each cell's run, one vector
// reduction per node and run.
constexpr int kRefLaneVecs = 2 * 9 + 5;  // shared vectors per particle
template <class T>
__global__ void __launch_bounds__(256, 1) p2g_lanes_ref_kernel(WorldDev<T> w) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nt = blockDim.x;
  V4* cu = reinterpret_cast<V4*>(smem);  // cu[q * 9 + j] = (u, wy)
  V4* cf = cu + 9 * nt;                  // cf[q * 9 + j] = (f, wz)
  V4* pw = cf + 9 * nt;                  // pw[q] = (wx0, wx1, wx2, m)
  V4* pc = pw + nt;                      // pc[q] = C[.][0]
  V4* po = pc + nt;                      // po[q] = (d_x of the three x nodes)
  V4* ps = po + nt;                      // ps[q] = dt sv[.][0]
  V4* pe = ps + nt;                      // pe[q] = (N'_x of the three x nodes) / dx
  int4* gk = reinterpret_cast<int4*>(pe + nt);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  const int n0 = sc.n[0], n1 = sc.n[1], n2 = sc.n[2];
  const int j = ch.y + tid;
  const bool live = j < ch.z;
  bool has = false;
  P2GPart<T> p;
  p.g[0] = p.g[1] = p.g[2] = 0;
  if (live) {
    const uint32_t src = w.perm ? w.perm[j] : uint32_t(j);
    p2g_setup<T, AE_MPM_MODE_REFERENCE>(w, sc, src, p);
    has = p.g[0] < n0 && p.g[1] < n1 && p.g[2] < n2;  // some stencil node inside the grid (g >= 0)
  }
  const uint32_t key = has ? uint32_t(p.g[0]) + uint32_t(n0) * (uint32_t(p.g[1]) + uint32_t(n1) * uint32_t(p.g[2]))
                           : 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(peers) - 1;
  const uint32_t lead_cnt = lane == leader ? uint32_t(__popc(peers)) : 0u;
  uint32_t incl = lead_cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t lead_off = incl - lead_cnt;
  const int pos = int(__shfl_sync(0xffffffffu, lead_off, leader)) + __popc(peers & ((1u << lane) - 1u));
  uint32_t starts = __reduce_or_sync(0xffffffffu, lane == leader ? (1u << lead_off) : 0u);
  const int q = warp * 32 + pos;
  if (has) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const T dy = p.o[1][b], dz = p.o[2][c], ey = p.dw[1][b], ez = p.dw[2][c];
        const T ux = p.v[0] + p.A[1] * dy + p.A[2] * dz;
        const T uy = p.v[1] + p.A[4] * dy + p.A[5] * dz;
        const T uz = p.v[2] + p.A[7] * dy + p.A[8] * dz;
        cu[q * 9 + b + 3 * c] = mk4(ux, uy, uz, p.w[1][b]);
        cf[q * 9 + b + 3 * c] =
            mk4(p.sv[1] * ey + p.sv[2] * ez, p.sv[4] * ey + p.sv[5] * ez, p.sv[7] * ey + p.sv[8] * ez, p.w[2][c]);
      }
    pw[q] = mk4(p.w[0][0], p.w[0][1], p.w[0][2], p.m);
    pc[q] = mk4(p.A[0], p.A[3], p.A[6], T(0));
    po[q] = mk4(p.o[0][0], p.o[0][1], p.o[0][2], T(0));
    ps[q] = mk4(p.sv[0], p.sv[3], p.sv[6], T(0));
    pe[q] = mk4(p.dw[0][0], p.dw[0][1], p.dw[0][2], T(0));
  }
  gk[q] = make_int4(p.g[0], p.g[1], p.g[2], int(key));
  __syncwarp();
  const int grp = lane < 27 ? lane / 9 : 2;
  const int jc = lane < 27 ? lane - 9 * grp : lane - 23;
  const int nb = jc % 3, nc = jc / 3;
  const int wb = warp * 32;
  while (starts) {
    const int s0 = __ffs(starts) - 1;
    starts &= starts - 1u;
    const int e0 = starts ? __ffs(starts) - 1 : 32;
    const int4 run = gk[wb + s0];
    if (uint32_t(run.w) == 0xffffffffu) continue;
    const int X = run.x, Y = run.y + nb, Z = run.z + nc;
    T acc[3][4];
#pragma unroll
    for (int a = 0; a < 3; ++a) acc[a][0] = acc[a][1] = acc[a][2] = acc[a][3] = T(0);
    for (int i = s0 + grp; i < e0; i += 3) {
      const V4 u = cu[(wb + i) * 9 + jc], f = cf[(wb + i) * 9 + jc];
      const V4 r = pw[wb + i], cx = pc[wb + i], dx = po[wb + i], sx = ps[wb + i], ex = pe[wb + i];
      const T wxs[3] = {r.x, r.y, r.z}, dxs[3] = {dx.x, dx.y, dx.z}, exs[3] = {ex.x, ex.y, ex.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const T wn = (wxs[a] * u.w) * f.w;  // (wx wy) wz, as the reference multiplies
        if (wn < T(1e-10)) continue;
        const T wm = wn * r.w;
        acc[a][0] += wm;
        acc[a][1] += wm * (u.x + cx.x * dxs[a]) + (f.x + sx.x * exs[a]);
        acc[a][2] += wm * (u.y + cx.y * dxs[a]) + (f.y + sx.y * exs[a]);
        acc[a][3] += wm * (u.z + cx.z * dxs[a]) + (f.z + sx.z * exs[a]);
      }
    }
    if (e0 - s0 > 1) {
      auto groups = [](T v) { return v + __shfl_down_sync(0xffffffffu, v, 9) + __shfl_down_sync(0xffffffffu, v, 18); };
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[a][k] = groups(acc[a][k]);
    }
    if (lane < 9 && Y < n1 && Z < n2) {
      const uint32_t row = ((sc.blk_off + (uint32_t(Z >> 2) * uint32_t(sc.nb[1]) + uint32_t(Y >> 2)) * uint32_t(sc.nb[0])) << 6) |
                           (uint32_t(Z & 3) << 4) | (uint32_t(Y & 3) << 2);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int xa = X + a;
        // a node every particle skipped has mass 0; one with a (skipped-weight) force only does not
        // exist: the force is added exactly where the mass is
        if (acc[a][0] != T(0) && xa < n0)
          atomic_add4(w.acc + (row + ((uint32_t(xa >> 2) << 6) | uint32_t(xa & 3))), acc[a][0], acc[a][1], acc[a][2],
                      acc[a][3]);
      }
    }
  }
  int B[3], NB[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int l = __reduce_min_sync(0xffffffffu, has ? p.g[a] : INT_MAX);
    const int h = __reduce_max_sync(0xffffffffu, has ? min(p.g[a] + 2, sc.n[a] - 1) : INT_MIN);
    B[a] = l >> 2;
    NB[a] = l == INT_MAX ? 0 : (h >> 2) - (l >> 2) + 1;
  }
  const int nblk = NB[0] * NB[1] * NB[2];
  for (int t = lane; t < nblk; t += 32) {
    const int bx = B[0] + t % NB[0], by = B[1] + (t / NB[0]) % NB[1], bz = B[2] + t / (NB[0] * NB[1]);
    mark_block(w, sc.blk_off + (uint32_t(bz) * uint32_t(sc.nb[1]) + uint32_t(by)) * uint32_t(sc.nb[0]) + uint32_t(bx));
  }
}

// shared bytes per particle of p2g_lanes_velonly_kernel
template <class T>
constexpr size_t velonly_lane_bytes() {
  return 2 * sizeof(typename V4T<T>::type) + sizeof(int4) + 9 * sizeof(T);
}

// ============================================================================================
// grid update (momentum -> velocity, gravity, walls); clears accumulator and touched flags
// ============================================================================================
template <class T, int MODE>
__device__ __forceinline__ void grid_velocity(const SceneDev<T>& sc, int i, int j, int k, T m, T px, T py, T pz,
                                              T& vx, T& vy, T& vz) {
  vx = vy = vz = T(0);
  if (MODE == AE_MPM_MODE_PHYSICS) {
    if (!(m > T(0))) return;
    vx = px / m + sc.dt * sc.grav[0];
    vy = py / m + sc.dt * sc.grav[1];
    vz = pz / m + sc.dt * sc.grav[2];
    const int mg = sc.wall_margin;
    const int id[3] = {i, j, k};
    if (sc.wall_mode == AE_MPM_WALL_STICKY) {
      bool wall = false;
#pragma unroll
      for (int a = 0; a < 3; ++a) wall = wall || id[a] < mg || id[a] >= sc.n[a] - mg;
      if (wall) vx = vy = vz = T(0);
    } else {
      T v[3] = {vx, vy, vz};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (id[a] < mg && v[a] < T(0)) v[a] = -v[a] * sc.restitution;
        if (id[a] >= sc.n[a] - mg && v[a] > T(0)) v[a] = -v[a] * sc.restitution;
      }
      vx = v[0];
      vy = v[1];
      vz = v[2];
    }
  } else {  // Grid::update_parallel (mpm_solver.rs:112-139), force folded into momentum
    if (!(m > T(1e-12))) return;
    vx = px / m + sc.grav[0] * sc.dt;
    vy = py / m + sc.grav[1] * sc.dt;
    vz = pz / m + sc.grav[2] * sc.dt;
    if (j == 0) {
      vy = t_max(vy, T(0));
      vx *= T(0.9);
      vz *= T(0.9);
    }
  }
}

template <class T>
__device__ __forceinline__ void block_coords(const SceneDev<T>& sc, uint32_t gb, int l, int& i, int& j, int& k) {
  uint32_t lb = gb - sc.blk_off;
  int bx = int(lb % uint32_t(sc.nb[0]));
  int by = int((lb / uint32_t(sc.nb[0])) % uint32_t(sc.nb[1]));
  int bz = int(lb / (uint32_t(sc.nb[0]) * uint32_t(sc.nb[1])));
  i = bx * 4 + (l & 3);
  j = by * 4 + ((l >> 2) & 3);
  k = bz * 4 + (l >> 4);
}

template <class T, int MODE>
__global__ void __launch_bounds__(256) grid_update_kernel(WorldDev<T> w, uint32_t* blk_epoch, const uint32_t* epoch,
                                                          uint32_t* zero_count) {
  using V4 = typename V4T<T>::type;
  const uint32_t count = launch_count(w.touched_count);
  const uint32_t ep = *epoch;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *w.clamp_count = 0u;  // G2P of this substep refills it
    // the fused G2P + P2G appends the next substep's blocks to the other list, whose previous
    // contents the grid update of the substep before consumed
    if (zero_count) *zero_count = 0u;
  }
  // each 64-thread group takes 4 touched blocks per iteration and issues their 4 accumulator loads
  // before using any, so a long touched list is not one latency-bound load after another
  constexpr int kU = 4;
  const int sub = threadIdx.x >> 6, l = threadIdx.x & 63;
  for (uint32_t t0 = (blockIdx.x * 4 + sub) * kU; t0 < count; t0 += gridDim.x * 4 * kU) {
    uint32_t gb[kU];
    V4 a[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) gb[u] = (t0 + u < count) ? w.touched[t0 + u] : 0xffffffffu;
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (gb[u] != 0xffffffffu) a[u] = w.acc[uint64_t(gb[u]) * 64u + l];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      if (gb[u] == 0xffffffffu) continue;
      const SceneDev<T>& sc = w.scenes[w.one_scene ? 0u : w.blk_scene[gb[u]]];  // one scene: no lookup
      int i, j, k;
      block_coords(sc, gb[u], l, i, j, k);
      const uint64_t gi = uint64_t(gb[u]) * 64u + l;
      w.acc[gi] = mk4(T(0), T(0), T(0), T(0));
      T vx, vy, vz;
      grid_velocity<T, MODE>(sc, i, j, k, a[u].x, a[u].y, a[u].z, a[u].w, vx, vy, vz);
      w.vel[gi] = mk4(vx, vy, vz, a[u].x);
      if (l == 0) {
        w.blk_flag[gb[u]] = 0u;
        blk_epoch[gb[u]] = ep;
      }
    }
  }
}

// ============================================================================================
// G2P
// ============================================================================================
template <class T>
struct G2POut {
  T x[3], v[3], C[9], F[9], J;
  uint32_t err;       // kErr* bits
  bool needs_clamp;   // snow: F left the elastic region; the clamp kernel finishes the update
  bool clamped;
};

// Node velocities for one block of particles: the block's bounding-box tile in shared memory
// (filled with coalesced loads before the gather), or the global array when the box is too big.
// The tile's x and y pitches are powers of two (2^p0 >= D0, 2^(sp-p0) >= D1), so slot indexes
// split into coordinates with shifts and masks.
template <class T>
struct VelTile {
  using V4 = typename V4T<T>::type;
  const V4* tile;
  const V4* vel;
  int L0, L1, L2, p0, sp;
  __device__ __forceinline__ V4 operator()(const SceneDev<T>& sc, int X, int Y, int Z) const {
    if (tile) return tile[((Z - L2) << sp) + ((Y - L1) << p0) + (X - L0)];
    return ld4(vel + node_index(sc, X, Y, Z));
  }
};

// Node velocities of the block-major grid by (y,z) row, through the read-only cache: row(Y, Z)
// once per stencil column, then at(row, X) for its three x nodes.  The block needs no bounding
// box, tile or barrier, so its warps never wait for one another.
template <class T>
struct GridRows {
  using V4 = typename V4T<T>::type;
  const V4* __restrict__ vel;
  uint32_t blk_off, nb0, nb1;
  __device__ __forceinline__ uint32_t row(int Y, int Z) const {
    return ((blk_off + (uint32_t(Z >> 2) * nb1 + uint32_t(Y >> 2)) * nb0) << 6) | (uint32_t(Z & 3) << 4) |
           (uint32_t(Y & 3) << 2);
  }
  __device__ __forceinline__ V4 at(uint32_t r, int X) const {
    return ld4(vel + (r + ((uint32_t(X >> 2) << 6) | uint32_t(X & 3))));
  }
  // row(Y, Z) == zpart(Z) + ypart(Y), and the node index of (X, Y, Z) == row + xpart(X)
  __device__ __forceinline__ uint32_t xpart(int X) const { return (uint32_t(X >> 2) << 6) | uint32_t(X & 3); }
  __device__ __forceinline__ uint32_t ypart(int Y) const {
    return ((uint32_t(Y >> 2) * nb0) << 6) | (uint32_t(Y & 3) << 2);
  }
  __device__ __forceinline__ uint32_t zpart(int Z) const {
    return ((blk_off + uint32_t(Z >> 2) * nb1 * nb0) << 6) | (uint32_t(Z & 3) << 4);
  }
  __device__ __forceinline__ V4 at_part(uint32_t r, uint32_t xp) const { return ld4(vel + (r + xp)); }
};
// Physics gather for a particle whose 27 stencil nodes are all inside the grid (every particle
// after its first substep: positions are clamped to [1, n-2] dx).  Separable: each (y,z) column
// is summed over x first,
//   S0 = sum_a wx[a] g(a,b,c),   S1 = sum_a wx[a] (a - fx) dx g(a,b,c),
// then v += wy wz S0, B[.][0] += wy wz S1, B[.][1] += wy (b - fy) dx wz S0,
// B[.][2] += wy wz (c - fz) dx S0: 36 instructions per column instead of 42 per node.
// Returns false (nothing written) when the particle does not qualify.
template <class T, class Rows>
__device__ __forceinline__ bool g2p_physics_gather_sep(const Rows& rows, const SceneDev<T>& sc, const T* x0, T* v,
                                                       T* C) {
  using V4 = typename V4T<T>::type;
  int b[3];
  T w[3][3], e[3][3];
  bool inside = true;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const T X = (x0[a] - sc.origin[a]) * sc.inv_dx;
    const int bb = floor_to_int(X - T(0.5));
    const T fx = X - T(bb);
    b[a] = bb;
    inside = inside && bb >= 0 && bb + 2 < sc.n[a];
    const T t0 = T(1.5) - fx, t1 = fx - T(1), t2 = fx - T(0.5);
    w[a][0] = T(0.5) * t0 * t0;
    w[a][1] = T(0.75) - t1 * t1;
    w[a][2] = T(0.5) * t2 * t2;
#pragma unroll
    for (int k = 0; k < 3; ++k) e[a][k] = w[a][k] * ((T(k) - fx) * sc.dx);
  }
  if (!inside) return false;
  T vv[3] = {0, 0, 0}, B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) {
      const uint32_t r = rows.row(b[1] + bb, b[2] + c);
      const V4 g0 = rows.at(r, b[0]), g1 = rows.at(r, b[0] + 1), g2 = rows.at(r, b[0] + 2);
      const T s0[3] = {w[0][0] * g0.x + w[0][1] * g1.x + w[0][2] * g2.x, w[0][0] * g0.y + w[0][1] * g1.y + w[0][2] * g2.y,
                       w[0][0] * g0.z + w[0][1] * g1.z + w[0][2] * g2.z};
      const T s1[3] = {e[0][0] * g0.x + e[0][1] * g1.x + e[0][2] * g2.x, e[0][0] * g0.y + e[0][1] * g1.y + e[0][2] * g2.y,
                       e[0][0] * g0.z + e[0][1] * g1.z + e[0][2] * g2.z};
      const T wbc = w[1][bb] * w[2][c], ebc = e[1][bb] * w[2][c], fbc = w[1][bb] * e[2][c];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        vv[k] += wbc * s0[k];
        B[k * 3 + 0] += wbc * s1[k];
        B[k * 3 + 1] += ebc * s0[k];
        B[k * 3 + 2] += fbc * s0[k];
      }
    }
  }
  const T cs = T(4) * sc.inv_dx * sc.inv_dx;
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = vv[k];
#pragma unroll
  for (int k = 0; k < 9; ++k) C[k] = cs * B[k];
  return true;
}

// The same separable gather in f32 with Blackwell's packed FMA (two lanes of a float2 per
// instruction): the x and y components of each column sum and accumulator travel as one pair, z
// alone.  Every pair op rounds like the scalar fused multiply-adds it replaces.
template <class Rows>
__device__ __forceinline__ bool g2p_physics_gather_sep_f2(const Rows& rows, const SceneDev<float>& sc, const float* x0,
                                                          float* v, float* C) {
  int b[3];
  float w[3][3], e[3][3];
  bool inside = true;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float X = (x0[a] - sc.origin[a]) * sc.inv_dx;
    const int bb = floor_to_int(X - 0.5f);
    const float fx = X - float(bb);
    b[a] = bb;
    inside = inside && bb >= 0 && bb + 2 < sc.n[a];
    const float t0 = 1.5f - fx, t1 = fx - 1.0f, t2 = fx - 0.5f;
    w[a][0] = 0.5f * t0 * t0;
    w[a][1] = 0.75f - t1 * t1;
    w[a][2] = 0.5f * t2 * t2;
#pragma unroll
    for (int k = 0; k < 3; ++k) e[a][k] = w[a][k] * ((float(k) - fx) * sc.dx);
  }
  if (!inside) return false;
  // only the x weights are kept as broadcast pairs; the y/z weight products are formed per
  // column and paired there (pairs of all six weight sets took 36 registers and spilled)
  float2 wx[3], ex[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    wx[k] = make_float2(w[0][k], w[0][k]);
    ex[k] = make_float2(e[0][k], e[0][k]);
  }
  float2 vxy = make_float2(0.f, 0.f), b0xy = vxy, b1xy = vxy, b2xy = vxy;
  float vz = 0.f, b0z = 0.f, b1z = 0.f, b2z = 0.f;
  // node index = z part + y part + x part: the three bit fields of the block-major index are
  // disjoint, so the 27 indexes come from 3 + 3 + 3 parts with one add each
  uint32_t xp[3], yp[3], zp[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    xp[k] = rows.xpart(b[0] + k);
    yp[k] = rows.ypart(b[1] + k);
    zp[k] = rows.zpart(b[2] + k);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) {
      const uint32_t r = zp[c] + yp[bb];
      const float4 g0 = rows.at_part(r, xp[0]), g1 = rows.at_part(r, xp[1]), g2 = rows.at_part(r, xp[2]);
      const float2 g0xy = make_float2(g0.x, g0.y), g1xy = make_float2(g1.x, g1.y), g2xy = make_float2(g2.x, g2.y);
      const float2 s0xy = __ffma2_rn(wx[2], g2xy, __ffma2_rn(wx[1], g1xy, __fmul2_rn(wx[0], g0xy)));
      const float2 s1xy = __ffma2_rn(ex[2], g2xy, __ffma2_rn(ex[1], g1xy, __fmul2_rn(ex[0], g0xy)));
      const float s0z = w[0][0] * g0.z + w[0][1] * g1.z + w[0][2] * g2.z;
      const float s1z = e[0][0] * g0.z + e[0][1] * g1.z + e[0][2] * g2.z;
      const float wbs = w[1][bb] * w[2][c], ebs = e[1][bb] * w[2][c], fbs = w[1][bb] * e[2][c];
      const float2 wbc = make_float2(wbs, wbs), ebc = make_float2(ebs, ebs), fbc = make_float2(fbs, fbs);
      vxy = __ffma2_rn(wbc, s0xy, vxy);
      b0xy = __ffma2_rn(wbc, s1xy, b0xy);
      b1xy = __ffma2_rn(ebc, s0xy, b1xy);
      b2xy = __ffma2_rn(fbc, s0xy, b2xy);
      vz += wbc.x * s0z;
      b0z += wbc.x * s1z;
      b1z += ebc.x * s0z;
      b2z += fbc.x * s0z;
    }
  }
  const float cs = 4.0f * sc.inv_dx * sc.inv_dx;
  v[0] = vxy.x;
  v[1] = vxy.y;
  v[2] = vz;
  // B[k][col]: column col of the affine sum for velocity component k
  C[0] = cs * b0xy.x;
  C[1] = cs * b1xy.x;
  C[2] = cs * b2xy.x;
  C[3] = cs * b0xy.y;
  C[4] = cs * b1xy.y;
  C[5] = cs * b2xy.y;
  C[6] = cs * b0z;
  C[7] = cs * b1z;
  C[8] = cs * b2z;
  return true;
}

// gather half of the physics G2P: grid velocity and APIC C at the particle
template <class T>
__device__ __forceinline__ void g2p_physics_gather(const VelTile<T>& vt, const SceneDev<T>& sc, const T* x0, T* v,
                                                   T* C) {
  using V4 = typename V4T<T>::type;
  int b[3];
  T wt[3][3], dp[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T X = (x0[a] - sc.origin[a]) * sc.inv_dx;
    int bb = floor_to_int(X - T(0.5));
    T fx = X - T(bb);
    b[a] = bb;
    T t0 = T(1.5) - fx, t1 = fx - T(1), t2 = fx - T(0.5);
    wt[a][0] = T(0.5) * t0 * t0;
    wt[a][1] = T(0.75) - t1 * t1;
    wt[a][2] = T(0.5) * t2 * t2;
#pragma unroll
    for (int k = 0; k < 3; ++k) dp[a][k] = (T(k) - fx) * sc.dx;
  }
  T B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  v[0] = v[1] = v[2] = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int bb = 0; bb < 3; ++bb)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        int X = b[0] + a, Y = b[1] + bb, Z = b[2] + c;
        if (X < 0 || Y < 0 || Z < 0 || X >= sc.n[0] || Y >= sc.n[1] || Z >= sc.n[2]) continue;
        T ww = wt[0][a] * wt[1][bb] * wt[2][c];
        V4 gv = vt(sc, X, Y, Z);
        T g3[3] = {gv.x, gv.y, gv.z};
        T d[3] = {dp[0][a], dp[1][bb], dp[2][c]};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          v[r] += ww * g3[r];
#pragma unroll
          for (int k = 0; k < 3; ++k) B[r * 3 + k] += ww * g3[r] * d[k];
        }
      }
  const T cs = T(4) * sc.inv_dx * sc.inv_dx;
#pragma unroll
  for (int k = 0; k < 9; ++k) C[k] = cs * B[k];
}

// update half of the physics G2P: advection, F update and the material's return mapping
template <class T>
__device__ __forceinline__ void g2p_physics_update(const SceneDev<T>& sc, const MatDev& md, const T* x0, const T* v,
                                                   const T* F, T J, T m, G2POut<T>& o) {
  bool nan = false, clamped = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T nx = x0[a] + sc.dt * v[a];
    if (!t_finite(nx)) nan = true;
    T lo = sc.origin[a] + sc.dx, hi = sc.origin[a] + T(sc.n[a] - 2) * sc.dx;
    T cx = t_fclamp(nx, lo, hi);
    if (cx != nx) clamped = true;
    o.x[a] = cx;
    o.v[a] = v[a];
  }
  o.err = (nan ? kErrNaN : 0u) | (clamped ? kErrDomain : 0u);
  o.clamped = clamped;
  o.needs_clamp = false;
  if (md.model == kPhysFluid) {
    T Jn = J * (T(1) + sc.dt * (o.C[0] + o.C[4] + o.C[8]));
    o.J = t_max(Jn, T(0.01));
#pragma unroll
    for (int k = 0; k < 9; ++k) o.F[k] = F[k];
    T A[9];
    affine_from_c(sc, md, m, o.C, o.F, o.J, A);
#pragma unroll
    for (int k = 0; k < 9; ++k) o.C[k] = A[k];
    return;
  }
  T G[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) G[k] = ((k % 4 == 0) ? T(1) : T(0)) + sc.dt * o.C[k];
  mm3(G, F, o.F);
  if (md.model == kPhysSnow) {
    // elastic region (every singular value provably inside the clamp interval): F_E and J_p
    // are final; otherwise the clamp kernel does the SVD, the return mapping and A
    o.J = J;
    o.needs_clamp = !clamp_is_identity(o.F, T(1) - T(md.theta_c), T(1) + T(md.theta_s));
  } else {
    o.J = det3(o.F);
  }
  if (!o.needs_clamp) {  // the C slot carries A from here on
    T A[9];
    affine_from_c(sc, md, m, o.C, o.F, o.J, A);
#pragma unroll
    for (int k = 0; k < 9; ++k) o.C[k] = A[k];
  }
}

// mpm_substep_serial_active / parallel_with_indices G2P (mpm_solver.rs:914-1053, 1206-1325)
template <class T>
__device__ __forceinline__ void g2p_reference(const VelTile<T>& vt, const SceneDev<T>& sc, const T* pos, const T* f,
                                              G2POut<T>& o) {
  using V4 = typename V4T<T>::type;
  int g[3];
  T fx[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T q = (pos[a] - sc.origin[a]) * sc.inv_dx - T(0.5);
    int gu = floor_to_int(q);
    fx[a] = q - T(gu);
    g[a] = max(gu, 0);
  }
  T nv[3] = {0, 0, 0}, nc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, gvm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
  for (int dk = 0; dk < 3; ++dk)
#pragma unroll 1
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
      for (int di = 0; di < 3; ++di) {
        T wx = b_spline(T(di) - fx[0]), wy = b_spline(T(dj) - fx[1]), wz = b_spline(T(dk) - fx[2]);
        T ww = wx * wy * wz;
        if (ww < T(1e-10)) continue;
        int X = g[0] + di, Y = g[1] + dj, Z = g[2] + dk;
        if (X >= sc.n[0] || Y >= sc.n[1] || Z >= sc.n[2]) continue;
        V4 gv = vt(sc, X, Y, Z);
        if (gv.w < T(1e-12)) continue;
        T g3[3] = {gv.x, gv.y, gv.z};
        nv[0] += ww * g3[0];
        nv[1] += ww * g3[1];
        nv[2] += ww * g3[2];
        T d3[3] = {(T(X) + T(0.5)) * sc.dx + sc.origin[0] - pos[0], (T(Y) + T(0.5)) * sc.dx + sc.origin[1] - pos[1],
                   (T(Z) + T(0.5)) * sc.dx + sc.origin[2] - pos[2]};
        T scale = T(4) * sc.inv_dx * sc.inv_dx * ww;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) nc[r * 3 + c] += scale * g3[r] * d3[c];
        T dw[3] = {b_spline_deriv(T(di) - fx[0]) * sc.inv_dx, b_spline_deriv(T(dj) - fx[1]) * sc.inv_dx,
                   b_spline_deriv(T(dk) - fx[2]) * sc.inv_dx};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) gvm[r * 3 + c] -= ww * g3[r] * dw[c];
      }
  if (!t_finite(nv[0]) || !t_finite(nv[1]) || !t_finite(nv[2])) {
    nv[0] = nv[1] = nv[2] = T(0);
#pragma unroll
    for (int k = 0; k < 9; ++k) nc[k] = T(0);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) nv[a] = t_clamp(nv[a], T(-50), T(50));
  T np[3] = {t_add_mul_rn(pos[0], nv[0], sc.dt), t_add_mul_rn(pos[1], nv[1], sc.dt), t_add_mul_rn(pos[2], nv[2], sc.dt)};
  if (!t_finite(np[0]) || !t_finite(np[1]) || !t_finite(np[2])) {
    np[0] = T(6);
    np[1] = T(5);
    np[2] = T(6);
    nv[0] = nv[1] = nv[2] = T(0);
  }
  if (np[1] < T(0)) {
    np[1] = T(0);
    nv[1] = t_max(nv[1], T(0)) * T(0.5);
  }
  const T gmx = T(sc.n[0] - 1) * sc.dx, gmz = T(sc.n[2] - 1) * sc.dx;
  const T lox = sc.wall_origin ? sc.origin[0] : T(0), loz = sc.wall_origin ? sc.origin[2] : T(0);
  if (np[0] < lox) {
    np[0] = lox;
    nv[0] = t_max(nv[0], T(0)) * T(0.5);
  } else if (np[0] > gmx + lox) {
    np[0] = gmx + lox;
    nv[0] = t_min(nv[0], T(0)) * T(0.5);
  }
  if (np[2] < loz) {
    np[2] = loz;
    nv[2] = t_max(nv[2], T(0)) * T(0.5);
  } else if (np[2] > gmz + loz) {
    np[2] = gmz + loz;
    nv[2] = t_min(nv[2], T(0)) * T(0.5);
  }
  T nf[9];
  bool valid = true;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T sum = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k) sum += (((r == k) ? T(1) : T(0)) + gvm[r * 3 + k] * sc.dt) * f[k * 3 + c];
      nf[r * 3 + c] = sum;
      if (!t_finite(sum) || t_abs(sum) > T(1e3)) valid = false;
    }
  if (valid) {
    o.J = t_clamp(det3(nf), T(0.1), T(10));
  } else {
    ident3(nf);
    o.J = T(1);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    o.v[a] = nv[a] * sc.damping;
    o.x[a] = np[a];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    o.C[k] = nc[k];
    o.F[k] = nf[k];
  }
  o.err = 0;
  o.needs_clamp = o.clamped = false;
}

// mpm_substep_velocity_only G2P (mpm_solver.rs:1465-1571); C, F and J are carried unchanged
template <class T>
__device__ __forceinline__ void g2p_velonly(const VelTile<T>& vt, const SceneDev<T>& sc, const T* pos, G2POut<T>& o) {
  using V4 = typename V4T<T>::type;
  int g[3];
  T wx[3], wy[3], wz[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T q = (pos[a] - sc.origin[a]) * sc.inv_dx - T(0.5);
    int gu = floor_to_int(q);
    T fx = q - T(gu);
    g[a] = max(gu, 0);
    T* wa = a == 0 ? wx : (a == 1 ? wy : wz);
#pragma unroll
    for (int k = 0; k < 3; ++k) wa[k] = b_spline(T(k) - fx);
  }
  T nv[3] = {0, 0, 0};
#pragma unroll
  for (int dk = 0; dk < 3; ++dk) {
    if (wz[dk] < T(1e-10)) continue;
    int Z = g[2] + dk;
    if (Z >= sc.n[2]) continue;
#pragma unroll
    for (int dj = 0; dj < 3; ++dj) {
      if (wy[dj] < T(1e-10)) continue;
      int Y = g[1] + dj;
      if (Y >= sc.n[1]) continue;
      T wyz = wy[dj] * wz[dk];
#pragma unroll
      for (int di = 0; di < 3; ++di) {
        T ww = wx[di] * wyz;
        if (ww < T(1e-10)) continue;
        int X = g[0] + di;
        if (X >= sc.n[0]) continue;
        V4 gv = vt(sc, X, Y, Z);
        if (gv.w < T(1e-12)) continue;
        nv[0] += ww * gv.x;
        nv[1] += ww * gv.y;
        nv[2] += ww * gv.z;
      }
    }
  }
  if (!t_finite(nv[0]) || !t_finite(nv[1]) || !t_finite(nv[2])) nv[0] = nv[1] = nv[2] = T(0);
#pragma unroll
  for (int a = 0; a < 3; ++a) nv[a] = t_clamp(nv[a], T(-50), T(50));
  T np[3] = {t_add_mul_rn(pos[0], nv[0], sc.dt), t_add_mul_rn(pos[1], nv[1], sc.dt), t_add_mul_rn(pos[2], nv[2], sc.dt)};
  if (!t_finite(np[0]) || !t_finite(np[1]) || !t_finite(np[2])) {
    np[0] = pos[0];
    np[1] = pos[1];
    np[2] = pos[2];
    nv[0] = nv[1] = nv[2] = T(0);
  }
  if (np[1] < T(0)) {
    np[1] = T(0);
    nv[1] = t_max(nv[1], T(0)) * T(0.5);
  }
  const T gmx = T(sc.n[0] - 1) * sc.dx, gmz = T(sc.n[2] - 1) * sc.dx;
  if (np[0] < T(0)) {
    np[0] = T(0);
    nv[0] = t_max(nv[0], T(0)) * T(0.5);
  } else if (np[0] > gmx + sc.origin[0]) {
    np[0] = gmx + sc.origin[0];
    nv[0] = t_min(nv[0], T(0)) * T(0.5);
  }
  if (np[2] < T(0)) {
    np[2] = T(0);
    nv[2] = t_max(nv[2], T(0)) * T(0.5);
  } else if (np[2] > gmz + sc.origin[2]) {
    np[2] = gmz + sc.origin[2];
    nv[2] = t_min(nv[2], T(0)) * T(0.5);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    o.v[a] = nv[a] * sc.damping;
    o.x[a] = np[a];
  }
  o.err = 0;
  o.needs_clamp = o.clamped = false;
}

// in-grid stencil node range of a position along one axis (empty when lo > hi)
template <class T, int MODE>
__device__ __forceinline__ void stencil_range(const SceneDev<T>& sc, T x, int a, int& lo, int& hi) {
  int g = floor_to_int((x - sc.origin[a]) * sc.inv_dx - T(0.5));
  if (MODE != AE_MPM_MODE_PHYSICS) g = max(g, 0);
  lo = max(g, 0);
  hi = min(g + 2, sc.n[a] - 1);
}

template <class T, int MODE>
__global__ void __launch_bounds__(256, (MODE == AE_MPM_MODE_PHYSICS && sizeof(T) == 4) ? 4 : 1) g2p_kernel(WorldDev<T> w, uint32_t* epoch,
                                                                                                    int write_keys) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  V4* tile = reinterpret_cast<V4*>(smem);
  // physics mode gathers straight from the grid (no block tile, no barriers)
  constexpr bool kTile = MODE != AE_MPM_MODE_PHYSICS;
  V4* stage = kTile ? tile + w.max_tile_nodes : tile;  // a1..a3 of this block's particles: stage[k * nt + tid]
  __shared__ int s_lo[3], s_hi[3];
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  const int tid = threadIdx.x, lane = tid & 31, nt = blockDim.x;
  const int j = ch.y + tid;
  const bool live = j < ch.z;
  if (blockIdx.x == 0 && tid == 0) {
    *w.touched_count = 0u;
    if (w.cell_count) *w.cell_count = 0u;
    *epoch += 1u;
  }
  if (kTile) {
    if (tid < 3) {
      s_lo[tid] = INT_MAX;
      s_hi[tid] = INT_MIN;
    }
    __syncthreads();
  }
  uint32_t src = 0;
  V4 a0 = mk4(T(0), T(0), T(0), T(0));
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  bool has = false;
  if (live) {
    src = w.perm ? w.perm[j] : uint32_t(j);
    // F, J and the material arrive in shared memory while the node velocities are gathered
#pragma unroll
    for (int k = 0; k < 3; ++k) cp_async_v4(stage + k * nt + tid, w.in[1 + k] + src);
    cp_async_commit();
    a0 = ld4(w.in[0] + src);
    const T x3[3] = {a0.x, a0.y, a0.z};
    has = true;
    if (kTile) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        stencil_range<T, MODE>(sc, x3[a], a, lo[a], hi[a]);
        if (lo[a] > hi[a]) has = false;
      }
    }
  }
  if (kTile) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int l = __reduce_min_sync(0xffffffffu, has ? lo[a] : INT_MAX);
      int h = __reduce_max_sync(0xffffffffu, has ? hi[a] : INT_MIN);
      if (lane == 0 && l != INT_MAX) {
        atomicMin(&s_lo[a], l);
        atomicMax(&s_hi[a], h);
      }
    }
    __syncthreads();
  }
  VelTile<T> vt;
  vt.tile = nullptr;
  vt.vel = w.vel;
  vt.L0 = kTile ? s_lo[0] : INT_MAX;
  vt.L1 = kTile ? s_lo[1] : INT_MAX;
  vt.L2 = kTile ? s_lo[2] : INT_MAX;
  if (kTile && vt.L0 != INT_MAX) {
    const int D0 = s_hi[0] - vt.L0 + 1, D1 = s_hi[1] - vt.L1 + 1, D2 = s_hi[2] - vt.L2 + 1;
    const int p0 = 32 - __clz(D0 - 1), p1 = 32 - __clz(D1 - 1);
    vt.p0 = p0;
    vt.sp = p0 + p1;
    const int slots = D2 << vt.sp;
    if (slots <= w.max_tile_nodes) {
      const int mx = (1 << p0) - 1, my = (1 << p1) - 1;
      for (int t = tid; t < slots; t += blockDim.x) {
        const int X = t & mx, Y = (t >> p0) & my;
        if (X < D0 && Y < D1) tile[t] = ld4(w.vel + node_index(sc, vt.L0 + X, vt.L1 + Y, vt.L2 + (t >> vt.sp)));
      }
      vt.tile = tile;
    }
  }
  if (kTile) __syncthreads();
  uint32_t err = 0;
  bool cl = false, need = false;
  if (live) {
    const T x0[3] = {a0.x, a0.y, a0.z};
    G2POut<T> o;
    T pv[3] = {0, 0, 0};
    if (MODE == AE_MPM_MODE_PHYSICS) {
      const bool done = g2p_physics_gather_sep<T>(
          GridRows<T>{w.vel, sc.blk_off, uint32_t(sc.nb[0]), uint32_t(sc.nb[1])}, sc, x0, pv, o.C);
      if (!done) g2p_physics_gather<T>(vt, sc, x0, pv, o.C);  // stencil partly outside the grid
    }
    cp_async_wait_all();
    const V4 a1 = stage[tid], a2 = stage[nt + tid], a3 = stage[2 * nt + tid];
    const T F[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
    if (MODE == AE_MPM_MODE_PHYSICS) {
      const MatDev& md = mat_of(w, sc, Bits<T>::unpack(a3.z) & 0xffffu);
      g2p_physics_update<T>(sc, md, x0, pv, F, a3.y, a0.w, o);
    } else if (MODE == AE_MPM_MODE_REFERENCE) {
      g2p_reference<T>(vt, sc, x0, F, o);
    } else {
      const V4 a4 = ld4(w.in[4] + src), a5 = ld4(w.in[5] + src), a6 = ld4(w.in[6] + src);
      g2p_velonly<T>(vt, sc, x0, o);
#pragma unroll
      for (int k = 0; k < 9; ++k) o.F[k] = F[k];
      o.J = a3.y;
      o.C[0] = a4.w;
      o.C[1] = a5.x;
      o.C[2] = a5.y;
      o.C[3] = a5.z;
      o.C[4] = a5.w;
      o.C[5] = a6.x;
      o.C[6] = a6.y;
      o.C[7] = a6.z;
      o.C[8] = a6.w;
    }
    w.out[0][j] = mk4(o.x[0], o.x[1], o.x[2], a0.w);
    w.out[1][j] = mk4(o.F[0], o.F[1], o.F[2], o.F[3]);
    w.out[2][j] = mk4(o.F[4], o.F[5], o.F[6], o.F[7]);
    w.out[3][j] = mk4(o.F[8], o.J, a3.z, a3.w);
    w.out[4][j] = mk4(o.v[0], o.v[1], o.v[2], o.C[0]);
    w.out[5][j] = mk4(o.C[1], o.C[2], o.C[3], o.C[4]);
    w.out[6][j] = mk4(o.C[5], o.C[6], o.C[7], o.C[8]);
    // the next substep's cell key, only when the next substep sorts (the world tracks this)
    if (write_keys) w.keys[j] = cell_key(sc, MODE, o.x[0], o.x[1], o.x[2]);
    err = o.err;
    cl = o.clamped;
    need = o.needs_clamp;
  } else if (j < ch.w && write_keys) {
    w.keys[j] = sc.dead_key;
  }
  // warp-aggregated error words, counters and clamp-queue appends
  const uint32_t e = __reduce_or_sync(0xffffffffu, err);
  const uint32_t ncl = __popc(__ballot_sync(0xffffffffu, cl));
  const uint32_t qmask = __ballot_sync(0xffffffffu, need);
  uint32_t qbase = 0;
  if (lane == 0) {
    if (e) atomicOr(w.err + 4 * ch.x, e);
    if (ncl) atomicAdd(w.err + 4 * ch.x + 2, ncl);
    if (qmask) qbase = atomicAdd(w.clamp_count, uint32_t(__popc(qmask)));
  }
  qbase = __shfl_sync(0xffffffffu, qbase, 0);
  if (need) w.clamp_queue[qbase + __popc(qmask & ((1u << lane) - 1u))] = make_uint2(uint32_t(j), uint32_t(ch.x));
}

// Snow return mapping for the particles G2P queued: F = U S V^T, singular values clamped to
// [1-theta_c, 1+theta_s], J_p *= prod(S)/prod(S_clamped) (ae_physics/src/mpm.rs:565-606 plus
// Stomakhin's J_p), with the FP64 SVD redo where a near-degenerate pair straddles a threshold.
// 64 registers, 8 blocks of 128 per SM: the FP64 redo, taken by few particles, would otherwise set
// the register count (94) and leave three quarters of the SM's warp slots empty.
template <class T>
__global__ void __launch_bounds__(128, 8) snow_clamp_kernel(WorldDev<T> w) {
  using V4 = typename V4T<T>::type;
  // the particle's mass and C slots arrive here while its SVD runs (each thread its own column)
  __shared__ V4 pre[4][128];
  const int tid = threadIdx.x;
  const uint32_t count = launch_count(w.clamp_count);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint2 q = w.clamp_queue[i];
    cp_async_v4(&pre[0][tid], w.out[0] + q.x);
    cp_async_v4(&pre[1][tid], w.out[4] + q.x);
    cp_async_v4(&pre[2][tid], w.out[5] + q.x);
    cp_async_v4(&pre[3][tid], w.out[6] + q.x);
    cp_async_commit();
    const SceneDev<T>& sc = w.scenes[q.y];
    V4 a1 = w.out[1][q.x], a2 = w.out[2][q.x], a3 = w.out[3][q.x];
    const MatDev& md = mat_of(w, sc, Bits<T>::unpack(a3.z) & 0xffffu);
    const T F[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
    const T lo = T(1) - T(md.theta_c), hi = T(1) + T(md.theta_s);
    T U[9], sg[3], V[9];
    const bool fb = svd3_fallback(F, U, sg, V, w.svd_fallback != 0, lo, hi);
    T scl[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) scl[k] = t_min(t_max(sg[k], lo), hi);
    const T J = a3.y * ((sg[0] * sg[1] * sg[2]) / (scl[0] * scl[1] * scl[2]));
    T nF[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        nF[r * 3 + c] = U[r * 3 + 0] * scl[0] * V[c * 3 + 0] + U[r * 3 + 1] * scl[1] * V[c * 3 + 1] + U[r * 3 + 2] * scl[2] * V[c * 3 + 2];
    w.out[1][q.x] = mk4(nF[0], nF[1], nF[2], nF[3]);
    w.out[2][q.x] = mk4(nF[4], nF[5], nF[6], nF[7]);
    w.out[3][q.x] = mk4(nF[8], J, a3.z, a3.w);
    // G2P left C in the C slot of queued particles: turn it into A with the returned F and J_p
    cp_async_wait_all();
    const V4 a0 = pre[0][tid], a4 = pre[1][tid], a5 = pre[2][tid], a6 = pre[3][tid];
    const T C[9] = {a4.w, a5.x, a5.y, a5.z, a5.w, a6.x, a6.y, a6.z, a6.w};
    T A[9];
    affine_from_c(sc, md, a0.w, C, nF, J, A);
    w.out[4][q.x] = mk4(a4.x, a4.y, a4.z, A[0]);
    w.out[5][q.x] = mk4(A[1], A[2], A[3], A[4]);
    w.out[6][q.x] = mk4(A[5], A[6], A[7], A[8]);
    if (fb) atomicAdd(w.err + 4 * q.y + 1, 1u);
  }
}

// ============================================================================================
// fused G2P + P2G for physics mode (grid -> particle -> grid in one pass over the particles)
// ============================================================================================
// G2P of substep s computes each particle's new position, mass-weighted velocity and affine
// matrix A = m C - k tau; those are exactly the inputs of P2G for substep s + 1, so the same
// kernel scatters them into the (already cleared) accumulator of the next substep while they are
// still in registers.  P2G then never re-reads the particle state.  Snow particles whose F left
// the elastic region get A only after the return mapping: the clamp kernel scatters them.
//
// Per-warp shared staging of the column-lane scatter (the layout of p2g_lanes_kernel, one
// contiguous region per warp): 32 particles x (9 column vectors, x weights + mass, dx times A's x
// column) and 32 run records.  Per-thread data the warp stages before the scatter (the cp.async
// prefetch of F, J and the material) lives in the same region.
template <class T>
struct WarpStage {
  using V4 = typename V4T<T>::type;
  V4* col;   // col[pos * 9 + column]
  V4* wxm;   // wxm[pos] = (wx0, wx1, wx2, m)
  V4* acol;  // acol[pos] = dx * A[.][0]
  int4* gk;  // gk[pos] = (stencil base, cell key)
};
template <class T>
__host__ __device__ constexpr size_t warp_stage_bytes() {
  return sizeof(typename V4T<T>::type) * 32 * kLaneVecs + sizeof(int4) * 32;
}
template <class T>
__device__ __forceinline__ WarpStage<T> warp_stage(unsigned char* smem, int warp) {
  using V4 = typename V4T<T>::type;
  unsigned char* base = smem + size_t(warp) * warp_stage_bytes<T>();
  WarpStage<T> s;
  s.col = reinterpret_cast<V4*>(base);
  s.wxm = s.col + 32 * 9;
  s.acol = s.wxm + 32;
  s.gk = reinterpret_cast<int4*>(s.acol + 32);
  return s;
}

// The column-lane scatter of one warp (p2g_lanes_kernel's grouping, runs and vector reductions)
// for particles whose 27 stencil nodes all lie inside their scene's grid, which G2P's domain clamp
// guarantees.  Every lane of the warp calls it; has = false lanes contribute nothing.  x is the
// position, mv = m v, A = m C - k tau.  The cell key is the global index of the stencil's base
// node, unique across scenes.  kMixed: lanes may belong to different scenes (each run looks its
// scene up from its base node's block); otherwise every lane belongs to scene sc.
// runs of at most this many particles are summed one node per lane; longer ones by the column lanes
constexpr int kShortRun = 6;

template <class T, bool kMixed>
__device__ __forceinline__ void p2g_warp_scatter(const WorldDev<T>& w, const SceneDev<T>& sc, bool has, const T* x,
                                                 T m, const T* mv, const T* A, const WarpStage<T>& st) {
  using V4 = typename V4T<T>::type;
  const int lane = threadIdx.x & 31;
  int g[3] = {0, 0, 0};
  T fx[3] = {0, 0, 0}, wt[3][3];
  if (has) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T X = (x[a] - sc.origin[a]) * sc.inv_dx;
      const int b = floor_to_int(X - T(0.5));
      fx[a] = X - T(b);
      g[a] = b;
      const T t0 = T(1.5) - fx[a], t1 = fx[a] - T(1), t2 = fx[a] - T(0.5);
      wt[a][0] = T(0.5) * t0 * t0;
      wt[a][1] = T(0.75) - t1 * t1;
      wt[a][2] = T(0.5) * t2 * t2;
    }
  }
  const uint32_t key = has ? node_index(sc, g[0], g[1], g[2]) : 0xffffffffu;
  // equal keys anywhere in the warp form one group: groups in order of their first lane, lanes
  // within a group in lane order; pos is this particle's slot in that grouped order
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int leader = __ffs(peers) - 1;
  const uint32_t lead_cnt = lane == leader ? uint32_t(__popc(peers)) : 0u;
  uint32_t incl = lead_cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t lead_off = incl - lead_cnt;
  const int pos = int(__shfl_sync(0xffffffffu, lead_off, leader)) + __popc(peers & ((1u << lane) - 1u));
  uint32_t starts = __reduce_or_sync(0xffffffffu, lane == leader ? (1u << lead_off) : 0u);
  if (has) {
    const T dx = sc.dx;
    T c0[3], c1[3], c2[3], qv[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      c0[r] = dx * A[3 * r + 0];
      c1[r] = dx * A[3 * r + 1];
      c2[r] = dx * A[3 * r + 2];
      qv[r] = mv[r] - (c0[r] * fx[0] + c1[r] * fx[1] + c2[r] * fx[2]);
    }
    V4* cq = st.col + pos * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const T ux = qv[0] + T(b) * c1[0] + T(c) * c2[0];
        const T uy = qv[1] + T(b) * c1[1] + T(c) * c2[1];
        const T uz = qv[2] + T(b) * c1[2] + T(c) * c2[2];
        cq[b + 3 * c] = mk4(ux, uy, uz, wt[1][b] * wt[2][c]);
      }
    }
    st.wxm[pos] = mk4(wt[0][0], wt[0][1], wt[0][2], m);
    st.acol[pos] = mk4(c0[0], c0[1], c0[2], T(0));
  }
  st.gk[pos] = make_int4(g[0], g[1], g[2], int(key));
  __syncwarp();
  // lanes 0..26 are 3 particle groups x 9 (y,z) columns; lanes 27..31 mirror lanes 22..26
  // (in-bounds reads, results never used)
  const int grp = lane < 27 ? lane / 9 : 2;
  const int jc = lane < 27 ? lane - 9 * grp : lane - 23;
  const int nb = jc % 3, nc = jc / 3;
  const V4* colw = st.col + jc;
  while (starts) {
    const int s0 = __ffs(starts) - 1;
    starts &= starts - 1u;
    const int e0 = starts ? __ffs(starts) - 1 : 32;
    const int4 run = st.gk[s0];
    if (uint32_t(run.w) == 0xffffffffu) continue;
    const SceneDev<T>& rs = kMixed ? w.scenes[w.blk_scene[uint32_t(run.w) >> 6]] : sc;
    if (e0 - s0 <= kShortRun) {
      // a short run: one lane per stencil node (27 lanes), each summing every particle of the run
      // for its node; no combine across lane groups, one vector reduction per lane
      const int ln = lane < 27 ? lane : 26;
      const int xa = ln % 3, jn = ln / 3;
      const T fa = T(xa);
      const V4* cn = st.col + jn;
      T m = 0, px = 0, py = 0, pz = 0;
      if constexpr (sizeof(T) == 4) {  // x and y as one packed pair
        float2 pxy = make_float2(0.f, 0.f);
        const float2 fa2 = make_float2(fa, fa);
        for (int i = s0; i < e0; ++i) {
          const float4 u = cn[i * 9];
          const float4 r = st.wxm[i];
          const float4 a = st.acol[i];
          const float W = (xa == 0 ? r.x : (xa == 1 ? r.y : r.z)) * u.w;
          m += W * r.w;
          pxy = __ffma2_rn(make_float2(W, W), __ffma2_rn(fa2, make_float2(a.x, a.y), make_float2(u.x, u.y)), pxy);
          pz += W * (u.z + fa * a.z);
        }
        px = pxy.x;
        py = pxy.y;
      } else {
        for (int i = s0; i < e0; ++i) {
          const V4 u = cn[i * 9];
          const V4 r = st.wxm[i];
          const V4 a = st.acol[i];
          const T W = (xa == 0 ? r.x : (xa == 1 ? r.y : r.z)) * u.w;
          m += W * r.w;
          px += W * (u.x + fa * a.x);
          py += W * (u.y + fa * a.y);
          pz += W * (u.z + fa * a.z);
        }
      }
      if (lane < 27 && m != T(0)) {
        const int Xn = run.x + xa, Yn = run.y + jn % 3, Zn = run.z + jn / 3;
        const uint32_t node =
            ((rs.blk_off + (uint32_t(Zn >> 2) * uint32_t(rs.nb[1]) + uint32_t(Yn >> 2)) * uint32_t(rs.nb[0]) +
              uint32_t(Xn >> 2))
             << 6) |
            (uint32_t(Zn & 3) << 4) | (uint32_t(Yn & 3) << 2) | uint32_t(Xn & 3);
        atomic_add4(w.acc + node, m, px, py, pz);
      }
      if (kMixed && lane >= 27) {  // the run's stencil blocks (at most 2 per axis): lanes 27..31 and
        for (int o = lane - 27; o < 8; o += 5) {  // 27..29 again
          const int bx = (run.x + 2 * (o & 1)) >> 2, by = (run.y + (o & 2)) >> 2, bz = (run.z + ((o >> 1) & 2)) >> 2;
          mark_block(w, rs.blk_off + (uint32_t(bz) * uint32_t(rs.nb[1]) + uint32_t(by)) * uint32_t(rs.nb[0]) + uint32_t(bx));
        }
      }
      continue;
    }
    const int X = run.x, Y = run.y + nb, Z = run.z + nc;
    T m0 = 0, x0 = 0, y0 = 0, z0 = 0, m1 = 0, x1 = 0, y1 = 0, z1 = 0, m2 = 0, x2 = 0, y2 = 0, z2 = 0;
    if constexpr (sizeof(T) == 4) {  // x and y of each node as one packed pair
      float2 q0 = make_float2(0.f, 0.f), q1 = q0, q2 = q0;
#pragma unroll 2
      for (int i = s0 + grp; i < e0; i += 3) {
        const float4 u = colw[i * 9];
        const float4 r = st.wxm[i];
        const float4 a = st.acol[i];
        const float W0 = r.x * u.w, W1 = r.y * u.w, W2 = r.z * u.w;
        const float2 axy = make_float2(a.x, a.y), u0 = make_float2(u.x, u.y);
        const float2 u1 = __fadd2_rn(u0, axy), u2 = __fadd2_rn(u1, axy);
        m0 += W0 * r.w;
        m1 += W1 * r.w;
        m2 += W2 * r.w;
        q0 = __ffma2_rn(make_float2(W0, W0), u0, q0);
        q1 = __ffma2_rn(make_float2(W1, W1), u1, q1);
        q2 = __ffma2_rn(make_float2(W2, W2), u2, q2);
        const float uz1 = u.z + a.z;
        z0 += W0 * u.z;
        z1 += W1 * uz1;
        z2 += W2 * (uz1 + a.z);
      }
      x0 = q0.x, y0 = q0.y, x1 = q1.x, y1 = q1.y, x2 = q2.x, y2 = q2.y;
    } else
#pragma unroll 2
    for (int i = s0 + grp; i < e0; i += 3) {
      const V4 u = colw[i * 9];
      const V4 r = st.wxm[i];
      const V4 a = st.acol[i];
      const T W0 = r.x * u.w, W1 = r.y * u.w, W2 = r.z * u.w;
      m0 += W0 * r.w;
      x0 += W0 * u.x;
      y0 += W0 * u.y;
      z0 += W0 * u.z;
      const T ux = u.x + a.x, uy = u.y + a.y, uz = u.z + a.z;
      m1 += W1 * r.w;
      x1 += W1 * ux;
      y1 += W1 * uy;
      z1 += W1 * uz;
      m2 += W2 * r.w;
      x2 += W2 * (ux + a.x);
      y2 += W2 * (uy + a.y);
      z2 += W2 * (uz + a.z);
    }
    if (e0 - s0 > 1) {
      auto groups = [](T v) { return v + __shfl_down_sync(0xffffffffu, v, 9) + __shfl_down_sync(0xffffffffu, v, 18); };
      m0 = groups(m0), x0 = groups(x0), y0 = groups(y0), z0 = groups(z0);
      m1 = groups(m1), x1 = groups(x1), y1 = groups(y1), z1 = groups(z1);
      m2 = groups(m2), x2 = groups(x2), y2 = groups(y2), z2 = groups(z2);
    }
    if (lane < 9) {
      const uint32_t row = ((rs.blk_off + (uint32_t(Z >> 2) * uint32_t(rs.nb[1]) + uint32_t(Y >> 2)) * uint32_t(rs.nb[0])) << 6) |
                           (uint32_t(Z & 3) << 4) | (uint32_t(Y & 3) << 2);
      auto node = [row](int xa) { return row + ((uint32_t(xa >> 2) << 6) | uint32_t(xa & 3)); };
      if (m0 != T(0)) atomic_add4(w.acc + node(X), m0, x0, y0, z0);
      if (m1 != T(0)) atomic_add4(w.acc + node(X + 1), m1, x1, y1, z1);
      if (m2 != T(0)) atomic_add4(w.acc + node(X + 2), m2, x2, y2, z2);
    }
    if (kMixed && lane >= 9 && lane < 17) {  // the run's stencil blocks (at most 2 per axis)
      const int o = lane - 9;
      const int bx = (run.x + 2 * (o & 1)) >> 2, by = (run.y + (o & 2)) >> 2, bz = (run.z + ((o >> 1) & 2)) >> 2;
      mark_block(w, rs.blk_off + (uint32_t(bz) * uint32_t(rs.nb[1]) + uint32_t(by)) * uint32_t(rs.nb[0]) + uint32_t(bx));
    }
  }
  if (!kMixed) {  // grid blocks of the warp's stencil bounding box (all inside the grid)
    int B[3], NB[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int l = __reduce_min_sync(0xffffffffu, has ? g[a] : INT_MAX);
      const int h = __reduce_max_sync(0xffffffffu, has ? g[a] + 2 : INT_MIN);
      B[a] = l >> 2;
      NB[a] = l == INT_MAX ? 0 : (h >> 2) - (l >> 2) + 1;
    }
    const int nblk = NB[0] * NB[1] * NB[2];
    for (int t = lane; t < nblk; t += 32) {
      const int bx = B[0] + t % NB[0], by = B[1] + (t / NB[0]) % NB[1], bz = B[2] + t / (NB[0] * NB[1]);
      mark_block(w, sc.blk_off + (uint32_t(bz) * uint32_t(sc.nb[1]) + uint32_t(by)) * uint32_t(sc.nb[0]) + uint32_t(bx));
    }
  }
  __syncwarp();  // the staging region is free again
}

// G2P of substep s and P2G of substep s + 1 (physics mode).  The grid update of substep s ran
// before; w.touched / w.touched_count are the touched-block list of substep s + 1.
template <class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) g2p2g_kernel(WorldDev<T> w, uint32_t* epoch,
                                                                              int write_keys) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  const int tid = threadIdx.x, lane = tid & 31;
  const WarpStage<T> st = warp_stage<T>(smem, tid >> 5);
  V4* pre = st.col;  // F, J and the material of the warp's particles (pre[k * 32 + lane]) until the scatter
  const int j = ch.y + tid;
  const bool live = j < ch.z;
  if (blockIdx.x == 0 && tid == 0) *epoch += 1u;
  uint32_t err = 0;
  bool cl = false, need = false, has = false;
  T xs[3] = {0, 0, 0}, m = 0, mv[3] = {0, 0, 0}, A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (live) {
    const uint32_t src = w.perm ? w.perm[j] : uint32_t(j);
#pragma unroll
    for (int k = 0; k < 3; ++k) cp_async_v4(pre + k * 32 + lane, w.in[1 + k] + src);
    cp_async_commit();
    const V4 a0 = ld4(w.in[0] + src);
    const T x0[3] = {a0.x, a0.y, a0.z};
    G2POut<T> o;
    T pv[3] = {0, 0, 0};
    bool done;
    if constexpr (sizeof(T) == 4)
      done = g2p_physics_gather_sep_f2(GridRows<T>{w.vel, sc.blk_off, uint32_t(sc.nb[0]), uint32_t(sc.nb[1])}, sc, x0,
                                       pv, o.C);
    else
      done = g2p_physics_gather_sep<T>(GridRows<T>{w.vel, sc.blk_off, uint32_t(sc.nb[0]), uint32_t(sc.nb[1])}, sc, x0,
                                       pv, o.C);
    if (!done) {  // stencil partly outside the grid (a particle's first substep)
      VelTile<T> vt;
      vt.tile = nullptr;
      vt.vel = w.vel;
      g2p_physics_gather<T>(vt, sc, x0, pv, o.C);
    }
    cp_async_wait_all();
    const V4 a1 = pre[lane], a2 = pre[32 + lane], a3 = pre[64 + lane];
    const T F[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
    const MatDev& md = mat_of(w, sc, Bits<T>::unpack(a3.z) & 0xffffu);
    g2p_physics_update<T>(sc, md, x0, pv, F, a3.y, a0.w, o);
    w.out[0][j] = mk4(o.x[0], o.x[1], o.x[2], a0.w);
    w.out[1][j] = mk4(o.F[0], o.F[1], o.F[2], o.F[3]);
    w.out[2][j] = mk4(o.F[4], o.F[5], o.F[6], o.F[7]);
    w.out[3][j] = mk4(o.F[8], o.J, a3.z, a3.w);
    w.out[4][j] = mk4(o.v[0], o.v[1], o.v[2], o.C[0]);
    w.out[5][j] = mk4(o.C[1], o.C[2], o.C[3], o.C[4]);
    w.out[6][j] = mk4(o.C[5], o.C[6], o.C[7], o.C[8]);
    if (write_keys) w.keys[j] = cell_key(sc, AE_MPM_MODE_PHYSICS, o.x[0], o.x[1], o.x[2]);
    err = o.err;
    cl = o.clamped;
    need = o.needs_clamp;
    has = !need;
    m = a0.w;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      xs[a] = o.x[a];
      mv[a] = m * o.v[a];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) A[k] = o.C[k];
  } else if (j < ch.w && write_keys) {
    w.keys[j] = sc.dead_key;
  }
  const uint32_t e = __reduce_or_sync(0xffffffffu, err);
  const uint32_t ncl = __popc(__ballot_sync(0xffffffffu, cl));
  const uint32_t qmask = __ballot_sync(0xffffffffu, need);
  uint32_t qbase = 0;
  if (lane == 0) {
    if (e) atomicOr(w.err + 4 * ch.x, e);
    if (ncl) atomicAdd(w.err + 4 * ch.x + 2, ncl);
    if (qmask) qbase = atomicAdd(w.clamp_count, uint32_t(__popc(qmask)));
  }
  qbase = __shfl_sync(0xffffffffu, qbase, 0);
  if (need) w.clamp_queue[qbase + __popc(qmask & ((1u << lane) - 1u))] = make_uint2(uint32_t(j), uint32_t(ch.x));
  __syncwarp();  // every lane has read its F, J and material: the scatter may reuse the region
  p2g_warp_scatter<T, false>(w, sc, has, xs, m, mv, A, st);
}

// The snow return mapping of snow_clamp_kernel for the particles the fused kernel queued, each
// then scattered into the next substep's accumulator with its final A.  A warp takes 32
// consecutive queue entries (possibly of several scenes of a world).
template <class T>
__global__ void __launch_bounds__(128, 8) snow_clamp_scatter_kernel(WorldDev<T> w) {
  using V4 = typename V4T<T>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const WarpStage<T> st = warp_stage<T>(smem, threadIdx.x >> 5);
  V4* pre = st.col;  // position+mass, velocity+A of the queued particle: pre[k * 32 + lane], until the scatter
  const uint32_t count = launch_count(w.clamp_count);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
    const uint32_t i = base + lane;
    const bool valid = i < count;
    const uint2 q = valid ? w.clamp_queue[i] : make_uint2(0u, 0u);
    const SceneDev<T>& sc = w.scenes[q.y];
    T xs[3] = {0, 0, 0}, m = 0, mv[3] = {0, 0, 0}, A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (valid) {
      cp_async_v4(pre + lane, w.out[0] + q.x);
      cp_async_v4(pre + 32 + lane, w.out[4] + q.x);
      cp_async_v4(pre + 64 + lane, w.out[5] + q.x);
      cp_async_v4(pre + 96 + lane, w.out[6] + q.x);
      cp_async_commit();
      const V4 a1 = w.out[1][q.x], a2 = w.out[2][q.x], a3 = w.out[3][q.x];
      const MatDev& md = mat_of(w, sc, Bits<T>::unpack(a3.z) & 0xffffu);
      const T F[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
      const T lo = T(1) - T(md.theta_c), hi = T(1) + T(md.theta_s);
      T U[9], sg[3], V[9];
      const bool fb = svd3_fallback(F, U, sg, V, w.svd_fallback != 0, lo, hi);
      T scl[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) scl[k] = t_min(t_max(sg[k], lo), hi);
      const T J = a3.y * ((sg[0] * sg[1] * sg[2]) / (scl[0] * scl[1] * scl[2]));
      T nF[9];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          nF[r * 3 + c] = U[r * 3 + 0] * scl[0] * V[c * 3 + 0] + U[r * 3 + 1] * scl[1] * V[c * 3 + 1] +
                          U[r * 3 + 2] * scl[2] * V[c * 3 + 2];
      w.out[1][q.x] = mk4(nF[0], nF[1], nF[2], nF[3]);
      w.out[2][q.x] = mk4(nF[4], nF[5], nF[6], nF[7]);
      w.out[3][q.x] = mk4(nF[8], J, a3.z, a3.w);
      cp_async_wait_all();
      const V4 a0 = pre[lane], a4 = pre[32 + lane], a5 = pre[64 + lane], a6 = pre[96 + lane];
      const T C[9] = {a4.w, a5.x, a5.y, a5.z, a5.w, a6.x, a6.y, a6.z, a6.w};
      affine_from_c(sc, md, a0.w, C, nF, J, A);
      w.out[4][q.x] = mk4(a4.x, a4.y, a4.z, A[0]);
      w.out[5][q.x] = mk4(A[1], A[2], A[3], A[4]);
      w.out[6][q.x] = mk4(A[5], A[6], A[7], A[8]);
      if (fb) atomicAdd(w.err + 4 * q.y + 1, 1u);
      m = a0.w;
      xs[0] = a0.x, xs[1] = a0.y, xs[2] = a0.z;
      mv[0] = m * a4.x, mv[1] = m * a4.y, mv[2] = m * a4.z;
    }
    __syncwarp();  // prefetched data consumed: the scatter may reuse the region
    p2g_warp_scatter<T, true>(w, sc, valid, xs, m, mv, A, st);
  }
}

// Drops a scatter that was queued for the next substep (the particle state it came from changed):
// zeroes the accumulator and the flags of the blocks on its touched list.
template <class T>
__global__ void discard_scatter_kernel(typename V4T<T>::type* acc, uint32_t* blk_flag, const uint32_t* list,
                                       const uint32_t* count) {
  const uint32_t n = launch_count(count);
  for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
    const uint32_t gb = list[t];
    if (threadIdx.x < 64) acc[uint64_t(gb) * 64u + threadIdx.x] = mk4(T(0), T(0), T(0), T(0));
    if (threadIdx.x == 0) blk_flag[gb] = 0u;
  }
}

// ============================================================================================
// deterministic mode: per-cell fixed-order sums, per-node fixed-order gather
// ============================================================================================
__global__ void det_heads_kernel(const uint32_t* __restrict__ skeys, uint64_t n, const uint32_t* __restrict__ dead_flag,
                                 uint32_t* cell_slot, uint32_t* seg_start, uint32_t* cell_count) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = skeys[i];
  if (dead_flag[k >> 6]) return;  // spare blocks hold dead and off-grid particles
  if (i > 0 && skeys[i - 1] == k) return;
  uint32_t s = atomicAdd(cell_count, 1u);
  cell_slot[k] = s;
  seg_start[s] = uint32_t(i);
}

template <class T, int MODE>
__global__ void __launch_bounds__(128) det_cellsum_kernel(WorldDev<T> w, uint64_t n_sorted) {
  using V4 = typename V4T<T>::type;
  const uint32_t count = launch_count(w.cell_count);
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x) {
    const uint32_t start = w.seg_start[s];
    const uint32_t key = w.sorted_keys[start];
    const SceneDev<T>& sc = w.scenes[w.blk_scene[key >> 6]];
    T acc[27][4];
#pragma unroll
    for (int o = 0; o < 27; ++o) acc[o][0] = acc[o][1] = acc[o][2] = acc[o][3] = T(0);
    int g0 = 0, g1 = 0, g2 = 0;
    for (uint64_t i = start; i < n_sorted && w.sorted_keys[i] == key; ++i) {
      P2GPart<T> p;
      p2g_setup<T, MODE>(w, sc, w.perm[i], p);
      g0 = p.g[0];
      g1 = p.g[1];
      g2 = p.g[2];
#pragma unroll
      for (int o = 0; o < 27; ++o) {
        T cm, cx, cy, cz;
        if (p2g_contrib<T, MODE>(sc, p, o % 3, (o / 3) % 3, o / 9, cm, cx, cy, cz)) {
          acc[o][0] += cm;
          acc[o][1] += cx;
          acc[o][2] += cy;
          acc[o][3] += cz;
        }
      }
    }
#pragma unroll
    for (int o = 0; o < 27; ++o) w.cell_rec[uint64_t(s) * 27 + o] = mk4(acc[o][0], acc[o][1], acc[o][2], acc[o][3]);
    // the cell's stencil spans at most two blocks per axis
    for (int t = 0; t < 8; ++t) {
      int X = (t & 1) ? min(g0 + 2, sc.n[0] - 1) : max(g0, 0);
      int Y = (t & 2) ? min(g1 + 2, sc.n[1] - 1) : max(g1, 0);
      int Z = (t & 4) ? min(g2 + 2, sc.n[2] - 1) : max(g2, 0);
      mark_block(w, sc.blk_off + (uint32_t(Z >> 2) * sc.nb[1] + (Y >> 2)) * sc.nb[0] + (X >> 2));
    }
  }
}

template <class T, int MODE>
__global__ void __launch_bounds__(256) det_gather_kernel(WorldDev<T> w, uint32_t* blk_epoch, const uint32_t* epoch) {
  using V4 = typename V4T<T>::type;
  const uint32_t count = launch_count(w.touched_count);
  const uint32_t ep = *epoch;
  if (blockIdx.x == 0 && threadIdx.x == 0) *w.clamp_count = 0u;
  const int sub = threadIdx.x >> 6, l = threadIdx.x & 63;
  for (uint32_t t = blockIdx.x * 4 + sub; t < count; t += gridDim.x * 4) {
    const uint32_t gb = w.touched[t];
    const SceneDev<T>& sc = w.scenes[w.blk_scene[gb]];
    int i, j, k;
    block_coords(sc, gb, l, i, j, k);
    T m = 0, px = 0, py = 0, pz = 0;
    if (i < sc.n[0] && j < sc.n[1] && k < sc.n[2]) {
      // node (i,j,k) receives offset (a,b,c) of the cell based at (i-a, j-b, k-c), in fixed order
#pragma unroll 1
      for (int o = 0; o < 27; ++o) {
        const int a = o % 3, b = (o / 3) % 3, c = o / 9;
        int X = i - a, Y = j - b, Z = k - c;
        if (X < 0 || Y < 0 || Z < 0) continue;
        uint32_t s = w.cell_slot[node_index(sc, X, Y, Z)];
        if (s == 0xffffffffu) continue;
        V4 r = w.cell_rec[uint64_t(s) * 27 + o];
        m += r.x;
        px += r.y;
        py += r.z;
        pz += r.w;
      }
    }
    T vx, vy, vz;
    grid_velocity<T, MODE>(sc, i, j, k, m, px, py, pz, vx, vy, vz);
    w.vel[uint64_t(gb) * 64u + l] = mk4(vx, vy, vz, m);
    if (l == 0) {
      w.blk_flag[gb] = 0u;
      blk_epoch[gb] = ep;
    }
  }
}

__global__ void det_reset_kernel(const uint32_t* __restrict__ seg_start, const uint32_t* __restrict__ skeys,
                                 const uint32_t* cell_count, uint32_t* cell_slot) {
  const uint32_t count = launch_count(cell_count);
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < count; s += gridDim.x * blockDim.x)
    cell_slot[skeys[seg_start[s]]] = 0xffffffffu;
}

// ============================================================================================
// keys, pack/unpack, totals, grid export
// ============================================================================================
template <class T, int MODE>
__global__ void init_keys_kernel(WorldDev<T> w) {
  const int4 ch = cta_chunk(w);
  const SceneDev<T>& sc = w.scenes[ch.x];
  const int j = ch.y + threadIdx.x;
  if (j < ch.z) {
    auto a0 = ld4(w.in[0] + j);
    w.keys[j] = cell_key(sc, MODE, a0.x, a0.y, a0.z);
  } else if (j < ch.w) {
    w.keys[j] = sc.dead_key;
  }
}

// staging layout (elements of T): pos 3n | vel 3n | F 9n | J n | C 9n | mass n | then u16 mat n
template <class T>
__global__ void pack_kernel(typename V4T<T>::type* const* dst, const T* __restrict__ st, uint64_t n, uint32_t p_off,
                            const SceneDev<T>* scp, const MatDev* mats) {
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T* pos = st;
  const T* vel = st + 3 * n;
  const T* F = st + 6 * n;
  const T* J = st + 15 * n;
  const T* C = st + 16 * n;
  const T* mass = st + 25 * n;
  const uint16_t* mat = reinterpret_cast<const uint16_t*>(st + 26 * n);
  uint64_t s = p_off + i;
  dst[0][s] = mk4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mass[i]);
  dst[1][s] = mk4(F[9 * i], F[9 * i + 1], F[9 * i + 2], F[9 * i + 3]);
  dst[2][s] = mk4(F[9 * i + 4], F[9 * i + 5], F[9 * i + 6], F[9 * i + 7]);
  dst[3][s] = mk4(F[9 * i + 8], J[i], Bits<T>::pack(uint32_t(mat[i])), Bits<T>::pack(uint32_t(i)));
  T c[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) c[k] = C[9 * i + k];
  const SceneDev<T>& sc = *scp;
  if (sc.mode == AE_MPM_MODE_PHYSICS) {  // the C slot holds A = m C - k tau on the device
    const uint32_t mi = mat[i];
    const MatDev& md = mats[sc.mat_off + (mi < sc.n_mat ? mi : sc.n_mat)];
    T f[9], a[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = F[9 * i + k];
    affine_from_c(sc, md, mass[i], c, f, J[i], a);
#pragma unroll
    for (int k = 0; k < 9; ++k) c[k] = a[k];
  }
  dst[4][s] = mk4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], c[0]);
  dst[5][s] = mk4(c[1], c[2], c[3], c[4]);
  dst[6][s] = mk4(c[5], c[6], c[7], c[8]);
}

template <class T>
__global__ void unpack_kernel(const typename V4T<T>::type* const* src, T* __restrict__ st, uint64_t n, uint32_t p_off,
                              const SceneDev<T>* scp, const MatDev* mats) {
  using V4 = typename V4T<T>::type;
  uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t s = p_off + i;
  V4 a0 = src[0][s], a1 = src[1][s], a2 = src[2][s], a3 = src[3][s], a4 = src[4][s], a5 = src[5][s], a6 = src[6][s];
  uint64_t o = Bits<T>::unpack(a3.w);
  if (o >= n) return;
  T* pos = st;
  T* vel = st + 3 * n;
  T* F = st + 6 * n;
  T* J = st + 15 * n;
  T* C = st + 16 * n;
  T* mass = st + 25 * n;
  uint16_t* mat = reinterpret_cast<uint16_t*>(st + 26 * n);
  pos[3 * o] = a0.x;
  pos[3 * o + 1] = a0.y;
  pos[3 * o + 2] = a0.z;
  mass[o] = a0.w;
  const T f[9] = {a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w, a3.x};
  T c[9] = {a4.w, a5.x, a5.y, a5.z, a5.w, a6.x, a6.y, a6.z, a6.w};
  const SceneDev<T>& sc = *scp;
  if (sc.mode == AE_MPM_MODE_PHYSICS) {  // C = (A + k tau) / m
    const uint32_t mi = Bits<T>::unpack(a3.z) & 0xffffu;
    const MatDev& md = mats[sc.mat_off + (mi < sc.n_mat ? mi : sc.n_mat)];
    T tau[9];
    phys_tau(md, f, a3.y, tau);
    const T k = affine_k(sc, md, a0.w);
#pragma unroll
    for (int q = 0; q < 9; ++q) c[q] = (c[q] + k * tau[q]) / a0.w;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    F[9 * o + k] = f[k];
    C[9 * o + k] = c[k];
  }
  J[o] = a3.y;
  vel[3 * o] = a4.x;
  vel[3 * o + 1] = a4.y;
  vel[3 * o + 2] = a4.z;
  mat[o] = uint16_t(Bits<T>::unpack(a3.z) & 0xffffu);
}

// per-chunk FP64 partial sums [mass, px, py, pz, ke]; fixed reduction order (deterministic)
template <class T>
__global__ void __launch_bounds__(256) totals_kernel(WorldDev<T> w, double* partial) {
  __shared__ double sm[8][5];
  const int4 ch = cta_chunk(w);
  const int j = ch.y + threadIdx.x;
  double v[5] = {0, 0, 0, 0, 0};
  if (j < ch.z) {
    auto a0 = ld4(w.in[0] + j);
    auto a4 = ld4(w.in[4] + j);
    double m = double(a0.w), vx = double(a4.x), vy = double(a4.y), vz = double(a4.z);
    v[0] = m;
    v[1] = m * vx;
    v[2] = m * vy;
    v[3] = m * vz;
    v[4] = 0.5 * m * (vx * vx + vy * vy + vz * vz);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 5; ++k) sm[wi][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) / 32;
    for (int k = 0; k < 5; ++k) {
      double s = 0;
      for (int q = 0; q < nw; ++q) s += sm[q][k];
      partial[uint64_t(blockIdx.x) * 5 + k] = s;
    }
  }
}

// dense reference-order grid export of scene 0's last substep (mass, velocity)
template <class T>
__global__ void grid_export_kernel(const typename V4T<T>::type* vel, const SceneDev<T>* scp, const uint32_t* blk_epoch,
                                   const uint32_t* epoch, float* mass_out, float* vel_out) {
  const SceneDev<T>& sc = *scp;
  uint64_t idx = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  uint64_t nn = uint64_t(sc.n[0]) * sc.n[1] * sc.n[2];
  if (idx >= nn) return;
  int i = int(idx % sc.n[0]), j = int((idx / sc.n[0]) % sc.n[1]), k = int(idx / (uint64_t(sc.n[0]) * sc.n[1]));
  uint32_t gi = node_index(sc, i, j, k);
  bool fresh = blk_epoch[gi >> 6] + 1u == *epoch;
  auto v = vel[gi];
  mass_out[idx] = fresh ? float(v.w) : 0.0f;
  vel_out[3 * idx] = fresh ? float(v.x) : 0.0f;
  vel_out[3 * idx + 1] = fresh ? float(v.y) : 0.0f;
  vel_out[3 * idx + 2] = fresh ? float(v.z) : 0.0f;
}

// ============================================================================================
// host side
// ============================================================================================
int device_sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = v > 0 ? v : 148;
  }
  return cached[dev];
}

static MatDev mat_dev(const ae_mpm_material& m, int model) {
  MatDev d{};
  float nu = std::min(std::max(m.poisson_ratio, -0.999f), 0.4999f);
  d.model = model;
  d.lambda = m.young_modulus * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
  d.mu = m.young_modulus / (2.0f * (1.0f + nu));
  d.bulk = m.young_modulus / (3.0f * (1.0f - 2.0f * nu));
  if (model >= kPhysJelly && m.bulk_modulus > 0.0f) d.bulk = m.bulk_modulus;
  d.rho = m.density;
  d.yield_stress = m.yield_stress;
  d.friction_angle = m.friction_angle;
  d.cohesion = m.cohesion;
  d.theta_c = m.theta_c;
  d.theta_s = m.theta_s;
  d.xi = m.hardening_xi;
  return d;
}

static uint64_t blocks_of(const ae_mpm_scene_desc& d) {
  return uint64_t((d.n[0] + 3) / 4) * ((d.n[1] + 3) / 4) * ((d.n[2] + 3) / 4) + 1;  // + spare block
}

uint64_t scene_device_bytes(const ae_mpm_scene_desc& d, int precision) {
  uint64_t es = precision == 64 ? 8 : 4;
  uint64_t parts = d.max_particles * (2 * 7 * 4 * es + 5 * 4 + 26 * es + 2);
  uint64_t grid = blocks_of(d) * 64 * (2 * 4 * es) + blocks_of(d) * 16;
  return parts + grid;
}

#define AE_TRY(call)                                                                           \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                                \
      return (e_ == cudaErrorMemoryAllocation) ? AE_MPM_ENOMEM : AE_MPM_ECUDA;                 \
    }                                                                                          \
  } while (0)

// the caller's arrays, from an ae_mpm_particles (f32) or ae_mpm_particles_f64 (f64) view
template <class T>
struct HostView {
  T* f[6];  // pos, vel, strain, jacobian, c, mass
  uint16_t* mat;
};
template <class T>
HostView<T> host_view(const void* host);
template <>
HostView<float> host_view<float>(const void* host) {
  const auto* h = static_cast<const ae_mpm_particles*>(host);
  return HostView<float>{{h->pos, h->vel, h->strain, h->jacobian, h->c, h->mass}, h->material_idx};
}
template <>
HostView<double> host_view<double>(const void* host) {
  const auto* h = static_cast<const ae_mpm_particles_f64*>(host);
  return HostView<double>{{h->pos, h->vel, h->strain, h->jacobian, h->c, h->mass}, h->material_idx};
}

template <class T>
class World final : public WorldBase {
 public:
  using V4 = typename V4T<T>::type;

  ~World() override { release(); }

  int init(const ae_mpm_scene_desc* sc, uint32_t n, const ae_mpm_exec_opts& o) {
    opts_ = o;
    if (n == 0) {
      err = "a world needs at least one scene";
      return AE_MPM_EINVAL;
    }
    mode_ = sc[0].mode;
    if (mode_ < AE_MPM_MODE_PHYSICS || mode_ > AE_MPM_MODE_VELOCITY_ONLY) {
      err = "unknown substep mode";
      return AE_MPM_EINVAL;
    }
    uint64_t blk = 0, cap = 0;
    for (uint32_t s = 0; s < n; ++s) {
      const ae_mpm_scene_desc& d = sc[s];
      if (d.mode != mode_) {
        err = "all scenes of a world must use the same substep mode";
        return AE_MPM_EINVAL;
      }
      const uint32_t nmin = mode_ == AE_MPM_MODE_PHYSICS ? 4u : 1u;
      if (d.n[0] < nmin || d.n[1] < nmin || d.n[2] < nmin || !(d.dx > 0.0f) || !(d.dt >= 0.0f)) {
        err = "scene " + std::to_string(s) + ": grid needs >= " + std::to_string(nmin) +
              " nodes per axis, dx > 0 and dt >= 0";
        return AE_MPM_EINVAL;
      }
      if (d.n_materials == 0 || !d.materials) {
        err = "scene " + std::to_string(s) + ": material table is empty";
        return AE_MPM_EINVAL;
      }
      if (mode_ == AE_MPM_MODE_PHYSICS && d.wall_margin < 1) {
        err = "physics mode needs wall_margin >= 1";
        return AE_MPM_EINVAL;
      }
      if (mode_ == AE_MPM_MODE_PHYSICS && (d.n[0] > 1024 || d.n[1] > 1024 || d.n[2] > 1024)) {
        err = "physics-mode grids are limited to 1024 nodes per axis";
        return AE_MPM_EINVAL;
      }
      descs_.push_back(d);
      mats_.emplace_back(d.materials, d.materials + d.n_materials);
      blk += blocks_of(d);
      cap += d.max_particles;
    }
    if (blk * 64 >= (1ull << 31) || cap >= (1ull << 31)) {
      err = "world too large for 32-bit keys";
      return AE_MPM_EINVAL;
    }
    total_blocks_ = blk;
    total_cap_ = cap;
    key_bits_ = 1;
    while ((1ull << key_bits_) < blk * 64) ++key_bits_;
    if (opts_.precision != 32 && opts_.precision != 64) opts_.precision = sizeof(T) == 8 ? 64 : 32;
    if (opts_.sort_interval < 1) opts_.sort_interval = 1;
    if (opts_.block_threads != 128 && opts_.block_threads != 256) opts_.block_threads = 256;
    if (opts_.p2g_variant < kVarTile || opts_.p2g_variant > kVarLanes) opts_.p2g_variant = kVarLanes;
    AE_TRY(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    // scene table and materials
    uint64_t mat_off = 0, boff = 0, poff = 0;
    std::vector<uint32_t> blk_scene(blk), dead(blk, 0u);
    for (uint32_t s = 0; s < n; ++s) {
      const ae_mpm_scene_desc& d = descs_[s];
      SceneDev<T> h{};
      h.mode = d.mode;
      h.wall_mode = d.wall_mode;
      h.wall_margin = d.wall_margin;
      h.wall_origin = d.wall_origin;
      for (int a = 0; a < 3; ++a) {
        h.n[a] = int(d.n[a]);
        h.nb[a] = int((d.n[a] + 3) / 4);
      }
      h.blk_off = uint32_t(boff);
      uint64_t nbk = blocks_of(d);
      h.dead_key = uint32_t((boff + nbk - 1) * 64);
      for (uint64_t b = 0; b < nbk; ++b) blk_scene[boff + b] = s;
      dead[boff + nbk - 1] = 1u;
      boff += nbk;
      h.mat_off = uint32_t(mat_off);
      h.n_mat = d.n_materials;
      for (uint32_t k = 0; k < d.n_materials; ++k) {
        h_mats_.push_back(mat_dev(d.materials[k], d.materials[k].model));
        if (d.materials[k].model == kPhysSnow) has_snow_ = true;
      }
      // out-of-range material index: materials[0]'s parameters; the reference pairs them with
      // the neo-Hookean model (mpm_solver.rs:840-841)
      h_mats_.push_back(mat_dev(d.materials[0], mode_ == AE_MPM_MODE_PHYSICS ? d.materials[0].model : kNeoHookean));
      mat_off += d.n_materials + 1;
      h.p_off = uint32_t(poff);
      h.p_cap = uint32_t(d.max_particles);
      h.p_count = 0;
      poff += d.max_particles;
      fill_scene_params(h, d);
      h_scenes_.push_back(h);
    }
    AE_TRY(dmalloc(&d_scenes_, sizeof(SceneDev<T>) * n));
    AE_TRY(dmalloc(&d_mats_, sizeof(MatDev) * h_mats_.size()));
    AE_TRY(cudaMemcpy(d_mats_, h_mats_.data(), sizeof(MatDev) * h_mats_.size(), cudaMemcpyHostToDevice));
    AE_TRY(dmalloc(&blk_scene_, sizeof(uint32_t) * blk));
    AE_TRY(cudaMemcpy(blk_scene_, blk_scene.data(), sizeof(uint32_t) * blk, cudaMemcpyHostToDevice));
    AE_TRY(dmalloc(&dead_blk_, sizeof(uint32_t) * blk));
    AE_TRY(cudaMemcpy(dead_blk_, dead.data(), sizeof(uint32_t) * blk, cudaMemcpyHostToDevice));
    // particles
    const uint64_t pc = std::max<uint64_t>(cap, 1);
    // particle slots past a scene's count are never read (every kernel gates on the live range),
    // so the particle arrays need no clearing
    for (int k = 0; k < 7; ++k) {
      AE_TRY(dmalloc(&bufA_[k], sizeof(V4) * pc));
      AE_TRY(dmalloc(&bufB_[k], sizeof(V4) * pc));
    }
    AE_TRY(dmalloc(&d_ptrA_, sizeof(V4*) * 7));
    AE_TRY(dmalloc(&d_ptrB_, sizeof(V4*) * 7));
    AE_TRY(cudaMemcpy(d_ptrA_, bufA_, sizeof(V4*) * 7, cudaMemcpyHostToDevice));
    AE_TRY(cudaMemcpy(d_ptrB_, bufB_, sizeof(V4*) * 7, cudaMemcpyHostToDevice));
    AE_TRY(dmalloc(&keys_, sizeof(uint32_t) * pc));
    AE_TRY(sort_scratch_alloc(sort_, pc, alloc_ ? &World::sort_alloc : nullptr, alloc_));
    // grid
    const uint64_t nodes = blk * 64;
    AE_TRY(dmalloc(&acc_, sizeof(V4) * nodes));
    AE_TRY(cudaMemset(acc_, 0, sizeof(V4) * nodes));
    AE_TRY(dmalloc(&vel_, sizeof(V4) * nodes));
    AE_TRY(cudaMemset(vel_, 0, sizeof(V4) * nodes));
    AE_TRY(dmalloc(&blk_flag_, sizeof(uint32_t) * blk));
    AE_TRY(cudaMemset(blk_flag_, 0, sizeof(uint32_t) * blk));
    AE_TRY(dmalloc(&blk_epoch_, sizeof(uint32_t) * blk));
    AE_TRY(cudaMemset(blk_epoch_, 0xff, sizeof(uint32_t) * blk));
    // two touched-block lists: the fused G2P + P2G fills the next substep's while the grid update
    // consumes the current one's
    AE_TRY(dmalloc(&touched_, sizeof(uint32_t) * 2 * blk));
    AE_TRY(dmalloc(&counters_, sizeof(uint32_t) * 8));
    AE_TRY(cudaMemset(counters_, 0, sizeof(uint32_t) * 8));
    AE_TRY(dmalloc(&clamp_queue_, sizeof(uint2) * pc));
    AE_TRY(dmalloc(&err_, sizeof(uint32_t) * 4 * n));
    AE_TRY(cudaMemset(err_, 0, sizeof(uint32_t) * 4 * n));
    if (opts_.deterministic) {
      AE_TRY(dmalloc(&cell_slot_, sizeof(uint32_t) * nodes));
      AE_TRY(cudaMemset(cell_slot_, 0xff, sizeof(uint32_t) * nodes));
      AE_TRY(dmalloc(&seg_start_, sizeof(uint32_t) * pc));
      AE_TRY(dmalloc(&cell_rec_, sizeof(V4) * 27 * pc));
    }
    return AE_MPM_OK;
  }

  void fill_scene_params(SceneDev<T>& h, const ae_mpm_scene_desc& d) {
    h.dx = T(d.dx);
    h.inv_dx = T(1) / T(d.dx);
    h.dt = T(d.dt);
    h.restitution = T(d.restitution);
    h.damping = T(d.damping);
    h.wall_mode = d.wall_mode;
    h.wall_margin = d.wall_margin;
    h.wall_origin = d.wall_origin;
    for (int a = 0; a < 3; ++a) {
      h.origin[a] = T(d.origin[a]);
      h.grav[a] = T(d.gravity[a]);
    }
    if (sizeof(T) == 4) h.inv_dx = T(1.0f / d.dx);  // f32: the reference's `1.0 / dx` in f32
  }

  int set_scene_params(uint32_t s, const ae_mpm_scene_desc& d) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    if (d.n[0] != uint32_t(h_scenes_[s].n[0]) || d.n[1] != uint32_t(h_scenes_[s].n[1]) || d.n[2] != uint32_t(h_scenes_[s].n[2])) {
      err = "grid size of a resident scene cannot change";
      return AE_MPM_EINVAL;
    }
    if (d.n_materials != h_scenes_[s].n_mat || !d.materials) {
      err = "material count of a resident scene cannot change";
      return AE_MPM_EINVAL;
    }
    if (d.mode != mode_ || !(d.dx > 0.0f) || !(d.dt >= 0.0f) || (mode_ == AE_MPM_MODE_PHYSICS && d.wall_margin < 1)) {
      err = "scene update needs the world's mode, dx > 0, dt >= 0 and (physics) wall_margin >= 1";
      return AE_MPM_EINVAL;
    }
    // physics mode stores A = m C - k tau, which depends on dt and the materials: convert the
    // resident particles back to C with the old tables and again to A with the new ones
    const uint64_t cnt = h_scenes_[s].p_count;
    const bool rebase = mode_ == AE_MPM_MODE_PHYSICS && cnt > 0;
    if (rebase) {
      int rc = ensure_stage(cnt);
      if (rc) return rc;
      if ((rc = sync_tables())) return rc;
      unpack_kernel<T><<<unsigned((cnt + 255) / 256), 256, 0, stream_>>>(in_ptrs_dev(), stage_, cnt, h_scenes_[s].p_off,
                                                                          d_scenes_ + s, d_mats_);
      AE_TRY(cudaGetLastError());
    }
    fill_scene_params(h_scenes_[s], d);
    for (uint32_t k = 0; k < d.n_materials; ++k) {
      h_mats_[h_scenes_[s].mat_off + k] = mat_dev(d.materials[k], d.materials[k].model);
      if (d.materials[k].model == kPhysSnow && !has_snow_) {
        has_snow_ = true;  // the substep gains the clamp kernel: recapture
        invalidate_graph();
      }
    }
    h_mats_[h_scenes_[s].mat_off + d.n_materials] =
        mat_dev(d.materials[0], mode_ == AE_MPM_MODE_PHYSICS ? d.materials[0].model : kNeoHookean);
    dirty_scene(s);
    dirty_mats(s);
    keys_stale_ = true;  // dx or origin may have moved the cells
    scatter_invalid_ = true;
    if (rebase) {
      int rc = sync_tables();
      if (rc) return rc;
      pack_kernel<T><<<unsigned((cnt + 255) / 256), 256, 0, stream_>>>(in_ptrs_dev(), stage_, cnt, h_scenes_[s].p_off,
                                                                        d_scenes_ + s, d_mats_);
      AE_TRY(cudaGetLastError());
      keys_stale_ = true;
    }
    return AE_MPM_OK;
  }

  // whether a particle view's seven arrays lie back to back in the staging order (pos, vel, F, J,
  // C, mass at 0, 3n, 6n, 15n, 16n, 25n elements, the material indices at 26n)
  static bool staging_layout(const HostView<T>& hv, uint64_t n) {
    const uintptr_t b = reinterpret_cast<uintptr_t>(hv.f[0]);
    const uint64_t at[6] = {0, 3, 6, 15, 16, 25};
    for (int k = 1; k < 6; ++k)
      if (reinterpret_cast<uintptr_t>(hv.f[k]) != b + sizeof(T) * at[k] * n) return false;
    return reinterpret_cast<uintptr_t>(hv.mat) == b + sizeof(T) * 26 * n;
  }

  int upload(uint32_t s, const void* host, uint64_t n, bool f64) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    if ((sizeof(T) == 8) != f64) {
      err = "particle view precision does not match the world precision";
      return AE_MPM_EINVAL;
    }
    if (n > h_scenes_[s].p_cap) {
      err = "scene " + std::to_string(s) + ": " + std::to_string(n) + " particles exceed max_particles " +
            std::to_string(h_scenes_[s].p_cap);
      return AE_MPM_EINVAL;
    }
    HostView<T> hv = host_view<T>(host);
    const T* const* f = hv.f;
    if (n > 0 && (!f[0] || !f[1] || !f[2] || !f[3] || !f[4] || !f[5] || !hv.mat)) {
      err = "particle view has a null array";
      return AE_MPM_EINVAL;
    }
    int rc = ensure_stage(n);
    if (rc) return rc;
    if (n > 0) {
      // the view's arrays may be host or device memory (unified addressing picks the direction);
      // a view laid out as the staging itself travels in one copy
      if (staging_layout(hv, n)) {
        AE_TRY(cudaMemcpyAsync(stage_, f[0], sizeof(T) * 26 * n + sizeof(uint16_t) * n, cudaMemcpyDefault, stream_));
      } else {
        AE_TRY(cudaMemcpyAsync(stage_, f[0], sizeof(T) * 3 * n, cudaMemcpyDefault, stream_));
        AE_TRY(cudaMemcpyAsync(stage_ + 3 * n, f[1], sizeof(T) * 3 * n, cudaMemcpyDefault, stream_));
        AE_TRY(cudaMemcpyAsync(stage_ + 6 * n, f[2], sizeof(T) * 9 * n, cudaMemcpyDefault, stream_));
        AE_TRY(cudaMemcpyAsync(stage_ + 15 * n, f[3], sizeof(T) * n, cudaMemcpyDefault, stream_));
        AE_TRY(cudaMemcpyAsync(stage_ + 16 * n, f[4], sizeof(T) * 9 * n, cudaMemcpyDefault, stream_));
        AE_TRY(cudaMemcpyAsync(stage_ + 25 * n, f[5], sizeof(T) * n, cudaMemcpyDefault, stream_));
        AE_TRY(cudaMemcpyAsync(stage_ + 26 * n, hv.mat, sizeof(uint16_t) * n, cudaMemcpyDefault, stream_));
      }
      rc = sync_tables();
      if (rc) return rc;
      pack_kernel<T><<<unsigned((n + 255) / 256), 256, 0, stream_>>>(in_ptrs_dev(), stage_, n, h_scenes_[s].p_off,
                                                                      d_scenes_ + s, d_mats_);
      AE_TRY(cudaGetLastError());
    }
    scatter_invalid_ = true;
    // the same count keeps the scene table, the chunks and the captured graph (which replays from
    // the upload's buffers); the cell keys are recomputed before the next substep either way
    if (h_scenes_[s].p_count != uint32_t(n)) {
      h_scenes_[s].p_count = uint32_t(n);
      count_changed(s);
    }
    keys_stale_ = true;
    return AE_MPM_OK;
  }

  int download(uint32_t s, void* host, bool f64) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    if ((sizeof(T) == 8) != f64) {
      err = "particle view precision does not match the world precision";
      return AE_MPM_EINVAL;
    }
    const uint64_t n = h_scenes_[s].p_count;
    HostView<T> hv = host_view<T>(host);
    T* const* f = hv.f;
    if (n == 0) return AE_MPM_OK;
    if (!f[0] || !f[1] || !f[2] || !f[3] || !f[4] || !f[5] || !hv.mat) {
      err = "particle view has a null array";
      return AE_MPM_EINVAL;
    }
    int rc = ensure_stage(n);
    if (rc) return rc;
    rc = sync_tables();
    if (rc) return rc;
    unpack_kernel<T><<<unsigned((n + 255) / 256), 256, 0, stream_>>>(in_ptrs_dev(), stage_, n, h_scenes_[s].p_off,
                                                                      d_scenes_ + s, d_mats_);
    AE_TRY(cudaGetLastError());
    if (staging_layout(hv, n)) {
      AE_TRY(cudaMemcpyAsync(f[0], stage_, sizeof(T) * 26 * n + sizeof(uint16_t) * n, cudaMemcpyDefault, stream_));
    } else {
      AE_TRY(cudaMemcpyAsync(f[0], stage_, sizeof(T) * 3 * n, cudaMemcpyDefault, stream_));
      AE_TRY(cudaMemcpyAsync(f[1], stage_ + 3 * n, sizeof(T) * 3 * n, cudaMemcpyDefault, stream_));
      AE_TRY(cudaMemcpyAsync(f[2], stage_ + 6 * n, sizeof(T) * 9 * n, cudaMemcpyDefault, stream_));
      AE_TRY(cudaMemcpyAsync(f[3], stage_ + 15 * n, sizeof(T) * n, cudaMemcpyDefault, stream_));
      AE_TRY(cudaMemcpyAsync(f[4], stage_ + 16 * n, sizeof(T) * 9 * n, cudaMemcpyDefault, stream_));
      AE_TRY(cudaMemcpyAsync(f[5], stage_ + 25 * n, sizeof(T) * n, cudaMemcpyDefault, stream_));
      AE_TRY(cudaMemcpyAsync(hv.mat, stage_ + 26 * n, sizeof(uint16_t) * n, cudaMemcpyDefault, stream_));
    }
    AE_TRY(cudaStreamSynchronize(stream_));
    return AE_MPM_OK;
  }

  // byte offset of each scene's region in a many-scene staging area (16-byte aligned regions in the
  // staging layout of upload)
  static uint64_t stage_region(uint64_t n) { return (sizeof(T) * 26 * n + sizeof(uint16_t) * n + 15) / 16 * 16; }

  // orders `later` after the work queued so far on `earlier`
  int stream_after(cudaStream_t later, cudaStream_t earlier) {
    if (!xfer_ev_) AE_TRY(cudaEventCreateWithFlags(&xfer_ev_, cudaEventDisableTiming));
    AE_TRY(cudaEventRecord(xfer_ev_, earlier));
    AE_TRY(cudaStreamWaitEvent(later, xfer_ev_, 0));
    return AE_MPM_OK;
  }

  int upload_many(uint32_t k, const uint32_t* scenes, const ae_mpm_particles* views, const uint64_t* counts,
                  cudaStream_t copy) override {
    if (sizeof(T) != 4) {
      err = "many-scene transfers are for f32 worlds";
      return AE_MPM_EINVAL;
    }
    if (k == 0) return AE_MPM_OK;
    if (!scenes || !views || !counts) {
      err = "null scene, view or count array";
      return AE_MPM_EINVAL;
    }
    uint64_t total = 0;
    for (uint32_t i = 0; i < k; ++i) {
      const uint32_t s = scenes[i];
      if (s >= h_scenes_.size()) {
        err = "unknown scene";
        return AE_MPM_ENOTFOUND;
      }
      if (counts[i] > h_scenes_[s].p_cap) {
        err = "scene " + std::to_string(s) + ": " + std::to_string(counts[i]) + " particles exceed max_particles " +
              std::to_string(h_scenes_[s].p_cap);
        return AE_MPM_EINVAL;
      }
      const ae_mpm_particles& v = views[i];
      if (counts[i] > 0 && (!v.pos || !v.vel || !v.strain || !v.jacobian || !v.c || !v.mass || !v.material_idx)) {
        err = "particle view has a null array";
        return AE_MPM_EINVAL;
      }
      total += stage_region(counts[i]);
    }
    {
      const int rs = ensure_stage_bytes(total);
      if (rs) return rs;
    }
    // all copies first, back to back on the copy stream (the world's own by default), then the packs
    const cudaStream_t cs = copy ? copy : stream_;
    if (copy) {  // the staging area is free once the world's queued work is done with it
      const int r = stream_after(cs, stream_);
      if (r) return r;
    }
    uint64_t off = 0;
    for (uint32_t i = 0; i < k; ++i) {
      const uint64_t n = counts[i];
      T* st = reinterpret_cast<T*>(reinterpret_cast<char*>(stage_) + off);
      HostView<T> hv = host_view<T>(&views[i]);
      if (n > 0) {
        if (staging_layout(hv, n)) {
          AE_TRY(cudaMemcpyAsync(st, hv.f[0], sizeof(T) * 26 * n + sizeof(uint16_t) * n, cudaMemcpyDefault, cs));
        } else {
          const uint64_t at[6] = {0, 3, 6, 15, 16, 25}, len[6] = {3, 3, 9, 1, 9, 1};
          for (int f = 0; f < 6; ++f)
            AE_TRY(cudaMemcpyAsync(st + at[f] * n, hv.f[f], sizeof(T) * len[f] * n, cudaMemcpyDefault, cs));
          AE_TRY(cudaMemcpyAsync(st + 26 * n, hv.mat, sizeof(uint16_t) * n, cudaMemcpyDefault, cs));
        }
      }
      off += stage_region(n);
    }
    if (copy) {
      const int r = stream_after(stream_, cs);
      if (r) return r;
    }
    for (uint32_t i = 0; i < k; ++i) {
      const uint32_t s = scenes[i];
      if (h_scenes_[s].p_count != uint32_t(counts[i])) {
        h_scenes_[s].p_count = uint32_t(counts[i]);
        count_changed(s);
      }
    }
    int rc = sync_tables();
    if (rc) return rc;
    off = 0;
    for (uint32_t i = 0; i < k; ++i) {
      const uint64_t n = counts[i];
      const T* st = reinterpret_cast<const T*>(reinterpret_cast<const char*>(stage_) + off);
      if (n > 0)
        pack_kernel<T><<<unsigned((n + 255) / 256), 256, 0, stream_>>>(in_ptrs_dev(), st, n, h_scenes_[scenes[i]].p_off,
                                                                        d_scenes_ + scenes[i], d_mats_);
      off += stage_region(n);
    }
    AE_TRY(cudaGetLastError());
    keys_stale_ = true;
    scatter_invalid_ = true;
    return AE_MPM_OK;
  }

  int download_many(uint32_t k, const uint32_t* scenes, ae_mpm_particles* views, cudaStream_t copy) override {
    if (sizeof(T) != 4) {
      err = "many-scene transfers are for f32 worlds";
      return AE_MPM_EINVAL;
    }
    if (k == 0) return AE_MPM_OK;
    if (!scenes || !views) {
      err = "null scene or view array";
      return AE_MPM_EINVAL;
    }
    uint64_t total = 0;
    for (uint32_t i = 0; i < k; ++i) {
      if (scenes[i] >= h_scenes_.size()) {
        err = "unknown scene";
        return AE_MPM_ENOTFOUND;
      }
      const ae_mpm_particles& v = views[i];
      if (h_scenes_[scenes[i]].p_count > 0 &&
          (!v.pos || !v.vel || !v.strain || !v.jacobian || !v.c || !v.mass || !v.material_idx)) {
        err = "particle view has a null array";
        return AE_MPM_EINVAL;
      }
      total += stage_region(h_scenes_[scenes[i]].p_count);
    }
    {
      const int rs = ensure_stage_bytes(total);
      if (rs) return rs;
    }
    int rc = sync_tables();
    if (rc) return rc;
    uint64_t off = 0;
    for (uint32_t i = 0; i < k; ++i) {
      const SceneDev<T>& h = h_scenes_[scenes[i]];
      T* st = reinterpret_cast<T*>(reinterpret_cast<char*>(stage_) + off);
      if (h.p_count > 0)
        unpack_kernel<T><<<unsigned((h.p_count + 255) / 256), 256, 0, stream_>>>(in_ptrs_dev(), st, h.p_count, h.p_off,
                                                                                 d_scenes_ + scenes[i], d_mats_);
      off += stage_region(h.p_count);
    }
    AE_TRY(cudaGetLastError());
    const cudaStream_t cs = copy ? copy : stream_;
    if (copy) {
      const int r = stream_after(cs, stream_);
      if (r) return r;
    }
    off = 0;
    for (uint32_t i = 0; i < k; ++i) {
      const uint64_t n = h_scenes_[scenes[i]].p_count;
      const T* st = reinterpret_cast<const T*>(reinterpret_cast<const char*>(stage_) + off);
      HostView<T> hv = host_view<T>(&views[i]);
      if (n > 0) {
        if (staging_layout(hv, n)) {
          AE_TRY(cudaMemcpyAsync(hv.f[0], st, sizeof(T) * 26 * n + sizeof(uint16_t) * n, cudaMemcpyDefault, cs));
        } else {
          const uint64_t at[6] = {0, 3, 6, 15, 16, 25}, len[6] = {3, 3, 9, 1, 9, 1};
          for (int f = 0; f < 6; ++f)
            AE_TRY(cudaMemcpyAsync(hv.f[f], st + at[f] * n, sizeof(T) * len[f] * n, cudaMemcpyDefault, cs));
          AE_TRY(cudaMemcpyAsync(hv.mat, st + 26 * n, sizeof(uint16_t) * n, cudaMemcpyDefault, cs));
        }
      }
      off += stage_region(n);
    }
    if (copy) {  // the next use of the staging area on the world's stream waits for these reads
      const int r = stream_after(stream_, cs);
      if (r) return r;
      return AE_MPM_OK;
    }
    AE_TRY(cudaStreamSynchronize(stream_));
    return AE_MPM_OK;
  }

  int step(uint32_t n) override {
    launches_ = 0;
    int rc = prepare();
    if (rc) return rc;
    if (n == 0) return AE_MPM_OK;
    if ((rc = sync_scatter())) return rc;
    if (keys_stale_) {
      WorldDev<T> w = dev(false);
      launch_init_keys(w);
      keys_stale_ = false;
      keys_fresh_ = true;
    }
    const int interval = opts_.deterministic ? 1 : opts_.sort_interval;
    const uint64_t period = (interval % 2 == 0) ? uint64_t(interval) : uint64_t(2 * interval);
    uint32_t left = n;
    if (opts_.use_graph) {
      while (left > 0 && substep_ % period != 0) {
        substep_eager();
        --left;
      }
      if (left >= period) {
        rc = ensure_graph(period);
        if (rc) return rc;
        while (left >= period) {
          AE_TRY(cudaGraphLaunch(graph_, stream_));
          launches_ += graph_launches_;
          substep_ += period;
          left -= uint32_t(period);
        }
      }
    }
    while (left > 0) {
      substep_eager();
      --left;
    }
    AE_TRY(cudaGetLastError());
    return AE_MPM_OK;
  }

  int sync() override {
    AE_TRY(cudaStreamSynchronize(stream_));
    std::vector<uint32_t> e(4 * h_scenes_.size());
    AE_TRY(cudaMemcpy(e.data(), err_, sizeof(uint32_t) * e.size(), cudaMemcpyDeviceToHost));
    uint32_t any = 0;
    for (size_t s = 0; s < h_scenes_.size(); ++s) any |= e[4 * s];
    if (any & kErrNaN) {
      err = "a particle position became non-finite";
      return AE_MPM_ENAN;
    }
    if (any & kErrDomain) {
      err = "particles reached the grid's outer ring and were clamped back";
      return AE_MPM_EDOMAIN;
    }
    return AE_MPM_OK;
  }

  int totals(uint32_t s, double out[5]) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    int rc = prepare();
    if (rc) return rc;
    if (n_chunks_ == 0) {
      for (int k = 0; k < 5; ++k) out[k] = 0;
      return AE_MPM_OK;
    }
    if (!partial_) AE_TRY(dmalloc(&partial_, sizeof(double) * 5 * n_chunks_alloc_));
    WorldDev<T> w = dev(false);
    totals_kernel<T><<<n_chunks_, chunk_threads_, 0, stream_>>>(w, partial_);
    AE_TRY(cudaGetLastError());
    std::vector<double> h(5 * size_t(n_chunks_));
    AE_TRY(cudaMemcpyAsync(h.data(), partial_, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream_));
    AE_TRY(cudaStreamSynchronize(stream_));
    for (int k = 0; k < 5; ++k) out[k] = 0;
    for (int c = 0; c < n_chunks_; ++c)
      if (uint32_t(h_chunks_[c].x) == s)
        for (int k = 0; k < 5; ++k) out[k] += h[5 * size_t(c) + k];
    return AE_MPM_OK;
  }

  int errors(uint32_t s, uint32_t* word, uint64_t counters[3]) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    uint32_t e[4];
    AE_TRY(cudaStreamSynchronize(stream_));
    AE_TRY(cudaMemcpy(e, err_ + 4 * s, sizeof(e), cudaMemcpyDeviceToHost));
    AE_TRY(cudaMemset(err_ + 4 * s, 0, sizeof(e)));
    if (word) *word = e[0];
    if (counters) {
      counters[0] = e[1];
      counters[1] = e[2];
      counters[2] = e[3];
    }
    return AE_MPM_OK;
  }

  int grid_download(uint32_t s, float* mass, float* vel, uint64_t n_nodes) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    const SceneDev<T>& h = h_scenes_[s];
    uint64_t nn = uint64_t(h.n[0]) * h.n[1] * h.n[2];
    if (n_nodes != nn || !mass || !vel) {
      err = "grid download needs nx*ny*nz nodes";
      return AE_MPM_EINVAL;
    }
    float *dm = nullptr, *dv = nullptr;
    AE_TRY(dmalloc(&dm, sizeof(float) * nn));
    AE_TRY(dmalloc(&dv, sizeof(float) * 3 * nn));
    grid_export_kernel<T><<<unsigned((nn + 255) / 256), 256, 0, stream_>>>(vel_, d_scenes_ + s, blk_epoch_, counters_ + 2,
                                                                           dm, dv);
    cudaError_t e1 = cudaMemcpyAsync(mass, dm, sizeof(float) * nn, cudaMemcpyDeviceToHost, stream_);
    cudaError_t e2 = cudaMemcpyAsync(vel, dv, sizeof(float) * 3 * nn, cudaMemcpyDeviceToHost, stream_);
    cudaError_t e3 = cudaStreamSynchronize(stream_);
    dfree(dm);
    dfree(dv);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      err = "grid download failed";
      return AE_MPM_ECUDA;
    }
    return AE_MPM_OK;
  }

  int snapshot(bool restore) override {
    const uint64_t pc = std::max<uint64_t>(total_cap_, 1);
    if (!restore) {
      for (int k = 0; k < 7; ++k) {
        if (!snap_[k]) AE_TRY(dmalloc(&snap_[k], sizeof(V4) * pc));
        AE_TRY(cudaMemcpyAsync(snap_[k], in_buf()[k], sizeof(V4) * pc, cudaMemcpyDeviceToDevice, stream_));
      }
      snap_substep_ = substep_;
    } else {
      if (!snap_[0]) {
        err = "no snapshot";
        return AE_MPM_EINVAL;
      }
      for (int k = 0; k < 7; ++k)
        AE_TRY(cudaMemcpyAsync(in_buf()[k], snap_[k], sizeof(V4) * pc, cudaMemcpyDeviceToDevice, stream_));
      keys_stale_ = true;
      scatter_invalid_ = true;
      AE_TRY(cudaMemsetAsync(err_, 0, sizeof(uint32_t) * 4 * h_scenes_.size(), stream_));
    }
    AE_TRY(cudaStreamSynchronize(stream_));
    return AE_MPM_OK;
  }

  uint64_t last_launches() const override { return launches_; }
  uint64_t particles() const override {
    uint64_t s = 0;
    for (auto& h : h_scenes_) s += h.p_count;
    return s;
  }
  cudaStream_t stream() const override { return stream_; }
  int set_stream_priority(int priority) override {
    if (graph_) {
      cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
    }
    AE_TRY(cudaStreamSynchronize(stream_));
    cudaStream_t s = nullptr;
    AE_TRY(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
    cudaStreamDestroy(stream_);
    stream_ = s;
    return AE_MPM_OK;
  }
  ae_mpm_exec_opts& opts() override { return opts_; }
  void invalidate_graph() override {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    chunks_dirty_ = true;
  }
  uint64_t device_bytes() const override { return device_bytes_; }

  int copy_scene_from(uint32_t dst, WorldBase* srcb, uint32_t s) override {
    auto* src = dynamic_cast<World<T>*>(srcb);
    if (!src || dst >= h_scenes_.size() || s >= src->h_scenes_.size()) {
      err = "scene copy between incompatible worlds";
      return AE_MPM_EINVAL;
    }
    const SceneDev<T>& a = src->h_scenes_[s];
    SceneDev<T>& b = h_scenes_[dst];
    if (a.n[0] != b.n[0] || a.n[1] != b.n[1] || a.n[2] != b.n[2] || a.p_count > b.p_cap) {
      err = "scene copy needs the same grid and enough particle capacity";
      return AE_MPM_EINVAL;
    }
    for (int k = 0; k < 7; ++k)
      if (a.p_count)
        AE_TRY(cudaMemcpyAsync(in_buf()[k] + b.p_off, src->in_buf()[k] + a.p_off, sizeof(V4) * a.p_count,
                               cudaMemcpyDeviceToDevice, stream_));
    // the scene's error word and counters move with it
    AE_TRY(cudaMemcpyAsync(err_ + 4 * dst, src->err_ + 4 * s, sizeof(uint32_t) * 4, cudaMemcpyDeviceToDevice, stream_));
    b.p_count = a.p_count;
    count_changed(dst);
    keys_stale_ = scatter_invalid_ = true;
    return AE_MPM_OK;
  }
  uint32_t scene_count(uint32_t s) const override { return s < h_scenes_.size() ? h_scenes_[s].p_count : 0; }

  int assign_scene(uint32_t s, const ae_mpm_scene_desc& d, const void* host, uint64_t n) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    SceneDev<T>& h = h_scenes_[s];
    const uint32_t nmin = mode_ == AE_MPM_MODE_PHYSICS ? 4u : 1u;
    if (d.mode != mode_ || d.n[0] < nmin || d.n[1] < nmin || d.n[2] < nmin || !(d.dx > 0.0f) || !(d.dt >= 0.0f) ||
        (mode_ == AE_MPM_MODE_PHYSICS && d.wall_margin < 1) || d.n_materials == 0 || !d.materials) {
      err = "slot scene needs the world's mode, >= " + std::to_string(nmin) +
            " nodes per axis, dx > 0, dt >= 0, materials and (physics) wall_margin >= 1";
      return AE_MPM_EINVAL;
    }
    if (blocks_of(d) > blocks_of(descs_[s]) || d.n_materials > descs_[s].n_materials || n > h.p_cap) {
      err = "scene does not fit slot " + std::to_string(s) + " (grid blocks, materials or particles)";
      return AE_MPM_EINVAL;
    }
    for (int a = 0; a < 3; ++a) {
      h.n[a] = int(d.n[a]);
      h.nb[a] = int((d.n[a] + 3) / 4);
    }
    h.mode = d.mode;
    h.n_mat = d.n_materials;  // the out-of-range fallback entry follows the scene's materials
    fill_scene_params(h, d);
    for (uint32_t k = 0; k < d.n_materials; ++k) {
      h_mats_[h.mat_off + k] = mat_dev(d.materials[k], d.materials[k].model);
      if (d.materials[k].model == kPhysSnow && !has_snow_) {
        has_snow_ = true;  // the substep gains the clamp kernel: recapture
        invalidate_graph();
      }
    }
    h_mats_[h.mat_off + d.n_materials] =
        mat_dev(d.materials[0], mode_ == AE_MPM_MODE_PHYSICS ? d.materials[0].model : kNeoHookean);
    dirty_scene(s);
    dirty_mats(s);
    keys_stale_ = true;
    AE_TRY(cudaMemsetAsync(err_ + 4 * s, 0, sizeof(uint32_t) * 4, stream_));
    if (!host) {
      h.p_count = 0;
      count_changed(s);
      return AE_MPM_OK;
    }
    // with the P2G of the next substep already queued for the other scenes (fused flow), add
    // only this scene's scatter instead of redoing everyone's
    const bool keep_queued = scatter_pending_ && !scatter_invalid_ && fused();
    int rc = upload(s, host, n, sizeof(T) == 8);
    if (rc || !keep_queued) return rc;
    scatter_invalid_ = false;
    // the slot's blocks may hold the last scatter of the scene that vacated it: zero them (their
    // flags stay set, so the touched list keeps each block once) and scatter the new particles
    AE_TRY(cudaMemsetAsync(acc_ + uint64_t(h.blk_off) * 64u, 0, sizeof(V4) * 64 * blocks_of(descs_[s]), stream_));
    if ((rc = prepare())) return rc;
    if (n == 0) return AE_MPM_OK;
    WorldDev<T> w = with_list(dev(false), int(substep_ & 1));
    const int c0 = chunk_first_[s], c1 = chunk_first_[s + 1];
    if (!w.one_scene) w.chunks = d_chunks_ + c0;
    const size_t per = sizeof(V4) * kLaneVecs + sizeof(int4);
    if (!lanes_smem_set_) {
      AE_TRY(cudaFuncSetAttribute(p2g_lanes_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(per * 256)));
      lanes_smem_set_ = true;
    }
    p2g_lanes_kernel<T><<<unsigned(c1 - c0), chunk_threads_, per * chunk_threads_, stream_>>>(w);
    AE_TRY(cudaGetLastError());
    return AE_MPM_OK;
  }

  int vacate_scene(uint32_t s) override {
    if (s >= h_scenes_.size()) {
      err = "unknown scene";
      return AE_MPM_ENOTFOUND;
    }
    // a scatter queued for the next substep may still hold the scene's contributions: they land in
    // the slot's own blocks, which the next grid update consumes and no particle reads
    h_scenes_[s].p_count = 0;
    count_changed(s);
    keys_stale_ = true;
    return AE_MPM_OK;
  }
  int precision() const override { return sizeof(T) == 8 ? 64 : 32; }

  int stage_times(uint32_t n, double out_us[6]) override {
    for (int k = 0; k < 6; ++k) out_us[k] = 0;
    int rc = prepare();
    if (rc) return rc;
    if (n == 0 || n_chunks_ == 0) return AE_MPM_OK;
    if ((rc = sync_scatter())) return rc;
    if (keys_stale_) {
      WorldDev<T> w = dev(false);
      launch_init_keys(w);
      keys_stale_ = false;
      keys_fresh_ = true;
    }
    // all substeps are queued before the one wait, so that (past the first) the stream is never
    // idle waiting for the host and the events measure device time, not launch latency
    // per substep: start, after the sort, after P2G, after the grid update, end, and after the
    // G2P (or fused) kernel alone, before the snow clamp (recorded between the last two)
    std::vector<cudaEvent_t> ev(6 * size_t(n), nullptr);
    int rc2 = AE_MPM_OK;
    for (auto& e : ev)
      if (cudaEventCreate(&e) != cudaSuccess) rc2 = AE_MPM_ECUDA;
    if (rc2 == AE_MPM_OK) {
      for (uint32_t i = 0; i < n; ++i) {
        stage_events_ = ev.data() + 6 * size_t(i);
        substep_eager();
      }
      stage_events_ = nullptr;
      if (cudaEventSynchronize(ev[6 * size_t(n - 1) + 4]) != cudaSuccess) rc2 = AE_MPM_ECUDA;
    }
    double acc[6] = {0, 0, 0, 0, 0, 0};
    // the first substep starts on an idle stream: skip it when there is more than one
    const uint32_t first = n > 1 ? 1u : 0u;
    for (uint32_t i = first; i < n && rc2 == AE_MPM_OK; ++i) {
      const cudaEvent_t* e = ev.data() + 6 * size_t(i);
      float ms;
      for (int k = 0; k < 4; ++k) {
        cudaEventElapsedTime(&ms, e[k], e[k + 1]);
        acc[k] += ms;
      }
      cudaEventElapsedTime(&ms, e[0], e[4]);
      acc[4] += ms;
      cudaEventElapsedTime(&ms, e[3], e[5]);
      acc[5] += ms;
    }
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (rc2 != AE_MPM_OK) {
      err = "stage timing events failed";
      return rc2;
    }
    for (int k = 0; k < 6; ++k) out_us[k] = 1000.0 * acc[k] / (n - first);
    return AE_MPM_OK;
  }

 private:
  template <class P>
  cudaError_t dmalloc(P** p, size_t bytes) {
    void* q = nullptr;
    cudaError_t e = alloc_ ? alloc_->alloc(&q, bytes) : cudaMalloc(&q, bytes);
    *p = static_cast<P*>(q);
    return e;
  }
  void dfree(const void* p) {
    if (!p) return;
    if (alloc_)
      alloc_->release(const_cast<void*>(p));
    else
      cudaFree(const_cast<void*>(p));
  }
  static cudaError_t sort_alloc(void* user, void** p, size_t bytes) { return static_cast<DevAlloc*>(user)->alloc(p, bytes); }
  static void sort_free(void* user, void* p) { static_cast<DevAlloc*>(user)->release(p); }

  V4** in_buf() { return a_in_ ? bufA_ : bufB_; }
  V4** out_buf() { return a_in_ ? bufB_ : bufA_; }
  V4* const* in_ptrs_dev() { return a_in_ ? d_ptrA_ : d_ptrB_; }

  int ensure_stage(uint64_t n) { return ensure_stage_bytes(sizeof(T) * 26 * n + sizeof(uint16_t) * n + 64); }
  int ensure_stage_bytes(size_t need) {
    if (need <= stage_bytes_) return AE_MPM_OK;
    // queued work may still read the old staging area
    AE_TRY(cudaStreamSynchronize(stream_));
    dfree(stage_);
    stage_ = nullptr;
    stage_bytes_ = 0;
    AE_TRY(dmalloc(&stage_, need));
    stage_bytes_ = need;
    return AE_MPM_OK;
  }

  int prepare() {
    if (opts_.block_threads != 128 && opts_.block_threads != 256) opts_.block_threads = 256;
    if (opts_.sort_interval < 1) opts_.sort_interval = 1;
    if (opts_.p2g_variant < kVarTile || opts_.p2g_variant > kVarLanes) opts_.p2g_variant = kVarLanes;
    if (opts_.block_threads != chunk_threads_) chunks_dirty_ = true;
    if (chunks_dirty_) {
      chunk_threads_ = opts_.block_threads;
      h_chunks_.clear();
      chunk_first_.assign(h_scenes_.size() + 1, 0);
      for (size_t s = 0; s < h_scenes_.size(); ++s) {
        chunk_first_[s] = int(h_chunks_.size());
        const SceneDev<T>& h = h_scenes_[s];
        for (uint64_t lo = h.p_off; lo < uint64_t(h.p_off) + h.p_cap; lo += chunk_threads_) {
          uint64_t hl = std::min<uint64_t>(lo + chunk_threads_, uint64_t(h.p_off) + h.p_count);
          uint64_t hc = std::min<uint64_t>(lo + chunk_threads_, uint64_t(h.p_off) + h.p_cap);
          h_chunks_.push_back(make_int4(int(s), int(lo), int(std::max(hl, lo)), int(hc)));
        }
      }
      n_chunks_ = int(h_chunks_.size());
      chunk_first_[h_scenes_.size()] = n_chunks_;
      count_dirty_.assign(h_scenes_.size(), 0);
      any_count_dirty_ = false;
      if (n_chunks_ > n_chunks_alloc_) {
        dfree(d_chunks_);
        d_chunks_ = nullptr;
        dfree(partial_);
        partial_ = nullptr;
        AE_TRY(dmalloc(&d_chunks_, sizeof(int4) * n_chunks_));
        n_chunks_alloc_ = n_chunks_;
      }
      if (n_chunks_ > 0)
        AE_TRY(cudaMemcpyAsync(d_chunks_, h_chunks_.data(), sizeof(int4) * n_chunks_, cudaMemcpyHostToDevice, stream_));
      if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
      }
      chunks_dirty_ = false;
    } else if (any_count_dirty_) {
      // particle counts changed, the chunk layout (by capacity) did not: rewrite those scenes'
      // slices of the chunk table only
      for (size_t s = 0; s < h_scenes_.size(); ++s) {
        if (!count_dirty_[s]) continue;
        const SceneDev<T>& h = h_scenes_[s];
        const int c0 = chunk_first_[s], c1 = chunk_first_[s + 1];
        for (int c = c0; c < c1; ++c) {
          const uint64_t lo = uint64_t(h_chunks_[c].y);
          const uint64_t hl = std::min<uint64_t>(lo + chunk_threads_, uint64_t(h.p_off) + h.p_count);
          h_chunks_[c].z = int(std::max(hl, lo));
        }
        if (c1 > c0)
          AE_TRY(cudaMemcpyAsync(d_chunks_ + c0, h_chunks_.data() + c0, sizeof(int4) * (c1 - c0), cudaMemcpyHostToDevice,
                                 stream_));
        count_dirty_[s] = 0;
      }
      any_count_dirty_ = false;
      if (graph_) {  // a one-scene world's graph carries the count in its launch parameters
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
      }
    }
    int rc = sync_tables();
    if (rc) return rc;
    // the tables are copied from pageable host memory, which the copy stages before returning
    return AE_MPM_OK;
  }

  // scene and material tables to the device (copied from pageable memory, staged at the call)
  int sync_tables() {
    if (scenes_dirty_) {
      const size_t lo = std::min(scene_lo_, h_scenes_.size()), hi = std::min(scene_hi_, h_scenes_.size());
      if (hi > lo)
        AE_TRY(cudaMemcpyAsync(d_scenes_ + lo, h_scenes_.data() + lo, sizeof(SceneDev<T>) * (hi - lo),
                               cudaMemcpyHostToDevice, stream_));
      scenes_dirty_ = false;
      scene_lo_ = SIZE_MAX;
      scene_hi_ = 0;
    }
    if (mats_dirty_) {
      const size_t lo = std::min(mat_lo_, h_mats_.size()), hi = std::min(mat_hi_, h_mats_.size());
      if (hi > lo)
        AE_TRY(cudaMemcpyAsync(d_mats_ + lo, h_mats_.data() + lo, sizeof(MatDev) * (hi - lo), cudaMemcpyHostToDevice,
                               stream_));
      mats_dirty_ = false;
      mat_lo_ = SIZE_MAX;
      mat_hi_ = 0;
    }
    return AE_MPM_OK;
  }

  WorldDev<T> dev(bool sorted) {
    WorldDev<T> w{};
    w.scenes = d_scenes_;
    w.mats = d_mats_;
    w.chunks = d_chunks_;
    if (h_scenes_.size() == 1) {
      const SceneDev<T>& h = h_scenes_[0];
      w.one_scene = 1u;
      w.one_off = h.p_off;
      w.one_live_end = h.p_off + h.p_count;
      w.one_cap_end = h.p_off + h.p_cap;
    }
    for (int k = 0; k < 7; ++k) {
      w.in[k] = in_buf()[k];
      w.out[k] = out_buf()[k];
    }
    w.perm = sorted ? perm_ : nullptr;
    w.keys = keys_;
    w.acc = acc_;
    w.vel = vel_;
    w.blk_flag = blk_flag_;
    w.touched = touched_;
    w.touched_count = counters_;
    w.blk_scene = blk_scene_;
    w.err = err_;
    w.svd_fallback = opts_.svd_fp64_fallback;
    w.max_tile_nodes = max_tile_nodes();
    w.sorted_keys = sorted ? sorted_keys_ : nullptr;
    w.cell_slot = cell_slot_;
    w.cell_rec = cell_rec_;
    w.cell_count = opts_.deterministic ? counters_ + 1 : nullptr;
    w.seg_start = seg_start_;
    w.clamp_queue = clamp_queue_;
    w.clamp_count = counters_ + 3;
    return w;
  }

  int max_tile_nodes() const { return sizeof(T) == 4 ? 1024 : 512; }

  void launch_init_keys(WorldDev<T>& w) {
    if (n_chunks_ == 0) return;
    switch (mode_) {
      case AE_MPM_MODE_PHYSICS: init_keys_kernel<T, AE_MPM_MODE_PHYSICS><<<n_chunks_, chunk_threads_, 0, stream_>>>(w); break;
      case AE_MPM_MODE_REFERENCE: init_keys_kernel<T, AE_MPM_MODE_REFERENCE><<<n_chunks_, chunk_threads_, 0, stream_>>>(w); break;
      default: init_keys_kernel<T, AE_MPM_MODE_VELOCITY_ONLY><<<n_chunks_, chunk_threads_, 0, stream_>>>(w); break;
    }
    ++launches_;
  }

  template <int MODE>
  void launch_p2g(WorldDev<T>& w) {
    const size_t sm = sizeof(V4) * max_tile_nodes();
    if (MODE == AE_MPM_MODE_PHYSICS && opts_.p2g_variant == kVarLanes) {
      const size_t per = sizeof(V4) * kLaneVecs + sizeof(int4);
      const size_t sm2 = per * chunk_threads_;
      if (!lanes_smem_set_) {  // sized for the largest block (256 threads) the world accepts
        cudaFuncSetAttribute(p2g_lanes_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(per * 256));
        lanes_smem_set_ = true;
      }
      p2g_lanes_kernel<T><<<n_chunks_, chunk_threads_, sm2, stream_>>>(w);
      return;
    }
    if (MODE == AE_MPM_MODE_REFERENCE && opts_.p2g_variant == kVarLanes) {
      const size_t per = sizeof(V4) * kRefLaneVecs + sizeof(int4);
      if (!ref_lanes_smem_set_) {  // sized for the largest block (256 threads) the world accepts
        cudaFuncSetAttribute(p2g_lanes_ref_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(per * 256));
        ref_lanes_smem_set_ = true;
      }
      p2g_lanes_ref_kernel<T><<<n_chunks_, chunk_threads_, per * chunk_threads_, stream_>>>(w);
      return;
    }
    if (MODE == AE_MPM_MODE_VELOCITY_ONLY && opts_.p2g_variant == kVarLanes) {
      p2g_lanes_velonly_kernel<T><<<n_chunks_, chunk_threads_, velonly_lane_bytes<T>() * chunk_threads_, stream_>>>(w);
      return;
    }
    switch (opts_.p2g_variant) {
      case kVarWarpAgg: p2g_kernel<T, MODE, kVarWarpAgg><<<n_chunks_, chunk_threads_, sm, stream_>>>(w); break;
      case kVarGlobal: p2g_kernel<T, MODE, kVarGlobal><<<n_chunks_, chunk_threads_, 0, stream_>>>(w); break;
      default: p2g_kernel<T, MODE, kVarTile><<<n_chunks_, chunk_threads_, sm, stream_>>>(w); break;
    }
  }

  template <int MODE>
  void substep_mode(WorldDev<T>& w, bool write_keys) {
    const int sms = device_sm_count();
    if (opts_.deterministic) {
      det_heads_kernel<<<unsigned((total_cap_ + 255) / 256), 256, 0, stream_>>>(w.sorted_keys, total_cap_, dead_blk_,
                                                                                 cell_slot_, seg_start_, counters_ + 1);
      det_cellsum_kernel<T, MODE><<<sms * 8, 128, 0, stream_>>>(w, total_cap_);
      det_gather_kernel<T, MODE><<<sms * 8, 256, 0, stream_>>>(w, blk_epoch_, counters_ + 2);
      mark(2);
      det_reset_kernel<<<sms * 4, 256, 0, stream_>>>(seg_start_, w.sorted_keys, counters_ + 1, cell_slot_);
      launches_ += 4;
    } else {
      launch_p2g<MODE>(w);
      mark(2);
      grid_update_kernel<T, MODE><<<sms * 4, 256, 0, stream_>>>(w, blk_epoch_, counters_ + 2, nullptr);
      launches_ += 2;
    }
    mark(3);
    const size_t g2p_smem = sizeof(V4) * ((MODE == AE_MPM_MODE_PHYSICS ? 0 : max_tile_nodes()) + 3 * chunk_threads_);
    g2p_kernel<T, MODE><<<n_chunks_, chunk_threads_, g2p_smem, stream_>>>(w, counters_ + 2, write_keys ? 1 : 0);
    ++launches_;
    mark(5);  // the G2P kernel alone ends here
    if (MODE == AE_MPM_MODE_PHYSICS && has_snow_) {
      snow_clamp_kernel<T><<<sms * 8, 128, 0, stream_>>>(w);
      ++launches_;
    }
    mark(4);
  }

  void mark(int k) {
    if (stage_events_) cudaEventRecord(stage_events_[k], stream_);
  }

  // ranges of the scene and material tables to copy to the device before the next launch
  void dirty_scene(size_t s) {
    scene_lo_ = std::min(scene_lo_, s);
    scene_hi_ = std::max(scene_hi_, s + 1);
    scenes_dirty_ = true;
  }
  void dirty_mats(size_t s) {
    const size_t lo = h_scenes_[s].mat_off, hi = lo + descs_[s].n_materials + 1;
    mat_lo_ = std::min(mat_lo_, lo);
    mat_hi_ = std::max(mat_hi_, hi);
    mats_dirty_ = true;
  }

  void count_changed(uint32_t s) {
    dirty_scene(s);
    if (count_dirty_.size() != h_scenes_.size()) {
      chunks_dirty_ = true;  // no table yet: the next prepare() builds it whole
      return;
    }
    count_dirty_[s] = 1;
    any_count_dirty_ = true;
  }

  // ---- fused G2P + P2G (physics mode, column-lane P2G, not deterministic) ----
  // The P2G of substep s + 1 is done by the G2P of substep s, so between substeps the grid
  // accumulator holds the scatter of the current particle state ("queued"), on touched list
  // (s + 1) & 1.  Anything that changes the particles or the flow drops it; the next step()
  // scatters the current state once with the stand-alone P2G before its first substep.
  bool fused() const {
    return mode_ == AE_MPM_MODE_PHYSICS && !opts_.deterministic && opts_.p2g_variant == kVarLanes;
  }
  uint32_t* touched_list(int par) { return touched_ + size_t(par) * total_blocks_; }
  uint32_t* touched_count(int par) { return counters_ + (par ? 4 : 0); }
  WorldDev<T> with_list(WorldDev<T> w, int par) {
    w.touched = touched_list(par);
    w.touched_count = touched_count(par);
    return w;
  }
  static size_t fused_smem(int threads) { return warp_stage_bytes<T>() * size_t(threads / 32); }

  int sync_scatter() {
    const int par = int(substep_ & 1);
    if (fused() && !fused_smem_set_) {  // sized for the largest block (256 threads) the world accepts
      AE_TRY(cudaFuncSetAttribute(g2p2g_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(fused_smem(256))));
      AE_TRY(cudaFuncSetAttribute(snow_clamp_scatter_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(fused_smem(128))));
      fused_smem_set_ = true;
    }
    if (scatter_pending_ && (!fused() || scatter_invalid_)) {
      discard_scatter_kernel<T><<<device_sm_count() * 8, 64, 0, stream_>>>(acc_, blk_flag_, touched_list(par),
                                                                            touched_count(par));
      AE_TRY(cudaMemsetAsync(counters_, 0, sizeof(uint32_t), stream_));
      AE_TRY(cudaMemsetAsync(counters_ + 4, 0, sizeof(uint32_t), stream_));
      ++launches_;
      scatter_pending_ = false;
    }
    scatter_invalid_ = false;
    if (fused() && !scatter_pending_ && n_chunks_ > 0) {
      AE_TRY(cudaMemsetAsync(touched_count(par), 0, sizeof(uint32_t), stream_));
      WorldDev<T> w = with_list(dev(false), par);
      launch_p2g<AE_MPM_MODE_PHYSICS>(w);
      ++launches_;
      scatter_pending_ = true;
    }
    AE_TRY(cudaGetLastError());
    return AE_MPM_OK;
  }

  void substep_fused(WorldDev<T>& w, bool write_keys) {
    const int sms = device_sm_count();
    const int par = int(substep_ & 1);
    mark(2);  // no stand-alone P2G: the previous substep's G2P scattered this one
    WorldDev<T> wg = with_list(w, par);
    grid_update_kernel<T, AE_MPM_MODE_PHYSICS><<<sms * 4, 256, 0, stream_>>>(wg, blk_epoch_, counters_ + 2,
                                                                          touched_count(par ^ 1));
    mark(3);
    WorldDev<T> wf = with_list(w, par ^ 1);
    g2p2g_kernel<T><<<n_chunks_, chunk_threads_, fused_smem(chunk_threads_), stream_>>>(wf, counters_ + 2,
                                                                                         write_keys ? 1 : 0);
    launches_ += 2;
    mark(5);  // the fused kernel alone ends here
    if (has_snow_) {
      snow_clamp_scatter_kernel<T><<<sms * 8, 128, fused_smem(128), stream_>>>(wf);
      ++launches_;
    }
    mark(4);
  }

  void substep_eager() {
    const int interval = opts_.deterministic ? 1 : opts_.sort_interval;
    const bool do_sort = (substep_ % uint64_t(interval)) == 0;
    // G2P writes the cell keys only for a substep that sorts next; a sort whose keys were not
    // written by the G2P just before it (sort interval changed, first substep) computes them first
    const bool next_sorts = ((substep_ + 1) % uint64_t(interval)) == 0;
    if (n_chunks_ > 0) {
      mark(0);
      if (do_sort) {
        if (!keys_fresh_) {
          WorldDev<T> wk = dev(false);
          launch_init_keys(wk);
        }
        // keys of a small grid in a mode whose results do not depend on the order of equal keys:
        // one counting pass instead of two radix passes
        if (!opts_.deterministic && key_bits_ <= kCountingSortBits && total_cap_ > uint64_t(kSmallSortMax))
          launches_ += counting_sort_pairs(keys_, total_cap_, key_bits_, sort_, stream_, &sorted_keys_, &perm_);
        else
          launches_ += radix_sort_pairs(keys_, total_cap_, key_bits_, sort_, stream_, &sorted_keys_, &perm_);
      }
      mark(1);
      WorldDev<T> w = dev(do_sort);
      switch (mode_) {
        case AE_MPM_MODE_PHYSICS:
          if (fused())
            substep_fused(w, next_sorts);
          else
            substep_mode<AE_MPM_MODE_PHYSICS>(w, next_sorts);
          break;
        case AE_MPM_MODE_REFERENCE: substep_mode<AE_MPM_MODE_REFERENCE>(w, next_sorts); break;
        default: substep_mode<AE_MPM_MODE_VELOCITY_ONLY>(w, next_sorts); break;
      }
      keys_fresh_ = next_sorts || opts_.deterministic;
      a_in_ = !a_in_;
    }
    ++substep_;
  }

  int ensure_graph(uint64_t period) {
    if (graph_ && graph_period_ == period && graph_variant_ == opts_.p2g_variant) return AE_MPM_OK;
    if (graph_) {
      cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
    }
    const bool a_in0 = a_in_;
    const uint64_t sub0 = substep_, l0 = launches_;
    AE_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    for (uint64_t k = 0; k < period; ++k) substep_eager();
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    a_in_ = a_in0;
    substep_ = sub0;
    graph_launches_ = launches_ - l0;
    launches_ = l0;
    if (e != cudaSuccess) {
      err = std::string("stream capture failed: ") + cudaGetErrorString(e);
      return AE_MPM_ECUDA;
    }
    e = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      err = std::string("graph instantiation failed: ") + cudaGetErrorString(e);
      graph_ = nullptr;
      return AE_MPM_ECUDA;
    }
    graph_period_ = period;
    graph_variant_ = opts_.p2g_variant;
    return AE_MPM_OK;
  }

  void release() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (xfer_ev_) cudaEventDestroy(xfer_ev_);
    for (int k = 0; k < 7; ++k) {
      dfree(bufA_[k]);
      dfree(bufB_[k]);
      dfree(snap_[k]);
    }
    dfree(d_ptrA_);
    dfree(d_ptrB_);
    dfree(keys_);
    sort_scratch_free(sort_, alloc_ ? &World::sort_free : nullptr, alloc_);
    dfree(acc_);
    dfree(vel_);
    dfree(blk_flag_);
    dfree(blk_epoch_);
    dfree(touched_);
    dfree(counters_);
    dfree(err_);
    dfree(cell_slot_);
    dfree(seg_start_);
    dfree(cell_rec_);
    dfree(clamp_queue_);
    dfree(d_scenes_);
    dfree(d_mats_);
    dfree(blk_scene_);
    dfree(dead_blk_);
    dfree(d_chunks_);
    dfree(partial_);
    dfree(stage_);
    if (stream_) cudaStreamDestroy(stream_);
  }

 public:
  DevAlloc* alloc_ = nullptr;
  int mode_ = 0;
  ae_mpm_exec_opts opts_{};
  std::vector<ae_mpm_scene_desc> descs_;
  std::vector<std::vector<ae_mpm_material>> mats_;
  std::vector<SceneDev<T>> h_scenes_;
  std::vector<MatDev> h_mats_;
  std::vector<int4> h_chunks_;
  std::vector<int> chunk_first_;  // first chunk of each scene (and the chunk count at the end)
  std::vector<uint8_t> count_dirty_;  // scenes whose particle count changed since the table was written
  bool any_count_dirty_ = false;
  SceneDev<T>* d_scenes_ = nullptr;
  MatDev* d_mats_ = nullptr;
  int4* d_chunks_ = nullptr;
  int n_chunks_ = 0, n_chunks_alloc_ = 0, chunk_threads_ = 0;
  V4* bufA_[7] = {};
  V4* bufB_[7] = {};
  V4* snap_[7] = {};
  V4** d_ptrA_ = nullptr;
  V4** d_ptrB_ = nullptr;
  bool a_in_ = true;
  uint32_t* keys_ = nullptr;
  SortScratch sort_;
  const uint32_t* perm_ = nullptr;
  const uint32_t* sorted_keys_ = nullptr;
  V4* acc_ = nullptr;
  V4* vel_ = nullptr;
  uint32_t *blk_flag_ = nullptr, *blk_epoch_ = nullptr, *touched_ = nullptr, *blk_scene_ = nullptr, *dead_blk_ = nullptr;
  uint32_t* counters_ = nullptr;  // [touched count, cell count, epoch, snow clamp queue count]
  uint32_t* err_ = nullptr;
  uint32_t *cell_slot_ = nullptr, *seg_start_ = nullptr;
  V4* cell_rec_ = nullptr;
  uint2* clamp_queue_ = nullptr;
  bool has_snow_ = false;
  T* stage_ = nullptr;
  size_t stage_bytes_ = 0;
  double* partial_ = nullptr;
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  uint64_t graph_period_ = 0, graph_launches_ = 0;
  int graph_variant_ = -1;
  bool lanes_smem_set_ = false, fused_smem_set_ = false, ref_lanes_smem_set_ = false;
  bool scatter_pending_ = false;  // the accumulator holds the P2G of the current particle state
  bool scatter_invalid_ = false;  // the particles changed since that scatter
  uint64_t substep_ = 0, snap_substep_ = 0, launches_ = 0;
  cudaEvent_t* stage_events_ = nullptr;
  cudaEvent_t xfer_ev_ = nullptr;  // orders copy streams against the world's stream
  uint64_t total_cap_ = 0, total_blocks_ = 0, device_bytes_ = 0;
  int key_bits_ = 1;
  bool keys_stale_ = true, chunks_dirty_ = true, scenes_dirty_ = true, mats_dirty_ = false;
  size_t scene_lo_ = 0, scene_hi_ = SIZE_MAX;  // dirty range of the scene table (all of it at first)
  size_t mat_lo_ = SIZE_MAX, mat_hi_ = 0;       // dirty range of the material table
  bool keys_fresh_ = false;  // keys_ hold the cell keys of the current positions
};

WorldBase* make_world(const ae_mpm_scene_desc* scenes, uint32_t n_scenes, const ae_mpm_exec_opts& opts, std::string& why,
                      int* status, DevAlloc* alloc) {
  size_t free0 = 0, total = 0;
  cudaMemGetInfo(&free0, &total);
  WorldBase* w = nullptr;
  int rc;
  if (opts.precision == 64) {
    auto* x = new World<double>();
    x->alloc_ = alloc;
    rc = x->init(scenes, n_scenes, opts);
    w = x;
  } else {
    auto* x = new World<float>();
    x->alloc_ = alloc;
    rc = x->init(scenes, n_scenes, opts);
    w = x;
  }
  if (rc != AE_MPM_OK) {
    why = w->err;
    delete w;
    if (status) *status = rc;
    return nullptr;
  }
  size_t free1 = 0;
  cudaMemGetInfo(&free1, &total);
  if (opts.precision == 64)
    static_cast<World<double>*>(w)->device_bytes_ = free0 > free1 ? free0 - free1 : 0;
  else
    static_cast<World<float>*>(w)->device_bytes_ = free0 > free1 ? free0 - free1 : 0;
  if (status) *status = AE_MPM_OK;
  return w;
}

}  // namespace aemp
