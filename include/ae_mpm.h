/*
 * ae_mpm.h -- C ABI of the B200 (sm_100a) MPM substep library `libae_mpm.so`.
 *
 * This is the drop-in boundary for AE-ENGINE's engine-driven MPM substep.  The engine calls
 *   ae_particle::mpm_solver::mpm_step_parallel_with_grid   (ae_particle/src/mpm_solver.rs:1063-1084)
 * from SimulationManager::update_fields_and_particles      (ae_engine/src/managers/simulation.rs:573-581)
 * and the mid-field LOD tier calls
 *   ae_particle::mpm_solver::mpm_step_velocity_only_parallel (ae_particle/src/mpm_solver.rs:1337-1351).
 * A Rust FFI crate binds these entry points exactly as ae_cpp_kernel binds its C++ kernel
 * (ae_cpp_kernel/src/lib.rs:21-32): raw pointers into the caller's SoA `Vec`s plus counts,
 * no Rust or torch types.  Unlike that template every call returns a status code.
 *
 * Besides the drop-in calls the library keeps scenes resident in HBM ("worlds": one or more
 * independent scenes stepped in lockstep by the same kernels), and runs a continuous-batching
 * server on top of worlds.  Nothing here allocates on the caller's behalf except through the
 * create functions, and every pointer argument is borrowed for the duration of the call only.
 *
 * Threading: an ae_mpm_ctx, and every world or server made from it, must be used from one host
 * thread at a time.  Work is queued on library-owned CUDA streams.
 */
#ifndef AE_MPM_H
#define AE_MPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AE_MPM_ABI_VERSION 1

/* ---- status codes (every function returns one; the message is in ae_mpm_last_error) ---- */
enum {
  AE_MPM_OK = 0,
  AE_MPM_EINVAL = 1,    /* bad argument (the reference panics or misbehaves instead)        */
  AE_MPM_ENOMEM = 2,    /* device or pinned host allocation failed                          */
  AE_MPM_ENAN = 3,      /* a particle position became non-finite on the device              */
  AE_MPM_ETIMEOUT = 4,  /* a bounded wait ran out (server wait, world sync with a deadline)  */
  AE_MPM_EBUDGET = 5,   /* admission refused: the scene does not fit the HBM budget          */
  AE_MPM_ECUDA = 6,     /* a CUDA runtime call failed                                       */
  AE_MPM_EDOMAIN = 7,   /* particles reached the grid's outer ring and were clamped back    */
  AE_MPM_ENOTFOUND = 8, /* unknown scene or request id                                      */
  AE_MPM_EAGAIN = 9     /* nothing ready yet (server poll)                                  */
};

/* ---- constitutive models ----
 * 0..6 are ae_particle::constitutive::ConstitutiveModel in declaration order
 * (ae_particle/src/constitutive.rs:12-27); they give Cauchy stress in the reference substep.
 * 16..18 are the physics-mode materials of the MLS-MPM substep:
 *   16 neo-Hookean jelly   tau = mu (F F^T - I) + lambda ln(J) I     (ae_physics/src/mpm.rs:429-454)
 *   17 Stomakhin snow      neo-Hookean on F_E, singular values of F_E clamped to
 *                          [1-theta_c, 1+theta_s] (ae_physics/src/mpm.rs:565-606), mu and lambda
 *                          scaled by exp(xi (1 - J_p)) (Stomakhin et al. 2013)
 *   18 J-only fluid        tau = K (J - 1) I, J <- J (1 + dt tr C)   (ae_compute/src/mpm_compute.rs:287-291,453-457)
 */
enum {
  AE_MPM_NEO_HOOKEAN = 0,
  AE_MPM_DRUCKER_PRAGER = 1,
  AE_MPM_VON_MISES = 2,
  AE_MPM_NEWTONIAN_FLUID = 3,
  AE_MPM_COROTATED = 4,
  AE_MPM_FIXED_COROTATED = 5,
  AE_MPM_RIGID = 6,
  AE_MPM_PHYS_JELLY = 16,
  AE_MPM_PHYS_SNOW = 17,
  AE_MPM_PHYS_FLUID = 18
};

/* ---- substep flavours ---- */
enum {
  /* MLS-MPM (Hu et al. 2018) with nodes at integer i*dx, base = floor(x/dx - 0.5), full F,
   * physics-mode materials and 3-cell walls (ae_compute/src/mpm_compute.rs:128-459 stencil). */
  AE_MPM_MODE_PHYSICS = 0,
  /* Bug-for-bug restatement of ae_particle::mpm_solver::mpm_substep_serial_active /
   * mpm_substep_parallel_with_indices (ae_particle/src/mpm_solver.rs:812-1054, 1088-1326):
   * nodes at (g+0.5)*dx, stencil g..g+2, reference Cauchy-stress models, floor-only grid rule,
   * particle wall clamps with x0.5 restitution, |v|<=50 clamp, NaN guards, damping. */
  AE_MPM_MODE_REFERENCE = 1,
  /* ae_particle::mpm_solver::mpm_substep_velocity_only (ae_particle/src/mpm_solver.rs:1353-1572). */
  AE_MPM_MODE_VELOCITY_ONLY = 2
};

/* ---- grid wall handling in physics mode ---- */
enum {
  AE_MPM_WALL_STICKY = 0, /* every velocity component zeroed on nodes within `wall_margin` of a face */
  AE_MPM_WALL_SLIP = 1    /* ae_compute rule (mpm_compute.rs:364-383): the outward normal component
                             is reflected with `restitution` */
};

/* Material parameters.  The first seven fields are ae_particle::constitutive::MaterialParams
 * (ae_particle/src/constitutive.rs:31-40) in order; mu/lambda/K derive from them exactly as
 * MaterialParams::{mu,lambda,bulk_modulus} (constitutive.rs:55-82, poisson_ratio clamped to
 * [-0.999, 0.4999]).  The trailing fields are used by the physics-mode materials only. */
typedef struct ae_mpm_material {
  float young_modulus;  /* E (Pa)                                  */
  float poisson_ratio;  /* nu                                      */
  float yield_stress;   /* sigma_y (Pa)                            */
  float hardening;      /* isotropic hardening coefficient         */
  float density;        /* rho (kg/m^3); particle volume = m / rho */
  float friction_angle; /* phi (degrees), Drucker-Prager           */
  float cohesion;       /* c (Pa), Drucker-Prager                  */
  int32_t model;        /* one of the AE_MPM_* model values above  */
  float theta_c;        /* snow critical compression (2.5e-2)      */
  float theta_s;        /* snow critical stretch (7.5e-3)          */
  float hardening_xi;   /* snow hardening exponent xi (10)         */
  float bulk_modulus;   /* fluid K; <= 0 means E / (3 (1 - 2 nu))  */
} ae_mpm_material;

/* ae_particle::mpm_solver::MpmConfig (ae_particle/src/mpm_solver.rs:46-55), field for field. */
typedef struct ae_mpm_config {
  float grid_dx;
  uint64_t grid_size[3];
  uint64_t substeps;
  float gravity[3];
  float damping;
  uint8_t enable_plasticity;
  uint8_t enable_contact;
  uint8_t use_sparse_grid;
} ae_mpm_config;

/* The parts of ae_particle::mpm_solver::Grid (mpm_solver.rs:73-86) that a substep reads:
 * node counts, spacing and the moving-window origin.  The node arrays themselves live on the
 * device; ae_mpm_grid_download copies mass and velocity back when a caller wants them. */
typedef struct ae_mpm_grid {
  uint64_t nx, ny, nz;
  float dx;
  float origin[3];
} ae_mpm_grid;

/* Borrowed views of the MPM fields of ae_particle::mpss::MpssBuffer (ae_particle/src/mpss.rs:105-157),
 * in its strides: pos/vel are [f32;3] per particle, strain (F) and c (APIC C) are row-major [f32;9].
 * In physics mode `jacobian` carries det F for jelly, J for fluid and the plastic J_p for snow. */
typedef struct ae_mpm_particles {
  float* pos;
  float* vel;
  float* strain;
  float* jacobian;
  float* c;
  float* mass;
  uint16_t* material_idx;
} ae_mpm_particles;

/* Same view in double precision, for FP64 worlds (error reference runs of the same kernels). */
typedef struct ae_mpm_particles_f64 {
  double* pos;
  double* vel;
  double* strain;
  double* jacobian;
  double* c;
  double* mass;
  uint16_t* material_idx;
} ae_mpm_particles_f64;

/* One scene of a world. */
typedef struct ae_mpm_scene_desc {
  int32_t mode;          /* AE_MPM_MODE_*                                         */
  uint32_t n[3];         /* grid nodes per axis (each >= 4)                        */
  float dx;              /* node spacing                                          */
  float origin[3];       /* world position of node (0,0,0) (ref: minus 0.5 dx)     */
  float gravity[3];
  float dt;              /* substep length                                        */
  int32_t wall_mode;     /* physics mode: AE_MPM_WALL_*                            */
  int32_t wall_margin;   /* physics mode: cells of wall at each face (3)           */
  float restitution;     /* physics mode, slip walls                              */
  float damping;         /* reference modes: velocity damping (0.995)             */
  int32_t wall_origin;   /* reference modes: 1 = particle walls offset by origin
                            (parallel path, mpm_solver.rs:1290-1297), 0 = walls at 0
                            (serial path, mpm_solver.rs:998-1015)                  */
  uint32_t n_materials;
  const ae_mpm_material* materials; /* indexed by particle material_idx; an index past the end
                                       uses materials[0] (mpm_solver.rs:840-841)          */
  uint64_t max_particles;
} ae_mpm_scene_desc;

/* Execution options of a world. */
/* P2G variants: TILE = per-particle shared-tile atomics; WARP_AGG = same-cell runs reduced with
 * __match_any_sync + shuffles first; GLOBAL = vector atomics straight to HBM; LANES = warp walks
 * its sorted particles with one lane per stencil node (physics mode; others use TILE). */
enum { AE_MPM_P2G_AUTO = 0, AE_MPM_P2G_TILE = 1, AE_MPM_P2G_WARP_AGG = 2, AE_MPM_P2G_GLOBAL = 3, AE_MPM_P2G_LANES = 4 };
typedef struct ae_mpm_exec_opts {
  int32_t precision;      /* 32 or 64                                                        */
  int32_t deterministic;  /* 1: fixed-order segmented sums, no float atomics (bitwise replay) */
  int32_t sort_interval;  /* radix sort every k substeps (>=1; deterministic mode forces 1)   */
  int32_t p2g_variant;    /* AE_MPM_P2G_*; AUTO takes the autotuned choice                    */
  int32_t block_threads;  /* particles per P2G/G2P block (128 or 256); 0 = autotuned          */
  int32_t use_graph;      /* 1: replay substeps from a captured CUDA graph                    */
  int32_t track_totals;   /* 1: accumulate FP64 mass/momentum totals every substep            */
  int32_t svd_fp64_fallback; /* 1 (default): snow SVD redone in FP64 near degenerate sigma    */
} ae_mpm_exec_opts;

typedef struct ae_mpm_ctx ae_mpm_ctx;
typedef struct ae_mpm_world ae_mpm_world;
typedef struct ae_mpm_server ae_mpm_server;

/* ---------------------------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------------------------- */
int ae_mpm_ctx_create(int device, ae_mpm_ctx** out);
void ae_mpm_ctx_destroy(ae_mpm_ctx* ctx);
/* Text of the last failure on this context (never NULL). */
const char* ae_mpm_last_error(const ae_mpm_ctx* ctx);
/* Fills the default execution options (autotuned fields left at 0). */
void ae_mpm_exec_opts_default(ae_mpm_exec_opts* opts);
int ae_mpm_abi_version(void);

/* ---------------------------------------------------------------------------------------------
 * Drop-in entry points (host buffers in the reference's layout; state copied in, stepped on the
 * device, copied back).  `capacity` is the length of the MpssBuffer arrays; `particle_indices`
 * select the particles to step, as in the reference.  The reference's trailing
 * buffer.update_lifetimes(total_dt) (mpm_solver.rs:1083) manipulates the MpssBuffer free list and
 * stays with the host wrapper.  An empty index list returns AE_MPM_OK without touching anything
 * (mpm_solver.rs:1072-1074).  An empty material table is AE_MPM_EINVAL (the reference panics at
 * material_table[0], mpm_solver.rs:840).
 * ------------------------------------------------------------------------------------------- */

/* Replaces mpm_step_parallel_with_grid (ae_particle/src/mpm_solver.rs:1063-1084): config.substeps
 * substeps of total_dt/config.substeps, each the serial-path rules below 50 000 particles and the
 * parallel-path rules at or above (mpm_solver.rs:1077). */
int ae_mpm_step_parallel_with_grid(ae_mpm_ctx* ctx, const ae_mpm_particles* buffer,
                                   uint64_t capacity, const ae_mpm_grid* grid,
                                   const ae_mpm_config* config,
                                   const ae_mpm_material* material_table, uint32_t n_materials,
                                   const int32_t* model_table, uint32_t n_models,
                                   float total_dt, const uint64_t* particle_indices,
                                   uint64_t n_indices);

/* Replaces mpm_step_velocity_only_parallel (ae_particle/src/mpm_solver.rs:1337-1351). */
int ae_mpm_step_velocity_only_parallel(ae_mpm_ctx* ctx, const ae_mpm_particles* buffer,
                                       uint64_t capacity, const ae_mpm_grid* grid,
                                       const ae_mpm_config* config, float total_dt,
                                       const uint64_t* particle_indices, uint64_t n_indices);

/* Grid mass and velocity (after the grid update of the last substep of the last drop-in call),
 * dense in the reference's index order i + j*nx + k*nx*ny (mpm_solver.rs:157-159).
 * mass: nx*ny*nz floats; vel: nx*ny*nz*3 floats. */
int ae_mpm_grid_download(ae_mpm_ctx* ctx, float* mass, float* vel, uint64_t n_nodes);

/* ---------------------------------------------------------------------------------------------
 * Device-resident worlds: one or more independent scenes stepped in lockstep by one set of
 * launches (the batched path).  A world with one scene is the plain path.
 * ------------------------------------------------------------------------------------------- */
int ae_mpm_world_create(ae_mpm_ctx* ctx, const ae_mpm_scene_desc* scenes, uint32_t n_scenes,
                        const ae_mpm_exec_opts* opts, ae_mpm_world** out);
int ae_mpm_world_destroy(ae_mpm_world* world);
/* Copy n particles (indices 0..n-1 of the view) into scene `scene`; n <= max_particles.
 * The view's arrays may be host memory or memory of the world's device.
 * The _f64 variants are for precision-64 worlds. */
int ae_mpm_world_upload(ae_mpm_world* world, uint32_t scene, const ae_mpm_particles* host, uint64_t n);
int ae_mpm_world_upload_f64(ae_mpm_world* world, uint32_t scene, const ae_mpm_particles_f64* host, uint64_t n);
/* Change a resident scene's dt, gravity, walls, damping, origin or material parameters (grid size
 * and material count stay), e.g. a CFL-adapted dt per frame as the reference's total_dt per call. */
int ae_mpm_world_set_scene(ae_mpm_world* world, uint32_t scene, const ae_mpm_scene_desc* desc);
/* Queue n substeps of every scene (asynchronous; returns after queueing). */
int ae_mpm_world_step(ae_mpm_world* world, uint32_t n_substeps);
/* Wait for queued work; returns AE_MPM_ENAN / AE_MPM_EDOMAIN if a scene raised its error word. */
int ae_mpm_world_sync(ae_mpm_world* world);
/* Copy scene particles back in their upload order (into host memory or memory of the world's device). */
int ae_mpm_world_download(ae_mpm_world* world, uint32_t scene, ae_mpm_particles* host);
int ae_mpm_world_download_f64(ae_mpm_world* world, uint32_t scene, ae_mpm_particles_f64* host);
/* Many scenes in one call (f32 worlds; no counterpart in the reference, whose engine moves one
 * MpssBuffer per call).  upload_many copies counts[i] particles of views[i] into scene scenes[i]
 * for i < n, as n calls of ae_mpm_world_upload would, but queues every host-to-device copy back
 * to back through one device staging area before unpacking, so pinned views (best laid out as
 * pos 3n | vel 3n | strain 9n | jacobian n | c 9n | mass n floats, then n u16 material indices,
 * which travels in one copy) stream at link speed; asynchronous like ae_mpm_world_upload.
 * download_many copies scene scenes[i] back into views[i] the same way and returns once all of
 * them are in place. */
int ae_mpm_world_upload_many(ae_mpm_world* world, uint32_t n, const uint32_t* scenes,
                             const ae_mpm_particles* views, const uint64_t* counts);
int ae_mpm_world_download_many(ae_mpm_world* world, uint32_t n, const uint32_t* scenes, ae_mpm_particles* views);

/* ---------------------------------------------------------------------------------------------
 * Pipelined batch (no counterpart in the reference): scenes that live in host memory, advanced
 * n_substeps per call with the PCIe copies hidden behind the substeps.  ae_mpm_batch_create
 * splits the n_scenes scenes into n_groups consecutive groups of about equal particle capacity
 * (max_particles), one f32 world each (opts as for ae_mpm_world_create; precision 64 is
 * AE_MPM_EINVAL; n_groups is clamped to 1..n_scenes).  ae_mpm_batch_run copies counts[i]
 * particles of in[i] into scene i, runs every group n_substeps substeps and writes each scene's
 * particles into out[i] (out may be in): group g's inputs cross while group g - 1 computes, and
 * its results cross back while group g + 1 computes, so a call costs about the substeps of all
 * groups plus one group's copies each way.  Host views should be pinned (page-locked) memory
 * for the copies to overlap.  Groups compute one after another, each scene's results the same
 * as in one world of all scenes (bitwise so in deterministic mode).  Returns once every result
 * is in place; an error word of any group (AE_MPM_ENAN, AE_MPM_EDOMAIN) is returned after all
 * results are written.  ae_mpm_batch_groups writes the first scene of every group and then
 * n_scenes into first_scene (n_groups + 1 entries) when it is not null, and returns n_groups. */
typedef struct ae_mpm_batch ae_mpm_batch;
int ae_mpm_batch_create(ae_mpm_ctx* ctx, const ae_mpm_scene_desc* scenes, uint32_t n_scenes,
                        const ae_mpm_exec_opts* opts, uint32_t n_groups, ae_mpm_batch** out);
int ae_mpm_batch_run(ae_mpm_batch* batch, const ae_mpm_particles* in, const uint64_t* counts, ae_mpm_particles* out,
                     uint32_t n_substeps);
uint32_t ae_mpm_batch_groups(const ae_mpm_batch* batch, uint32_t* first_scene);
/* The grouping ae_mpm_batch_create uses, on the host (no device needed): writes the first scene
 * of each of the min(max(n_groups, 1), n_scenes) groups and then n_scenes into first_scene
 * (n_scenes + 1 entries suffice) for scenes of the given particle capacities, and returns the
 * group count (0 for no scenes or null arrays). */
uint32_t ae_mpm_batch_partition(const uint64_t* capacities, uint32_t n_scenes, uint32_t n_groups,
                                uint32_t* first_scene);
int ae_mpm_batch_destroy(ae_mpm_batch* batch);
/* FP64 totals of a scene: [mass, px, py, pz, kinetic energy] of its particles, now. */
int ae_mpm_world_totals(ae_mpm_world* world, uint32_t scene, double out[5]);
/* Per-scene error word (bit 0 NaN, bit 1 domain clamp) and counters
 * [svd_fp64_fallbacks, domain_clamps, tile_overflow_blocks]; clears them. */
int ae_mpm_world_errors(ae_mpm_world* world, uint32_t scene, uint32_t* error_word, uint64_t counters[3]);
/* Number of kernels the last ae_mpm_world_step queued (graph nodes count as launches). */
int ae_mpm_world_launch_count(const ae_mpm_world* world, uint64_t* launches);
/* Runs n substeps eagerly with CUDA events between the stages on the world's stream and returns
 * the mean device time per substep of each stage in microseconds:
 * out_us = [sort, P2G (deterministic: cell sums + gather), grid update, G2P, whole substep]. */
int ae_mpm_world_stage_times(ae_mpm_world* world, uint32_t n_substeps, double out_us[5]);
/* The same measurement with a sixth entry: out_us[5] = the G2P kernel alone (in physics mode with
 * the column-lane P2G, the fused G2P + P2G kernel alone), without the snow clamp that out_us[3]
 * includes. */
int ae_mpm_world_stage_times_split(ae_mpm_world* world, uint32_t n_substeps, double out_us[6]);
/* CUDA stream the world queues on (cudaStream_t), so callers can time it with events. */
void* ae_mpm_world_stream(ae_mpm_world* world);
/* Particle count of every scene summed. */
uint64_t ae_mpm_world_particles(const ae_mpm_world* world);
/* Particle count of scene `scene` (0 for an unknown scene): the number of particles a download
 * of it writes, so the caller's arrays must hold at least that many. */
uint64_t ae_mpm_world_scene_particles(const ae_mpm_world* world, uint32_t scene);

/* ---------------------------------------------------------------------------------------------
 * Radix sort by cell key, exposed for parity testing: stable ascending sort of n 32-bit keys
 * (only the low `key_bits` bits are compared).  Host buffers.  perm_out[i] = index of the i-th
 * smallest key; equal keys keep their input order.
 * ------------------------------------------------------------------------------------------- */
int ae_mpm_radix_sort_keys(ae_mpm_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t key_bits,
                           uint32_t* sorted_keys_out, uint32_t* perm_out);

/* The grouping sort that non-deterministic worlds with keys of at most 16 bits use (a 32^3 grid):
 * one histogram, one scan and one scatter instead of radix passes.  Same buffers as
 * ae_mpm_radix_sort_keys; sorted_keys_out comes out ascending, but equal keys in no defined order,
 * and perm_out is a permutation with keys[perm_out[i]] == sorted_keys_out[i].  Up to 16384 keys the
 * call sorts stably in one CTA.  key_bits above 16 is AE_MPM_EINVAL.  No reference counterpart. */
int ae_mpm_counting_sort_keys(ae_mpm_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t key_bits,
                              uint32_t* sorted_keys_out, uint32_t* perm_out);

/* The same sort for callers that cannot allocate GPU memory: an engine frame loop living on
 * memory it reserved up front, work queued during CUDA stream capture, a host whose own pool owns
 * all of HBM.  This entry point has no counterpart in the reference.  keys_dev, sorted_keys_dev
 * and perm_dev are device buffers the caller owns; the scratch is a fixed array compiled into the
 * library (about 9 MB per GPU that loads it, held until exit), so at most
 * AE_MPM_NOALLOC_MAX_KEYS keys are accepted and larger n is AE_MPM_EINVAL.  Nothing is allocated
 * or freed.  The work is queued on `stream` (a cudaStream_t; NULL = default stream).  ctx may be
 * NULL; when given, its device is made current and failures leave their text in it.  The first
 * call on a device looks up the array's device address, so make that first call before any stream
 * capture; the address is kept for the life of the process, so a device that was reset
 * (cudaDeviceReset) must not be given to this call again.  All calls on a device share the
 * scratch: calls whose work overlaps on the GPU race.  keys_dev, sorted_keys_dev and perm_dev
 * must not overlap (AE_MPM_EINVAL otherwise): no in-place sort. */
#define AE_MPM_NOALLOC_MAX_KEYS (1u << 20)
int ae_mpm_radix_sort_keys_noalloc(ae_mpm_ctx* ctx, const uint32_t* keys_dev, uint64_t n, uint32_t key_bits,
                                   uint32_t* sorted_keys_dev, uint32_t* perm_dev, void* stream);

/* ---------------------------------------------------------------------------------------------
 * The engine tick's particle passes around the substep (ae_engine/src/managers/simulation.rs,
 * SimulationManager::update_fields_and_particles).  Arrays are MpssBuffer's: pos and vel are
 * count x 3 floats, temperature and mass count floats, active count bytes (0/1; NULL = all
 * active).  Index lists are usize (uint64).  The pointers of one call are either all host memory
 * (staged through the context) or all device memory (used in place, no copies); which one is
 * decided from `pos`.  Results equal the reference's f32 arithmetic bit for bit (the order of the
 * near list aside, below).
 * ------------------------------------------------------------------------------------------- */

/* LOD classification, simulation.rs:495-532 (the reclassify branch; its Vec<(usize, f32)> /
 * Vec<usize> lists become near_out / mid_out / far_out, each with room for count entries).
 * near: active particles with |pos - player|^2 < near_dist^2, capped to the max_near closest, in
 * ascending index order (the reference's select_nth_unstable_by leaves their order unspecified; on
 * equal distances at the cap the lower index stays near).  mid: |pos - player|^2 < mid_dist^2, in
 * ascending index order, followed by the near particles over the cap in ascending index order.
 * far: the rest, ascending. */
int ae_mpm_lod_classify(ae_mpm_ctx* ctx, const float* pos, const uint8_t* active, uint64_t count,
                        const float player[3], float near_dist, float mid_dist, uint64_t max_near,
                        uint64_t* near_out, uint64_t* n_near, uint64_t* mid_out, uint64_t* n_mid,
                        uint64_t* far_out, uint64_t* n_far);

/* Far-field update, simulation.rs:612-679: for each far particle v.y -= 9.81 far_dt,
 * pos.y += v.y far_dt, and its temperature relaxes (rate 0.02 far_dt) toward the nearest cell
 * ((pos - origin) / dx truncated toward zero) of the coarse_n^3 coarse temperature field (x
 * fastest) when that cell exists.  Host indices are checked against count (AE_MPM_EINVAL). */
int ae_mpm_far_field_update(ae_mpm_ctx* ctx, float* pos, float* vel, float* temperature, uint64_t count,
                            const uint64_t* far_idx, uint64_t n_far, const float* coarse_temperature,
                            uint32_t coarse_n, float coarse_dx, const float coarse_origin[3], float far_dt);

/* Coarse temperature field update, SimulationManager::update_coarse_field (simulation.rs:877-966):
 * mass-weighted temperature of the active near particles per cell, relaxation of the field toward
 * it (rate min(0.1 dt, 1)), then one 6-neighbour FTCS diffusion step (coefficient
 * min(10 dt / dx^2, 0.16)).  coarse_temperature (coarse_n^3 floats) is updated in place.  Host
 * indices are checked against count (AE_MPM_EINVAL). */
int ae_mpm_coarse_field_update(ae_mpm_ctx* ctx, const float* pos, const float* mass, const float* temperature,
                               const uint8_t* active, uint64_t count, const uint64_t* near_idx, uint64_t n_near,
                               float* coarse_temperature, uint32_t coarse_n, float coarse_dx,
                               const float coarse_origin[3], float dt);

/* MpssBuffer housekeeping after the substep, the three calls of ae_engine/src/lib.rs:347-358 in
 * their order, over particles 0..count (active ones only):
 *   passes & 1  MpssBuffer::apply_boundary_conditions_par (ae_particle/src/mpss.rs:449-476): a
 *               coordinate outside [bounds_min, bounds_max] is clamped and its velocity component,
 *               when it points outward, reversed and halved;
 *   passes & 2  MpssBuffer::clamp_temperatures_par (mpss.rs:479-497) to [min_temp, max_temp];
 *   passes & 4  MpssBuffer::apply_phase_transitions_par (mpss.rs:500-548): material 1 water, 3
 *               iron, 0 wood, 2 concrete, up to 3 hops; phase holds MpssPhase values (Solid 0,
 *               Liquid 1, Gas 2, ...) as bytes, material_idx MpssBuffer::material_idx.
 * *transitions receives the number of particles whose phase changed (the u32 the reference
 * returns).  pos/vel are count x 3 floats.  Host or device pointers, as above (decided by pos). */
int ae_mpm_mpss_housekeeping(ae_mpm_ctx* ctx, float* pos, float* vel, float* temperature, uint8_t* phase,
                             const uint16_t* material_idx, const uint8_t* active, uint64_t count,
                             const float bounds_min[3], const float bounds_max[3], float min_temp, float max_temp,
                             uint32_t passes, uint32_t* transitions);

/* ---------------------------------------------------------------------------------------------
 * CK-MPM, the compact-kernel MPM solver (ae_compute/src/ck_mpm.rs, CkMpmSolver): C^2 kernel
 * w(x) = (1 - (x/h)^2)^3 / h on the 2 nodes per axis around a particle (nodes at (i + 1/2) h,
 * i = floor(x/h) + {0, 1}, 0 <= i < grid_n), APIC transfer, neo-Hookean forces, guarded grid and
 * particle updates.  Particles are CkMpmParticle records; matrices are glam Mat3, column-major.
 * The particle pointer of a call is host memory (staged through the context) or device memory
 * (updated in place); which one is decided from the pointer.
 * ------------------------------------------------------------------------------------------- */
typedef struct ae_mpm_ck_config {  /* CkMpmConfig, ck_mpm.rs:41-59                          */
  float dt;
  float grid_h;
  uint32_t grid_n;                 /* usize in the reference; at most 1024 here            */
  float gravity[3];
  float youngs_modulus;
  float poissons_ratio;
  float density;                   /* carried, read by no step (as in the reference)       */
  float bounds_min[3];
  float bounds_max[3];
  float restitution;
  uint8_t dual_grid;               /* carried, read by no step (as in the reference)       */
  uint8_t pad[3];
} ae_mpm_ck_config;

typedef struct ae_mpm_ck_particle {  /* CkMpmParticle, ck_mpm.rs:84-95; 104 bytes            */
  float position[3];
  float velocity[3];
  float affine[9];                   /* APIC matrix B, columns x_axis, y_axis, z_axis         */
  float deformation[9];              /* deformation gradient F, same layout                   */
  float rest_volume;
  float mass;
} ae_mpm_ck_particle;

typedef struct ae_mpm_ck_stats {
  float kinetic_energy;        /* CkMpmSolver::kinetic_energy, ck_mpm.rs:484-486        */
  float average_velocity[3];   /* CkMpmSolver::average_velocity, :489-494               */
  float average_volume_ratio;  /* CkMpmSolver::average_volume_ratio, :497-503           */
} ae_mpm_ck_stats;

/* CkMpmConfig::default() (ck_mpm.rs:61-77). */
void ae_mpm_ck_config_default(ae_mpm_ck_config* out);

/* `steps` calls of CkMpmSolver::step (ck_mpm.rs:187-480) over particles[0..n), in place.  Each
 * particle's contribution to a node and each particle update from the node velocities round as
 * the reference's f32 arithmetic does; node sums are accumulated in atomic order (not particle
 * order), so results agree with the reference to rounding, not bit for bit, where several
 * particles share a node.  Invalid: null config, grid_n > 1024 (AE_MPM_EINVAL). */
int ae_mpm_ck_step(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config* config,
                   uint32_t steps);

/* ae_mpm_ck_step with CUDA events around each kernel: kernel_ms[0] receives the summed duration
 * of the particle kernels (G2P fused with the next step's P2G and force scatter), kernel_ms[1]
 * that of the grid kernels (touched-block compaction and grid update), in milliseconds. */
int ae_mpm_ck_step_timed(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n, const ae_mpm_ck_config* config,
                         uint32_t steps, double kernel_ms[2]);

/* ae_mpm_ck_step with each node's sums added in particle order, as the reference's serial loops
 * add them (a per-node merge over particles sorted by cell instead of atomics): results are the
 * same bits on every run, and equal the reference's bit for bit wherever ln(det F) agrees (the
 * device takes the correctly rounded logarithm; glibc's logf differs from it by one ulp for a few
 * percent of arguments).  Slower than ae_mpm_ck_step; at most 2^32 - 1 particles, and
 * (grid_n + 1)^3 x 8 bytes of cell table on the device. */
int ae_mpm_ck_step_deterministic(ae_mpm_ctx* ctx, ae_mpm_ck_particle* particles, uint64_t n,
                                 const ae_mpm_ck_config* config, uint32_t steps);

/* The solver's diagnostics over particles[0..n), summed on the device in double precision;
 * n = 0 gives 0, (0, 0, 0) and 1, as the reference's empty-solver cases do. */
int ae_mpm_ck_stats_compute(ae_mpm_ctx* ctx, const ae_mpm_ck_particle* particles, uint64_t n,
                            ae_mpm_ck_stats* out);

/* CkMpmSolver::weight and weight_grad (ck_mpm.rs:163-185) at x[0..n) with support h, evaluated
 * by the device code the solver uses.  Host or device arrays (decided from x). */
int ae_mpm_ck_weights(ae_mpm_ctx* ctx, const float* x, uint64_t n, float h, float* w, float* dw);

/* ---------------------------------------------------------------------------------------------
 * Autotuner: times the P2G variants, block sizes and sort intervals on a world and writes the
 * fastest choice back into the world's options.  Choices are cached per workload signature.
 * ------------------------------------------------------------------------------------------- */
typedef struct ae_mpm_tune_result {
  int32_t p2g_variant;
  int32_t block_threads;
  int32_t sort_interval;
  float us_per_substep;
} ae_mpm_tune_result;
int ae_mpm_world_autotune(ae_mpm_world* world, uint32_t substeps_per_trial, ae_mpm_tune_result* out);

/* ---------------------------------------------------------------------------------------------
 * Continuous-batching server.  Requests (a physics-mode scene plus its particles and a substep
 * count) run in one resident world of scene *slots*, each made with a grid, material and particle
 * capacity (the request's size class: axes rounded up to 16 nodes, particles and materials to
 * powers of two).  A request is admitted, first come first served, into a free slot that fits it;
 * when none does, the world grows by slots of its class (doubling per class) as long as the
 * slots' device state fits the HBM budget, dropping vacant slots first if needed.  Admitted
 * scenes are uploaded into their slots in place and stepped together with every other resident
 * scene; a finished scene is copied back and vacates its slot for the next request.  Inputs and
 * results travel through page-locked staging, and results reach the callers' buffers while the
 * device runs the next batch of substeps.  One host thread per server drives the device.
 * ------------------------------------------------------------------------------------------- */
typedef struct ae_mpm_server_opts {
  uint64_t hbm_budget_bytes;   /* budget for the slots' device state                         */
  uint32_t substeps_per_tick;  /* substeps run between admission checks (default 10)         */
  uint32_t max_scenes;         /* cap on resident scenes (default 4096)                      */
  ae_mpm_exec_opts exec;
} ae_mpm_server_opts;

typedef struct ae_mpm_request_result {
  uint64_t request_id;
  int32_t status;          /* AE_MPM_OK or the scene's error                          */
  double submit_s;         /* host steady-clock seconds at submit                      */
  double admit_s;          /* ... when admitted to the device                          */
  double done_s;           /* ... when its results were in the caller's buffers         */
} ae_mpm_request_result;

int ae_mpm_server_create(ae_mpm_ctx* ctx, const ae_mpm_server_opts* opts, ae_mpm_server** out);
/* Submit: the particles are copied at submit time; results are written into `out` (which must
 * stay valid until the request's result has been polled).  A request whose slot class alone
 * exceeds the budget is refused with AE_MPM_EBUDGET; one that is not physics mode, or whose grid
 * is outside 4..1024 nodes per axis, with AE_MPM_EINVAL. */
int ae_mpm_server_submit(ae_mpm_server* server, const ae_mpm_scene_desc* scene,
                         const ae_mpm_particles* in, uint64_t n, uint32_t substeps,
                         ae_mpm_particles* out, uint64_t* request_id);
/* Cancel a request that has not finished; its result reports AE_MPM_ENOTFOUND-free status
 * AE_MPM_EINVAL ("cancelled") and its buffers are left untouched. */
int ae_mpm_server_cancel(ae_mpm_server* server, uint64_t request_id);
/* Collect finished results (up to max); returns AE_MPM_EAGAIN when none are ready. */
int ae_mpm_server_poll(ae_mpm_server* server, ae_mpm_request_result* results, uint32_t max,
                       uint32_t* n_out);
/* Wait until every submitted request has finished, at most timeout_s seconds. */
int ae_mpm_server_drain(ae_mpm_server* server, double timeout_s);
/* Device bytes of the slots and scenes resident right now; ticks run; particle-substeps run. */
int ae_mpm_server_stats(ae_mpm_server* server, uint64_t* resident_bytes, uint32_t* resident_scenes,
                        uint64_t* ticks, uint64_t* particle_substeps);
int ae_mpm_server_destroy(ae_mpm_server* server);
/* The size class of the slot a request of `scene` with n_particles takes (host only, no device
 * needed): grid axes rounded up to multiples of 16 nodes (at least 16), a particle capacity of
 * the first quarter-octave step 2^(k/4) * 2^j >= n_particles (j >= 10, rounded up to 256), and a
 * power-of-two material count of at least 4. */
int ae_mpm_server_slot_class(const ae_mpm_scene_desc* scene, uint64_t n_particles, uint32_t grid_out[3],
                             uint64_t* particles_out, uint32_t* materials_out);

#ifdef __cplusplus
}
#endif
#endif /* AE_MPM_H */
