//! ae_mpm_cuda -- Rust binding of include/ae_mpm.h (the B200 MPM substep library).
//!
//! The raw `extern "C"` block mirrors the header one to one.  The safe layer keeps the
//! reference's argument shapes: `mpm_step_parallel_with_grid` takes the MpssBuffer field slices
//! (`pos`, `vel`, `strain`, `jacobian`, `c`, `mass`, `material_idx`), the grid's node counts,
//! spacing and origin, `MpmConfig`, the material and model tables, `total_dt` and the particle
//! indices, exactly like ae_particle::mpm_solver::mpm_step_parallel_with_grid
//! (ae_particle/src/mpm_solver.rs:1063-1084).  Errors come back as `Result`; the reference panics
//! instead, and ae_particle's wrapper keeps that by unwrapping.

#![allow(non_camel_case_types)]
use std::ffi::CStr;
use std::os::raw::{c_char, c_int, c_void};
use std::sync::OnceLock;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ae_mpm_material {
    pub young_modulus: f32,
    pub poisson_ratio: f32,
    pub yield_stress: f32,
    pub hardening: f32,
    pub density: f32,
    pub friction_angle: f32,
    pub cohesion: f32,
    pub model: i32,
    pub theta_c: f32,
    pub theta_s: f32,
    pub hardening_xi: f32,
    pub bulk_modulus: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ae_mpm_config {
    pub grid_dx: f32,
    pub grid_size: [u64; 3],
    pub substeps: u64,
    pub gravity: [f32; 3],
    pub damping: f32,
    pub enable_plasticity: u8,
    pub enable_contact: u8,
    pub use_sparse_grid: u8,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ae_mpm_grid {
    pub nx: u64,
    pub ny: u64,
    pub nz: u64,
    pub dx: f32,
    pub origin: [f32; 3],
}

#[repr(C)]
pub struct ae_mpm_particles {
    pub pos: *mut f32,
    pub vel: *mut f32,
    pub strain: *mut f32,
    pub jacobian: *mut f32,
    pub c: *mut f32,
    pub mass: *mut f32,
    pub material_idx: *mut u16,
}

#[repr(C)]
pub struct ae_mpm_ctx {
    _private: [u8; 0],
}

pub const AE_MPM_OK: c_int = 0;

/// CkMpmConfig (ae_compute/src/ck_mpm.rs:41-59) in the library's layout.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ae_mpm_ck_config {
    pub dt: f32,
    pub grid_h: f32,
    pub grid_n: u32,
    pub gravity: [f32; 3],
    pub youngs_modulus: f32,
    pub poissons_ratio: f32,
    pub density: f32,
    pub bounds_min: [f32; 3],
    pub bounds_max: [f32; 3],
    pub restitution: f32,
    pub dual_grid: u8,
    pub pad: [u8; 3],
}

/// CkMpmParticle (ck_mpm.rs:84-95): glam Vec3 / Mat3 are #[repr(C)] (Mat3 = three column Vec3s),
/// so a CkMpmParticle declared #[repr(C)] has exactly this layout and its slice can be passed as is.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ae_mpm_ck_particle {
    pub position: [f32; 3],
    pub velocity: [f32; 3],
    pub affine: [f32; 9],
    pub deformation: [f32; 9],
    pub rest_volume: f32,
    pub mass: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ae_mpm_ck_stats {
    pub kinetic_energy: f32,
    pub average_velocity: [f32; 3],
    pub average_volume_ratio: f32,
}

extern "C" {
    pub fn ae_mpm_ctx_create(device: c_int, out: *mut *mut ae_mpm_ctx) -> c_int;
    pub fn ae_mpm_ctx_destroy(ctx: *mut ae_mpm_ctx);
    pub fn ae_mpm_last_error(ctx: *const ae_mpm_ctx) -> *const c_char;
    pub fn ae_mpm_step_parallel_with_grid(
        ctx: *mut ae_mpm_ctx,
        buffer: *const ae_mpm_particles,
        capacity: u64,
        grid: *const ae_mpm_grid,
        config: *const ae_mpm_config,
        material_table: *const ae_mpm_material,
        n_materials: u32,
        model_table: *const i32,
        n_models: u32,
        total_dt: f32,
        particle_indices: *const u64,
        n_indices: u64,
    ) -> c_int;
    pub fn ae_mpm_step_velocity_only_parallel(
        ctx: *mut ae_mpm_ctx,
        buffer: *const ae_mpm_particles,
        capacity: u64,
        grid: *const ae_mpm_grid,
        config: *const ae_mpm_config,
        total_dt: f32,
        particle_indices: *const u64,
        n_indices: u64,
    ) -> c_int;
    pub fn ae_mpm_grid_download(ctx: *mut ae_mpm_ctx, mass: *mut f32, vel: *mut f32, n_nodes: u64) -> c_int;
    pub fn ae_mpm_lod_classify(
        ctx: *mut ae_mpm_ctx,
        pos: *const f32,
        active: *const u8,
        count: u64,
        player: *const f32,
        near_dist: f32,
        mid_dist: f32,
        max_near: u64,
        near_out: *mut u64,
        n_near: *mut u64,
        mid_out: *mut u64,
        n_mid: *mut u64,
        far_out: *mut u64,
        n_far: *mut u64,
    ) -> c_int;
    pub fn ae_mpm_far_field_update(
        ctx: *mut ae_mpm_ctx,
        pos: *mut f32,
        vel: *mut f32,
        temperature: *mut f32,
        count: u64,
        far_idx: *const u64,
        n_far: u64,
        coarse_temperature: *const f32,
        coarse_n: u32,
        coarse_dx: f32,
        coarse_origin: *const f32,
        far_dt: f32,
    ) -> c_int;
    pub fn ae_mpm_coarse_field_update(
        ctx: *mut ae_mpm_ctx,
        pos: *const f32,
        mass: *const f32,
        temperature: *const f32,
        active: *const u8,
        count: u64,
        near_idx: *const u64,
        n_near: u64,
        coarse_temperature: *mut f32,
        coarse_n: u32,
        coarse_dx: f32,
        coarse_origin: *const f32,
        dt: f32,
    ) -> c_int;
    pub fn ae_mpm_mpss_housekeeping(
        ctx: *mut ae_mpm_ctx,
        pos: *mut f32,
        vel: *mut f32,
        temperature: *mut f32,
        phase: *mut u8,
        material_idx: *const u16,
        active: *const u8,
        count: u64,
        bounds_min: *const f32,
        bounds_max: *const f32,
        min_temp: f32,
        max_temp: f32,
        passes: u32,
        transitions: *mut u32,
    ) -> c_int;
    pub fn ae_mpm_ck_config_default(out: *mut ae_mpm_ck_config);
    pub fn ae_mpm_ck_step(
        ctx: *mut ae_mpm_ctx,
        particles: *mut ae_mpm_ck_particle,
        n: u64,
        config: *const ae_mpm_ck_config,
        steps: u32,
    ) -> c_int;
    pub fn ae_mpm_ck_step_deterministic(
        ctx: *mut ae_mpm_ctx,
        particles: *mut ae_mpm_ck_particle,
        n: u64,
        config: *const ae_mpm_ck_config,
        steps: u32,
    ) -> c_int;
    pub fn ae_mpm_ck_step_timed(
        ctx: *mut ae_mpm_ctx,
        particles: *mut ae_mpm_ck_particle,
        n: u64,
        config: *const ae_mpm_ck_config,
        steps: u32,
        kernel_ms: *mut f64,
    ) -> c_int;
    pub fn ae_mpm_ck_stats_compute(
        ctx: *mut ae_mpm_ctx,
        particles: *const ae_mpm_ck_particle,
        n: u64,
        out: *mut ae_mpm_ck_stats,
    ) -> c_int;
    pub fn ae_mpm_ck_weights(ctx: *mut ae_mpm_ctx, x: *const f32, n: u64, h: f32, w: *mut f32, dw: *mut f32) -> c_int;
}

/// Library context on device 0, created on first use (one per process, like the rayon pool).
struct Ctx(*mut ae_mpm_ctx);
unsafe impl Send for Ctx {}
unsafe impl Sync for Ctx {}

fn ctx() -> *mut ae_mpm_ctx {
    static CTX: OnceLock<Ctx> = OnceLock::new();
    CTX.get_or_init(|| {
        let mut p = std::ptr::null_mut();
        let rc = unsafe { ae_mpm_ctx_create(0, &mut p) };
        assert_eq!(rc, AE_MPM_OK, "ae_mpm: no usable CUDA device");
        Ctx(p)
    })
    .0
}

fn check(rc: c_int) -> Result<(), String> {
    if rc == AE_MPM_OK {
        Ok(())
    } else {
        Err(unsafe { CStr::from_ptr(ae_mpm_last_error(ctx())) }.to_string_lossy().into_owned())
    }
}

/// The MpssBuffer fields one substep reads and writes.
pub struct ParticleSlices<'a> {
    pub pos: &'a mut [[f32; 3]],
    pub vel: &'a mut [[f32; 3]],
    pub strain: &'a mut [[f32; 9]],
    pub jacobian: &'a mut [f32],
    pub c: &'a mut [[f32; 9]],
    pub mass: &'a mut [f32],
    pub material_idx: &'a mut [u16],
}

impl<'a> ParticleSlices<'a> {
    fn raw(&mut self) -> ae_mpm_particles {
        ae_mpm_particles {
            pos: self.pos.as_mut_ptr() as *mut f32,
            vel: self.vel.as_mut_ptr() as *mut f32,
            strain: self.strain.as_mut_ptr() as *mut f32,
            jacobian: self.jacobian.as_mut_ptr(),
            c: self.c.as_mut_ptr() as *mut f32,
            mass: self.mass.as_mut_ptr(),
            material_idx: self.material_idx.as_mut_ptr(),
        }
    }
    fn capacity(&self) -> u64 {
        self.pos.len() as u64
    }
}

/// Same semantics as ae_particle::mpm_solver::mpm_step_parallel_with_grid minus the trailing
/// `buffer.update_lifetimes(total_dt)`, which stays with the caller (it edits the free list).
pub fn mpm_step_parallel_with_grid(
    p: &mut ParticleSlices,
    grid: &ae_mpm_grid,
    config: &ae_mpm_config,
    material_table: &[ae_mpm_material],
    model_table: &[i32],
    total_dt: f32,
    particle_indices: &[usize],
) -> Result<(), String> {
    let idx: Vec<u64> = particle_indices.iter().map(|&i| i as u64).collect();
    let raw = p.raw();
    check(unsafe {
        ae_mpm_step_parallel_with_grid(
            ctx(),
            &raw,
            p.capacity(),
            grid,
            config,
            material_table.as_ptr(),
            material_table.len() as u32,
            model_table.as_ptr(),
            model_table.len() as u32,
            total_dt,
            idx.as_ptr(),
            idx.len() as u64,
        )
    })
}

/// Same semantics as ae_particle::mpm_solver::mpm_step_velocity_only_parallel.
pub fn mpm_step_velocity_only_parallel(
    p: &mut ParticleSlices,
    grid: &ae_mpm_grid,
    config: &ae_mpm_config,
    total_dt: f32,
    particle_indices: &[usize],
) -> Result<(), String> {
    let idx: Vec<u64> = particle_indices.iter().map(|&i| i as u64).collect();
    let raw = p.raw();
    check(unsafe {
        ae_mpm_step_velocity_only_parallel(ctx(), &raw, p.capacity(), grid, config, total_dt, idx.as_ptr(), idx.len() as u64)
    })
}

/// Grid mass and velocity after the last drop-in step (reference node order i + j nx + k nx ny).
pub fn grid_download(mass: &mut [f32], vel: &mut [[f32; 3]]) -> Result<(), String> {
    assert_eq!(mass.len(), vel.len());
    check(unsafe { ae_mpm_grid_download(ctx(), mass.as_mut_ptr(), vel.as_mut_ptr() as *mut f32, mass.len() as u64) })
}

/// The reclassify branch of SimulationManager::update_fields_and_particles (simulation.rs:495-532):
/// returns (near, mid, far).  `active` is MpssBuffer::active (Vec<bool>, one byte per entry).
/// The near list comes back in ascending index order; the engine's Vec<(usize, f32)> keeps
/// only the indices downstream.
pub fn lod_classify(
    pos: &[[f32; 3]],
    active: &[bool],
    player: [f32; 3],
    near_dist: f32,
    mid_dist: f32,
    max_near: usize,
) -> Result<(Vec<usize>, Vec<usize>, Vec<usize>), String> {
    let n = pos.len();
    assert_eq!(active.len(), n);
    let (mut near, mut mid, mut far) = (vec![0u64; n], vec![0u64; n], vec![0u64; n]);
    let (mut nn, mut nm, mut nf) = (0u64, 0u64, 0u64);
    check(unsafe {
        ae_mpm_lod_classify(
            ctx(),
            pos.as_ptr() as *const f32,
            active.as_ptr() as *const u8,
            n as u64,
            player.as_ptr(),
            near_dist,
            mid_dist,
            max_near as u64,
            near.as_mut_ptr(),
            &mut nn,
            mid.as_mut_ptr(),
            &mut nm,
            far.as_mut_ptr(),
            &mut nf,
        )
    })?;
    let cut = |v: Vec<u64>, k: u64| v[..k as usize].iter().map(|&i| i as usize).collect::<Vec<usize>>();
    Ok((cut(near, nn), cut(mid, nm), cut(far, nf)))
}

/// The far-field pass of update_fields_and_particles (simulation.rs:612-679) over `far_idx`.
pub fn far_field_update(
    pos: &mut [[f32; 3]],
    vel: &mut [[f32; 3]],
    temperature: &mut [f32],
    far_idx: &[usize],
    coarse_temperature: &[f32],
    coarse_n: usize,
    coarse_dx: f32,
    coarse_origin: [f32; 3],
    far_dt: f32,
) -> Result<(), String> {
    let idx: Vec<u64> = far_idx.iter().map(|&i| i as u64).collect();
    check(unsafe {
        ae_mpm_far_field_update(
            ctx(),
            pos.as_mut_ptr() as *mut f32,
            vel.as_mut_ptr() as *mut f32,
            temperature.as_mut_ptr(),
            pos.len() as u64,
            idx.as_ptr(),
            idx.len() as u64,
            coarse_temperature.as_ptr(),
            coarse_n as u32,
            coarse_dx,
            coarse_origin.as_ptr(),
            far_dt,
        )
    })
}

/// SimulationManager::update_coarse_field (simulation.rs:877-966) with the near indices.
pub fn coarse_field_update(
    pos: &[[f32; 3]],
    mass: &[f32],
    temperature: &[f32],
    active: &[bool],
    near_idx: &[usize],
    coarse_temperature: &mut [f32],
    coarse_n: usize,
    coarse_dx: f32,
    coarse_origin: [f32; 3],
    dt: f32,
) -> Result<(), String> {
    let idx: Vec<u64> = near_idx.iter().map(|&i| i as u64).collect();
    check(unsafe {
        ae_mpm_coarse_field_update(
            ctx(),
            pos.as_ptr() as *const f32,
            mass.as_ptr(),
            temperature.as_ptr(),
            active.as_ptr() as *const u8,
            pos.len() as u64,
            idx.as_ptr(),
            idx.len() as u64,
            coarse_temperature.as_mut_ptr(),
            coarse_n as u32,
            coarse_dx,
            coarse_origin.as_ptr(),
            dt,
        )
    })
}

/// The three MpssBuffer calls of ae_engine/src/lib.rs:347-358 (apply_boundary_conditions_par,
/// clamp_temperatures_par, apply_phase_transitions_par) in one device pass; returns the number of
/// phase transitions.  `phase` holds MpssPhase discriminants as bytes (`p as u8` and back, or
/// MpssPhase declared #[repr(u8)] and the slice reinterpreted).
pub fn mpss_housekeeping(
    pos: &mut [[f32; 3]],
    vel: &mut [[f32; 3]],
    temperature: &mut [f32],
    phase: &mut [u8],
    material_idx: &[u16],
    active: &[bool],
    bounds_min: [f32; 3],
    bounds_max: [f32; 3],
    min_temp: f32,
    max_temp: f32,
) -> Result<u32, String> {
    let mut transitions = 0u32;
    check(unsafe {
        ae_mpm_mpss_housekeeping(
            ctx(),
            pos.as_mut_ptr() as *mut f32,
            vel.as_mut_ptr() as *mut f32,
            temperature.as_mut_ptr(),
            phase.as_mut_ptr(),
            material_idx.as_ptr(),
            active.as_ptr() as *const u8,
            pos.len() as u64,
            bounds_min.as_ptr(),
            bounds_max.as_ptr(),
            min_temp,
            max_temp,
            7,
            &mut transitions,
        )
    })?;
    Ok(transitions)
}

/// `steps` x CkMpmSolver::step (ck_mpm.rs:187-480) on the caller's particles, in place.
pub fn ck_step(particles: &mut [ae_mpm_ck_particle], config: &ae_mpm_ck_config, steps: u32) -> Result<(), String> {
    check(unsafe { ae_mpm_ck_step(ctx(), particles.as_mut_ptr(), particles.len() as u64, config, steps) })
}

/// The same steps with node sums in the reference's particle order: bitwise reproducible.
pub fn ck_step_deterministic(
    particles: &mut [ae_mpm_ck_particle],
    config: &ae_mpm_ck_config,
    steps: u32,
) -> Result<(), String> {
    check(unsafe { ae_mpm_ck_step_deterministic(ctx(), particles.as_mut_ptr(), particles.len() as u64, config, steps) })
}

/// kinetic_energy, average_velocity, average_volume_ratio (ck_mpm.rs:484-503).
pub fn ck_stats(particles: &[ae_mpm_ck_particle]) -> Result<ae_mpm_ck_stats, String> {
    let mut out = ae_mpm_ck_stats::default();
    check(unsafe { ae_mpm_ck_stats_compute(ctx(), particles.as_ptr(), particles.len() as u64, &mut out) })?;
    Ok(out)
}

#[allow(dead_code)]
fn _assert_ffi_safe(_: *const c_void) {}
