/*
 * emerge_oracle.h -- C API of the CPU oracle for the emerge-engine MLS-MPM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a C++17 restatement of the
 * reference crate's CPU step (Rust, M1thieu/emerge-engine 0.1.0), used as the
 * parity checker for the CUDA backend and as the timed CPU baseline.  Only the
 * test suite, the smoke check and bench.py's CPU-baseline leg may load it.
 * The product library (libemerge_cuda.so) never links or calls it.
 *
 * Parity status: the reference cannot be compiled here (no Rust toolchain),
 * and it ships no golden trajectories.  The oracle is pinned against every
 * known-answer unit test the reference holds for this path (ported into
 * tests/test_oracle_known_answers.py); bit-level agreement with the Rust
 * build is not claimed (glam arithmetic and Rust's libm calls are restated,
 * not executed).
 *
 * Struct layouts that cross the ABI (particle, config, spawn, body state) are
 * byte-identical to include/emerge_cuda.h so one ctypes definition serves
 * both libraries.  The material descriptor here is the oracle's own: it holds
 * every field of the reference material structs (not only the 96-byte
 * MaterialParams), because the reference CPU step reads the structs.
 */
#ifndef EMERGE_ORACLE_H
#define EMERGE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as emerge_particle (reference matter/particle.rs:13-138, 128 B). */
typedef struct oracle_particle {
    float x[2];
    float v[2];
    float c[4];          /* velocity_gradient, column-major (x_axis, y_axis) */
    float f[4];          /* deformation_gradient, column-major */
    float mass;
    float initial_volume;
    float volume;
    float density;
    uint32_t material_id;
    float plastic_volume_ratio;
    float hardening_scale;
    float friction_hardening;
    float log_volume_strain;
    float temperature;
    uint32_t user_tag;
    float activation;
    float activation_dir[2];
    uint32_t muscle_group_id;
    uint32_t contact_group;
    uint32_t sleeping;
    uint32_t pinned;
    float scalar_field;
    uint32_t pad_;
} oracle_particle;

/* Same layout as emerge_sim_config (reference spacetime/solver/config.rs:26-121). */
typedef struct oracle_config {
    uint64_t grid_res;
    float grid_cell_size;
    float dt;
    uint32_t adaptive_timestep;
    uint32_t cfl_include_affine_speed;
    float cfl_coefficient;
    float material_cfl_coefficient;
    float viscous_timestep_coefficient;
    float min_dt;
    uint32_t project_invalid_state;
    float projection_min_density;
    float projection_min_volume;
    float projection_min_deformation_j;
    float gravity[2];
    uint64_t boundary_thickness;
    float default_initial_volume;
    uint32_t recompute_density_each_step;
    float particle_mass;
    uint32_t pad0_;
    uint64_t max_substeps_per_step;
    float apic_blend;
    float j_max;
    float sleep_threshold;
    float contact_friction;
    float asflip_blend;
    float mixture_drag_coefficient;
    uint32_t mixture_pressure_iterations;
    float dx_meters;
    float dt_seconds;
    uint32_t pad1_;
} oracle_config;

/* Same layout as emerge_spawn_region (reference config.rs:317-346). */
typedef struct oracle_spawn {
    float spacing;
    int32_t box_size[2];
    float box_center[2];
    uint32_t shape;              /* 0 = Box, 1 = Disk */
    float disk_radius;
    float initial_deformation_gradient[4];
    uint32_t precompute_initial_volumes;
    float initial_velocity_scale;
    float position_jitter;
    uint32_t rng_seed;
    uint32_t material_id;
    uint32_t has_mass_override;
    float mass_override;
} oracle_spawn;

/* Same layout as emerge_body_state (reference solver/query.rs:17-32). */
typedef struct oracle_body_state {
    uint64_t count;
    float avg_volume_ratio;
    float max_volume_ratio;
    float avg_speed;
    float avg_det_f;
    float avg_density;
    float centroid[2];
    uint32_t pad_;
} oracle_body_state;

/* Full field set of the reference material structs.  `model` is the
 * ConstitutiveModel discriminant (materials/mod.rs:53-66). */
typedef struct oracle_material {
    uint32_t model;
    /* NeoHookean (elastic.rs:20-48); DP/Snow share lambda/mu */
    float lambda, mu, min_density, thermal_expansion, active_stress_coeff,
          damage_softening_rate, viscosity;
    /* NewtonianFluid (fluid.rs:10-45) */
    float rest_density, dynamic_viscosity, eos_stiffness, eos_power,
          pressure_floor, fluid_min_density, fluid_min_volume,
          thermal_viscosity_coeff, bulk_viscosity, surface_tension_coeff,
          settling_damping;
    /* DruckerPrager (sand.rs:11-75) */
    float friction_angle, hardening_peak, hardening_decay, friction_residual,
          volume_correction, dilatancy_angle, cohesion, min_volume_jacobian;
    /* Stomakhin snow (snow.rs:19-37) */
    float hardening_exponent, compression_limit, stretch_limit,
          min_plastic_jacobian, max_plastic_jacobian, cohesion_coeff;
    /* NACC (nacc.rs:34-60) */
    float kappa, friction, nacc_cohesion, hardening_factor;
    uint32_t hardening_enabled;
    float nacc_min_density;
    /* Corotated (corotated.rs:16-27) reuses lambda, mu, thermal_expansion,
     * active_stress_coeff; VonMises (von_mises.rs:29-38) */
    float yield_stress, hardening_modulus;
    /* Rankine (rankine.rs) */
    float tensile_strength, softening_rate;
    /* MuIRheology (sand_mui.rs) */
    float mu_static, mu_dynamic, inertial_q;
    /* Viscoelastic (viscoelastic.rs) reuses lambda, mu, viscosity, active_stress_coeff,
     * thermal_expansion */
    float j_min;
    /* BinghamFluid (bingham.rs): model FLUID with bingham = 1; reuses the fluid fields */
    float bingham_yield_stress, critical_shear_rate;
    uint32_t bingham;
    /* GranularFluid (granular_fluid.rs) reuses lambda, mu, rest_density, eos_stiffness,
     * eos_power, pressure_floor and the snow fields hardening_exponent, compression_limit,
     * stretch_limit, min_plastic_jacobian, max_plastic_jacobian */
    /* WithMixturePhase (materials/mod.rs:296-357): 0 none, 1 solid, 2 fluid */
    uint32_t mixture_phase;
} oracle_material;

/* One built-in force field (forces/fields/); kinds and data layout as
 * emerge_force_field in include/emerge_cuda.h (same 48-byte layout). */
typedef struct oracle_force_field {
    uint32_t kind, material_mask, material_filter, count, data_offset, n_charges;
    float params[6];
} oracle_force_field;

typedef struct oracle_sim oracle_sim;

/* Simulation::empty (lifecycle.rs:26): validates the config (error -> NULL),
 * registers the fallback material at id 0 and one SlipBoundary of
 * config.boundary_thickness. */
oracle_sim *oracle_create(const oracle_config *cfg);
void oracle_destroy(oracle_sim *s);
/* MaterialRegistry::insert / set_default (registry.rs:29-60). Returns 0 or -1
 * (non-contiguous id / id >= 64). id 0 replaces the default and re-runs
 * init_particle on every particle (with_default_material, lifecycle.rs:107). */
int oracle_set_material(oracle_sim *s, uint32_t id, const oracle_material *m);
/* with_boundary(SlipBoundary::new(t)) (lifecycle.rs:114); clear=1 removes all first. */
int oracle_add_slip_boundary(oracle_sim *s, uint64_t thickness, int clear_first);
/* add_body (particles.rs:355-423).  Returns 0 and writes the tag, or -1 if the
 * region does not fit (validate_for_sim panics in the reference). */
int oracle_add_body(oracle_sim *s, const oracle_spawn *spawn, uint32_t *tag_out);
/* Simulation::new's particle set-up (lifecycle.rs:57-71): spawn the region as
 * tag 0 into an empty sim and run the full volume estimate when
 * spawn.precompute_initial_volumes is set. */
int oracle_init_with_spawn(oracle_sim *s, const oracle_spawn *spawn);
/* Raw particle append (active, in order), no density pass. */
int oracle_push_particles(oracle_sim *s, const oracle_particle *p, uint64_t n);
void oracle_step(oracle_sim *s, uint32_t n_steps);
/* 0 (default): exp/log/pow/sin/sinh from the C library, as the Rust reference calls them;
 * 1: evaluated in double and rounded once to f32 (process-wide switch). */
void oracle_set_correctly_rounded(int on);
/* Replaces the force fields (application order); returns 0, or -1 for an unknown kind or
 * data out of range. */
int oracle_set_force_fields(oracle_sim *s, const oracle_force_field *fields, uint32_t n,
                            const float *data, uint64_t n_data);
/* The fields' summed Field::acceleration for every particle (out[2 i], out[2 i + 1]), the
 * n-body trees built from the current positions (n_body.rs:332-360). */
void oracle_field_accelerations(oracle_sim *s, float *out);
/* DirectionalContactGrip (grid/directional_grip.rs) for contact resolution:
 * on = 0 removes it (Coulomb friction with SimConfig::contact_friction). */
void oracle_set_contact_grip(oracle_sim *s, int on, float mu_easy, float mu_resist, float dir_x,
                             float dir_y);
/* fit_contact_normal_lr (grid/contact_normal.rs) on n points (x, y, label); returns 1 and the
 * normal, or 0 for no normal. */
int oracle_fit_contact_normal(const float *points, uint32_t n, float node_x, float node_y,
                              float cell, float normal[2]);
/* Field::acceleration of one field at one particle. */
void oracle_field_acceleration(const oracle_force_field *f, const float *data,
                               const oracle_particle *p, float out[2]);
uint64_t oracle_particle_count(const oracle_sim *s);
/* active_count (solver/mod.rs:40-42): particles [0, active_count) are awake. */
uint64_t oracle_active_count(const oracle_sim *s);
/* Replaces the particle array (reference order) and the active-zone size. */
int oracle_replace_particles(oracle_sim *s, const oracle_particle *p, uint64_t n, uint64_t active_count);
void oracle_wake_tag(oracle_sim *s, uint32_t tag);
void oracle_sleep_tag(oracle_sim *s, uint32_t tag);
void oracle_read_particles(const oracle_sim *s, oracle_particle *out);
void oracle_write_particles(oracle_sim *s, const oracle_particle *in);
void oracle_region_state(const oracle_sim *s, float cx, float cy, float r,
                         oracle_body_state *out);
float oracle_effective_dt(const oracle_sim *s);
uint64_t oracle_last_substeps(const oracle_sim *s);
uint64_t oracle_last_vel_clamp_count(const oracle_sim *s);
uint64_t oracle_last_j_projection_count(const oracle_sim *s);
/* Per-phase CPU time of the last step in microseconds:
 * [cfl, project, density, p2g, grid_update, g2p, total]. */
void oracle_last_timing_us(const oracle_sim *s, double out[7]);
/* Worker threads for G2P phase 1 (0 = all hardware threads); returns the count in use. */
int oracle_set_threads(int n);

/* ---- unit-level entry points for known-answer tests ---- */
void oracle_svd2(const float f[4], float u[4], float sigma[2], float vt[4]);
void oracle_polar(const float f[4], float r[4]);
void oracle_axis_weights(float d, float w[3]);
void oracle_kirchhoff(const oracle_material *m, const oracle_particle *p, float tau[4]);
void oracle_update_particle(const oracle_material *m, oracle_particle *p, float dt);
void oracle_init_particle(const oracle_material *m, oracle_particle *p);
float oracle_timestep_bound(const oracle_material *m, float density, float h,
                            float cell, float mat_cfl, float visc_cfl);
/* NaccMaterial::project (nacc.rs:129-223). */
void oracle_nacc_project(const oracle_material *m, const float f[4], float alpha,
                         float f_out[4], float *alpha_out);
/* DruckerPragerMaterial::project (sand.rs:156-194); returns 1 = Some, 0 = None. */
int oracle_dp_project(const oracle_material *m, const float sigma[2], float lvs,
                      float q, float sigma_out[2], float *dq_out);
void oracle_slip_velocity(uint64_t thickness, uint64_t cell_index, uint64_t res, float v[2]);
/* particle_sort.wgsl:94-102 block_index key (reference GPU sort key). */
uint32_t oracle_block_index(float px, float py, uint32_t grid_res);
/* Stable sort of keys by value (ties by index) -> permutation. */
void oracle_stable_argsort_u32(const uint32_t *keys, uint64_t n, uint32_t *perm_out);
/* Project one particle to the admissible set (step.rs:347-429); returns 1 if changed. */
int oracle_project_particle(const oracle_config *cfg, oracle_particle *p);
/* choose_substep_dt (step.rs:434-468) over the sim's current particles. */
float oracle_choose_substep_dt(const oracle_sim *s, float max_dt);

#ifdef __cplusplus
}
#endif
#endif
