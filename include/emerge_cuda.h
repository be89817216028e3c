/*
 * emerge_cuda.h -- C ABI of the B200 (sm_100a) MLS-MPM backend for emerge-engine.
 *
 * This library is a drop-in `cuda` backend for the reference crate's CPU step
 * (M1thieu/emerge-engine 0.1.0, Rust).  Every entry point below names the
 * reference item it stands in for (path:line inside the reference crate).
 * Signatures use plain pointers, sizes and POD structs only.
 *
 * Conventions
 *  - Every function returns an emerge_status (0 = EMERGE_OK).  On failure the
 *    message is available from emerge_cuda_last_error(sim) (or, for create,
 *    emerge_cuda_last_global_error()).  The reference panics in the same
 *    situations (invalid config, spawn out of bounds, non-contiguous material
 *    ids); a Rust shim turns the codes back into those panics.
 *  - The library owns all device memory of a simulation.  Reads copy into
 *    caller memory; no caller pointer is retained after a call returns.
 *  - One CUDA stream per simulation.  Calls on one simulation must be
 *    serialised by the caller (the reference Simulation is `&mut self`);
 *    different simulations are independent.
 *  - There is no CPU fallback: a missing or unusable GPU is an error.
 */
#ifndef EMERGE_CUDA_H
#define EMERGE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum emerge_status {
    EMERGE_OK = 0,
    EMERGE_ERR_INVALID_ARG = 1,  /* config.rs:247-299 / :485-505, registry.rs:31-46 asserts */
    EMERGE_ERR_UNSUPPORTED = 2,  /* model / feature with no device implementation */
    EMERGE_ERR_CUDA = 3,         /* CUDA runtime error (message has the CUDA error string) */
    EMERGE_ERR_TIMEOUT = 4,      /* a bounded device wait gave up */
    EMERGE_ERR_NONFINITE = 5,    /* non-finite state where the reference would NaN-cascade */
    EMERGE_ERR_OOM = 6           /* device allocation failed */
} emerge_status;

/* Particle, byte-identical to the reference `Particle` (matter/particle.rs:13-138,
 * size asserted 128 at :144).  Matrices are column-major (glam Mat2 x_axis, y_axis). */
typedef struct emerge_particle {
    float x[2];
    float v[2];
    float c[4];               /* velocity_gradient (APIC C) */
    float f[4];               /* deformation_gradient */
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
    uint32_t contact_group;   /* != 0: in the grip field of multi-field contact */
    uint32_t sleeping;
    uint32_t pinned;
    float scalar_field;
    uint32_t pad_;
} emerge_particle;

/* SimConfig, field for field (spacetime/solver/config.rs:26-121); usize -> uint64,
 * bool -> uint32, Vec2 -> float[2].  Explicit padding keeps the layout fixed. */
typedef struct emerge_sim_config {
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
    float sleep_threshold;          /* sleep scoring speed (step.rs:299-315); 0 = off */
    float contact_friction;
    float asflip_blend;             /* ASFLIP FLIP blend (transfer/g2p.rs:263-296); 0 = APIC only */
    float mixture_drag_coefficient;
    uint32_t mixture_pressure_iterations;
    float dx_meters;
    float dt_seconds;
    uint32_t pad1_;
} emerge_sim_config;

/* MaterialParams (matter/materials/params.rs:10-101, 96 bytes).  `model` carries
 * MaterialModel::constitutive_model() (materials/mod.rs:53-66), NOT params().model:
 * NaccMaterial::params() reports NeoHookean (nacc.rs:300-314).  Every model id 0-11 runs
 * on the device, each reading its own params() packing.  A Fluid slot with
 * compression_limit > 0 is a BinghamFluidMaterial (bingham.rs params() puts yield_stress
 * there); its critical shear rate is the constructor's 1e-4.  Viscoelastic reads
 * thermal_expansion from the thermal_expansion field, which its params() leaves 0. */
typedef struct emerge_material_params {
    uint32_t model;
    float lambda;
    float mu;
    float hardening_exponent;
    float compression_limit;
    float stretch_limit;
    float rest_density;
    float eos_stiffness;
    float eos_power;
    float dynamic_viscosity;
    float volume_ratio_min;
    float volume_ratio_max;
    float dp_h0;
    float dp_h1;
    float dp_h2;
    float dp_h3;
    float active_stress_coeff;
    float hardening_modulus;
    float thermal_viscosity_coeff;
    float thermal_expansion;
    float pressure_floor;
    float bulk_viscosity;
    float surface_tension_coeff;
    float cohesion_coeff;
} emerge_material_params;

/* SpawnRegion (spacetime/solver/config.rs:317-346). shape: 0 = Box, 1 = Disk. */
typedef struct emerge_spawn_region {
    float spacing;
    int32_t box_size[2];
    float box_center[2];
    uint32_t shape;
    float disk_radius;
    float initial_deformation_gradient[4];
    uint32_t precompute_initial_volumes;
    float initial_velocity_scale;
    float position_jitter;
    uint32_t rng_seed;
    uint32_t material_id;
    uint32_t has_mass_override;
    float mass_override;
} emerge_spawn_region;

/* BodyState (spacetime/solver/query.rs:17-32). */
typedef struct emerge_body_state {
    uint64_t count;
    float avg_volume_ratio;
    float max_volume_ratio;
    float avg_speed;
    float avg_det_f;
    float avg_density;
    float centroid[2];
    uint32_t pad_;
} emerge_body_state;

/* StepTiming (systems/diagnostics/snapshot.rs:82-105), microseconds of GPU time
 * measured with CUDA events on the simulation's stream.  Filled per phase only
 * when the simulation runs in the instrumented (non-graph) mode; in graph mode
 * only total_us is filled.  fields/thermal/spatial_hash/phase_sleep are 0. */
typedef struct emerge_step_timing {
    uint64_t p2g_us;
    uint64_t grid_update_us;
    uint64_t g2p_us;
    uint64_t fields_us;
    uint64_t thermal_us;
    uint64_t cfl_us;
    uint64_t spatial_hash_us;
    uint64_t phase_sleep_us;
    uint64_t project_us;
    uint64_t density_us;
    uint64_t total_us;
} emerge_step_timing;

typedef struct emerge_sim emerge_sim;

/* ---- lifecycle -------------------------------------------------------------- */

/* Simulation::empty(config) (spacetime/solver/lifecycle.rs:26-54): validates the
 * config (SimConfig::validate, config.rs:247-299), registers the fallback material
 * at id 0 and one SlipBoundary(config.boundary_thickness) (lifecycle.rs:29-30). */
emerge_status emerge_cuda_create(const emerge_sim_config *config, int device, emerge_sim **out);
/* Drop for Simulation. */
emerge_status emerge_cuda_destroy(emerge_sim *sim);
/* Message for the last failed call on `sim` (never NULL). */
const char *emerge_cuda_last_error(const emerge_sim *sim);
/* Message for the last failed emerge_cuda_create on this thread. */
const char *emerge_cuda_last_global_error(void);

/* MaterialRegistry contents (materials/registry.rs:12-112; all_params :110).
 * Replaces the whole registry with `count` entries, ids 0..count-1 (count <= 64,
 * MAX_MATERIAL_SLOTS registry.rs:6).  Entry 0 replaces the default material and,
 * like with_default_material (lifecycle.rs:107-111), re-runs init_particle on
 * every particle whose material changed. */
emerge_status emerge_cuda_set_materials(emerge_sim *sim, const emerge_material_params *params,
                                        uint32_t count);
/* Boundary list (Simulation::boundaries, solver/mod.rs:50): `n` SlipBoundary
 * thicknesses applied in order (with_boundary lifecycle.rs:114 appends;
 * set_boundary_condition :353 replaces). */
emerge_status emerge_cuda_set_slip_boundaries(emerge_sim *sim, const uint64_t *thickness,
                                              uint32_t n);

/* ---- sleep partition ---------------------------------------------------------- */

/* Simulation::active_count (particles.rs:314): reference indices [0, active) are awake.
 * With SimConfig::sleep_threshold > 0 particles below the speed threshold with zero
 * activation sleep at the end of every substep and sleeping particles whose stencil meets
 * a cell of a substep's P2G wake (step.rs:107-131, 299-315); sleep_particle / wake_particle
 * swap reference indices exactly as the reference (particles.rs:227-268). */
emerge_status emerge_cuda_active_count(emerge_sim *sim, uint64_t *active_count);

/* Replaces every particle (reference order) and the active-zone size: the write-back of
 * the reference's particle-set edits that take host predicates (remove_particles
 * particles.rs:177-205, retain_particles lifecycle.rs:237-253, split_particles :271-310,
 * wake_tag / sleep_tag particles.rs:271-312), which a shim runs on the host copy. */
emerge_status emerge_cuda_replace_particles(emerge_sim *sim, const emerge_particle *particles,
                                            uint64_t n, uint64_t active_count);

/* ---- force fields ------------------------------------------------------------- */

/* Built-in force fields (forces/fields/): per particle v += sub_dt * sum of the
 * fields' accelerations after G2P, then the G2P speed clamp again (step.rs:212-259).
 * The reference's Field trait objects can hold arbitrary code; the device runs these
 * kinds, which cover every built-in field except SpatialDragField (a host function
 * pointer). */
enum {
    EMERGE_FIELD_GRAVITY_WELL = 1,       /* gravity.rs: params {G, softening, cutoff, switch_on};
                                            data: count sources (x, y, mass) */
    EMERGE_FIELD_BUOYANCY = 2,           /* buoyancy.rs: {fluid_density, gravity.x, gravity.y,
                                            min_density} */
    EMERGE_FIELD_LINEAR_DRAG = 3,        /* drag.rs: {target.x, target.y, drag_coefficient};
                                            material_mask */
    EMERGE_FIELD_RADIAL_CONFINEMENT = 4, /* confinement.rs: {center.x, center.y, radius, stiffness} */
    EMERGE_FIELD_AABB_CONFINEMENT = 5,   /* confinement.rs: {min.x, min.y, max.x, max.y, stiffness} */
    EMERGE_FIELD_COULOMB = 6,            /* coulomb.rs: {k, softening, cutoff, switch_on}; data: count
                                            sources (x, y, charge), then n_charges charges by
                                            material id */
    EMERGE_FIELD_UNIFORM_ELECTRIC = 7,   /* em.rs: {field.x, field.y}; data: n_charges charges by
                                            material id */
    EMERGE_FIELD_CHEMOTAXIS = 8,         /* chemotaxis.rs: {sensitivity}; material_filter; data:
                                            count x count potential phi[x * count + y] */
    EMERGE_FIELD_NBODY_GRAVITY = 9       /* n_body.rs: {G, softening, theta, max_depth,
                                            max_bodies_per_node}: the particles' own Plummer-softened
                                            gravity through a Barnes-Hut quadtree over every
                                            particle of positive mass, rebuilt on the device each
                                            substep after G2P.  theta in (0, 1]; max_depth an
                                            integer in 0..10 (the reference takes any usize);
                                            max_bodies_per_node a non-negative integer.  All
                                            NBody fields of a simulation share max_depth and
                                            max_bodies_per_node (one tree) */
};
#define EMERGE_FIELD_ALL_MATERIALS 0xFFFFFFFFu

/* One field (48 bytes).  Material charge maps (HashMap<u32, f32>) are flattened to a table
 * indexed by material id; ids at or past n_charges have no charge. */
typedef struct emerge_force_field {
    uint32_t kind;             /* EMERGE_FIELD_* */
    uint32_t material_mask;    /* LinearDrag: bit (id & 31) set = applies; ALL_MATERIALS = all */
    uint32_t material_filter;  /* Chemotaxis: only this material id; ALL_MATERIALS = no filter */
    uint32_t count;            /* sources (GravityWell, Coulomb) or grid_res (Chemotaxis) */
    uint32_t data_offset;      /* first float of this field's data in the data array */
    uint32_t n_charges;        /* Coulomb, UniformElectric */
    float params[6];
} emerge_force_field;

/* Replaces the simulation's force fields (Simulation::add_force_field / add_named_force_field /
 * remove_force_field / clear_force_fields, lifecycle.rs:368-392: the caller keeps the named
 * list and passes it in application order).  `data` holds every field's sources, charge
 * tables and potentials; n = 0 clears. */
emerge_status emerge_cuda_set_force_fields(emerge_sim *sim, const emerge_force_field *fields,
                                           uint32_t n, const float *data, uint64_t n_data);
/* Field::acceleration (forces/fields/force_field.rs) summed over the simulation's fields in
 * application order, for every particle at its current state: out[2 i], out[2 i + 1] for
 * reference index i (n = the particle count).  NBodyGravityField builds its tree from the
 * current positions first, as prepare() does. */
emerge_status emerge_cuda_field_accelerations(emerge_sim *sim, float *out, uint64_t n);

/* ---- multi-field contact and two-phase mixture ---------------------------------- */

/* Multi-field contact (spacetime/grid/contact.rs) runs when some particle has
 * contact_group != 0, the two-phase mixture coupling (spacetime/grid/mixture.rs) when some
 * material slot has a phase.  With EMERGE_OPT_DETERMINISTIC the cell-sorted scatter records
 * give each contact cell its point cloud in particle index order (the reference's sums, bit
 * for bit); otherwise the fused step sums the fields with the total and gathers each
 * contact cell's points from per-cell particle lists.  After the grid update (step.rs:166-197)
 * every grip cell gets a logistic-regression interface normal (grid/contact_normal.rs) or
 * the grip-mass gradient, Coulomb friction or the directional grip, and the overlap
 * correction; every mixture cell the implicit Darcy drag between the phases and, with
 * SimConfig::mixture_pressure_iterations > 0, the Jacobi pressure projection.  G2P reads
 * the resolved velocities (transfer/g2p.rs:219-238). */

/* Simulation::with_contact_grip (lifecycle.rs:125-131): DirectionalContactGrip
 * (grid/directional_grip.rs) replaces contact_friction with mu_easy / mu_resist by slip
 * direction.  (dir_x, dir_y) is the grip's stored easy direction, already normalised as
 * DirectionalContactGrip::new / set_easy_direction store it (normalize_or_zero).
 * enabled = 0 removes the grip.  mu outside [0, 1] is EMERGE_ERR_INVALID_ARG. */
emerge_status emerge_cuda_set_contact_grip(emerge_sim *sim, int enabled, float mu_easy, float mu_resist,
                                          float dir_x, float dir_y);
/* MaterialModel::mixture_phase per material slot (matter/materials/mod.rs:170-172,
 * WithMixturePhase :296-357): 0 none, 1 solid, 2 fluid; slots at or past `count` have none.
 * The caller passes the table again whenever the registry changes. */
emerge_status emerge_cuda_set_mixture_phases(emerge_sim *sim, const uint32_t *phases, uint32_t count);

/* ---- particles ---------------------------------------------------------------- */

/* Simulation::add_body (spacetime/solver/particles.rs:355-423): lattice spawn with
 * the LCG (solver/mod.rs:88-175), tag stamping, init_particle, and the local
 * initial-volume estimate (density.rs:81-144) on the device. */
emerge_status emerge_cuda_add_body(emerge_sim *sim, const emerge_spawn_region *spawn,
                                   uint32_t *tag_out);
/* Simulation::new (lifecycle.rs:57-99) particle set-up for an empty simulation:
 * spawns the region with tag 0 and, if spawn->precompute_initial_volumes, runs the
 * full estimate_particle_volumes (density.rs:41-72) on the device. */
emerge_status emerge_cuda_init_with_spawn(emerge_sim *sim, const emerge_spawn_region *spawn);
/* GpuSimulation::new(config, Vec<Particle>, registry) particle upload
 * (systems/gpu/solver/mod.rs:246): appends `n` particles as-is.  When
 * estimate_volumes != 0 the appended group gets add_body's local volume estimate. */
emerge_status emerge_cuda_add_particles(emerge_sim *sim, const emerge_particle *particles,
                                        uint64_t n, int estimate_volumes);
/* Particles::len (matter/particle.rs:300). */
emerge_status emerge_cuda_particle_count(const emerge_sim *sim, uint64_t *n_out);
/* Simulation::particles() (lifecycle.rs:214): copies all particles, in the
 * reference's index order, into `out` (n must equal the particle count). */
emerge_status emerge_cuda_read_particles(emerge_sim *sim, emerge_particle *out, uint64_t n);
/* Asynchronous Simulation::particles() (no reference counterpart: the reference's read is a
 * borrow of host memory).  Enqueues the copy of every particle into `out` (reference index
 * order, n = particle count) after the work already queued, and returns at once.  The copy
 * runs on a stream of its own: later steps and uploads wait only for its device-side
 * gather, so the device-to-host transfer overlaps them.  `out` is complete after the next
 * emerge_cuda_synchronize; page-locked memory (emerge_cuda_host_alloc) lets the transfer
 * run asynchronously.  Successive calls complete in order. */
emerge_status emerge_cuda_read_particles_async(emerge_sim *sim, emerge_particle *out, uint64_t n);
/* Simulation::particles_mut() (lifecycle.rs:233) write-back: replaces every
 * particle's state from `in` (reference index order), after the work already queued.  The
 * host-to-device copy runs on a stream of its own and overlaps that work; the call returns
 * once `in` has been copied. */
emerge_status emerge_cuda_write_particles(emerge_sim *sim, const emerge_particle *in, uint64_t n);

/* ---- stepping ------------------------------------------------------------------ */

/* Simulation::step_n(n) (spacetime/solver/step.rs:327-331); each step is
 * Simulation::step (step.rs:23-60): adaptive substeps with CFL (step.rs:434-488),
 * state projection (:347-429), density recompute (density.rs:41-72), P2G
 * (transfer/p2g.rs:24-72), grid update (grid/mod.rs:264-291, step.rs:150-165),
 * G2P + constitutive update (transfer/g2p.rs:151-343).  Asynchronous: returns
 * once the work is queued.  `timing` (nullable) receives the last step's timing
 * and forces a synchronisation. */
emerge_status emerge_cuda_step(emerge_sim *sim, uint32_t n_steps, emerge_step_timing *timing);
/* Simulation::last_substeps (step.rs:323). Synchronises. */
emerge_status emerge_cuda_last_substeps(emerge_sim *sim, uint64_t *out);
/* Simulation::effective_dt (step.rs:319). Synchronises. */
emerge_status emerge_cuda_effective_dt(emerge_sim *sim, float *out);
/* last_vel_clamp_count / last_j_projection_count (solver/mod.rs:63-64) and
 * last_sim_time_dropped (:65) of the last step. Synchronises. */
emerge_status emerge_cuda_last_counters(emerge_sim *sim, uint64_t *vel_clamp_count,
                                        uint64_t *j_projection_count, float *sim_time_dropped);
/* Blocks until all queued work of `sim` is done, asynchronous readbacks included. */
emerge_status emerge_cuda_synchronize(emerge_sim *sim);

/* ---- queries --------------------------------------------------------------------- */

/* Simulation::region_state(center, radius) (spacetime/solver/queries.rs:125-141):
 * device reduction (f64 accumulators) over active particles with |x-c|^2 <= r^2. */
emerge_status emerge_cuda_region_state(emerge_sim *sim, float cx, float cy, float radius,
                                       emerge_body_state *out);

/* ---- options and diagnostics ------------------------------------------------------- */

/* Tuning knobs that change no result beyond float summation order:
 *   EMERGE_OPT_USE_GRAPH       1 = capture each step in a CUDA graph with a device-side
 *                              substep loop (default), 0 = host-driven substep loop with
 *                              per-phase event timing.
 *   EMERGE_OPT_SORT_INTERVAL   re-sort particles by tile every N steps (default 16;
 *                              0 = only before the first step after particles are added;
 *                              see emerge_cuda_sort_now).
 *   EMERGE_OPT_P2G_AGGREGATE   0 = one global reduction per contribution (default, the
 *                              fastest measured: reductions in L2 cost less than combining
 *                              contributions first); 1 = contributions of lanes sharing a
 *                              base cell are summed in the warp before one global reduction
 *                              per cell; 2 = lane pairs and quads sharing a base cell are
 *                              summed first.
 *   EMERGE_OPT_DETERMINISTIC   1 = reference-order mode: every grid cell sums its P2G and
 *                              density contributions sequentially in the reference's
 *                              particle index order (transfer/p2g.rs:16-23), so results
 *                              do not depend on thread scheduling; slower (for parity
 *                              checks and reproducible runs).  0 = fast fused path
 *                              (default).  Set it before adding particles for the
 *                              spawn-time volume estimate to use it too.
 *   EMERGE_OPT_PRECISE_MATH    1 = evaluate exp/log/sin/sinh/pow in double and round once
 *                              to f32 (agrees with the reference's glibc f32 results in
 *                              nearly all cases), 0 = CUDA single-precision functions,
 *                              -1 = follow EMERGE_OPT_DETERMINISTIC (default). */
enum {
    EMERGE_OPT_USE_GRAPH = 1,
    EMERGE_OPT_SORT_INTERVAL = 2,
    EMERGE_OPT_P2G_AGGREGATE = 3,
    EMERGE_OPT_DETERMINISTIC = 4,
    EMERGE_OPT_PRECISE_MATH = 5,
    EMERGE_OPT_TILE_SHAPE = 7,      /* batches: the particle order the sort gives each scene (what
                                     * patch of grid a CTA covers): 0 8 x 8-cell tiles in Morton
                                     * order, cells row by row (default); 1 the same tiles, cells
                                     * in Morton order; 2 16 x 16 blocks of four 16 x 4 strips;
                                     * 3 16 x 16 blocks of four 4 x 16 strips */
    EMERGE_OPT_CHUNKS_PER_CTA = 8   /* batches: particles per CTA of the particle and density
                                     * passes, in chunks of 256: 1 (default), 2 or 4 */
};
emerge_status emerge_cuda_set_option(emerge_sim *sim, int option, int64_t value);

/* Particle sort (reference GPU path: systems/gpu/shaders/particle_sort.wgsl:124-245,
 * counting sort by block_index, non-deterministic within a block).  Here: stable
 * device LSD radix sort of the current particles by key, applied as a permutation
 * of the device particle storage.  key_mode 0 = tile key (8x8-cell tiles in Morton
 * order, cell within tile), 1 = the reference's block_index key
 * (particle_sort.wgsl:94-102).  Host-visible particle order is unchanged. */
emerge_status emerge_cuda_sort_now(emerge_sim *sim, int key_mode);
/* Test hook for the sort: computes keys for `n` positions (key_mode as above, for a
 * grid of `grid_res` cells) and the stable sort permutation, on the device.
 * keys_out[i] = key of xy[i]; perm_out = stable argsort of the keys. */
emerge_status emerge_cuda_sort_keys(const float *xy, uint64_t n, uint32_t grid_res, int key_mode,
                                    uint32_t *keys_out, uint32_t *perm_out);

/* Allocation-free variant of emerge_cuda_sort_keys (no counterpart in the reference).
 * For callers that must not let a library allocate: cudaMalloc/cudaFree synchronise the
 * whole device, stalling the caller's other streams, and fail outright when the caller's
 * memory pool has reserved the device's memory.  Same keys and the same stable
 * permutation as emerge_cuda_sort_keys, but every buffer is the caller's DEVICE memory
 * (current device, or managed) and the work is enqueued on the caller's stream:
 *   xy_dev    n (x, y) float pairs, 8-byte aligned
 *   keys_dev  n uint32: key of xy[i];  perm_dev  n uint32: stable argsort of the keys
 *   stream    cudaStream_t as void* (NULL = the legacy default stream)
 * The library allocates nothing; it works in one fixed array of about 1 MiB inside its
 * device image, so n is limited to EMERGE_SORT_NOALLOC_MAX and a larger n returns
 * EMERGE_ERR_INVALID_ARG before any device work.  grid_res must lie in 1..32768 (the
 * keys then fit in 30 bits) and key_mode be 0 or 1; other values return
 * EMERGE_ERR_INVALID_ARG, also before any device work.  Nothing needs to start at zero
 * (the outputs need no initial contents; the working array is written before it is read).
 * Returns once the work is enqueued; results are ready when the stream reaches it.
 * The first call on each device (and the first after that device's context was destroyed,
 * e.g. by cudaDeviceReset) looks up the working array's address (cudaGetSymbolAddress):
 * make that first call before any stream capture begins.  With CUDA's lazy module loading
 * (the default since CUDA 12.2) that first call is also when the driver loads this part of
 * the library's device image and reserves the fixed array, so a caller whose memory pool
 * will reserve the whole device should make the first call before the pool does, or set
 * CUDA_MODULE_LOADING=EAGER.
 * Launch errors: an error that earlier, unrelated work left pending on the calling thread
 * is not reported here as this call's failure and stays pending for its owner; a launch
 * of this call that fails with that same error code cannot be told apart from it.
 * All calls on one device share the one working array, so calls whose work may overlap
 * in time (unordered streams, several host threads) race and corrupt each other's
 * results: order them on one stream or with events. */
#define EMERGE_SORT_NOALLOC_MAX 65536u
emerge_status emerge_cuda_sort_keys_noalloc(const float *xy_dev, uint32_t n, uint32_t grid_res,
                                            int key_mode, uint32_t *keys_dev, uint32_t *perm_dev,
                                            void *stream);

/* The CUDA stream the simulation's work runs on (cudaStream_t as void*). */
void *emerge_cuda_stream(emerge_sim *sim);

/* ---- measurement helpers (no reference counterpart) --------------------------------- */

/* Records CUDA event `slot` (0..15) on the simulation's stream. */
emerge_status emerge_cuda_event_record(emerge_sim *sim, int slot);
/* Milliseconds between two recorded events (synchronises on `to`). */
emerge_status emerge_cuda_event_elapsed(emerge_sim *sim, int from, int to, float *ms);
/* Evicts the L2 cache: writes a device buffer larger than L2 on the simulation's stream. */
emerge_status emerge_cuda_flush_l2(emerge_sim *sim);
/* Page-locked host memory for fast uploads/readbacks (cudaMallocHost). */
emerge_status emerge_cuda_host_alloc(size_t bytes, void **out);
emerge_status emerge_cuda_host_free(void *ptr);

/* Lifetime counters of a simulation. Synchronises. */
typedef struct emerge_stats {
    uint64_t steps;              /* Simulation::step calls executed */
    uint64_t substeps;           /* substeps executed */
    uint64_t kernel_launches;    /* kernels of this library executed (see emerge_cuda_kernel_launches) */
    uint64_t p2g_blocks;         /* CTAs of the particle/density passes */
    uint64_t p2g_fallback_blocks;/* of which scattered with global reductions (window did not fit) */
    uint64_t sorts;              /* particle re-sorts */
} emerge_stats;
emerge_status emerge_cuda_stats(emerge_sim *sim, emerge_stats *out);
/* Number of kernels this library launched on `sim` since creation (graph launches
 * count every kernel node executed, substep loops included). Synchronises. */
emerge_status emerge_cuda_kernel_launches(emerge_sim *sim, uint64_t *out);

/* ---- learned return-mapping closure (no counterpart in the reference) --------------
 * A 6 -> 64 -> 64 -> 64 -> 3 SiLU network replaces the smooth plastic branch of the
 * Drucker-Prager (sand.rs:156-194, model 0) and NACC (nacc.rs:129-223, model 1) return
 * mappings inside the particle pass, evaluated on the tensor cores in BF16 with FP32
 * accumulation.  The exact branch decisions (yield test, DP tip, NACC caps) stay exact;
 * inputs outside the training box use the plain mapping; a hashed sample of network
 * evaluations (one in judge_stride) is also run through the plain mapping and the relative
 * error of the principal Kirchhoff stress is recorded.  Workflow: closure_log (run steps with
 * the plain mapping while logging), closure_train per model, closure_enable. */
typedef struct emerge_closure_stats {
    uint64_t smooth;         /* particles that reached a smooth plastic branch */
    uint64_t net;            /* of which the network evaluated */
    uint64_t hull_fallback;  /* of which fell outside the training box (plain mapping) */
    uint64_t judged;         /* network results also computed by the plain mapping */
    uint64_t logged[2];      /* samples logged per model (capped at the capacity) */
    double err_mean;         /* mean relative stress error of the judged results */
    float err_max;           /* max relative stress error of the judged results */
    uint32_t pad_;
    uint64_t judge_replaced; /* judged results above the judge's bar, replaced by the plain one */
    float err_p50, err_p99;  /* percentiles of the judged errors (quarter-decade bins: upper edge) */
} emerge_closure_stats;

typedef struct emerge_closure_train_config {
    uint32_t epochs;
    uint32_t batch;          /* <= 65536 */
    float lr;                /* Adam learning rate */
    float lr_decay;          /* per-epoch factor (0 = none) */
    float beta1, beta2, eps; /* Adam */
    float val_fraction;      /* held-out share, seeded split */
    uint64_t seed;
    uint64_t max_samples;    /* 0 = all logged */
} emerge_closure_train_config;

typedef struct emerge_closure_train_report {
    uint64_t n_train, n_val;
    float train_loss;        /* MSE of normalised outputs, last epoch */
    float val_loss;          /* MSE of normalised outputs, held out, tensor-core inference */
    float val_err_mean, val_err_p50, val_err_p99, val_err_max;  /* relative stress error */
    float val_err_trial_mean;  /* the same error when the mapping is skipped (trial state kept) */
    float seconds;
    uint32_t steps;          /* Adam steps */
} emerge_closure_train_report;

/* Log (inputs, targets) of the plain mapping on the smooth branches from the following
 * steps: up to `capacity` samples per model, one evaluation in `stride` (hashed).
 * capacity 0 stops logging. */
emerge_status emerge_cuda_closure_log(emerge_sim *sim, uint64_t capacity, uint32_t stride);
/* Trains the network of `model` (0 Drucker-Prager, 1 NACC) on its logged samples with the
 * library's own forward, backward and Adam kernels, then installs it. */
emerge_status emerge_cuda_closure_train(emerge_sim *sim, int model, const emerge_closure_train_config *cfg,
                                        emerge_closure_train_report *report);
/* Turns network inference on or off for the following steps. */
emerge_status emerge_cuda_closure_enable(emerge_sim *sim, int on, uint32_t judge_stride);
/* Lifetime counters; reset != 0 zeroes them (the logged counts are kept). */
emerge_status emerge_cuda_closure_stats(emerge_sim *sim, emerge_closure_stats *out, int reset);
/* How the enabled closure runs.  defer = 1 (default): the particle pass queues the particles
 * the network maps and a tile kernel evaluates them 128 at a time on the tcgen05 tensor cores
 * (accumulators in tensor memory) and finishes their update and P2G; the particle pass keeps
 * the plain pass's register budget.  Scenes with force fields, ASFLIP, a sleep partition or
 * multi-field sums, and batches, evaluate inside the particle pass (defer = 0: always).
 * judge_bar: a judged result whose relative stress error exceeds it is replaced by the plain
 * mapping's (default 1e-3; +inf keeps every network result). */
emerge_status emerge_cuda_closure_set_mode(emerge_sim *sim, int defer, float judge_bar);
/* FP32 master parameters (8963 floats: W1[6][64] b1 W2[64][64] b2 W3[64][64] b3 W4[64][3] b4)
 * and normalisation (in_shift[6] in_scale[6] out_shift[3] out_scale[3]) of a network. */
emerge_status emerge_cuda_closure_get_params(emerge_sim *sim, int model, float *params, float *norm);
/* Installs a network: parameters, normalisation as above, and the training box of the
 * normalised inputs (hull_lo[6] hull_hi[6]). */
emerge_status emerge_cuda_closure_set_params(emerge_sim *sim, int model, const float *params,
                                             const float *norm, const float *hull);
/* Copies up to `max` logged samples of `model` (x: max x 6 raw inputs, t: max x 3 targets);
 * *n receives the number copied. */
emerge_status emerge_cuda_closure_get_log(emerge_sim *sim, int model, float *x, float *t, uint64_t max,
                                          uint64_t *n);
/* Test hooks on host arrays (they allocate device memory): loss and gradient of the MSE
 * of normalised outputs over a batch; one Adam step; the BF16 tensor-core inference. */
emerge_status emerge_cuda_mlp_loss_grad(const float *params, const float *x, const float *t, uint32_t batch,
                                        float *loss, float *grad);
emerge_status emerge_cuda_mlp_adam(float *params, float *m, float *v, const float *grad, uint32_t n,
                                   uint32_t step, float lr, float beta1, float beta2, float eps);
emerge_status emerge_cuda_mlp_infer_bf16(const float *params, const float *x, uint32_t n, float *y);
/* The same network evaluated as the closure's tile kernel does it: 128 inputs per tile on the
 * tcgen05 tensor cores (BF16 operands in shared memory, FP32 accumulators in tensor memory,
 * SiLU from the hardware tanh).  EMERGE_ERR_TIMEOUT if a bounded wait gave up. */
emerge_status emerge_cuda_mlp_infer_tc(const float *params, const float *x, uint32_t n, float *y);
/* Test hook (no reference counterpart): the tile kernel's SiLU, z (1 + tanh(z / 2)) / 2 with
 * the hardware tanh, on n host values. */
emerge_status emerge_cuda_silu_fast(const float *x, uint32_t n, float *y);

/* ---- batched scenes (no counterpart in the reference) -----------------------------
 * Many independent scenes advanced together: every substep is one launch per kernel for
 * all scenes (the passes find their scene from CTA and tile tables), and each scene keeps
 * its own grid size, materials, boundaries, configuration and CFL substep schedule.  A
 * batch is built from simulations set up with the single-scene API (their particles are
 * copied; the simulations stay usable and independent).  Scenes run the fast path. */
typedef struct emerge_batch emerge_batch;

#define EMERGE_TUNE_MAX_TRIALS 16
typedef struct emerge_batch_tune_report {
    int32_t sort_interval;       /* chosen */
    int32_t aggregate;           /* chosen P2G warp aggregation (0 / 1) */
    int32_t tile_shape;          /* chosen EMERGE_OPT_TILE_SHAPE */
    int32_t chunks_per_cta;      /* chosen EMERGE_OPT_CHUNKS_PER_CTA */
    uint32_t n_trials;
    uint32_t from_cache;         /* 1: taken from the cache file, no trials run */
    float best_ms;               /* GPU ms per frame of the chosen setting (from the cache: as
                                    stored when it was tuned) */
    int32_t trial_sort_interval[EMERGE_TUNE_MAX_TRIALS];
    int32_t trial_aggregate[EMERGE_TUNE_MAX_TRIALS];
    int32_t trial_tile_shape[EMERGE_TUNE_MAX_TRIALS];
    int32_t trial_chunks[EMERGE_TUNE_MAX_TRIALS];
    float trial_ms[EMERGE_TUNE_MAX_TRIALS];  /* GPU ms per frame of each trial */
} emerge_batch_tune_report;

emerge_status emerge_cuda_batch_create(emerge_sim *const *sims, uint32_t n_sims, emerge_batch **out);
emerge_status emerge_cuda_batch_destroy(emerge_batch *batch);
/* Message for the last failed call on `batch` (or the last failed create when NULL). */
const char *emerge_cuda_batch_last_error(const emerge_batch *batch);
/* Simulation::step() for every scene, n_steps times (synchronises at the end). */
emerge_status emerge_cuda_batch_step(emerge_batch *batch, uint32_t n_steps);
/* Steps n_steps times, timing each frame with CUDA events on the batch's stream (optionally
 * writing a buffer larger than L2 before each frame); *ms_total = sum of frame times. */
emerge_status emerge_cuda_batch_time_steps(emerge_batch *batch, uint32_t n_steps, int flush_l2, float *ms_total);
emerge_status emerge_cuda_batch_scene_count(const emerge_batch *batch, uint32_t *n);
emerge_status emerge_cuda_batch_particle_count(const emerge_batch *batch, uint32_t scene, uint64_t *n);
/* particles() of one scene, reference index order. */
emerge_status emerge_cuda_batch_read_particles(emerge_batch *batch, uint32_t scene, emerge_particle *out, uint64_t n);
emerge_status emerge_cuda_batch_region_state(emerge_batch *batch, uint32_t scene, float cx, float cy, float radius,
                                             emerge_body_state *out);
/* Per scene: substeps of the last frame (last) and lifetime substeps (total); either may be NULL. */
emerge_status emerge_cuda_batch_substeps(emerge_batch *batch, uint64_t *last, uint64_t *total);
/* EMERGE_OPT_USE_GRAPH, EMERGE_OPT_SORT_INTERVAL, EMERGE_OPT_P2G_AGGREGATE,
 * EMERGE_OPT_TILE_SHAPE, EMERGE_OPT_CHUNKS_PER_CTA. */
emerge_status emerge_cuda_batch_set_option(emerge_batch *batch, int option, int64_t value);
/* Autotuner (no reference counterpart): picks the tile shape, the particles per CTA, the
 * sort interval and the P2G warp aggregation for this batch by coordinate descent -- each knob
 * in turn takes every value (4 + 3 + 3 + 2 trials; each re-sorts, runs one untimed frame
 * and times steps_per_trial frames), keeping the fastest -- and applies the result; the batch advances by those
 * frames.  None of the knobs changes a result beyond float summation order.  cache_path
 * (NULL or "" = none): a text file of tuned settings keyed by the batch's signature (device
 * name, SM count, every scene's grid size, particle count and model set); a hit applies the
 * stored setting without trials, a tuned setting is stored. */
emerge_status emerge_cuda_batch_autotune(emerge_batch *batch, uint32_t steps_per_trial, const char *cache_path,
                                         emerge_batch_tune_report *report);

#ifdef __cplusplus
}
#endif
#endif /* EMERGE_CUDA_H */
