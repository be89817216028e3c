// sim.cu -- host runtime of the CUDA backend and the C ABI (include/emerge_cuda.h).
//
// One emerge_sim owns: the particle SoA (two slot-order copies, swapped by the
// sort), the tiled grid, the sort scratch, the device step controller, an AoS
// staging buffer for uploads/readbacks, a stream, and a CUDA graph per step.
// The graph is [k_step_begin] -> while(cont){k_substep_begin, k_grid_update,
// k_particle, k_density?}: the adaptive substep loop of Simulation::step
// (spacetime/solver/step.rs:34-49) runs on the device with no host round trip.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "closure_host.h"
#include "device_state.cuh"
#include "kernels.h"

using namespace emerge;

namespace {

thread_local std::string g_global_error;

struct Buffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    ~Buffer() { reset(); }
    void reset() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Bump allocator over one device allocation, 256-byte aligned pieces.
struct Carver {
    uintptr_t p;
    explicit Carver(void *base) : p(reinterpret_cast<uintptr_t>(base)) {}
    template <class T>
    T *take(size_t n) {
        p = (p + 255) & ~static_cast<uintptr_t>(255);
        T *r = reinterpret_cast<T *>(p);
        p += n * sizeof(T);
        return r;
    }
};

DevParticles carve_particles(Carver &c, size_t cap) {
    DevParticles P;
    P.x = c.take<float2>(cap);
    P.v = c.take<float2>(cap);
    P.c = c.take<float4>(cap);
    P.f = c.take<float4>(cap);
    P.mass = c.take<float>(cap);
    P.v0 = c.take<float>(cap);
    P.vol = c.take<float>(cap);
    P.rho = c.take<float>(cap);
    P.mat = c.take<uint32_t>(cap);
    P.jp = c.take<float>(cap);
    P.h = c.take<float>(cap);
    P.q = c.take<float>(cap);
    P.lvs = c.take<float>(cap);
    P.temperature = c.take<float>(cap);
    P.activation = c.take<float>(cap);
    P.act_dir = c.take<float2>(cap);
    P.pinned = c.take<uint32_t>(cap);
    P.user_tag = c.take<uint32_t>(cap);
    P.muscle = c.take<uint32_t>(cap);
    P.contact = c.take<uint32_t>(cap);
    P.sleeping = c.take<uint32_t>(cap);
    P.scalar = c.take<float>(cap);
    P.slot_to_index = c.take<uint32_t>(cap);
    P.rho_dp = c.take<float>(cap);
    return P;
}

// Exact size of one particle set: a dry-run carve from address 0, so the allocation
// and carve_particles can never disagree.
size_t particle_set_bytes(size_t cap) {
    Carver c(nullptr);
    carve_particles(c, cap);
    return static_cast<size_t>(c.p) + 256;
}

bool model_supported(uint32_t m) {
    return m <= M_GRANULAR_FLUID;  // every ConstitutiveModel id (materials/mod.rs:53-66)
}

// LcgRng (spacetime/solver/mod.rs:154-175)
struct Lcg {
    uint32_t state;
    uint32_t next_u32() {
        state = state * 1664525u + 1013904223u;
        return state;
    }
    float next_f32() { return static_cast<float>(next_u32()) / 4294967296.0f; }
};

size_t sat_sub_sz(size_t a, size_t b) { return a > b ? a - b : 0; }

}  // namespace

struct emerge_sim {
    emerge_sim_config cfg{};
    DevConfig dcfg{};
    int device = 0;
    int sm_count = 0;        // streaming multiprocessors of the device (persistent grids)
    cudaStream_t stream = nullptr;
    std::string error;

    // particles
    size_t n = 0, cap = 0;
    Buffer pbuf;             // two particle sets
    DevParticles P[2];
    int cur = 0;
    Buffer staging;          // AoS staging (cap * 128 B)
    emerge_particle *d_aos = nullptr;
    // asynchronous readback: its own AoS staging and stream, so a step's device-to-host copy
    // overlaps the next step's upload and work
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_gathered = nullptr;
    Buffer staging_rb;
    // uploads: their own AoS staging and stream, so a write-back's host-to-device copy
    // overlaps the work already queued (the step before it)
    cudaStream_t up_stream = nullptr;
    cudaEvent_t ev_up_done = nullptr, ev_up_free = nullptr;
    Buffer staging_up;
    bool up_used = false;
    uint32_t next_tag = 1;
    LoadFlagsHost lf;
    std::vector<uint8_t> host_pinned_flag;  // not used for stepping; kept for add/write scans

    // grid
    int res = 0, tpd = 0;
    Buffer gbuf;
    GridView g{};

    // materials / boundaries / force fields
    std::vector<emerge_material_params> mats;
    Buffer mbuf;
    std::vector<uint64_t> bounds;
    int n_fields = 0;
    Buffer fbuf;  // force field table, then its data
    NBodyTreeHost nb;        // NBodyGravityField's tree (nb.depth < 0: none)
    Buffer nbbuf;            // its arrays, sized for nb_cap particles and nb_alloc_depth
    size_t nb_cap = 0;
    int nb_alloc_fields = 0;  // NBody fields the accel blocks were allocated for
    int nb_alloc_depth = -1;

    // sleep partition (solver/mod.rs:40-42): reference indices [0, active) are awake
    uint64_t active = 0;
    Buffer zbuf;            // event count, event log, index remap table
    uint32_t zlog_cap = 0;
    std::vector<uint32_t> pos_of_base, base_of_pos;  // index swaps since the last commit
    bool perm_dirty = false;

    // controller
    Buffer sbuf;
    StepState *d_state = nullptr;
    StepState *h_state = nullptr;  // pinned mirror
    StepState *h_state_dev = nullptr;  // its device address (nullptr: not mapped)
    Buffer region_buf;

    // sort
    Buffer sortbuf;
    SortScratch sort;
    size_t sort_cap = 0;
    uint64_t steps_since_sort = 0;
    bool sorted_once = false;
    unsigned long long fallback_at_sort = 0, blocks_at_sort = 0;

    // multi-field contact (grid/contact.rs) and two-phase mixture (grid/mixture.rs)
    bool contact_seen = false;       // some particle has contact_group != 0
    std::vector<uint32_t> phases;    // MixturePhase per material slot: 0 none, 1 solid, 2 fluid
    int grip_on = 0;                 // Simulation::contact_grip (solver/mod.rs:55)
    float grip_mu_easy = 0.0f, grip_mu_resist = 0.0f, grip_dir[2] = {0.0f, 0.0f};
    Buffer mfbuf;                    // the multi-field grid arrays and the phase table
    Buffer ptsbuf;                   // the contact point cloud, one entry per scatter record
    size_t pts_cap = 0;
    Buffer listbuf;                  // fast pipeline: the contact list nodes, one per particle slot
    size_t list_cap = 0;
    float4 *det_points() const { return static_cast<float4 *>(ptsbuf.ptr); }

    // reference-order (deterministic) mode
    int deterministic = 0;
    int precise_opt = -1;  // -1: precise math follows `deterministic`
    Buffer detbuf;
    SortScratch det_sort;
    float4 *det_payload = nullptr;
    uint8_t *det_fmask = nullptr;   // each record's fields (multi-field scenes)
    size_t det_cap = 0;
    int det_sorted = 0;             // which key / value buffer holds the last sort's result

    // step pipeline
    bool pending_valid = false;  // the next substep's P2G (+density) is already on the grid
    int use_graph = 1;
    int use_window = 0;
    int64_t sort_interval = 16;  // re-sort every N steps; 0 = keep the first sort
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_dirty = true;
    unsigned long long host_launches = 0;
    unsigned long long graph_launches = 0;
    unsigned long long sorts = 0;
    ClosureHost *closure = nullptr;  // learned return-mapping closure (closure.cu)
    cudaEvent_t ev[8] = {};
    cudaEvent_t user_ev[16] = {};
    Buffer flushbuf;
    emerge_step_timing last_timing{};

    int fail(emerge_status st, const std::string &msg) {
        error = msg;
        return st;
    }
};

namespace {

bool cuda_ok(emerge_sim *s, cudaError_t e, const char *what, emerge_status *out) {
    if (e == cudaSuccess) return true;
    s->error = std::string(what) + ": " + cudaGetErrorString(e);
    *out = (e == cudaErrorMemoryAllocation) ? EMERGE_ERR_OOM : EMERGE_ERR_CUDA;
    return false;
}

#define CK(call)                                                    \
    do {                                                            \
        emerge_status st_ = EMERGE_OK;                              \
        if (!cuda_ok(s, (call), #call, &st_)) return st_;           \
    } while (0)

// SimConfig::validate (config.rs:247-299) plus the device path's feature gates.
emerge_status validate_config(const emerge_sim_config &c, std::string &msg) {
    auto bad = [&](const char *m) {
        msg = m;
        return EMERGE_ERR_INVALID_ARG;
    };
    if (c.grid_res < 4) return bad("grid_res must be >= 4");
    if (!(c.grid_cell_size > 0.0f)) return bad("grid_cell_size must be positive");
    if (!(c.dt > 0.0f)) return bad("dt must be positive");
    if (!(c.cfl_coefficient > 0.0f)) return bad("cfl_coefficient must be positive");
    if (!(c.material_cfl_coefficient > 0.0f)) return bad("material_cfl_coefficient must be positive");
    if (!(c.viscous_timestep_coefficient > 0.0f))
        return bad("viscous_timestep_coefficient must be positive");
    if (!(c.min_dt > 0.0f)) return bad("min_dt must be positive");
    if (!(c.min_dt <= c.dt)) return bad("min_dt must be <= dt");
    if (!(c.projection_min_density > 0.0f)) return bad("projection_min_density must be positive");
    if (!(c.projection_min_volume > 0.0f)) return bad("projection_min_volume must be positive");
    if (!(c.projection_min_deformation_j > 0.0f))
        return bad("projection_min_deformation_j must be positive");
    if (!(c.particle_mass > 0.0f)) return bad("particle_mass must be positive");
    if (!(c.contact_friction >= 0.0f)) return bad("contact_friction must be non-negative");
    if (c.max_substeps_per_step == 0) return bad("max_substeps_per_step must be > 0");
    if (!(c.default_initial_volume > 0.0f)) return bad("default_initial_volume must be positive");
    if (!(c.j_max > 1.0f)) return bad("j_max must be > 1.0");
    if (!(c.apic_blend >= 0.0f && c.apic_blend <= 1.0f)) return bad("apic_blend must be in [0, 1]");
    if (!(c.boundary_thickness > 0 && c.boundary_thickness < c.grid_res - 1))
        return bad("boundary_thickness must be in [1, grid_res-2]");
    if (c.grid_res > 32768) {
        msg = "grid_res above 32768 is not supported by the device grid";
        return EMERGE_ERR_UNSUPPORTED;
    }
    if (!(c.asflip_blend >= 0.0f)) return bad("asflip_blend must be >= 0");
    if (c.max_substeps_per_step > 0x7fffffffull) {
        msg = "max_substeps_per_step too large";
        return EMERGE_ERR_INVALID_ARG;
    }
    return EMERGE_OK;
}

DevConfig make_dev_config(const emerge_sim_config &c, const std::vector<uint64_t> &bounds,
                          int precise) {
    DevConfig d{};
    d.precise_math = precise;
    d.res = static_cast<int>(c.grid_res);
    d.cell = c.grid_cell_size;
    d.dt = c.dt;
    d.adaptive = c.adaptive_timestep ? 1 : 0;
    d.affine_cfl = c.cfl_include_affine_speed ? 1 : 0;
    d.cfl = c.cfl_coefficient;
    d.mat_cfl = c.material_cfl_coefficient;
    d.visc_cfl = c.viscous_timestep_coefficient;
    d.min_dt = c.min_dt;
    d.project = c.project_invalid_state ? 1 : 0;
    d.min_density = c.projection_min_density;
    d.min_volume = c.projection_min_volume;
    d.min_j = c.projection_min_deformation_j;
    d.gravity = make_float2(c.gravity[0], c.gravity[1]);
    d.thickness = static_cast<int>(c.boundary_thickness);
    d.default_v0 = c.default_initial_volume;
    d.particle_mass = c.particle_mass;
    d.max_substeps = static_cast<int>(c.max_substeps_per_step);
    d.apic_blend = c.apic_blend;
    d.j_max = c.j_max;
    d.n_bound = static_cast<int>(bounds.size());
    for (size_t k = 0; k < bounds.size() && k < static_cast<size_t>(MAX_BOUNDARIES); ++k)
        d.bound_t[k] = static_cast<int>(bounds[k]);
    d.asflip = c.asflip_blend;
    return d;
}

bool mixture_on(const emerge_sim *s) {
    for (uint32_t ph : s->phases)
        if (ph != 0) return true;
    return false;
}
// Multi-field contact or mixture in use.  In the reference-order pipeline the cell-sorted
// scatter records give every contact cell its point cloud in particle index order; the fast
// pipeline sums the fields with the total and lists the particles per base cell.
bool multi_on(const emerge_sim *s) { return s->contact_seen || mixture_on(s); }
bool det_pipeline(const emerge_sim *s) { return s->deterministic != 0; }

// The sleep partition is in use: sleep scoring is on, or some particle is outside the
// active zone.
bool zones_on(const emerge_sim *s) { return s->cfg.sleep_threshold > 0.0f || s->active < s->n; }
emerge_status drain_zone_log(emerge_sim *s);
emerge_status commit_perm(emerge_sim *s);
emerge_status update_multi(emerge_sim *s);
emerge_status update_zones(emerge_sim *s);

// The simulation's device configuration: config, boundaries, force-field table, sleep
// partition.
void refresh_dev_config(emerge_sim *s) {
    s->dcfg = make_dev_config(s->cfg, s->bounds, s->dcfg.precise_math);
    s->dcfg.sleep_thr = s->cfg.sleep_threshold;
    s->dcfg.zones = (zones_on(s) && s->zbuf.ptr) ? 1 : 0;
    if (s->zbuf.ptr) {
        char *z = static_cast<char *>(s->zbuf.ptr);
        s->dcfg.zone_log_count = reinterpret_cast<uint32_t *>(z);
        s->dcfg.zone_log = reinterpret_cast<unsigned long long *>(z + 256);
        s->dcfg.zone_log_cap = s->zlog_cap;
    }
    s->dcfg.multi = (multi_on(s) && s->mfbuf.ptr) ? 1 : 0;
    s->dcfg.contact_friction = s->cfg.contact_friction;
    s->dcfg.grip_on = s->grip_on;
    s->dcfg.grip_mu_easy = s->grip_mu_easy;
    s->dcfg.grip_mu_resist = s->grip_mu_resist;
    s->dcfg.grip_dir = make_float2(s->grip_dir[0], s->grip_dir[1]);
    s->dcfg.mix_drag = s->cfg.mixture_drag_coefficient;
    s->dcfg.mix_iters = static_cast<int>(s->cfg.mixture_pressure_iterations);
    s->dcfg.mat_phase = s->mfbuf.ptr ? static_cast<const uint32_t *>(s->mfbuf.ptr) : nullptr;
    s->dcfg.mf_fast = (s->dcfg.multi && !s->deterministic) ? 1 : 0;
    s->dcfg.mf_fields = (s->contact_seen ? 1 : 0) | (mixture_on(s) ? 2 : 0);
    // One kind of field: its particles scatter into their field only and the grid update forms
    // the total.  With both kinds a particle may sit in two fields and scatters into the total
    // as well.
    s->dcfg.mf_excl = (s->dcfg.mf_fast && (s->dcfg.mf_fields == 1 || s->dcfg.mf_fields == 2)) ? 1 : 0;
    s->dcfg.nbody = NBodyView{};
    if (s->nb.depth >= 0 && s->nbbuf.ptr && s->nb_alloc_depth == s->nb.depth) {
        s->dcfg.nbody.depth = s->nb.depth;
        s->dcfg.nbody.max_bodies = s->nb.max_bodies;
        s->dcfg.nbody.root = s->nb.root;
        s->dcfg.nbody.bdata = s->nb.bdata;
        s->dcfg.nbody.order = s->nb.order;
        // the fast pipeline's build leaves one body order for all levels
        s->dcfg.nbody.stride = det_pipeline(s) ? s->nb.stride : 0;
        s->dcfg.nbody.range = s->nb.range;
        s->dcfg.nbody.com = s->nb.com;
        s->dcfg.nbody.error = &s->d_state->error_flags;
        s->dcfg.nbody.fast = det_pipeline(s) ? 0 : 1;
        s->dcfg.nbody.accel = s->nb.accel;
        s->dcfg.nbody.accel_stride = s->nb.stride;
    }
    s->dcfg.n_fields = s->n_fields;
    s->dcfg.fields = s->n_fields ? static_cast<const emerge_force_field *>(s->fbuf.ptr) : nullptr;
    s->dcfg.field_data = s->n_fields ? reinterpret_cast<const float *>(
                                           static_cast<const char *>(s->fbuf.ptr) +
                                           align_up(s->n_fields * sizeof(emerge_force_field), 256))
                                     : nullptr;
}

StepLaunch make_launch(emerge_sim *s) {
    StepLaunch L;
    L.P = s->P[s->cur];
    L.n = static_cast<int>(s->n);
    L.mats = static_cast<const MatP *>(s->mbuf.ptr);
    L.n_mats = static_cast<int>(s->mats.size());
    L.cfg = s->dcfg;
    L.st = s->d_state;
    L.g = s->g;
    int density = s->cfg.recompute_density_each_step ? 1 : 0;
    for (const auto &m : s->mats)
        if (m.model == M_FLUID) density = 1;  // needs_density_recompute (fluid.rs:261-263)
    L.density_mode = density;
    L.use_window = s->use_window;
    L.model_mask = 1u << M_FALLBACK;
    for (const auto &m : s->mats) L.model_mask |= model_bits(m);
    if (s->dcfg.n_fields > 0 || s->dcfg.asflip > 0.0f || s->dcfg.zones || s->dcfg.multi)
        L.model_mask |= 1u << M_EXTRAS_BIT;
    L.fast = det_pipeline(s) ? 0 : 1;
    L.cl = closure_args(s->closure, s->n);
    L.stream = s->stream;
    return L;
}

void update_material_flags(emerge_sim *s) {
    s->lf.temperature = 0;
    s->lf.activation = 0;
    for (const auto &m : s->mats) {
        const bool thermal_solid = m.model == M_NEOHOOKEAN || m.model == M_COROTATED ||
                                   m.model == M_VISCOELASTIC;
        if (thermal_solid && m.thermal_expansion != 0.0f) s->lf.temperature = 1;
        if (m.model == M_FLUID && m.thermal_viscosity_coeff > 0.0f) s->lf.temperature = 1;
        if (activation_scale(m) > 0.0f) s->lf.activation = 1;
    }
}

emerge_status ensure_capacity(emerge_sim *s, size_t need) {
    if (need <= s->cap) return EMERGE_OK;
    if (s->copy_stream) CK(cudaStreamSynchronize(s->copy_stream));  // a readback may read the old sets
    size_t cap = s->cap ? s->cap : 1024;
    while (cap < need) cap *= 2;
    const size_t set_bytes = particle_set_bytes(cap);
    size_t bytes = 2 * set_bytes;
    void *ptr = nullptr;
    CK(cudaMalloc(&ptr, bytes));
    Carver c(ptr);
    DevParticles np[2];
    np[0] = carve_particles(c, cap);
    c.p = reinterpret_cast<uintptr_t>(ptr) + set_bytes;
    np[1] = carve_particles(c, cap);
    if (c.p > reinterpret_cast<uintptr_t>(ptr) + bytes) {
        cudaFree(ptr);
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_OOM, "particle carve exceeds allocation"));
    }
    if (s->n > 0) {
        // move the live set into np[0] (same slot order)
        std::vector<uint32_t> ident;  // identity permutation via a device copy of slots
        uint32_t *d_perm = nullptr;
        CK(cudaMalloc(&d_perm, s->n * sizeof(uint32_t)));
        ident.resize(s->n);
        for (size_t i = 0; i < s->n; ++i) ident[i] = static_cast<uint32_t>(i);
        CK(cudaMemcpyAsync(d_perm, ident.data(), s->n * sizeof(uint32_t), cudaMemcpyHostToDevice,
                           s->stream));
        launch_permute(s->P[s->cur], np[0], d_perm, static_cast<int>(s->n), s->stream);
        s->host_launches += 1;
        CK(cudaStreamSynchronize(s->stream));
        cudaFree(d_perm);
    }
    s->pbuf.reset();
    s->pbuf.ptr = ptr;
    s->pbuf.bytes = bytes;
    s->P[0] = np[0];
    s->P[1] = np[1];
    s->cur = 0;
    s->cap = cap;
    s->staging.reset();
    CK(cudaMalloc(&s->staging.ptr, cap * sizeof(emerge_particle)));
    s->staging.bytes = cap * sizeof(emerge_particle);
    s->d_aos = static_cast<emerge_particle *>(s->staging.ptr);
    // the write-back's own staging buffer, sized with the particle sets so that a write-back
    // does not allocate (a large cudaMalloc can take tens of milliseconds)
    if (s->up_stream) CK(cudaStreamSynchronize(s->up_stream));
    s->staging_up.reset();
    CK(cudaMalloc(&s->staging_up.ptr, cap * sizeof(emerge_particle)));
    s->staging_up.bytes = cap * sizeof(emerge_particle);
    s->up_used = false;
    s->sortbuf.reset();
    size_t sb = sort_scratch_bytes(cap);
    CK(cudaMalloc(&s->sortbuf.ptr, sb));
    s->sortbuf.bytes = sb;
    sort_scratch_bind(s->sort, s->sortbuf.ptr, cap);
    s->graph_dirty = true;
    return EMERGE_OK;
}

emerge_status upload_materials(emerge_sim *s) {
    CK(cudaMemcpyAsync(s->mbuf.ptr, s->mats.data(), s->mats.size() * sizeof(emerge_material_params),
                       cudaMemcpyHostToDevice, s->stream));
    update_material_flags(s);
    s->graph_dirty = true;
    return EMERGE_OK;
}

void destroy_graph(emerge_sim *s) {
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->graph_exec = nullptr;
    s->graph = nullptr;
}

// Kernels the fast pipeline adds to a substep for multi-field scenes: the clear, the two
// contact kernels, the mixture kernels.
int multi_fast_launches(const DevConfig &c) {
    if (!c.mf_fast) return 0;
    int k = 1;
    if (c.mf_fields & 1) k += 2;
    if (c.mf_fields & 2) k += (c.mix_drag <= 0.0f || c.mix_iters <= 0) ? 1 : 3 + c.mix_iters;
    return k;
}

// After the grid update: contact and mixture coupling (step.rs:166-197) on the fast pipeline.
void enqueue_multi_resolves(const StepLaunch &L) {
    if (!L.cfg.mf_fast) return;
    if (L.cfg.mf_fields & 1) launch_contact_resolve_lists(L);
    if (L.cfg.mf_fields & 2) launch_mixture_resolve(L);
}

bool nbody_live(const emerge_sim *s) {
    return s->nb.depth >= 0 && s->nbbuf.ptr != nullptr && s->nb_alloc_depth == s->nb.depth;
}

// Kernels a substep's particle pass takes beyond the one pass: with an NBodyGravityField, the
// tree build, the walk and the fields half.
int nbody_extra_kernels(const emerge_sim *s) {
    return nbody_live(s) ? nbody_build_kernels(s->nb.depth, static_cast<int>(s->n), det_pipeline(s)) + 2 : 0;
}

// The particle pass of a substep (G2P of substep k, fields, CFL bound, and with emit_p2g the
// projection and P2G of k + 1).  With an NBodyGravityField the fields need the tree of every
// particle's post-G2P position (step.rs:221-226): the pass runs as its G2P half, the tree
// build, the walk (each particle's n-body acceleration) and its fields half.
void launch_particle_pass_fields(emerge_sim *s, const StepLaunch &L, int project_in, int emit_p2g) {
    if (!nbody_live(s)) {
        launch_particle_pass(L, s->lf, 1, project_in, emit_p2g);
        return;
    }
    launch_particle_pass(L, s->lf, 1, project_in, 0, 1);
    launch_nbody_build(s->nb, L.P, L.n, s->sort, det_pipeline(s), L.stream);
    launch_nbody_walk(s->nb, L.cfg, L.P, L.n, false, L.stream);
    launch_particle_pass(L, s->lf, 0, 0, emit_p2g, 2);
}

// The tree's arrays for the current capacity and depth (allocated before a step).
emerge_status nbody_prepare(emerge_sim *s) {
    if (s->nb.depth < 0) return EMERGE_OK;
    if (s->nbbuf.ptr && s->nb_cap >= s->cap && s->nb_alloc_depth == s->nb.depth &&
        s->nb_alloc_fields == s->nb.n_fields)
        return EMERGE_OK;
    CK(cudaStreamSynchronize(s->stream));  // queued kernels may still read the old arrays
    s->nbbuf.reset();
    const size_t cap = std::max<size_t>(s->cap, 1);
    const size_t slots = static_cast<size_t>(nbody_slots(s->nb.depth));
    const size_t stride = align_up(cap, 64);
    const size_t b_bounds = align_up(sizeof(NBodyBounds), 256), b_root = 256;
    const size_t b_bdata = align_up(cap * sizeof(float4), 256), b_path = align_up(cap * sizeof(uint2), 256);
    const size_t b_order = static_cast<size_t>(s->nb.depth + 1) * stride * sizeof(uint32_t);
    const size_t b_range = align_up(slots * sizeof(uint2), 256), b_com = align_up(slots * sizeof(float4), 256);
    const size_t b_accel = static_cast<size_t>(std::max(s->nb.n_fields, 1)) * stride * sizeof(float2);
    const size_t bytes = b_bounds + b_root + b_bdata + b_path + b_order + b_range + b_com + b_accel;
    CK(cudaMalloc(&s->nbbuf.ptr, bytes));
    s->nbbuf.bytes = bytes;
    char *p = static_cast<char *>(s->nbbuf.ptr);
    s->nb.bounds = reinterpret_cast<NBodyBounds *>(p);
    p += b_bounds;
    s->nb.root = reinterpret_cast<float4 *>(p);
    p += b_root;
    s->nb.bdata = reinterpret_cast<float4 *>(p);
    p += b_bdata;
    s->nb.path = reinterpret_cast<uint2 *>(p);
    p += b_path;
    s->nb.order = reinterpret_cast<uint32_t *>(p);
    s->nb.stride = stride;
    p += b_order;
    s->nb.range = reinterpret_cast<uint2 *>(p);
    p += b_range;
    s->nb.com = reinterpret_cast<float4 *>(p);
    p += b_com;
    s->nb.accel = reinterpret_cast<float2 *>(p);
    s->nb.walk_ctas = nbody_walk_ctas();
    s->nb_cap = cap;
    s->nb_alloc_depth = s->nb.depth;
    s->nb_alloc_fields = s->nb.n_fields;
    refresh_dev_config(s);
    s->graph_dirty = true;
    return EMERGE_OK;
}

emerge_status build_graph(emerge_sim *s) {
    destroy_graph(s);
    StepLaunch L = make_launch(s);
    cudaGraph_t graph;
    CK(cudaGraphCreate(&graph, 0));
    s->graph = graph;
    // node 1: k_step_begin (captured into the top-level graph)
    CK(cudaStreamBeginCaptureToGraph(s->stream, graph, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    launch_step_begin(L);
    CK(cudaStreamEndCapture(s->stream, &graph));
    size_t nn = 0;
    CK(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
    cudaGraphConditionalHandle handle;
    CK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CK(cudaGraphAddNode(&wnode, graph, nodes.data(), nn, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const int kps = 3 + (L.density_mode ? 1 : 0) + multi_fast_launches(L.cfg) + (closure_tiles_on(L) ? 1 : 0) +
                    nbody_extra_kernels(s);
    CK(cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    launch_substep_begin(L, 1, static_cast<unsigned long long>(handle), kps);
    if (L.cfg.mf_fast) launch_multi_clear(L);
    launch_grid_update(L);
    enqueue_multi_resolves(L);
    launch_particle_pass_fields(s, L, L.cfg.project, 1);
    if (closure_tiles_on(L)) launch_closure_tiles(L, s->lf, s->sm_count);
    if (L.density_mode) launch_density_pass(L, s->lf);
    CK(cudaStreamEndCapture(s->stream, &body));
    CK(cudaGraphInstantiate(&s->graph_exec, graph, 0));
    s->graph_dirty = false;
    return EMERGE_OK;
}

emerge_status prime(emerge_sim *s) {
    StepLaunch L = make_launch(s);
    launch_prime_setup(L);
    if (L.cfg.mf_fast) {  // the lists and field sums the prime's scatter fills
        launch_multi_clear(L);
        s->host_launches += 1;
    }
    if (det_pipeline(s)) {  // CFL reduction only; the substep scatters after dt is known
        launch_particle_pass(L, s->lf, 0, 0, 0);
        s->host_launches += 2;
        CK(cudaGetLastError());
        s->pending_valid = true;
        return EMERGE_OK;
    }
    launch_particle_pass(L, s->lf, 0, 0, 1);
    s->host_launches += 2;
    if (L.density_mode) {
        launch_density_pass(L, s->lf);
        s->host_launches += 1;
    }
    CK(cudaGetLastError());
    s->pending_valid = true;
    return EMERGE_OK;
}

emerge_status sort_particles(emerge_sim *s, int key_mode) {
    if (s->n < 2) return EMERGE_OK;
    int n = static_cast<int>(s->n);
    launch_sort_keys(s->P[s->cur].x, n, s->res, key_mode, s->sort.keys[0], s->sort.vals[0],
                     s->stream);
    int bits = sort_key_bits(s->res, key_mode);
    int r = radix_sort_pairs(s->sort, n, bits, s->stream);
    launch_permute(s->P[s->cur], s->P[s->cur ^ 1], s->sort.vals[r], n, s->stream);
    s->host_launches += 2 + 5 * ((bits + 7) / 8);
    s->cur ^= 1;
    s->sorts += 1;
    s->graph_dirty = true;
    s->sorted_once = true;
    s->steps_since_sort = 0;
    CK(cudaGetLastError());
    return EMERGE_OK;
}

// Particle order policy: sort by tile before the first step after particles are
// added, then every sort_interval steps (0: never again).  Sorting changes no result
// beyond float summation order; it keeps each warp's particles in few cells so the
// warp-aggregated P2G issues few reductions and the G2P gather stays cache-local.
emerge_status maybe_sort(emerge_sim *s) {
    bool need = !s->sorted_once;
    if (!need && s->sort_interval > 0)
        need = s->steps_since_sort >= static_cast<uint64_t>(s->sort_interval);
    if (!need) return EMERGE_OK;
    return sort_particles(s, 0);
}

emerge_status run_host_loop_step(emerge_sim *s, bool timed) {
    StepLaunch L = make_launch(s);
    float t_cfl = 0, t_grid = 0, t_part = 0, t_dens = 0;
    if (timed) CK(cudaEventRecord(s->ev[0], s->stream));
    launch_step_begin(L);
    s->host_launches += 1;
    CK(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(StepState), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    while (s->h_state->cont) {
        // Wake after this substep's P2G (step.rs:107-131), which the previous pass (or the
        // prime) already scattered.  It runs here, inside the step the substep belongs to,
        // so that between steps the state is the reference's.
        if (L.cfg.zones) {
            launch_wake(L, 1);
            s->host_launches += 1;
        }
        CK(cudaEventRecord(s->ev[1], s->stream));
        launch_substep_begin(L, 0, 0ull, 0);
        if (L.cfg.mf_fast) launch_multi_clear(L);
        CK(cudaEventRecord(s->ev[2], s->stream));
        launch_grid_update(L);
        enqueue_multi_resolves(L);
        CK(cudaEventRecord(s->ev[3], s->stream));
        launch_particle_pass_fields(s, L, L.cfg.project, 1);
        s->host_launches += nbody_extra_kernels(s);
        if (closure_tiles_on(L)) {
            launch_closure_tiles(L, s->lf, s->sm_count);
            s->host_launches += 1;
        }
        CK(cudaEventRecord(s->ev[4], s->stream));
        s->host_launches += 3 + multi_fast_launches(L.cfg);
        if (L.density_mode) {
            launch_density_pass(L, s->lf);
            s->host_launches += 1;
        }
        CK(cudaEventRecord(s->ev[5], s->stream));
        CK(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(StepState), cudaMemcpyDeviceToHost,
                           s->stream));
        CK(cudaStreamSynchronize(s->stream));
        CK(cudaGetLastError());
        {
            emerge_status zst = drain_zone_log(s);
            if (zst != EMERGE_OK) return zst;
        }
        float a, b, c, d;
        cudaEventElapsedTime(&a, s->ev[1], s->ev[2]);
        cudaEventElapsedTime(&b, s->ev[2], s->ev[3]);
        cudaEventElapsedTime(&c, s->ev[3], s->ev[4]);
        cudaEventElapsedTime(&d, s->ev[4], s->ev[5]);
        t_cfl += a;
        t_grid += b;
        t_part += c;
        t_dens += d;
    }
    if (timed) {
        CK(cudaEventRecord(s->ev[6], s->stream));
        CK(cudaEventSynchronize(s->ev[6]));
        float tot;
        cudaEventElapsedTime(&tot, s->ev[0], s->ev[6]);
        emerge_step_timing &t = s->last_timing;
        std::memset(&t, 0, sizeof(t));
        t.cfl_us = static_cast<uint64_t>(t_cfl * 1000.0f);
        t.grid_update_us = static_cast<uint64_t>(t_grid * 1000.0f);
        t.g2p_us = static_cast<uint64_t>(t_part * 1000.0f);  // fused G2P+update+projection+P2G pass
        t.density_us = static_cast<uint64_t>(t_dens * 1000.0f);
        t.total_us = static_cast<uint64_t>(tot * 1000.0f);
    }
    return EMERGE_OK;
}

// ---------------------------------------------------------------- sleep partition
// Sizes the event log for the particle capacity (one wake and one sleep per particle per
// substep at most: the log is drained after every substep) and switches the device
// configuration to the partition's state.
emerge_status update_zones(emerge_sim *s) {
    const bool on = zones_on(s);
    const uint32_t need = static_cast<uint32_t>(2 * std::max<size_t>(s->cap, 1) + 64);
    if (on && s->zlog_cap < need) {
        CK(cudaStreamSynchronize(s->stream));
        s->zbuf.reset();
        const size_t bytes = 256 + need * sizeof(unsigned long long) + std::max<size_t>(s->cap, 1) * sizeof(uint32_t);
        CK(cudaMalloc(&s->zbuf.ptr, bytes));
        s->zbuf.bytes = bytes;
        s->zlog_cap = need;
        CK(cudaMemsetAsync(s->zbuf.ptr, 0, 256, s->stream));
    }
    const int want = (on && s->zbuf.ptr) ? 1 : 0;
    if (want != s->dcfg.zones || (want && s->dcfg.zone_log_cap != s->zlog_cap)) {
        refresh_dev_config(s);
        s->graph_dirty = true;
    }
    return EMERGE_OK;
}

void perm_init(emerge_sim *s) {
    if (s->pos_of_base.size() == s->n) return;
    s->pos_of_base.resize(s->n);
    s->base_of_pos.resize(s->n);
    for (size_t k = 0; k < s->n; ++k) s->pos_of_base[k] = s->base_of_pos[k] = static_cast<uint32_t>(k);
}

void perm_swap(emerge_sim *s, uint32_t a, uint32_t b) {
    if (a == b) return;
    const uint32_t ba = s->base_of_pos[a], bb = s->base_of_pos[b];
    s->base_of_pos[a] = bb;
    s->base_of_pos[b] = ba;
    s->pos_of_base[ba] = b;
    s->pos_of_base[bb] = a;
}

// Replays the logged wake / sleep events of the finished substep(s) on the reference
// indices: per event key in order, wakes in ascending index order swap with the first
// sleeping particle (particles.rs:252-268), sleeps in descending order with the last active
// particle (particles.rs:227-245).  The device's indices are updated by commit_perm.
emerge_status drain_zone_log(emerge_sim *s) {
    if (!s->dcfg.zones) return EMERGE_OK;
    uint32_t count = 0;
    CK(cudaMemcpyAsync(&count, s->dcfg.zone_log_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (count == 0) return EMERGE_OK;
    if (count > s->zlog_cap)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_CUDA, "sleep partition event log overflow"));
    std::vector<unsigned long long> ev(count);
    CK(cudaMemcpyAsync(ev.data(), s->dcfg.zone_log, count * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       s->stream));
    CK(cudaMemsetAsync(s->dcfg.zone_log_count, 0, sizeof(uint32_t), s->stream));
    CK(cudaStreamSynchronize(s->stream));
    std::sort(ev.begin(), ev.end());
    perm_init(s);
    std::vector<uint32_t> idx;
    for (size_t a = 0; a < ev.size();) {
        const uint32_t key = static_cast<uint32_t>(ev[a] >> 32);
        size_t b = a;
        idx.clear();
        for (; b < ev.size() && static_cast<uint32_t>(ev[b] >> 32) == key; ++b)
            idx.push_back(s->pos_of_base[static_cast<uint32_t>(ev[b])]);
        if ((key & 1u) == 0u) {  // wake
            std::sort(idx.begin(), idx.end());
            for (uint32_t i : idx) {
                perm_swap(s, i, static_cast<uint32_t>(s->active));
                s->active += 1;
            }
        } else {  // sleep
            std::sort(idx.begin(), idx.end(), std::greater<uint32_t>());
            for (uint32_t i : idx) {
                perm_swap(s, i, static_cast<uint32_t>(s->active - 1));
                s->active -= 1;
            }
        }
        a = b;
    }
    s->perm_dirty = true;
    return EMERGE_OK;
}

// Moves the replayed swaps into the device's reference indices.
emerge_status commit_perm(emerge_sim *s) {
    if (!s->perm_dirty) return EMERGE_OK;
    uint32_t *table = reinterpret_cast<uint32_t *>(static_cast<char *>(s->zbuf.ptr) + 256 +
                                                   s->zlog_cap * sizeof(unsigned long long));
    CK(cudaMemcpyAsync(table, s->pos_of_base.data(), s->n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
    launch_remap_index(s->P[s->cur], static_cast<int>(s->n), table, s->stream);
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaGetLastError());
    for (size_t k = 0; k < s->n; ++k) s->pos_of_base[k] = s->base_of_pos[k] = static_cast<uint32_t>(k);
    s->perm_dirty = false;
    return EMERGE_OK;
}

emerge_status ensure_det_scratch(emerge_sim *s) {
    size_t need = 9 * (s->cap > 0 ? s->cap : 1);
    if (s->det_cap >= need) return EMERGE_OK;
    s->detbuf.reset();
    size_t bytes = sort_scratch_bytes(need) + need * (sizeof(float4) + sizeof(uint8_t)) + 1024;
    CK(cudaMalloc(&s->detbuf.ptr, bytes));
    s->detbuf.bytes = bytes;
    sort_scratch_bind(s->det_sort, s->detbuf.ptr, need);
    uintptr_t p = reinterpret_cast<uintptr_t>(s->detbuf.ptr) + sort_scratch_bytes(need);
    p = (p + 255) & ~static_cast<uintptr_t>(255);
    s->det_payload = reinterpret_cast<float4 *>(p);
    p = (p + need * sizeof(float4) + 255) & ~static_cast<uintptr_t>(255);
    s->det_fmask = reinterpret_cast<uint8_t *>(p);
    s->det_cap = need;
    return EMERGE_OK;
}

uint32_t det_invalid_key(const emerge_sim *s) {
    return static_cast<uint32_t>(s->res) * static_cast<uint32_t>(s->res);
}

int det_key_bits(const emerge_sim *s) {
    uint64_t top = static_cast<uint64_t>(det_invalid_key(s));
    int b = 0;
    while ((1ull << b) <= top) ++b;
    return b;
}

// Records -> stable sort by cell -> sequential per-cell sums (see det_kernels.cu).
// reuse_sort: the positions are those of the previous call, whose sorted keys stand (only
// the payload is written).  The full scatter can also write each record's fields (`fmask`,
// for det_field_sum), the contact point cloud (`points`), each cell's record range and, in
// `sorted_vals`, the cell-sorted record order they index.
emerge_status det_scatter(emerge_sim *s, const StepLaunch &L, int mode, int filter, float lox,
                          float loy, float hix, float hiy, bool reuse_sort = false,
                          uint8_t *fmask = nullptr, float4 *points = nullptr, int2 *range = nullptr,
                          const uint32_t **sorted_vals = nullptr) {
    emerge_status st = ensure_det_scratch(s);
    if (st != EMERGE_OK) return st;
    const uint32_t inv = det_invalid_key(s);
    const int n_rec = 9 * L.n;
    launch_det_records(L, mode, inv, s->det_sort.keys[0], s->det_sort.vals[0], s->det_payload, filter,
                       lox, loy, hix, hiy, reuse_sort ? 0 : 1, fmask, points);
    int bits = det_key_bits(s);
    if (!reuse_sort) {
        s->det_sorted = radix_sort_pairs(s->det_sort, n_rec, bits, s->stream);
        s->host_launches += 5 * ((bits + 7) / 8);
    }
    const int r = s->det_sorted;
    launch_segsum(s->det_sort.keys[r], s->det_sort.vals[r], s->det_payload, n_rec, inv, s->g,
                  mode == 0 ? 1 : 0, s->stream, range);
    if (sorted_vals) *sorted_vals = s->det_sort.vals[r];
    s->host_launches += 2;
    CK(cudaGetLastError());
    return EMERGE_OK;
}

emerge_status clear_grid(emerge_sim *s) {
    size_t cells = static_cast<size_t>(s->tpd) * s->tpd * TILE_CELLS;
    CK(cudaMemsetAsync(s->g.acc_a, 0, cells * sizeof(float4), s->stream));
    CK(cudaMemsetAsync(s->g.acc_s, 0, cells * sizeof(float2), s->stream));
    CK(cudaMemsetAsync(s->g.tile_flag, 0, static_cast<size_t>(s->tpd) * s->tpd, s->stream));
    return EMERGE_OK;
}

// Contact point cloud storage: one (x, y, label) per scatter record.
emerge_status ensure_points(emerge_sim *s) {
    const size_t need = 9 * (s->cap > 0 ? s->cap : 1);
    if (s->pts_cap >= need) return EMERGE_OK;
    s->ptsbuf.reset();
    CK(cudaMalloc(&s->ptsbuf.ptr, need * sizeof(float4)));
    s->ptsbuf.bytes = need * sizeof(float4);
    s->pts_cap = need;
    return EMERGE_OK;
}

// The per-substep clear of the field sums, the pressure scratch (zero is the pressure of a
// cell outside the mixture) and the contact flag (Grid::clear, grid/mod.rs:163-176).
emerge_status clear_multi(emerge_sim *s) {
    const size_t cells = static_cast<size_t>(s->tpd) * s->tpd * TILE_CELLS;
    CK(cudaMemsetAsync(s->g.acc_grip, 0, cells * sizeof(float4), s->stream));
    CK(cudaMemsetAsync(s->g.acc_sol, 0, cells * sizeof(float4), s->stream));
    CK(cudaMemsetAsync(s->g.acc_flu, 0, cells * sizeof(float4), s->stream));
    CK(cudaMemsetAsync(s->g.mx_k, 0, cells * sizeof(float), s->stream));
    CK(cudaMemsetAsync(s->g.mx_p[0], 0, cells * sizeof(float), s->stream));
    CK(cudaMemsetAsync(s->g.mx_p[1], 0, cells * sizeof(float), s->stream));
    CK(cudaMemsetAsync(&s->d_state->contact_active, 0, sizeof(uint32_t), s->stream));
    return EMERGE_OK;
}

int mixture_launches(const DevConfig &c) {
    return (c.mix_drag <= 0.0f || c.mix_iters <= 0) ? 1 : 3 + c.mix_iters;
}

// One Simulation::step in reference order (step.rs:23-60, 62-210), host-driven.
emerge_status run_det_step(emerge_sim *s, bool timed) {
    StepLaunch L = make_launch(s);
    float t_cfl = 0, t_grid = 0, t_part = 0, t_dens = 0, t_p2g = 0, t_proj = 0;
    if (timed) CK(cudaEventRecord(s->ev[0], s->stream));
    launch_step_begin(L);
    s->host_launches += 1;
    CK(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(StepState), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    emerge_status st = EMERGE_OK;
    const bool contact = L.cfg.multi && s->contact_seen;
    const bool mixture = L.cfg.multi && mixture_on(s);
    if (contact) {
        st = ensure_points(s);
        if (st != EMERGE_OK) return st;
    }
    while (s->h_state->cont) {
        CK(cudaEventRecord(s->ev[1], s->stream));
        launch_substep_begin(L, 0, 0ull, 0);
        if (L.cfg.multi) {
            st = clear_multi(s);
            if (st != EMERGE_OK) return st;
        }
        CK(cudaEventRecord(s->ev[2], s->stream));
        if (L.cfg.project) launch_project(L);
        CK(cudaEventRecord(s->ev[3], s->stream));
        s->host_launches += 2;
        if (L.density_mode) {  // estimate_particle_volumes(.., false) (density.rs:41-72)
            st = det_scatter(s, L, 0, 0, 0, 0, 0, 0);
            if (st != EMERGE_OK) return st;
            launch_mass_gather(L.P, 0, L.n, L.g, 0, s->stream, L.cfg.zones);
            s->host_launches += 1;
            st = clear_grid(s);
            if (st != EMERGE_OK) return st;
        }
        CK(cudaEventRecord(s->ev[4], s->stream));
        // P2G at the positions the density scatter sorted, when there was one; the grip and
        // mixture-phase fields take the same contributions as the total (p2g.rs:60-66),
        // summed per field over the same sorted records in particle index order
        const uint32_t *sorted_vals = nullptr;
        st = det_scatter(s, L, 1, 0, 0, 0, 0, 0, L.density_mode != 0, (contact || mixture) ? s->det_fmask : nullptr,
                         contact ? s->det_points() : nullptr, contact ? s->g.rec_range : nullptr, &sorted_vals);
        if (st != EMERGE_OK) return st;
        const int r = s->det_sorted;
        const uint32_t inv = det_invalid_key(s);
        auto field_sum = [&](uint32_t bit, float4 *target, uint32_t *any) {
            launch_segsum_field(s->det_sort.keys[r], s->det_sort.vals[r], s->det_payload, s->det_fmask, bit,
                                9 * L.n, inv, s->g, target, any, s->stream);
            s->host_launches += 1;
        };
        if (contact) field_sum(1u, s->g.acc_grip, &s->d_state->contact_active);
        if (mixture) {
            field_sum(2u, s->g.acc_sol, nullptr);
            field_sum(4u, s->g.acc_flu, nullptr);
        }
        CK(cudaGetLastError());
        if (L.cfg.zones) {  // wake after this substep's P2G (step.rs:107-131)
            launch_wake(L, 0);
            s->host_launches += 1;
        }
        CK(cudaEventRecord(s->ev[5], s->stream));
        launch_grid_update(L);
        if (contact) {  // step.rs:166-183
            launch_contact_resolve(L, sorted_vals, s->det_points());
            s->host_launches += 1;
        }
        if (mixture) {  // step.rs:185-197
            launch_mixture_resolve(L);
            s->host_launches += mixture_launches(L.cfg);
        }
        CK(cudaEventRecord(s->ev[6], s->stream));
        launch_particle_pass_fields(s, L, 0, 0);
        CK(cudaEventRecord(s->ev[7], s->stream));
        s->host_launches += 2 + nbody_extra_kernels(s);
        CK(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(StepState), cudaMemcpyDeviceToHost,
                           s->stream));
        CK(cudaStreamSynchronize(s->stream));
        CK(cudaGetLastError());
        if (L.cfg.zones) {  // the next substep's records follow the new index order
            st = drain_zone_log(s);
            if (st == EMERGE_OK) st = commit_perm(s);
            if (st != EMERGE_OK) return st;
        }
        float a, b, c, d, e, f;
        cudaEventElapsedTime(&a, s->ev[1], s->ev[2]);
        cudaEventElapsedTime(&b, s->ev[2], s->ev[3]);
        cudaEventElapsedTime(&c, s->ev[3], s->ev[4]);
        cudaEventElapsedTime(&d, s->ev[4], s->ev[5]);
        cudaEventElapsedTime(&e, s->ev[5], s->ev[6]);
        cudaEventElapsedTime(&f, s->ev[6], s->ev[7]);
        t_cfl += a;
        t_proj += b;
        t_dens += c;
        t_p2g += d;
        t_grid += e;
        t_part += f;
    }
    if (timed) {
        CK(cudaEventRecord(s->ev[7], s->stream));
        CK(cudaEventSynchronize(s->ev[7]));
        float tot;
        cudaEventElapsedTime(&tot, s->ev[0], s->ev[7]);
        emerge_step_timing &t = s->last_timing;
        std::memset(&t, 0, sizeof(t));
        t.cfl_us = static_cast<uint64_t>(t_cfl * 1000.0f);
        t.project_us = static_cast<uint64_t>(t_proj * 1000.0f);
        t.density_us = static_cast<uint64_t>(t_dens * 1000.0f);
        t.p2g_us = static_cast<uint64_t>(t_p2g * 1000.0f);
        t.grid_update_us = static_cast<uint64_t>(t_grid * 1000.0f);
        t.g2p_us = static_cast<uint64_t>(t_part * 1000.0f);
        t.total_us = static_cast<uint64_t>(tot * 1000.0f);
    }
    return EMERGE_OK;
}

emerge_status spawn_region(emerge_sim *s, const emerge_spawn_region &sp, uint32_t tag,
                           std::vector<emerge_particle> &out) {
    // initialize_particles (spacetime/solver/mod.rs:88-151)
    if (!(sp.spacing > 0.0f) || sp.box_size[0] <= 0 || sp.box_size[1] <= 0)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "spawn: spacing and box_size must be positive"));
    float hx = static_cast<float>(sp.box_size[0]) * 0.5f, hy = static_cast<float>(sp.box_size[1]) * 0.5f;
    float mnx = sp.box_center[0] - hx, mny = sp.box_center[1] - hy;
    float mxx = sp.box_center[0] + hx, mxy = sp.box_center[1] + hy;
    // SpawnRegion::fits_in_sim (config.rs:472-482)
    float dmin = static_cast<float>(s->cfg.boundary_thickness);
    float dmax = static_cast<float>(sat_sub_sz(s->cfg.grid_res, s->cfg.boundary_thickness));
    if (!(mnx >= dmin && mny >= dmin && mxx <= dmax && mxy <= dmax))
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG,
                                                  "spawn region must stay inside the simulation domain"));
    float mass = sp.has_mass_override ? sp.mass_override : s->cfg.particle_mass;
    float v0 = s->cfg.default_initial_volume;
    Lcg rng{sp.rng_seed};
    const emerge_material_params *mat =
        sp.material_id < s->mats.size() ? &s->mats[sp.material_id] : nullptr;
    for (float i = mnx; i < mxx; i += sp.spacing) {
        for (float j = mny; j < mxy; j += sp.spacing) {
            bool inside = true;
            if (sp.shape == 1) {
                float dx = i - sp.box_center[0], dy = j - sp.box_center[1];
                inside = std::sqrt(dx * dx + dy * dy) <= sp.disk_radius;
            }
            if (!inside) continue;
            float jitter_mag = sp.position_jitter * sp.spacing;
            float jx = (rng.next_f32() - 0.5f) * 2.0f * jitter_mag;
            float jy = (rng.next_f32() - 0.5f) * 2.0f * jitter_mag;
            float rx = rng.next_f32();
            float ry = rng.next_f32();
            emerge_particle q;
            std::memset(&q, 0, sizeof(q));
            q.x[0] = i + jx;
            q.x[1] = j + jy;
            q.v[0] = (rx - 0.5f) * sp.initial_velocity_scale;
            q.v[1] = (ry - 0.5f) * sp.initial_velocity_scale;
            std::memcpy(q.f, sp.initial_deformation_gradient, sizeof(q.f));
            q.mass = mass;
            q.initial_volume = v0;
            q.volume = v0;
            q.density = mass / v0;
            q.material_id = sp.material_id;
            q.plastic_volume_ratio = 1.0f;
            q.hardening_scale = 1.0f;
            q.user_tag = tag;
            if (mat) init_particle(*mat, q);  // add_body stamps + init (particles.rs:383-392)
            out.push_back(q);
        }
    }
    return EMERGE_OK;
}

// Appends host particles and optionally runs the local (add_body) or full
// (Simulation::new) initial-volume estimate on the device.
emerge_status append_particles(emerge_sim *s, const emerge_particle *src, size_t count,
                               int volume_mode /*0 none, 1 local, 2 full*/) {
    if (s->n + count > 0x7fffffffull)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "too many particles"));
    emerge_status st = ensure_capacity(s, s->n + count);
    if (st != EMERGE_OK) return st;
    for (size_t k = 0; k < count; ++k)
        if (src[k].pinned) s->lf.pinned = 1;
    st = commit_perm(s);
    if (st != EMERGE_OK) return st;
    const int n_old = static_cast<int>(s->n), n_new = static_cast<int>(s->n + count);
    const uint64_t old_active = s->active;
    if (count > 0) {
        CK(cudaMemcpyAsync(s->d_aos, src, count * sizeof(emerge_particle), cudaMemcpyHostToDevice,
                           s->stream));
        launch_append_aos(s->P[s->cur], n_old, n_new, s->d_aos, s->stream);
        s->host_launches += 1;
        // new particles go before the sleeping zone (particles.rs:389-410)
        if (old_active < static_cast<uint64_t>(n_old))
            launch_insert_index(s->P[s->cur], n_old, n_new, static_cast<uint32_t>(old_active), s->stream);
    }
    s->n = static_cast<size_t>(n_new);
    s->active = old_active + count;
    s->pos_of_base.clear();
    s->base_of_pos.clear();
    st = update_zones(s);
    if (st != EMERGE_OK) return st;
    bool contact = false;
    for (size_t k = 0; k < count && !contact; ++k) contact = src[k].contact_group != 0;
    if (contact && !s->contact_seen) {
        s->contact_seen = true;
        st = update_multi(s);
        if (st != EMERGE_OK) return st;
    }
    if (s->dcfg.zones) launch_zone_bits(s->P[s->cur], n_new, static_cast<uint32_t>(s->active), s->stream);
    if (volume_mode != 0 && count > 0) {
        // estimate_particle_volumes_local (density.rs:81-144) / estimate_particle_volumes (:41-72)
        int filter = 0;
        float lox = 0, loy = 0, hix = 0, hiy = 0;
        if (volume_mode == 1) {
            float lo[2] = {3.402823466e38f, 3.402823466e38f};
            float hi[2] = {-3.402823466e38f, -3.402823466e38f};
            for (size_t k = 0; k < count; ++k)
                for (int d = 0; d < 2; ++d) {
                    lo[d] = std::fmin(lo[d], src[k].x[d]);
                    hi[d] = std::fmax(hi[d], src[k].x[d]);
                }
            lox = lo[0] - 3.0f;
            loy = lo[1] - 3.0f;
            hix = hi[0] + 3.0f;
            hiy = hi[1] + 3.0f;
            filter = 1;
        }
        size_t cells = static_cast<size_t>(s->tpd) * s->tpd * TILE_CELLS;
        CK(cudaMemsetAsync(s->g.acc_a, 0, cells * sizeof(float4), s->stream));
        if (s->deterministic) {
            StepLaunch L = make_launch(s);
            L.n = n_new;
            emerge_status dst = det_scatter(s, L, 0, filter, lox, loy, hix, hiy);
            if (dst != EMERGE_OK) return dst;
        } else {
            launch_mass_scatter(s->P[s->cur], n_new, s->g, filter, lox, loy, hix, hiy, s->stream,
                                s->dcfg.zones);
        }
        launch_mass_gather(s->P[s->cur], volume_mode == 1 ? n_old : 0, n_new, s->g, 1, s->stream,
                           s->dcfg.zones);
        CK(cudaMemsetAsync(s->g.acc_a, 0, cells * sizeof(float4), s->stream));
        CK(cudaMemsetAsync(s->g.acc_s, 0, cells * sizeof(float2), s->stream));
        CK(cudaMemsetAsync(s->g.tile_flag, 0, static_cast<size_t>(s->tpd) * s->tpd, s->stream));
        s->host_launches += 2;
    }
    CK(cudaGetLastError());
    s->pending_valid = false;
    s->graph_dirty = true;
    s->sorted_once = false;
    return EMERGE_OK;
}

emerge_status invalidate_pending(emerge_sim *s) {
    if (!s->pending_valid) return EMERGE_OK;
    size_t cells = static_cast<size_t>(s->tpd) * s->tpd * TILE_CELLS;
    CK(cudaMemsetAsync(s->g.acc_a, 0, cells * sizeof(float4), s->stream));
    CK(cudaMemsetAsync(s->g.acc_s, 0, cells * sizeof(float2), s->stream));
    CK(cudaMemsetAsync(s->g.tile_flag, 0, static_cast<size_t>(s->tpd) * s->tpd, s->stream));
    if (s->mfbuf.ptr)  // the fast pipeline's field sums of the pending scatter
        for (int f = 0; f < 3; ++f) {
            CK(cudaMemsetAsync(s->g.fa[f], 0, cells * sizeof(float4), s->stream));
            CK(cudaMemsetAsync(s->g.fs[f], 0, cells * sizeof(float2), s->stream));
        }
    s->pending_valid = false;
    return EMERGE_OK;
}

// Uploads the material phase table (MAX_MATERIALS entries, unset slots 0).
emerge_status upload_phases(emerge_sim *s) {
    if (!s->mfbuf.ptr) return EMERGE_OK;
    std::vector<uint32_t> table(MAX_MATERIALS, 0u);
    for (size_t k = 0; k < s->phases.size() && k < static_cast<size_t>(MAX_MATERIALS); ++k) table[k] = s->phases[k];
    CK(cudaMemcpyAsync(s->mfbuf.ptr, table.data(), table.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                       s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return EMERGE_OK;
}

// Switches the multi-field pipeline on (allocating its grid arrays the first time) or off
// after a change of the particles' contact groups or the materials' phases.
emerge_status update_multi(emerge_sim *s) {
    const int was = s->dcfg.multi, was_fast = s->dcfg.mf_fast, was_fields = s->dcfg.mf_fields;
    if (multi_on(s) && !s->mfbuf.ptr) {
        const size_t cells = static_cast<size_t>(s->tpd) * s->tpd * TILE_CELLS;
        const size_t flat = static_cast<size_t>(s->res) * s->res;
        const size_t bytes = MAX_MATERIALS * sizeof(uint32_t) +
                             cells * (3 * sizeof(float4) + 4 * sizeof(float2) + sizeof(float) + sizeof(int2) +
                                      6 * sizeof(float) + sizeof(uint8_t) +
                                      3 * (sizeof(float4) + sizeof(float2))) +
                             3 * flat * sizeof(int) + 30 * 256;
        CK(cudaMalloc(&s->mfbuf.ptr, bytes));
        s->mfbuf.bytes = bytes;
        CK(cudaMemsetAsync(s->mfbuf.ptr, 0, bytes, s->stream));
        Carver c(s->mfbuf.ptr);
        c.take<uint32_t>(MAX_MATERIALS);  // the phase table, at the start
        s->g.acc_grip = c.take<float4>(cells);
        s->g.acc_sol = c.take<float4>(cells);
        s->g.acc_flu = c.take<float4>(cells);
        s->g.grip_v = c.take<float2>(cells);
        s->g.rest_v = c.take<float2>(cells);
        s->g.sol_v = c.take<float2>(cells);
        s->g.flu_v = c.take<float2>(cells);
        s->g.grid_m = c.take<float>(cells);
        s->g.rec_range = c.take<int2>(cells);
        s->g.mx_as = c.take<float>(cells);
        s->g.mx_af = c.take<float>(cells);
        s->g.mx_k = c.take<float>(cells);
        s->g.mx_rhs = c.take<float>(cells);
        s->g.mx_p[0] = c.take<float>(cells);
        s->g.mx_p[1] = c.take<float>(cells);
        s->g.mx_sig = c.take<uint8_t>(cells);
        for (int f = 0; f < 3; ++f) {
            s->g.fa[f] = c.take<float4>(cells);
            s->g.fs[f] = c.take<float2>(cells);
        }
        s->g.chead[0] = c.take<int>(flat);
        s->g.chead[1] = c.take<int>(flat);
        s->g.iface = c.take<int>(flat);
        emerge_status st = upload_phases(s);
        if (st != EMERGE_OK) return st;
    }
    refresh_dev_config(s);
    if (s->dcfg.multi != was || s->dcfg.mf_fast != was_fast || s->dcfg.mf_fields != was_fields) {
        // the pending scatter was made without (or with other) field sums and point lists
        s->graph_dirty = true;
        return invalidate_pending(s);
    }
    return EMERGE_OK;
}

}  // namespace

// =============================================================== C ABI
namespace emerge {
// Message returned by emerge_cuda_last_global_error for entry points in other files.
void set_global_error(const char *msg) { g_global_error = msg; }

cudaStream_t sim_stream(emerge_sim *s) { return s->stream; }

SimView sim_view(emerge_sim *s) {
    SimView v;
    v.cfg = s->cfg;
    v.bounds = s->bounds;
    v.mats = s->mats;
    v.lf = s->lf;
    v.dcfg = s->dcfg;
    v.deterministic = s->deterministic;
    v.n = s->n;
    v.device = s->device;
    return v;
}

size_t particle_set_size(size_t cap) { return particle_set_bytes(cap); }

DevParticles particle_set_carve(void *base, size_t cap) {
    Carver c(base);
    return carve_particles(c, cap);
}
ClosureHost *&sim_closure(emerge_sim *s) { return s->closure; }
size_t sim_capacity(emerge_sim *s) { return std::max<size_t>(s->cap, std::max<size_t>(s->n, 1)); }
void sim_invalidate_graph(emerge_sim *s) { s->graph_dirty = true; }
emerge_status sim_fail(emerge_sim *s, emerge_status st, const std::string &msg) {
    return static_cast<emerge_status>(s->fail(st, msg));
}
}  // namespace emerge

extern "C" {

const char *emerge_cuda_last_error(const emerge_sim *sim) {
    return sim ? sim->error.c_str() : "null simulation handle";
}

const char *emerge_cuda_last_global_error(void) { return g_global_error.c_str(); }

emerge_status emerge_cuda_create(const emerge_sim_config *config, int device, emerge_sim **out) {
    if (!config || !out) {
        g_global_error = "null argument";
        return EMERGE_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::string msg;
    emerge_status vs = validate_config(*config, msg);
    if (vs != EMERGE_OK) {
        g_global_error = msg;
        return vs;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        g_global_error = std::string("no CUDA device available: ") + cudaGetErrorString(e);
        return EMERGE_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) {
        g_global_error = "device index out of range";
        return EMERGE_ERR_INVALID_ARG;
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_global_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return EMERGE_ERR_CUDA;
    }
    emerge_sim *s = new emerge_sim();
    s->cfg = *config;
    s->device = device;
    if (cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        s->sm_count = 0;  // the persistent grids then assume 148
    s->bounds.push_back(config->boundary_thickness);  // default SlipBoundary (lifecycle.rs:29-30)
    s->dcfg = make_dev_config(s->cfg, s->bounds, 0);
    emerge_material_params fallback;
    std::memset(&fallback, 0, sizeof(fallback));
    s->mats.push_back(fallback);
    auto bail = [&](emerge_status st) {
        g_global_error = s->error;
        emerge_cuda_destroy(s);
        return st;
    };
    emerge_status st = EMERGE_OK;
    if (!cuda_ok(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream", &st))
        return bail(st);
    for (auto &ev : s->ev)
        if (!cuda_ok(s, cudaEventCreate(&ev), "event", &st)) return bail(st);
    s->res = static_cast<int>(config->grid_res);
    s->tpd = (s->res + TILE - 1) / TILE;
    size_t cells = static_cast<size_t>(s->tpd) * s->tpd * TILE_CELLS;
    const bool asflip = config->asflip_blend > 0.0f;
    size_t gbytes = cells * (sizeof(float4) + (asflip ? 3 : 2) * sizeof(float2)) +
                    static_cast<size_t>(s->tpd) * s->tpd + 5 * 256;
    if (!cuda_ok(s, cudaMalloc(&s->gbuf.ptr, gbytes), "grid alloc", &st)) return bail(st);
    s->gbuf.bytes = gbytes;
    Carver c(s->gbuf.ptr);
    s->g.res = s->res;
    s->g.tpd = s->tpd;
    s->g.acc_a = c.take<float4>(cells);
    s->g.acc_s = c.take<float2>(cells);
    s->g.grid_v = c.take<float2>(cells);
    s->g.tile_flag = c.take<uint8_t>(static_cast<size_t>(s->tpd) * s->tpd);
    s->g.grid_vpre = asflip ? c.take<float2>(cells) : nullptr;
    if (!cuda_ok(s, cudaMemsetAsync(s->gbuf.ptr, 0, gbytes, s->stream), "grid clear", &st)) return bail(st);
    if (!cuda_ok(s, cudaMalloc(&s->mbuf.ptr, MAX_MATERIALS * sizeof(emerge_material_params)), "mat alloc", &st))
        return bail(st);
    if (!cuda_ok(s, cudaMalloc(&s->sbuf.ptr, sizeof(StepState)), "state alloc", &st)) return bail(st);
    s->d_state = static_cast<StepState *>(s->sbuf.ptr);
    if (!cuda_ok(s, cudaMallocHost(&s->h_state, sizeof(StepState)), "pinned alloc", &st)) return bail(st);
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&s->h_state_dev), s->h_state, 0) != cudaSuccess) {
        s->h_state_dev = nullptr;  // an unmapped mirror: its words are read back with copies
        (void)cudaGetLastError();
    }
    std::memset(s->h_state, 0, sizeof(StepState));
    s->h_state->last_step_dt = config->dt;
    s->h_state->min_mdt_bits[0] = s->h_state->min_mdt_bits[1] = 0x7f800000u;
    if (!cuda_ok(s, cudaMemcpyAsync(s->d_state, s->h_state, sizeof(StepState), cudaMemcpyHostToDevice, s->stream),
                 "state init", &st))
        return bail(st);
    if (!cuda_ok(s, cudaMalloc(&s->region_buf.ptr, region_acc_bytes()), "region alloc", &st)) return bail(st);
    if (upload_materials(s) != EMERGE_OK) return bail(EMERGE_ERR_CUDA);
    if (ensure_capacity(s, 1024) != EMERGE_OK) return bail(EMERGE_ERR_OOM);
    if (!cuda_ok(s, cudaStreamSynchronize(s->stream), "create sync", &st)) return bail(st);
    const char *env = std::getenv("EMERGE_CUDA_USE_GRAPH");
    if (env) s->use_graph = std::atoi(env) != 0;
    *out = s;
    return EMERGE_OK;
}

emerge_status emerge_cuda_destroy(emerge_sim *s) {
    if (!s) return EMERGE_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    if (s->up_stream) cudaStreamSynchronize(s->up_stream);
    destroy_graph(s);
    for (auto &ev : s->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto &ev : s->user_ev)
        if (ev) cudaEventDestroy(ev);
    s->flushbuf.reset();
    if (s->h_state) cudaFreeHost(s->h_state);
    s->pbuf.reset();
    s->staging.reset();
    s->staging_rb.reset();
    s->staging_up.reset();
    if (s->ev_up_done) cudaEventDestroy(s->ev_up_done);
    if (s->ev_up_free) cudaEventDestroy(s->ev_up_free);
    if (s->up_stream) cudaStreamDestroy(s->up_stream);
    if (s->ev_ready) cudaEventDestroy(s->ev_ready);
    if (s->ev_gathered) cudaEventDestroy(s->ev_gathered);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    s->detbuf.reset();
    s->gbuf.reset();
    s->mbuf.reset();
    s->fbuf.reset();
    s->zbuf.reset();
    s->sbuf.reset();
    s->sortbuf.reset();
    s->region_buf.reset();
    closure_destroy(s->closure);
    s->closure = nullptr;
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return EMERGE_OK;
}

emerge_status emerge_cuda_set_materials(emerge_sim *s, const emerge_material_params *params,
                                        uint32_t count) {
    if (!s || (!params && count)) return EMERGE_ERR_INVALID_ARG;
    if (count == 0 || count > MAX_MATERIALS)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "material count must be in [1, 64]"));
    for (uint32_t k = 0; k < count; ++k)
        if (!model_supported(params[k].model))
            return static_cast<emerge_status>(
                s->fail(EMERGE_ERR_UNSUPPORTED, "material " + std::to_string(k) + ": constitutive model " +
                                                    std::to_string(params[k].model) + " is not on the device path"));
    bool default_changed = s->mats.empty() || std::memcmp(&s->mats[0], &params[0], sizeof(emerge_material_params)) != 0;
    s->mats.assign(params, params + count);
    emerge_status st = upload_materials(s);
    if (st != EMERGE_OK) return st;
    if (default_changed && s->n > 0) {
        launch_reinit(s->P[s->cur], static_cast<int>(s->n), static_cast<const MatP *>(s->mbuf.ptr),
                      static_cast<int>(count), s->stream);
        s->host_launches += 1;
    }
    st = invalidate_pending(s);
    CK(cudaGetLastError());
    return st;
}

emerge_status emerge_cuda_set_slip_boundaries(emerge_sim *s, const uint64_t *thickness, uint32_t n) {
    if (!s || (!thickness && n)) return EMERGE_ERR_INVALID_ARG;
    if (n > static_cast<uint32_t>(MAX_BOUNDARIES))
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_UNSUPPORTED, "at most 8 boundaries"));
    for (uint32_t k = 0; k < n; ++k)
        if (thickness[k] + 1 > s->cfg.grid_res)
            return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "boundary thickness exceeds grid"));
    s->bounds.assign(thickness, thickness + n);
    refresh_dev_config(s);
    s->graph_dirty = true;
    return EMERGE_OK;
}

emerge_status emerge_cuda_set_force_fields(emerge_sim *s, const emerge_force_field *fields, uint32_t n,
                                           const float *data, uint64_t n_data) {
    if (!s || (!fields && n) || (!data && n_data)) return EMERGE_ERR_INVALID_ARG;
    for (uint32_t k = 0; k < n; ++k) {
        const emerge_force_field &f = fields[k];
        uint64_t need = 0;
        switch (f.kind) {
        case EMERGE_FIELD_GRAVITY_WELL: need = 3ull * f.count; break;
        case EMERGE_FIELD_COULOMB: need = 3ull * f.count + f.n_charges; break;
        case EMERGE_FIELD_UNIFORM_ELECTRIC: need = f.n_charges; break;
        case EMERGE_FIELD_CHEMOTAXIS: need = static_cast<uint64_t>(f.count) * f.count; break;
        case EMERGE_FIELD_BUOYANCY:
        case EMERGE_FIELD_LINEAR_DRAG:
        case EMERGE_FIELD_RADIAL_CONFINEMENT:
        case EMERGE_FIELD_AABB_CONFINEMENT: break;
        case EMERGE_FIELD_NBODY_GRAVITY: {
            // NBodyGravityField::new asserts theta in (0, 1] (n_body.rs:306-311)
            const float theta = f.params[2], depth = f.params[3], maxb = f.params[4];
            if (!(theta > 0.0f && theta <= 1.0f))
                return static_cast<emerge_status>(
                    s->fail(EMERGE_ERR_INVALID_ARG, "force field " + std::to_string(k) + ": theta must be in (0, 1]"));
            if (!(maxb >= 0.0f && maxb <= 2147483647.0f && maxb == std::floor(maxb)) || !(depth >= 0.0f) ||
                depth != std::floor(depth))
                return static_cast<emerge_status>(s->fail(
                    EMERGE_ERR_INVALID_ARG,
                    "force field " + std::to_string(k) + ": max_depth and max_bodies_per_node must be non-negative integers"));
            if (depth > static_cast<float>(NBODY_MAX_DEPTH))
                return static_cast<emerge_status>(
                    s->fail(EMERGE_ERR_UNSUPPORTED, "force field " + std::to_string(k) + ": max_depth above " +
                                                        std::to_string(NBODY_MAX_DEPTH)));
            break;
        }
        default:
            return static_cast<emerge_status>(
                s->fail(EMERGE_ERR_UNSUPPORTED, "force field " + std::to_string(k) + ": unknown kind"));
        }
        if (static_cast<uint64_t>(f.data_offset) + need > n_data)
            return static_cast<emerge_status>(
                s->fail(EMERGE_ERR_INVALID_ARG, "force field " + std::to_string(k) + ": data out of range"));
    }
    // NBody fields share one tree: the same max_depth and max_bodies_per_node
    NBodyTreeHost tree;
    for (uint32_t k = 0; k < n; ++k) {
        const emerge_force_field &f = fields[k];
        if (f.kind != EMERGE_FIELD_NBODY_GRAVITY) continue;
        const int depth = static_cast<int>(f.params[3]), maxb = static_cast<int>(f.params[4]);
        if (tree.depth >= 0 && (tree.depth != depth || tree.max_bodies != maxb))
            return static_cast<emerge_status>(s->fail(
                EMERGE_ERR_UNSUPPORTED, "n-body fields with different max_depth or max_bodies_per_node"));
        tree.depth = depth;
        tree.max_bodies = maxb;
        tree.theta_max = std::max(tree.theta_max, f.params[2]);
        ++tree.n_fields;
    }
    if (s->stream) CK(cudaStreamSynchronize(s->stream));  // kernels in flight may read the old table
    if (tree.depth < 0) {
        s->nbbuf.reset();
        s->nb = NBodyTreeHost{};
        s->nb_cap = 0;
        s->nb_alloc_depth = -1;
    } else {
        s->nb.depth = tree.depth;
        s->nb.max_bodies = tree.max_bodies;
        s->nb.theta_max = tree.theta_max;
        s->nb.n_fields = tree.n_fields;
        if (s->nb_alloc_depth != tree.depth || s->nb_alloc_fields != tree.n_fields)
            s->nbbuf.reset();  // reallocated for the new depth or field count
        s->nb_alloc_depth = s->nbbuf.ptr ? tree.depth : -1;
    }
    s->fbuf.reset();
    s->n_fields = 0;
    if (n > 0) {
        const size_t table = align_up(n * sizeof(emerge_force_field), 256);
        const size_t bytes = table + std::max<uint64_t>(n_data, 1) * sizeof(float);
        CK(cudaMalloc(&s->fbuf.ptr, bytes));
        s->fbuf.bytes = bytes;
        CK(cudaMemcpy(s->fbuf.ptr, fields, n * sizeof(emerge_force_field), cudaMemcpyHostToDevice));
        if (n_data)
            CK(cudaMemcpy(static_cast<char *>(s->fbuf.ptr) + table, data, n_data * sizeof(float),
                          cudaMemcpyHostToDevice));
        s->n_fields = static_cast<int>(n);
    }
    refresh_dev_config(s);
    s->graph_dirty = true;
    return EMERGE_OK;
}

static emerge_status sync_state(emerge_sim *s);

emerge_status emerge_cuda_field_accelerations(emerge_sim *s, float *out, uint64_t n) {
    if (!s || (!out && n)) return EMERGE_ERR_INVALID_ARG;
    if (n != s->n)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "n must equal the particle count"));
    if (n == 0) return EMERGE_OK;
    emerge_status st = nbody_prepare(s);
    if (st != EMERGE_OK) return st;
    StepLaunch L = make_launch(s);
    if (nbody_live(s)) {
        launch_nbody_build(s->nb, L.P, L.n, s->sort, det_pipeline(s), s->stream);
        launch_nbody_walk(s->nb, L.cfg, L.P, L.n, true, s->stream);
    }
    float2 *d_out = nullptr;
    CK(cudaMalloc(&d_out, n * sizeof(float2)));
    launch_field_accelerations(L, s->lf, d_out);
    cudaError_t e = cudaMemcpyAsync(out, d_out, n * sizeof(float2), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(d_out);
    CK(e);
    return sync_state(s);
}

emerge_status emerge_cuda_set_contact_grip(emerge_sim *s, int enabled, float mu_easy, float mu_resist,
                                          float dir_x, float dir_y) {
    if (!s) return EMERGE_ERR_INVALID_ARG;
    if (enabled && !(mu_easy >= 0.0f && mu_easy <= 1.0f && mu_resist >= 0.0f && mu_resist <= 1.0f))
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "mu_easy and mu_resist must be in [0.0, 1.0]"));
    if (enabled && !(std::isfinite(dir_x) && std::isfinite(dir_y)))
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "easy direction must be finite"));
    s->grip_on = enabled ? 1 : 0;
    s->grip_mu_easy = enabled ? mu_easy : 0.0f;
    s->grip_mu_resist = enabled ? mu_resist : 0.0f;
    s->grip_dir[0] = enabled ? dir_x : 0.0f;
    s->grip_dir[1] = enabled ? dir_y : 0.0f;
    refresh_dev_config(s);
    s->graph_dirty = true;
    return EMERGE_OK;
}

emerge_status emerge_cuda_set_mixture_phases(emerge_sim *s, const uint32_t *phases, uint32_t count) {
    if (!s || (!phases && count)) return EMERGE_ERR_INVALID_ARG;
    if (count > static_cast<uint32_t>(MAX_MATERIALS))
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "at most 64 material slots"));
    for (uint32_t k = 0; k < count; ++k)
        if (phases[k] > 2u)
            return static_cast<emerge_status>(
                s->fail(EMERGE_ERR_INVALID_ARG, "material " + std::to_string(k) + ": phase must be 0, 1 or 2"));
    if (s->stream) CK(cudaStreamSynchronize(s->stream));  // kernels in flight may read the old table
    s->phases.assign(phases, phases + count);
    emerge_status st = upload_phases(s);
    if (st != EMERGE_OK) return st;
    return update_multi(s);
}

emerge_status emerge_cuda_add_body(emerge_sim *s, const emerge_spawn_region *spawn, uint32_t *tag_out) {
    if (!s || !spawn) return EMERGE_ERR_INVALID_ARG;
    std::vector<emerge_particle> ps;
    uint32_t tag = s->next_tag;
    emerge_status st = spawn_region(s, *spawn, tag, ps);
    if (st != EMERGE_OK) return st;
    s->next_tag += 1;
    st = append_particles(s, ps.data(), ps.size(), 1);
    if (st != EMERGE_OK) return st;
    if (tag_out) *tag_out = tag;
    return EMERGE_OK;
}

emerge_status emerge_cuda_init_with_spawn(emerge_sim *s, const emerge_spawn_region *spawn) {
    if (!s || !spawn) return EMERGE_ERR_INVALID_ARG;
    if (s->n != 0)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "init_with_spawn needs an empty simulation"));
    std::vector<emerge_particle> ps;
    emerge_status st = spawn_region(s, *spawn, 0, ps);
    if (st != EMERGE_OK) return st;
    // Simulation::new does not run init_particle (lifecycle.rs:57-99): undo it.
    for (auto &q : ps) {
        q.plastic_volume_ratio = 1.0f;
        q.hardening_scale = 1.0f;
        q.friction_hardening = 0.0f;
        q.log_volume_strain = 0.0f;
    }
    return append_particles(s, ps.data(), ps.size(), spawn->precompute_initial_volumes ? 2 : 0);
}

emerge_status emerge_cuda_add_particles(emerge_sim *s, const emerge_particle *particles, uint64_t n,
                                        int estimate_volumes) {
    if (!s || (!particles && n)) return EMERGE_ERR_INVALID_ARG;
    return append_particles(s, particles, static_cast<size_t>(n), estimate_volumes ? 1 : 0);
}

emerge_status emerge_cuda_particle_count(const emerge_sim *s, uint64_t *n_out) {
    if (!s || !n_out) return EMERGE_ERR_INVALID_ARG;
    *n_out = s->n;
    return EMERGE_OK;
}

emerge_status emerge_cuda_read_particles(emerge_sim *s, emerge_particle *out, uint64_t n) {
    if (!s || (!out && n)) return EMERGE_ERR_INVALID_ARG;
    if (n != s->n) return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "n must equal the particle count"));
    if (n == 0) return EMERGE_OK;
    launch_gather_aos(s->P[s->cur], static_cast<int>(n), s->d_aos, s->stream);
    s->host_launches += 1;
    CK(cudaMemcpyAsync(out, s->d_aos, n * sizeof(emerge_particle), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_read_particles_async(emerge_sim *s, emerge_particle *out, uint64_t n) {
    if (!s || (!out && n)) return EMERGE_ERR_INVALID_ARG;
    if (n != s->n) return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "n must equal the particle count"));
    if (n == 0) return EMERGE_OK;
    if (!s->copy_stream) {
        CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&s->ev_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s->ev_gathered, cudaEventDisableTiming));
    }
    const size_t bytes = s->cap * sizeof(emerge_particle);
    if (s->staging_rb.bytes < bytes) {
        CK(cudaStreamSynchronize(s->copy_stream));  // the old buffer may still be copied out
        s->staging_rb.reset();
        CK(cudaMalloc(&s->staging_rb.ptr, bytes));
        s->staging_rb.bytes = bytes;
    }
    emerge_particle *rb = static_cast<emerge_particle *>(s->staging_rb.ptr);
    // gather on the copy stream once the queued steps are done; later work on the
    // simulation's stream waits for the gather only, not for the copy-out
    CK(cudaEventRecord(s->ev_ready, s->stream));
    CK(cudaStreamWaitEvent(s->copy_stream, s->ev_ready, 0));
    launch_gather_aos(s->P[s->cur], static_cast<int>(n), rb, s->copy_stream);
    s->host_launches += 1;
    CK(cudaEventRecord(s->ev_gathered, s->copy_stream));
    CK(cudaStreamWaitEvent(s->stream, s->ev_gathered, 0));
    CK(cudaMemcpyAsync(out, rb, n * sizeof(emerge_particle), cudaMemcpyDeviceToHost, s->copy_stream));
    CK(cudaGetLastError());
    return EMERGE_OK;
}

emerge_status emerge_cuda_write_particles(emerge_sim *s, const emerge_particle *in, uint64_t n) {
    if (!s || (!in && n)) return EMERGE_ERR_INVALID_ARG;
    if (n != s->n) return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "n must equal the particle count"));
    if (n == 0) return EMERGE_OK;
    // Upload into a staging buffer of its own on a stream of its own, so the copy overlaps
    // the work already queued on the simulation's stream (which waits for it before the
    // check), then check it there (contact groups switch the multi-field pipeline on,
    // pinned particles the pinned load).
    if (!s->up_stream) {
        CK(cudaStreamCreateWithFlags(&s->up_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&s->ev_up_done, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s->ev_up_free, cudaEventDisableTiming));
    }
    const size_t up_bytes = s->cap * sizeof(emerge_particle);
    if (s->staging_up.bytes < up_bytes) {
        CK(cudaStreamSynchronize(s->stream));  // the previous upload's scatter reads the old buffer
        s->staging_up.reset();
        CK(cudaMalloc(&s->staging_up.ptr, up_bytes));
        s->staging_up.bytes = up_bytes;
        s->up_used = false;
    }
    emerge_particle *up = static_cast<emerge_particle *>(s->staging_up.ptr);
    if (s->up_used) CK(cudaStreamWaitEvent(s->up_stream, s->ev_up_free, 0));  // read by the last scatter
    CK(cudaMemcpyAsync(up, in, n * sizeof(emerge_particle), cudaMemcpyHostToDevice, s->up_stream));
    CK(cudaEventRecord(s->ev_up_done, s->up_stream));
    CK(cudaStreamWaitEvent(s->stream, s->ev_up_done, 0));
    CK(cudaMemsetAsync(&s->d_state->upload_flags, 0, sizeof(uint32_t), s->stream));
    launch_check_aos(up, static_cast<int>(n), &s->d_state->upload_flags, s->stream);
    // The flags come back by a store into the mapped mirror, not by a copy: a device-to-host
    // copy here would queue behind a readback still in flight (emerge_cuda_read_particles_async
    // of the previous step) and hold this call up until it lands.
    if (s->h_state_dev) {
        launch_copy_word_to_host(&s->d_state->upload_flags, &s->h_state_dev->upload_flags, s->stream);
        s->host_launches += 1;
    } else {
        CK(cudaMemcpyAsync(&s->h_state->upload_flags, &s->d_state->upload_flags, sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, s->stream));
    }
    CK(cudaStreamSynchronize(s->stream));
    s->host_launches += 1;
    const uint32_t flags = s->h_state->upload_flags;
    if (((flags & 1u) != 0) != s->contact_seen) {  // the upload replaces every particle
        s->contact_seen = (flags & 1u) != 0;
        emerge_status st = update_multi(s);
        if (st != EMERGE_OK) return st;
    }
    const int pinned = (flags & 2u) ? 1 : 0;  // the upload replaces every particle
    if (pinned != s->lf.pinned) {
        s->lf.pinned = pinned;
        s->graph_dirty = true;  // the particle kernels' load flags are baked into the graph
    }
    launch_scatter_aos(s->P[s->cur], static_cast<int>(n), up, s->stream);
    CK(cudaEventRecord(s->ev_up_free, s->stream));
    s->up_used = true;
    s->host_launches += 1;
    if (s->dcfg.zones) launch_zone_bits(s->P[s->cur], static_cast<int>(n), static_cast<uint32_t>(s->active), s->stream);
    CK(cudaGetLastError());
    return invalidate_pending(s);
}

emerge_status emerge_cuda_active_count(emerge_sim *s, uint64_t *out) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    *out = s->active;
    return EMERGE_OK;
}

emerge_status emerge_cuda_replace_particles(emerge_sim *s, const emerge_particle *in, uint64_t n,
                                            uint64_t active_count) {
    if (!s || (!in && n)) return EMERGE_ERR_INVALID_ARG;
    if (active_count > n)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "active_count above the particle count"));
    if (s->stream) CK(cudaStreamSynchronize(s->stream));
    s->n = 0;
    s->active = 0;
    s->lf.pinned = 0;
    s->contact_seen = false;
    emerge_status st = append_particles(s, in, n, 0);
    if (st == EMERGE_OK && !s->contact_seen && s->dcfg.multi) st = update_multi(s);
    if (st != EMERGE_OK) return st;
    s->active = active_count;
    st = update_zones(s);
    if (st != EMERGE_OK) return st;
    if (s->dcfg.zones) launch_zone_bits(s->P[s->cur], static_cast<int>(n), static_cast<uint32_t>(active_count), s->stream);
    s->graph_dirty = true;
    CK(cudaGetLastError());
    return invalidate_pending(s);
}

emerge_status emerge_cuda_step(emerge_sim *s, uint32_t n_steps, emerge_step_timing *timing) {
    if (!s) return EMERGE_ERR_INVALID_ARG;
    // An empty simulation still runs the substep loop (step.rs:34-49): with no particles the
    // CFL bound leaves the whole frame as one substep, and last_substeps / effective_dt report
    // it as the reference does; every particle kernel launcher returns at n == 0.
    if (s->dcfg.mf_fast && (s->dcfg.mf_fields & 1)) {  // the contact lists' nodes, one per slot
        float4 *before = s->g.cpts;
        if (s->list_cap < s->cap) {
            CK(cudaStreamSynchronize(s->stream));  // queued kernels may still walk the old nodes
            s->listbuf.reset();
            CK(cudaMalloc(&s->listbuf.ptr, std::max<size_t>(s->cap, 1) * sizeof(float4)));
            s->listbuf.bytes = std::max<size_t>(s->cap, 1) * sizeof(float4);
            s->list_cap = s->cap;
        }
        s->g.cpts = static_cast<float4 *>(s->listbuf.ptr);
        if (s->g.cpts != before) {
            s->graph_dirty = true;
            emerge_status st = invalidate_pending(s);
            if (st != EMERGE_OK) return st;
        }
    }
    {
        emerge_status st = nbody_prepare(s);
        if (st != EMERGE_OK) return st;
    }
    for (uint32_t k = 0; k < n_steps; ++k) {
        emerge_status st = maybe_sort(s);
        if (st != EMERGE_OK) return st;
        if (!s->pending_valid) {
            st = prime(s);
            if (st != EMERGE_OK) return st;
        }
        st = update_zones(s);
        if (st != EMERGE_OK) return st;
        if (det_pipeline(s)) {
            st = run_det_step(s, timing != nullptr);
            if (st != EMERGE_OK) return st;
        } else if (s->use_graph && !s->dcfg.zones) {
            if (s->graph_dirty || !s->graph_exec) {
                st = build_graph(s);
                if (st != EMERGE_OK) return st;
            }
            bool timed = timing && k + 1 == n_steps;
            if (timed) CK(cudaEventRecord(s->ev[0], s->stream));
            CK(cudaGraphLaunch(s->graph_exec, s->stream));
            s->graph_launches += 1;
            if (timed) {
                CK(cudaEventRecord(s->ev[6], s->stream));
                CK(cudaEventSynchronize(s->ev[6]));
                float tot;
                cudaEventElapsedTime(&tot, s->ev[0], s->ev[6]);
                std::memset(&s->last_timing, 0, sizeof(s->last_timing));
                s->last_timing.total_us = static_cast<uint64_t>(tot * 1000.0f);
            }
        } else {
            st = run_host_loop_step(s, timing != nullptr);
            if (st != EMERGE_OK) return st;
        }
        CK(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(StepState), cudaMemcpyDeviceToHost, s->stream));
        s->steps_since_sort += 1;
        if (s->dcfg.zones) {  // the step's wakes and sleeps into the reference indices
            st = drain_zone_log(s);
            if (st == EMERGE_OK) st = commit_perm(s);
            if (st == EMERGE_OK) st = update_zones(s);
            if (st != EMERGE_OK) return st;
        }
    }
    CK(cudaGetLastError());
    if (timing) {
        CK(cudaStreamSynchronize(s->stream));
        *timing = s->last_timing;
    }
    return EMERGE_OK;
}

static emerge_status sync_state(emerge_sim *s) {
    CK(cudaMemcpyAsync(s->h_state, s->d_state, sizeof(StepState), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (s->h_state->error_flags & ERR_CLOSURE_WAIT)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_TIMEOUT,
                                                  "learned closure: a tensor-core wait gave up (tile kernel returned)"));
    if (s->h_state->error_flags & ERR_CONTACT_LIST)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_CUDA, "contact point list walk cut short"));
    if (s->h_state->error_flags & ERR_NBODY_SKIPPED)
        return static_cast<emerge_status>(s->fail(EMERGE_ERR_CUDA, "n-body field: a far node had no center of mass"));
    return EMERGE_OK;
}

emerge_status emerge_cuda_last_substeps(emerge_sim *s, uint64_t *out) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    emerge_status st = sync_state(s);
    if (st != EMERGE_OK) return st;
    *out = s->h_state->substeps;
    return EMERGE_OK;
}

emerge_status emerge_cuda_effective_dt(emerge_sim *s, float *out) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    emerge_status st = sync_state(s);
    if (st != EMERGE_OK) return st;
    *out = s->h_state->last_step_dt;
    return EMERGE_OK;
}

emerge_status emerge_cuda_last_counters(emerge_sim *s, uint64_t *vel_clamp, uint64_t *jproj,
                                        float *dropped) {
    if (!s) return EMERGE_ERR_INVALID_ARG;
    emerge_status st = sync_state(s);
    if (st != EMERGE_OK) return st;
    if (vel_clamp) *vel_clamp = s->h_state->vel_clamp;
    if (jproj) *jproj = s->h_state->jproj;
    if (dropped) *dropped = s->h_state->dropped;
    return EMERGE_OK;
}

emerge_status emerge_cuda_synchronize(emerge_sim *s) {
    if (!s) return EMERGE_ERR_INVALID_ARG;
    CK(cudaStreamSynchronize(s->stream));
    if (s->copy_stream) CK(cudaStreamSynchronize(s->copy_stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_region_state(emerge_sim *s, float cx, float cy, float radius,
                                       emerge_body_state *out) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    std::vector<unsigned char> acc(region_acc_bytes(), 0);
    // max_jp starts at the ordered encoding of 0.0f (BodyState::default)
    CK(cudaMemsetAsync(s->region_buf.ptr, 0, region_acc_bytes(), s->stream));
    uint32_t zero_ordered = 0x80000000u;
    CK(cudaMemcpyAsync(static_cast<char *>(s->region_buf.ptr) + region_acc_bytes() - 8, &zero_ordered, 4,
                       cudaMemcpyHostToDevice, s->stream));
    launch_region_state(s->P[s->cur], static_cast<int>(s->n), cx, cy, radius * radius, s->region_buf.ptr,
                        s->stream, s->dcfg.zones);
    s->host_launches += 1;
    CK(cudaMemcpyAsync(acc.data(), s->region_buf.ptr, acc.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    region_acc_finalize(acc.data(), out);
    return EMERGE_OK;
}

emerge_status emerge_cuda_set_option(emerge_sim *s, int option, int64_t value) {
    if (!s) return EMERGE_ERR_INVALID_ARG;
    switch (option) {
    case EMERGE_OPT_USE_GRAPH: s->use_graph = value != 0; return EMERGE_OK;
    case EMERGE_OPT_SORT_INTERVAL:
        if (value < 0) return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "sort interval < 0"));
        s->sort_interval = value;
        return EMERGE_OK;
    case EMERGE_OPT_P2G_AGGREGATE:
        if (value < 0 || value > 2)
            return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "P2G aggregation mode must be 0, 1 or 2"));
        s->use_window = static_cast<int>(value);
        s->graph_dirty = true;
        return EMERGE_OK;
    case EMERGE_OPT_DETERMINISTIC: {
        int v = value != 0;
        if (v != s->deterministic) {
            emerge_status st = invalidate_pending(s);
            if (st != EMERGE_OK) return st;
            s->deterministic = v;
            if (v) {
                st = ensure_det_scratch(s);
                if (st != EMERGE_OK) return st;
            }
        }
        s->dcfg.precise_math = s->precise_opt >= 0 ? s->precise_opt : s->deterministic;
        refresh_dev_config(s);  // the multi-field pipeline follows the mode
        s->graph_dirty = true;
        return EMERGE_OK;
    }
    case EMERGE_OPT_PRECISE_MATH:
        s->precise_opt = value < 0 ? -1 : (value != 0);
        s->dcfg.precise_math = s->precise_opt >= 0 ? s->precise_opt : s->deterministic;
        s->graph_dirty = true;
        return invalidate_pending(s);
    default: return static_cast<emerge_status>(s->fail(EMERGE_ERR_INVALID_ARG, "unknown option"));
    }
}

emerge_status emerge_cuda_sort_now(emerge_sim *s, int key_mode) {
    if (!s || (key_mode != 0 && key_mode != 1)) return EMERGE_ERR_INVALID_ARG;
    emerge_status st = sort_particles(s, key_mode);
    if (st != EMERGE_OK) return st;
    CK(cudaStreamSynchronize(s->stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_sort_keys(const float *xy, uint64_t n, uint32_t grid_res, int key_mode,
                                    uint32_t *keys_out, uint32_t *perm_out) {
    if ((!xy && n) || (key_mode != 0 && key_mode != 1) || grid_res < 1 || n > 0x7fffffffull) {
        g_global_error = "invalid argument";
        return EMERGE_ERR_INVALID_ARG;
    }
    if (n == 0) return EMERGE_OK;
    cudaStream_t stream;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
        g_global_error = "stream create failed";
        return EMERGE_ERR_CUDA;
    }
    float2 *d_xy = nullptr;
    void *scratch = nullptr;
    emerge_status rc = EMERGE_OK;
    SortScratch sc;
    int r = 0;
    if (cudaMalloc(&d_xy, n * sizeof(float2)) != cudaSuccess ||
        cudaMalloc(&scratch, sort_scratch_bytes(n)) != cudaSuccess) {
        rc = EMERGE_ERR_OOM;
        goto done;
    }
    sort_scratch_bind(sc, scratch, n);
    cudaMemcpyAsync(d_xy, xy, n * sizeof(float2), cudaMemcpyHostToDevice, stream);
    launch_sort_keys(d_xy, static_cast<int>(n), static_cast<int>(grid_res), key_mode, sc.keys[0], sc.vals[0],
                     stream);
    cudaMemcpyAsync(keys_out, sc.keys[0], n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    r = radix_sort_pairs(sc, static_cast<int>(n), sort_key_bits(static_cast<int>(grid_res), key_mode), stream);
    cudaMemcpyAsync(perm_out, sc.vals[r], n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = EMERGE_ERR_CUDA;
done:
    if (rc != EMERGE_OK) g_global_error = "sort_keys failed";
    if (d_xy) cudaFree(d_xy);
    if (scratch) cudaFree(scratch);
    cudaStreamDestroy(stream);
    return rc;
}

void *emerge_cuda_stream(emerge_sim *s) { return s ? static_cast<void *>(s->stream) : nullptr; }

emerge_status emerge_cuda_event_record(emerge_sim *s, int slot) {
    if (!s || slot < 0 || slot >= 16) return EMERGE_ERR_INVALID_ARG;
    if (!s->user_ev[slot]) CK(cudaEventCreate(&s->user_ev[slot]));
    CK(cudaEventRecord(s->user_ev[slot], s->stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_event_elapsed(emerge_sim *s, int from, int to, float *ms) {
    if (!s || !ms || from < 0 || from >= 16 || to < 0 || to >= 16 || !s->user_ev[from] ||
        !s->user_ev[to])
        return EMERGE_ERR_INVALID_ARG;
    CK(cudaEventSynchronize(s->user_ev[to]));
    CK(cudaEventElapsedTime(ms, s->user_ev[from], s->user_ev[to]));
    return EMERGE_OK;
}

emerge_status emerge_cuda_flush_l2(emerge_sim *s) {
    if (!s) return EMERGE_ERR_INVALID_ARG;
    const size_t bytes = size_t(512) << 20;  // 512 MiB > 126 MB L2
    if (!s->flushbuf.ptr) {
        CK(cudaMalloc(&s->flushbuf.ptr, bytes));
        s->flushbuf.bytes = bytes;
    }
    CK(cudaMemsetAsync(s->flushbuf.ptr, static_cast<int>(s->host_launches & 0xff), bytes, s->stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_host_alloc(size_t bytes, void **out) {
    if (!out) return EMERGE_ERR_INVALID_ARG;
    cudaError_t e = cudaMallocHost(out, bytes);
    if (e != cudaSuccess) {
        g_global_error = cudaGetErrorString(e);
        return EMERGE_ERR_OOM;
    }
    return EMERGE_OK;
}

emerge_status emerge_cuda_host_free(void *ptr) {
    if (ptr) cudaFreeHost(ptr);
    return EMERGE_OK;
}

emerge_status emerge_cuda_stats(emerge_sim *s, emerge_stats *out) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    emerge_status st = sync_state(s);
    if (st != EMERGE_OK) return st;
    out->steps = s->h_state->total_steps;
    out->substeps = s->h_state->total_substeps;
    out->kernel_launches = s->host_launches + s->graph_launches + s->h_state->graph_kernels;
    out->p2g_blocks = s->h_state->window_blocks;
    out->p2g_fallback_blocks = s->h_state->window_fallback;
    out->sorts = s->sorts;
    return EMERGE_OK;
}

emerge_status emerge_cuda_kernel_launches(emerge_sim *s, uint64_t *out) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    emerge_status st = sync_state(s);
    if (st != EMERGE_OK) return st;
    *out = s->host_launches + s->graph_launches + s->h_state->graph_kernels;
    return EMERGE_OK;
}

}  // extern "C"
