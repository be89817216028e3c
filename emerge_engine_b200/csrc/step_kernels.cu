// step_kernels.cu -- the MLS-MPM substep on sm_100a.
//
// One substep k of the reference (spacetime/solver/step.rs:62-317) runs as:
//   k_substep_begin   1 thread: dt(k) from the CFL reduction (step.rs:434-479),
//                     loop bookkeeping, CUDA-graph loop condition.
//   k_grid_update     per active 8x8 tile: momentum = A + dt*S, normalise, gravity,
//                     slip walls, speed clamp (grid/mod.rs:264-291, step.rs:150-165),
//                     then zero the accumulators for the next scatter.
//   k_particle        per particle, fused: projection recompute, G2P gather
//                     (transfer/g2p.rs:151-328), constitutive update (:333-340),
//                     CFL contribution for substep k+1 (step.rs:447-466), projection
//                     for k+1 (step.rs:347-429), P2G scatter for k+1
//                     (transfer/p2g.rs:24-72) as vector reductions into L2.
//   k_density         only when a material needs it (step.rs:80-87): density gather
//                     (solver/density.rs:41-72) + the fluid stress scatter, which
//                     depends on that density (fluid.rs:157-162, 193-195).
// Particle state is read once and written once per substep by k_particle.
// The pass before the first substep of a step sequence (k_particle in prime
// mode) only projects and scatters.
#include <cfloat>
#include <cstdio>

#include "particle_pass.cuh"

namespace emerge {

// ---------------------------------------------------------------- k_particle (exact)
// Reference-order mode: cell-by-cell stencil sums, IEEE division and square root, no
// contraction (this file is compiled with -fmad=false).
template <unsigned MASK>
__global__ void __launch_bounds__(THREADS, 4) k_particle(ParticleKernelArgs a) {
    particle_pass<MASK, false>(a);
}

// ---------------------------------------------------------------- grid update
struct GridKernelArgs {
    GridView g;
    DevConfig cfg;
    StepState *st;
    int n_tiles;
};

// Grid::update_velocities (grid/mod.rs:264-291), boundaries (step.rs:150-152,
// 334-344; forces/boundary/mod.rs:78-101), speed clamp (step.rs:155-165) for one cell of
// an active tile, then the accumulators are zeroed for the next scatter.
// The fast pipeline's field sum of one cell: A + dt S as {m, px, py, w} (the form the
// reference-order scatter writes, w > 0 marking the field), the accumulators zeroed for the
// next scatter.  Each scatter adds exactly 1 to the w lanes, so `rest_w`, the scatters of the
// particles outside the field, is an exact count whatever the order of the sums: w = 2 marks
// a cell that also holds other particles, w = 1 a field-only cell, whose rest mass the
// reference computes as exactly 0 (its field and total sums run in the same order), while
// total - field here would be rounding noise.
__device__ __forceinline__ bool finalize_field(float4 *fa, float2 *fs, float4 *out, int ci, float dt,
                                               float rest_w) {
    const float4 a = fa[ci];
    if (!(a.w > 0.0f)) return false;
    const float2 s = fs[ci];
    out[ci] = make_float4(a.x, a.y + dt * s.x, a.z + dt * s.y, rest_w > 0.5f ? 2.0f : 1.0f);
    fa[ci] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    fs[ci] = v2(0.0f, 0.0f);
    return true;
}

__device__ __forceinline__ void grid_update_cell(const GridView &g, const DevConfig &cfg, float dt,
                                                 int tile, int local, uint32_t *contact_active) {
    const int ci = tile * TILE_CELLS + local;
    const int x = (tile / g.tpd) * TILE + (local >> 3);
    const int y = (tile % g.tpd) * TILE + (local & 7);
    float4 acc = g.acc_a[ci];
    float2 s = g.acc_s[ci];
    const float rest_w = acc.w;  // with exclusive field sums: the scatters of particles in no field
    if (cfg.mf_excl) {           // the fields' particles scattered into their fields only
        int k0 = 1, k1 = 2;      // the solid and fluid phases
        if (cfg.mf_fields & 1) k0 = k1 = 0;  // the grip field
        for (int k = k0; k <= k1; ++k) {
            const float4 f = g.fa[k][ci];
            const float2 fs = g.fs[k][ci];
            acc = make_float4(acc.x + f.x, acc.y + f.y, acc.z + f.z, acc.w + f.w);
            s = v2(s.x + fs.x, s.y + fs.y);
        }
    }
    float m = acc.x;
    float2 mom = v2(acc.y + dt * s.x, acc.z + dt * s.y);
    if (m > 0.0f) mom = vdivs(mom, m);
    // ASFLIP snapshot between normalisation and gravity (step.rs:140-147)
    if (cfg.asflip > 0.0f) g.grid_vpre[ci] = mom;
    if (m > 0.0f) {
        mom = vadd(mom, vmuls(cfg.gravity, dt));
        for (int k = 0; k < cfg.n_bound; ++k) slip_velocity(cfg.bound_t[k], x, y, g.res, mom);
        float vel_limit = cfg.cell / dt;
        float spd = vlen(mom);
        if (spd > vel_limit) mom = vmuls(mom, vel_limit / spd);
    }
    g.grid_v[ci] = mom;
    if (cfg.multi) {
        g.grid_m[ci] = m;  // the contact and mixture resolves read the total mass
        if (cfg.mf_fast) {
            if (cfg.mf_fields & 1) {
                float rest = rest_w;
                if (!cfg.mf_excl) rest = acc.w - g.fa[0][ci].w;
                if (finalize_field(g.fa[0], g.fs[0], g.acc_grip, ci, dt, rest))
                    *contact_active = 1u;  // Grid::has_contact_activity
            }
            if (cfg.mf_fields & 2) {
                finalize_field(g.fa[1], g.fs[1], g.acc_sol, ci, dt, 0.0f);
                finalize_field(g.fa[2], g.fs[2], g.acc_flu, ci, dt, 0.0f);
            }
        }
    }
    g.acc_a[ci] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    g.acc_s[ci] = v2(0.0f, 0.0f);
}

__global__ void __launch_bounds__(256) k_grid_update(GridKernelArgs a) {
    const int tile = blockIdx.x * 4 + (threadIdx.x >> 6);
    const int local = threadIdx.x & 63;
    uint8_t flag = 0;
    if (tile < a.n_tiles) flag = a.g.tile_flag[tile];
    __syncthreads();
    if (tile >= a.n_tiles || !flag) return;
    if (local == 0) a.g.tile_flag[tile] = 0;
    grid_update_cell(a.g, a.cfg, a.st->sub_dt, tile, local, &a.st->contact_active);
}

// Batched scenes: global tile t belongs to scene tile_scene[t] (local tile t - tile0).
// A tile's 64 cells span two warps, so the flag is cleared after a CTA barrier.
__global__ void __launch_bounds__(256) k_grid_update_batch(BatchView b, int n_tiles) {
    const int t = blockIdx.x * 4 + (threadIdx.x >> 6);
    const int local = threadIdx.x & 63;
    const SceneDesc *sd = nullptr;
    int tile = 0;
    uint8_t flag = 0;
    if (t < n_tiles) {
        sd = &b.scenes[b.tile_scene[t]];
        if (sd->st->active) {
            tile = t - sd->tile0;
            flag = sd->g.tile_flag[tile];
        }
    }
    __syncthreads();
    if (!flag) return;
    if (local == 0) sd->g.tile_flag[tile] = 0;
    grid_update_cell(sd->g, sd->cfg, sd->st->sub_dt, tile, local, &sd->st->contact_active);
}

// ---------------------------------------------------------------- controller
// Step start (step.rs:29-33).
__device__ __forceinline__ void step_begin_state(StepState &s, const DevConfig &cfg) {
    s.remaining = cfg.dt;
    s.substeps = 0;
    s.vel_clamp = 0;
    s.jproj = 0;
    s.dropped = fmaxf(cfg.dt, 0.0f);
    s.cont = (cfg.dt > F32_EPS && cfg.max_substeps > 0) ? 1u : 0u;
    s.total_steps += 1;
}

__global__ void k_step_begin(StepState *st, DevConfig cfg) { step_begin_state(*st, cfg); }

// Substep start: choose_substep_dt (step.rs:434-468) from the reduction of slot
// (parity), loop bookkeeping (step.rs:46-48); returns the loop condition (step.rs:34)
// for the next substep.
__device__ __forceinline__ uint32_t substep_begin_state(StepState &s, const DevConfig &cfg) {
    const uint32_t k = s.parity;
    const float rem = s.remaining;
    float dt;
    if (!cfg.adaptive) {
        dt = fminf(rem, cfg.dt);
    } else {
        float max_speed = __uint_as_float(s.max_speed_bits[k]);
        float min_mdt = __uint_as_float(s.min_mdt_bits[k]);
        dt = cfl_bound(cfg, max_speed, fminf(rem, min_mdt), rem);
    }
    s.sub_dt = dt;
    s.last_step_dt = dt;
    s.jproj += s.jproj_pending[k];
    const uint32_t k1 = k ^ 1u;
    s.max_speed_bits[k1] = 0u;
    s.min_mdt_bits[k1] = __float_as_uint(INFINITY);
    s.jproj_pending[k1] = 0ull;
    s.proj_changed[k1] = 0ull;
    for (int m = 0; m < CL_NMODELS; ++m) s.cl_queued[k1][m] = 0u;
    s.contact_active = 0u;
    s.acc_slot = k1;
    s.parity = k1;
    const float rem_after = rem - dt;
    s.remaining = rem_after;
    s.substeps += 1;
    s.total_substeps += 1;
    s.dropped = fmaxf(rem_after, 0.0f);
    s.cont = (rem_after > F32_EPS && s.substeps < static_cast<uint32_t>(cfg.max_substeps)) ? 1u : 0u;
    return s.cont;
}

__global__ void k_substep_begin(StepState *st, DevConfig cfg, int use_cond,
                                cudaGraphConditionalHandle handle, int kernels_per_substep) {
    StepState &s = *st;
    const uint32_t cont = substep_begin_state(s, cfg);
    s.active = 1u;
    if (use_cond) {
        s.graph_kernels += static_cast<unsigned long long>(kernels_per_substep);
        cudaGraphSetConditional(handle, cont);
    }
}

// Before a prime pass: the next k_substep_begin reads slot (parity).
__device__ __forceinline__ void prime_setup_state(StepState &s) {
    const uint32_t k = s.parity;
    s.max_speed_bits[k] = 0u;
    s.min_mdt_bits[k] = __float_as_uint(INFINITY);
    s.jproj_pending[k] = 0ull;
    s.proj_changed[k] = 0ull;
    s.acc_slot = k;
    s.active = 1u;
}

__global__ void k_prime_setup(StepState *st) { prime_setup_state(*st); }

// Batched controller, one thread per scene (one CTA).  A scene whose frame has ended
// (cont == 0) sits out the remaining substeps of the batch's frame (active = 0).
__global__ void k_step_begin_batch(BatchView b, StepState *batch_st) {
    int any = 0;
    for (int s = threadIdx.x; s < b.n_scenes; s += blockDim.x) {
        const SceneDesc &sd = b.scenes[s];
        step_begin_state(*sd.st, sd.cfg);
        any |= sd.st->cont ? 1 : 0;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        batch_st->total_steps += 1;
        batch_st->cont = any ? 1u : 0u;
    }
}

__global__ void k_substep_begin_batch(BatchView b, StepState *batch_st, int use_cond,
                                      cudaGraphConditionalHandle handle, int kernels_per_substep) {
    int any = 0;
    for (int s = threadIdx.x; s < b.n_scenes; s += blockDim.x) {
        StepState &st = *b.scenes[s].st;
        if (st.cont) {
            st.active = 1u;
            any |= substep_begin_state(st, b.scenes[s].cfg) ? 1 : 0;
        } else {
            st.active = 0u;
        }
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        batch_st->total_substeps += 1;
        batch_st->cont = any ? 1u : 0u;
        if (use_cond) {
            batch_st->graph_kernels += static_cast<unsigned long long>(kernels_per_substep);
            cudaGraphSetConditional(handle, any ? 1u : 0u);
        }
    }
}

__global__ void k_prime_setup_batch(BatchView b) {
    for (int s = threadIdx.x; s < b.n_scenes; s += blockDim.x) prime_setup_state(*b.scenes[s].st);
}

// ---------------------------------------------------------------- queries
struct RegionAcc {
    unsigned long long count;
    double sx, sy, speed, jp, det, rho;
    unsigned int max_jp_bits;  // ordered-int encoding of a float
    unsigned int pad;
};

__device__ __forceinline__ unsigned int float_to_ordered(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// region_state (queries.rs:125-141) as a device reduction (f64 partial sums).
__global__ void k_region_state(DevParticles P, int n, float cx, float cy, float r2,
                               RegionAcc *out, int zones) {
    __shared__ double sh[6][256 / 32];
    __shared__ unsigned long long shc[256 / 32];
    __shared__ unsigned int shm[256 / 32];
    double sx = 0, sy = 0, sp = 0, sjp = 0, sdet = 0, srho = 0;
    unsigned long long cnt = 0;
    unsigned int mjp = float_to_ordered(0.0f);  // BodyState::default max_volume_ratio = 0
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float2 x = P.x[i];
        float2 d = vsub(x, v2(cx, cy));
        // the spatial hash holds the active zone only (step.rs:53-56)
        if (vlen2(d) <= r2 && !(zones && (P.sleeping[i] & ZB_OUT))) {
            cnt += 1;
            sx += x.x;
            sy += x.y;
            sp += vlen(P.v[i]);
            float jp = P.jp[i];
            sjp += jp;
            unsigned int o = float_to_ordered(jp);
            if (!isnan(jp) && o > mjp) mjp = o;
            sdet += mdet(m_from4(P.f[i]));
            srho += P.rho[i];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sp += __shfl_xor_sync(0xffffffffu, sp, o);
        sjp += __shfl_xor_sync(0xffffffffu, sjp, o);
        sdet += __shfl_xor_sync(0xffffffffu, sdet, o);
        srho += __shfl_xor_sync(0xffffffffu, srho, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        mjp = max(mjp, __shfl_xor_sync(0xffffffffu, mjp, o));
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sh[0][w] = sx; sh[1][w] = sy; sh[2][w] = sp; sh[3][w] = sjp; sh[4][w] = sdet; sh[5][w] = srho;
        shc[w] = cnt;
        shm[w] = mjp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < 256 / 32; ++k) {
            sh[0][0] += sh[0][k]; sh[1][0] += sh[1][k]; sh[2][0] += sh[2][k];
            sh[3][0] += sh[3][k]; sh[4][0] += sh[4][k]; sh[5][0] += sh[5][k];
            shc[0] += shc[k];
            shm[0] = max(shm[0], shm[k]);
        }
        if (shc[0]) {
            atomicAdd(&out->count, shc[0]);
            atomicAdd(&out->sx, sh[0][0]);
            atomicAdd(&out->sy, sh[1][0]);
            atomicAdd(&out->speed, sh[2][0]);
            atomicAdd(&out->jp, sh[3][0]);
            atomicAdd(&out->det, sh[4][0]);
            atomicAdd(&out->rho, sh[5][0]);
            atomicMax(&out->max_jp_bits, shm[0]);
        }
    }
}

// ---------------------------------------------------------------- particle I/O
__global__ void k_gather_aos(DevParticles P, int n, emerge_particle *out) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    emerge_particle q;
    float2 x = P.x[s], v = P.v[s];
    float4 c = P.c[s], f = P.f[s];
    q.x[0] = x.x; q.x[1] = x.y;
    q.v[0] = v.x; q.v[1] = v.y;
    q.c[0] = c.x; q.c[1] = c.y; q.c[2] = c.z; q.c[3] = c.w;
    q.f[0] = f.x; q.f[1] = f.y; q.f[2] = f.z; q.f[3] = f.w;
    q.mass = P.mass[s];
    q.initial_volume = P.v0[s];
    q.volume = P.vol[s];
    q.density = P.rho[s];
    q.material_id = P.mat[s];
    q.plastic_volume_ratio = P.jp[s];
    q.hardening_scale = P.h[s];
    q.friction_hardening = P.q[s];
    q.log_volume_strain = P.lvs[s];
    q.temperature = P.temperature[s];
    q.user_tag = P.user_tag[s];
    q.activation = P.activation[s];
    float2 ad = P.act_dir[s];
    q.activation_dir[0] = ad.x; q.activation_dir[1] = ad.y;
    q.muscle_group_id = P.muscle[s];
    q.contact_group = P.contact[s];
    q.sleeping = P.sleeping[s] & ZB_FLAG;
    q.pinned = P.pinned[s];
    q.scalar_field = P.scalar[s];
    q.pad_ = 0;
    out[P.slot_to_index[s]] = q;
}

__device__ __forceinline__ void put_slot(const DevParticles &P, int s, const emerge_particle &q) {
    P.x[s] = v2(q.x[0], q.x[1]);
    P.v[s] = v2(q.v[0], q.v[1]);
    P.c[s] = make_float4(q.c[0], q.c[1], q.c[2], q.c[3]);
    P.f[s] = make_float4(q.f[0], q.f[1], q.f[2], q.f[3]);
    P.mass[s] = q.mass;
    P.v0[s] = q.initial_volume;
    P.vol[s] = q.volume;
    P.rho[s] = q.density;
    P.mat[s] = q.material_id;
    P.jp[s] = q.plastic_volume_ratio;
    P.h[s] = q.hardening_scale;
    P.q[s] = q.friction_hardening;
    P.lvs[s] = q.log_volume_strain;
    P.temperature[s] = q.temperature;
    P.user_tag[s] = q.user_tag;
    P.activation[s] = q.activation;
    P.act_dir[s] = v2(q.activation_dir[0], q.activation_dir[1]);
    P.muscle[s] = q.muscle_group_id;
    P.contact[s] = q.contact_group;
    P.sleeping[s] = q.sleeping;
    P.pinned[s] = q.pinned;
    P.scalar[s] = q.scalar_field;
    P.rho_dp[s] = 0.0f;
}

__global__ void k_scatter_aos(DevParticles P, int n, const emerge_particle *in) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    put_slot(P, s, in[P.slot_to_index[s]]);
}

// Flags of an uploaded particle array: bit 0 some contact_group != 0 (not on the device
// path), bit 1 some particle pinned.
__global__ void k_check_aos(const emerge_particle *in, int n, uint32_t *flags) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t f = 0;
    if (k < n) f = (in[k].contact_group != 0 ? 1u : 0u) | (in[k].pinned != 0 ? 2u : 0u);
    const unsigned any_c = __ballot_sync(0xffffffffu, (f & 1u) != 0u);
    const unsigned any_p = __ballot_sync(0xffffffffu, (f & 2u) != 0u);
    if ((threadIdx.x & 31) == 0 && (any_c | any_p))
        atomicOr(flags, (any_c ? 1u : 0u) | (any_p ? 2u : 0u));
}

__global__ void k_append_aos(DevParticles P, int n_old, int n_new, const emerge_particle *in) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int s = n_old + k;
    if (s >= n_new) return;
    put_slot(P, s, in[k]);
    P.slot_to_index[s] = static_cast<uint32_t>(s);
}

// init_particle for every particle (reinit_all_particle_state, lifecycle.rs:328-334)
__global__ void k_reinit(DevParticles P, int n, const MatP *mats, int n_mats) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t id = P.mat[s];
    const MatP &m = mats[id < static_cast<uint32_t>(n_mats) ? id : 0u];
    emerge_particle q;
    q.friction_hardening = P.q[s];
    q.plastic_volume_ratio = P.jp[s];
    q.hardening_scale = P.h[s];
    q.log_volume_strain = P.lvs[s];
    init_particle(m, q);
    P.q[s] = q.friction_hardening;
    P.jp[s] = q.plastic_volume_ratio;
    P.h[s] = q.hardening_scale;
    P.lvs[s] = q.log_volume_strain;
}

// Mass scatter of estimate_particle_volumes(_local) (density.rs:47-48, 105-120).
__global__ void k_mass_scatter(DevParticles P, int n, GridView g, int filter, float lox, float loy,
                               float hix, float hiy, int zones) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || (zones && (P.sleeping[s] & ZB_OUT))) return;
    float2 x = P.x[s];
    if (filter && (x.x < lox || x.y < loy || x.x > hix || x.y > hiy)) return;
    float mass = P.mass[s];
    QW w = quadratic_weights(x);
    for (int gx = 0; gx < 3; ++gx)
        for (int gy = 0; gy < 3; ++gy) {
            float weight = w.wx[gx] * w.wy[gy];
            int cx = w.bx + gx - 1, cy = w.by + gy - 1;
            if (!in_domain(cx, cy, g.res)) continue;
            atomicAdd(&g.acc_a[cell_index(cx, cy, g.tpd)].x, weight * mass);
        }
}

// Density gather of estimate_particle_volumes(_local) (density.rs:50-71, 122-143)
// for slots [lo, hi).
__global__ void k_mass_gather(DevParticles P, int lo, int hi, GridView g, int write_initial, int zones) {
    int s = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= hi || (zones && (P.sleeping[s] & ZB_OUT))) return;
    float2 x = P.x[s];
    float mass = P.mass[s];
    QW w = quadratic_weights(x);
    float density = 0.0f;
    for (int gx = 0; gx < 3; ++gx)
        for (int gy = 0; gy < 3; ++gy) {
            float weight = w.wx[gx] * w.wy[gy];
            int cx = w.bx + gx - 1, cy = w.by + gy - 1;
            float mc = in_domain(cx, cy, g.res) ? g.acc_a[cell_index(cx, cy, g.tpd)].x : 0.0f;
            density += mc * weight;
        }
    if (density > F32_EPS) {
        P.rho[s] = density;
        float vol = mass / density;
        P.vol[s] = vol;
        if (write_initial) P.v0[s] = vol;
    }
}

// ---------------------------------------------------------------- sleep partition
// Wake after P2G (step.rs:107-131): a particle outside the active zone whose stencil
// overlaps a cell of this substep's scatter (acc_a.w > 0) joins the active zone.  `key`
// is the event key of the substep the P2G belongs to.
__global__ void k_wake(DevParticles P, int n, GridView g, DevConfig cfg, const StepState *st,
                       int substep_offset) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || !(P.sleeping[s] & ZB_OUT)) return;
    const QW w = quadratic_weights(P.x[s]);
    bool hit = false;
    for (int gx = 0; gx < 3; ++gx)
        for (int gy = 0; gy < 3; ++gy) {
            const int cx = w.bx + gx - 1, cy = w.by + gy - 1;
            if (!in_domain(cx, cy, g.res)) continue;
            const int ci = cell_index(cx, cy, g.tpd);
            if (g.acc_a[ci].w > 0.0f) hit = true;
            // with exclusive field sums, a cell touched by field particles only
            if (cfg.mf_excl && (((cfg.mf_fields & 1) && g.fa[0][ci].w > 0.0f) ||
                                ((cfg.mf_fields & 2) && (g.fa[1][ci].w > 0.0f || g.fa[2][ci].w > 0.0f))))
                hit = true;
        }
    if (!hit) return;
    // The woken particle's G2P reads all 9 stencil cells, some of which this substep's P2G
    // may not have touched: flag their tiles so the grid update writes their velocity (zero
    // for an untouched cell, as Grid::velocity_at) instead of leaving an older substep's.
    mark_tiles(g, w.bx, w.by);
    P.sleeping[s] = ZB_WOKEN;  // wake_particle clears the flag (particles.rs:252-268)
    zone_log(cfg, 2u * static_cast<uint32_t>(st->total_substeps + substep_offset), P.slot_to_index[s]);
}

// Zone bits from the reference index: outside the active zone iff index >= active.
__global__ void k_zone_bits(DevParticles P, int n, uint32_t active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    P.sleeping[s] = (P.sleeping[s] & ZB_FLAG) | (P.slot_to_index[s] >= active ? ZB_OUT : 0u);
}

// Reference indices after the host replayed wake / sleep swaps: index := new_of_old[index].
__global__ void k_remap_index(DevParticles P, int n, const uint32_t *new_of_old) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) P.slot_to_index[s] = new_of_old[P.slot_to_index[s]];
}

// add_body with a sleeping zone (particles.rs:389-410): the new particles (slots [n_old,
// n_new)) take indices [old_active, old_active + count), the sleeping zone moves up.
__global__ void k_insert_index(DevParticles P, int n_old, int n_new, uint32_t old_active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_new) return;
    const uint32_t count = static_cast<uint32_t>(n_new - n_old);
    if (s >= n_old) {
        P.slot_to_index[s] = old_active + static_cast<uint32_t>(s - n_old);
    } else {
        const uint32_t idx = P.slot_to_index[s];
        if (idx >= old_active) P.slot_to_index[s] = idx + count;
    }
}

void launch_wake(const StepLaunch &L, int substep_offset) {
    if (L.n > 0) k_wake<<<blocks_for(L.n, 256), 256, 0, L.stream>>>(L.P, L.n, L.g, L.cfg, L.st, substep_offset);
}
void launch_zone_bits(const DevParticles &P, int n, uint32_t active, cudaStream_t stream) {
    if (n > 0) k_zone_bits<<<blocks_for(n, 256), 256, 0, stream>>>(P, n, active);
}
void launch_remap_index(const DevParticles &P, int n, const uint32_t *new_of_old, cudaStream_t stream) {
    if (n > 0) k_remap_index<<<blocks_for(n, 256), 256, 0, stream>>>(P, n, new_of_old);
}
void launch_insert_index(const DevParticles &P, int n_old, int n_new, uint32_t old_active, cudaStream_t stream) {
    if (n_new > 0) k_insert_index<<<blocks_for(n_new, 256), 256, 0, stream>>>(P, n_old, n_new, old_active);
}

// Field::acceleration summed over the force fields for every particle at its current state,
// written in reference index order (the dv of step.rs:232-236 before the dt factor).
__global__ void k_field_accelerations(DevParticles P, int n, LoadFlags lf, DevConfig cfg, float2 *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PState p = load_state(P, i, lf);
    const uint32_t ref = P.slot_to_index[i];
    if (ref < static_cast<uint32_t>(n)) out[ref] = force_field_sum(cfg, p, i);
}

// ---------------------------------------------------------------- launchers

void launch_field_accelerations(const StepLaunch &L, const LoadFlagsHost &lfh, float2 *out) {
    if (L.n == 0) return;
    LoadFlags lf;
    lf.temperature = lfh.temperature;
    lf.activation = lfh.activation;
    lf.pinned = lfh.pinned;
    k_field_accelerations<<<blocks_for(L.n, 256), 256, 0, L.stream>>>(L.P, L.n, lf, L.cfg, out);
}

void launch_particle_pass(const StepLaunch &L, const LoadFlagsHost &lfh, int mode_g2p,
                          int project_in, int emit_p2g, int split) {
    if (L.n == 0) return;
    ParticleKernelArgs a;
    fill_common(a, L, lfh);
    a.split = split;
    a.mode_g2p = mode_g2p;
    a.density_mode = L.density_mode;
    a.project_in = project_in;
    a.emit_p2g = emit_p2g;
    a.cl = L.cl;
    if (L.fast) {
        launch_particle_pass_fast(a, L.model_mask, L.stream);
        return;
    }
    const int grid = blocks_for(L.n, THREADS);
    switch (covering_mask(L.model_mask)) {
    case MASK_FLUID: k_particle<MASK_FLUID><<<grid, THREADS, 0, L.stream>>>(a); break;
    case MASK_SOLID: k_particle<MASK_SOLID><<<grid, THREADS, 0, L.stream>>>(a); break;
    case MASK_SOLID_FLUID: k_particle<MASK_SOLID_FLUID><<<grid, THREADS, 0, L.stream>>>(a); break;
    case MASK_GRANULAR: k_particle<MASK_GRANULAR><<<grid, THREADS, 0, L.stream>>>(a); break;
    case ALL_MODELS: k_particle<ALL_MODELS><<<grid, THREADS, 0, L.stream>>>(a); break;
    default: k_particle<FULL_MODELS><<<grid, THREADS, 0, L.stream>>>(a); break;
    }
}

void launch_density_pass(const StepLaunch &L, const LoadFlagsHost &lfh) {
    if (L.n == 0) return;
    DensityKernelArgs a;
    fill_common(a, L, lfh);
    // The density pass scatters two stress components per cell: there the warp-aggregated
    // reductions cost fewer L2 atomics than they add shuffles (dam break 1M: 47.7 -> 42.7 us
    // per launch), unlike the particle pass's mass + momentum scatter (74.5 -> 76.1 us).
    a.aggregate = L.use_window == 2 && !L.cfg.mf_fast ? 3 : (L.cfg.mf_excl ? 2 : 1);
    launch_density_pass_fast(a, L.model_mask, L.stream);
}

void launch_grid_update(const StepLaunch &L) {
    GridKernelArgs a;
    a.g = L.g;
    a.cfg = L.cfg;
    a.st = L.st;
    a.n_tiles = L.g.tpd * L.g.tpd;
    k_grid_update<<<blocks_for(a.n_tiles, 4), 256, 0, L.stream>>>(a);
}

void launch_step_begin(const StepLaunch &L) { k_step_begin<<<1, 1, 0, L.stream>>>(L.st, L.cfg); }

void launch_grid_update_batch(const BatchView &b, int n_tiles, cudaStream_t stream) {
    if (n_tiles > 0) k_grid_update_batch<<<blocks_for(n_tiles, 4), 256, 0, stream>>>(b, n_tiles);
}
void launch_step_begin_batch(const BatchView &b, StepState *batch_st, cudaStream_t stream) {
    k_step_begin_batch<<<1, 1024, 0, stream>>>(b, batch_st);
}
void launch_substep_begin_batch(const BatchView &b, StepState *batch_st, int use_cond,
                                unsigned long long handle, int kernels_per_substep, cudaStream_t stream) {
    k_substep_begin_batch<<<1, 1024, 0, stream>>>(b, batch_st, use_cond,
                                                 static_cast<cudaGraphConditionalHandle>(handle),
                                                 kernels_per_substep);
}
void launch_prime_setup_batch(const BatchView &b, cudaStream_t stream) {
    k_prime_setup_batch<<<1, 1024, 0, stream>>>(b);
}

void launch_substep_begin(const StepLaunch &L, int use_cond, unsigned long long handle,
                          int kernels_per_substep) {
    k_substep_begin<<<1, 1, 0, L.stream>>>(L.st, L.cfg, use_cond,
                                           static_cast<cudaGraphConditionalHandle>(handle),
                                           kernels_per_substep);
}

void launch_prime_setup(const StepLaunch &L) { k_prime_setup<<<1, 1, 0, L.stream>>>(L.st); }

void launch_region_state(const DevParticles &P, int n, float cx, float cy, float r2, void *acc,
                         cudaStream_t stream, int zones) {
    int blocks = blocks_for(n, 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    k_region_state<<<blocks, 256, 0, stream>>>(P, n, cx, cy, r2, static_cast<RegionAcc *>(acc), zones);
}

size_t region_acc_bytes() { return sizeof(RegionAcc); }

void region_acc_finalize(const void *acc, emerge_body_state *out) {
    const RegionAcc &a = *static_cast<const RegionAcc *>(acc);
    out->count = a.count;
    float sx = static_cast<float>(a.sx), sy = static_cast<float>(a.sy);
    float sp = static_cast<float>(a.speed), sjp = static_cast<float>(a.jp);
    float sdet = static_cast<float>(a.det), srho = static_cast<float>(a.rho);
    unsigned int o = a.max_jp_bits;
    unsigned int u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    float mjp;
    std::memcpy(&mjp, &u, sizeof(float));
    if (a.count > 0) {
        float n = static_cast<float>(a.count);
        sx /= n; sy /= n; sp /= n; sjp /= n; sdet /= n; srho /= n;
    }
    out->avg_volume_ratio = sjp;
    out->max_volume_ratio = mjp;
    out->avg_speed = sp;
    out->avg_det_f = sdet;
    out->avg_density = srho;
    out->centroid[0] = sx;
    out->centroid[1] = sy;
    out->pad_ = 0;
}

// One word from device memory into pinned host memory through its device address: a store
// from the SM, not a copy, so it does not queue behind device-to-host copies in flight.
__global__ void k_copy_word_to_host(const uint32_t *src, uint32_t *dst_mapped) { *dst_mapped = *src; }

void launch_copy_word_to_host(const uint32_t *src, uint32_t *dst_mapped, cudaStream_t stream) {
    k_copy_word_to_host<<<1, 1, 0, stream>>>(src, dst_mapped);
}

void launch_gather_aos(const DevParticles &P, int n, emerge_particle *out, cudaStream_t stream) {
    if (n) k_gather_aos<<<blocks_for(n, 256), 256, 0, stream>>>(P, n, out);
}
void launch_scatter_aos(const DevParticles &P, int n, const emerge_particle *in, cudaStream_t stream) {
    if (n) k_scatter_aos<<<blocks_for(n, 256), 256, 0, stream>>>(P, n, in);
}
void launch_check_aos(const emerge_particle *in, int n, uint32_t *flags, cudaStream_t stream) {
    if (n) k_check_aos<<<blocks_for(n, 256), 256, 0, stream>>>(in, n, flags);
}
void launch_append_aos(const DevParticles &P, int n_old, int n_new, const emerge_particle *in,
                       cudaStream_t stream) {
    if (n_new > n_old)
        k_append_aos<<<blocks_for(n_new - n_old, 256), 256, 0, stream>>>(P, n_old, n_new, in);
}
void launch_reinit(const DevParticles &P, int n, const MatP *mats, int n_mats, cudaStream_t stream) {
    if (n) k_reinit<<<blocks_for(n, 256), 256, 0, stream>>>(P, n, mats, n_mats);
}
void launch_mass_scatter(const DevParticles &P, int n, const GridView &g, int filter, float lox,
                         float loy, float hix, float hiy, cudaStream_t stream, int zones) {
    if (n) k_mass_scatter<<<blocks_for(n, 256), 256, 0, stream>>>(P, n, g, filter, lox, loy, hix, hiy, zones);
}
void launch_mass_gather(const DevParticles &P, int lo, int hi, const GridView &g, int write_initial,
                        cudaStream_t stream, int zones) {
    if (hi > lo) k_mass_gather<<<blocks_for(hi - lo, 256), 256, 0, stream>>>(P, lo, hi, g, write_initial, zones);
}

}  // namespace emerge
