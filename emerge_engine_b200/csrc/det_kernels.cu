// det_kernels.cu -- reference-order (deterministic) substep pieces.
//
// The reference sums P2G contributions into each grid cell sequentially, in
// particle index order (transfer/p2g.rs:16-23, 192-231), and keeps that order on
// purpose.  The fast path reduces with float atomics, whose order varies from run
// to run.  This mode reproduces the reference order on the device:
//   1. every (particle, stencil cell) pair becomes a record keyed by the cell's
//      flat index x*res+y (grid/mod.rs:89-99), numbered particle-major in the
//      reference's index order,
//   2. a stable radix sort groups the records by cell, keeping index order inside
//      a cell,
//   3. one thread per cell adds its records sequentially, exactly like
//      Grid::accumulate (grid/mod.rs:200-212).
// The rest of the substep runs unfused with dt known up front, as the reference
// does: projection in place (step.rs:67-73), density pass (density.rs:41-72),
// P2G with coeff = -V*4*dt, grid update, G2P + constitutive update.
#include "device_state.cuh"
#include "kernels.h"

namespace emerge {

__device__ __forceinline__ void count_warp_det(unsigned long long *ctr, bool pred) {
    unsigned ballot = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(ctr, (unsigned long long)__popc(ballot));
}

// project_particle_state_to_admissible in place (step.rs:67-73); counts corrections.
__global__ void k_project(DevParticles P, int n, DevConfig cfg, StepState *st) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool projected = false;
    if (i < n && !(cfg.zones && (P.sleeping[i] & ZB_OUT))) {
        PState p;
        p.x = P.x[i];
        p.v = P.v[i];
        p.c = m_from4(P.c[i]);
        p.f = m_from4(P.f[i]);
        p.mass = P.mass[i];
        p.v0 = P.v0[i];
        p.vol = P.vol[i];
        p.rho = P.rho[i];
        p.jp = P.jp[i];
        p.h = P.h[i];
        p.q = P.q[i];
        p.lvs = P.lvs[i];
        projected = project_state(cfg, p);
        P.x[i] = p.x;
        P.v[i] = p.v;
        P.c[i] = m_to4(p.c);
        P.f[i] = m_to4(p.f);
        P.mass[i] = p.mass;
        P.v0[i] = p.v0;
        P.vol[i] = p.vol;
        P.rho[i] = p.rho;
        P.jp[i] = p.jp;
        P.h[i] = p.h;
        P.q[i] = p.q;
        P.lvs[i] = p.lvs;
    }
    count_warp_det(&st->jproj, projected);
}

// Records of one substep's scatter.  mode 0: mass only (scatter_particle_mass,
// p2g.rs:230-243); mode 1: full P2G with dt (p2g.rs:192-213).
__global__ void k_det_records(DevParticles P, int n, const MatP *mats, int n_mats, DevConfig cfg,
                              const StepState *st, int mode, uint32_t invalid_key, uint32_t *keys,
                              uint32_t *vals, float4 *payload, int filter, float lox, float loy,
                              float hix, float hiy, int write_keys, uint8_t *fmask, float4 *points) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t hi = P.slot_to_index[s];
    PState p;
    p.x = P.x[s];
    p.mass = P.mass[s];
    // estimate_particle_volumes_local's AABB filter (density.rs:106-110); particles outside
    // the active zone take no part
    bool skip = (filter && (p.x.x < lox || p.x.y < loy || p.x.x > hix || p.x.y > hiy)) ||
                (cfg.zones && (P.sleeping[s] & ZB_OUT));
    // the fields the particle's contributions also go to (p2g.rs:60-66): bit 0 grip
    // (contact_group != 0), bit 1 / 2 the solid / fluid mixture phase
    const uint32_t cgroup = (fmask || points) ? P.contact[s] : 0u;
    uint8_t fbits = 0;
    if (fmask) {
        const uint32_t mat = P.mat[s];
        const uint32_t ph = cfg.mat_phase[mat < static_cast<uint32_t>(n_mats) ? mat : 0u];
        fbits = static_cast<uint8_t>((cgroup != 0u ? 1u : 0u) | (ph == 1u ? 2u : 0u) | (ph == 2u ? 4u : 0u));
    }
    float2 v = v2(0.0f, 0.0f);
    M2 c = mzero(), stress = mzero();
    float stress_coeff = 0.0f;
    if (mode == 1) {
        p.v = P.v[s];
        p.c = m_from4(P.c[s]);
        p.f = m_from4(P.f[s]);
        p.v0 = P.v0[s];
        p.vol = P.vol[s];
        p.rho = P.rho[s];
        p.mat = P.mat[s];
        p.jp = P.jp[s];
        p.h = P.h[s];
        p.q = P.q[s];
        p.lvs = P.lvs[s];
        p.temperature = P.temperature[s];
        p.activation = P.activation[s];
        p.act_dir = P.act_dir[s];
        p.pinned = 0;
        const MatP &m = mats[p.mat < static_cast<uint32_t>(n_mats) ? p.mat : 0u];
        v = p.v;
        c = p.c;
        stress = combined_kirchhoff_stress(m, p, cfg.precise_math != 0);
        stress_coeff = -stress_volume(m, p) * KERNEL_D_INVERSE * st->sub_dt;
    }
    QW w = quadratic_weights(p.x);
    for (int gx = 0; gx < 3; ++gx)
        for (int gy = 0; gy < 3; ++gy) {
            const uint32_t r = hi * 9u + static_cast<uint32_t>(gx * 3 + gy);
            float weight = w.wx[gx] * w.wy[gy];
            int cx = w.bx + gx - 1, cy = w.by + gy - 1;
            // write_keys = 0: the keys of an earlier call at the same positions are already sorted
            if (write_keys) vals[r] = r;
            if (skip || !in_domain(cx, cy, cfg.res)) {
                if (write_keys) keys[r] = invalid_key;
                payload[r] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                continue;
            }
            if (write_keys)
                keys[r] = static_cast<uint32_t>(cx) * static_cast<uint32_t>(cfg.res) + static_cast<uint32_t>(cy);
            if (fmask) fmask[r] = fbits;
            float2 mom = v2(0.0f, 0.0f);
            if (mode == 1) {
                float2 cell_dist = vadd(vsub(v2(static_cast<float>(cx), static_cast<float>(cy)), p.x),
                                        splat(0.5f));
                mom = svmul(weight, vadd(svmul(p.mass, vadd(v, mv(c, cell_dist))),
                                         svmul(stress_coeff, mv(stress, cell_dist))));
            }
            payload[r] = make_float4(weight * p.mass, mom.x, mom.y, 0.0f);
            // the contact point cloud (p2g.rs:54-74): position and label of every record
            if (points) points[r] = make_float4(p.x.x, p.x.y, cgroup != 0u ? 1.0f : -1.0f, 0.0f);
        }
}

// Sequential per-cell sums over the cell-sorted records (Grid::accumulate order).
__global__ void k_segsum(const uint32_t *keys, const uint32_t *vals, const float4 *payload, int n_rec,
                         uint32_t invalid_key, GridView g, int mass_only, int2 *range) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_rec) return;
    uint32_t key = keys[j];
    if (key == invalid_key) return;
    if (j > 0 && keys[j - 1] == key) return;  // not the head of its cell
    float4 first = payload[vals[j]];
    float m = first.x, px = first.y, py = first.z;
    int k = j + 1;
    for (; k < n_rec && keys[k] == key; ++k) {
        float4 q = payload[vals[k]];
        m += q.x;
        px += q.y;
        py += q.z;
    }
    int cx = static_cast<int>(key / static_cast<uint32_t>(g.res));
    int cy = static_cast<int>(key % static_cast<uint32_t>(g.res));
    int ci = cell_index(cx, cy, g.tpd);
    if (range) range[ci] = make_int2(j, k);  // the cell's records, in particle index order
    if (mass_only) {
        g.acc_a[ci].x = m;
    } else {
        g.acc_a[ci] = make_float4(m, px, py, 1.0f);  // w > 0: the cell is in the dirty set
    }
    int t = (cx >> 3) * g.tpd + (cy >> 3);
    g.tile_flag[t] = 1;
}

// One field's sums over the same sorted records (add_grip_mass_momentum contact.rs:41-72,
// add_mixture_mass_momentum mixture.rs:20-58): per cell, the records of the field's particles
// (fmask & fbit) in particle index order, the first set and the rest added, as the reference
// does in its own scatter loop.
__global__ void k_segsum_field(const uint32_t *keys, const uint32_t *vals, const float4 *payload,
                               const uint8_t *fmask, uint32_t fbit, int n_rec, uint32_t invalid_key,
                               GridView g, float4 *target, uint32_t *any) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_rec) return;
    uint32_t key = keys[j];
    if (key == invalid_key) return;
    if (j > 0 && keys[j - 1] == key) return;  // not the head of its cell
    bool found = false;
    float m = 0.0f, px = 0.0f, py = 0.0f;
    for (int k = j; k < n_rec && keys[k] == key; ++k) {
        const uint32_t r = vals[k];
        if (!(fmask[r] & fbit)) continue;
        const float4 q = payload[r];
        if (!found) {
            m = q.x;
            px = q.y;
            py = q.z;
            found = true;
        } else {
            m += q.x;
            px += q.y;
            py += q.z;
        }
    }
    if (!found) return;
    const int cx = static_cast<int>(key / static_cast<uint32_t>(g.res));
    const int cy = static_cast<int>(key % static_cast<uint32_t>(g.res));
    target[cell_index(cx, cy, g.tpd)] = make_float4(m, px, py, 1.0f);
    if (any) *any = 1u;
}

void launch_project(const StepLaunch &L) {
    if (L.n) k_project<<<(L.n + 255) / 256, 256, 0, L.stream>>>(L.P, L.n, L.cfg, L.st);
}

void launch_det_records(const StepLaunch &L, int mode, uint32_t invalid_key, uint32_t *keys,
                        uint32_t *vals, float4 *payload, int filter, float lox, float loy, float hix,
                        float hiy, int write_keys, uint8_t *fmask, float4 *points) {
    if (L.n)
        k_det_records<<<(L.n + 127) / 128, 128, 0, L.stream>>>(L.P, L.n, L.mats, L.n_mats, L.cfg, L.st,
                                                               mode, invalid_key, keys, vals, payload,
                                                               filter, lox, loy, hix, hiy, write_keys,
                                                               fmask, points);
}

void launch_segsum_field(const uint32_t *keys, const uint32_t *vals, const float4 *payload,
                         const uint8_t *fmask, uint32_t fbit, int n_rec, uint32_t invalid_key,
                         const GridView &g, float4 *target, uint32_t *any, cudaStream_t stream) {
    if (n_rec)
        k_segsum_field<<<(n_rec + 255) / 256, 256, 0, stream>>>(keys, vals, payload, fmask, fbit, n_rec,
                                                                invalid_key, g, target, any);
}

void launch_segsum(const uint32_t *keys, const uint32_t *vals, const float4 *payload, int n_rec,
                   uint32_t invalid_key, const GridView &g, int mass_only, cudaStream_t stream,
                   int2 *range) {
    if (n_rec)
        k_segsum<<<(n_rec + 255) / 256, 256, 0, stream>>>(keys, vals, payload, n_rec, invalid_key, g,
                                                          mass_only, range);
}

}  // namespace emerge
