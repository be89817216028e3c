// kernels.h -- host-side launchers of the device kernels (step_kernels.cu, sort.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "device_state.cuh"

namespace emerge {

struct LoadFlagsHost {
    int temperature = 0;
    int activation = 0;
    int pinned = 0;
};

// closure_tiles.cu: the learned closure's tile kernel (after the particle pass, when the
// pass queued particles for it: deferred closure, fast path, plastic models, no extras)
void launch_closure_tiles(const StepLaunch &L, const LoadFlagsHost &lf, int sm_count);
// test hook: the tile kernel's network on n normalised inputs (closure.cu, emerge_cuda_mlp_infer_tc)
cudaError_t launch_mlp_tiles(const ClosureNet *net, const float *x, int n, float *y, uint32_t *error,
                             cudaStream_t stream);
// The tile kernel's SiLU on n values (device pointers; test hook).
cudaError_t launch_silu_fast(const float *x, int n, float *y, cudaStream_t stream);
inline bool closure_tiles_on(const StepLaunch &L) {
    const unsigned plastic = (1u << M_DRUCKER_PRAGER) | (1u << M_NACC);
    return L.fast && L.cl.defer && (L.model_mask & plastic) && !(L.model_mask & (1u << M_EXTRAS_BIT));
}

// step_kernels.cu
// nbody.cu: NBodyGravityField's quadtree (NBodyView), rebuilt each substep.
struct SortScratch;
struct NBodyBounds {
    uint32_t lo[2], hi[2];          // order-preserving bits of the bodies' min / max x, y
    uint32_t all_lo[2], all_hi[2];  // ... of every particle's position
    uint32_t n_bodies;              // particles of positive mass
    uint32_t walk_next;             // k_nb_walk's next particle
};
struct NBodyTreeHost {
    int depth = -1;          // max_depth; -1: no NBodyGravityField
    int max_bodies = 0;      // max_bodies_per_node
    float theta_max = 0.0f;  // largest theta over the NBody fields (which nodes may be far)
    float4 *root = nullptr;
    float4 *bdata = nullptr;     // per particle slot (cap)
    uint2 *path = nullptr;       // per reference index: full quadrant path (or none), slot (cap)
    uint32_t *order = nullptr;   // (depth + 1) levels of `stride` entries
    size_t stride = 0;
    uint2 *range = nullptr;
    float4 *com = nullptr;
    NBodyBounds *bounds = nullptr;
    int n_fields = 0;            // NBody fields (one walk and one accel block each)
    float2 *accel = nullptr;     // n_fields blocks of `stride` float2 (per particle slot)
    int walk_ctas = 0;           // resident CTAs of k_nb_walk on the device (its grid)
};
// Builds the tree over the n particles of P on `stream` (the level sorts use `sort`, which
// must hold n entries); exact: centers of mass folded in insertion order (reference order).
void launch_nbody_build(const NBodyTreeHost &t, const DevParticles &P, int n, SortScratch &sort, bool exact,
                        cudaStream_t stream);
// Every particle's acceleration from each NBody field of `cfg` (the tree built), into
// t.accel; particles outside the sleep partition's active zone are skipped unless
// all_particles.
void launch_nbody_walk(const NBodyTreeHost &t, const DevConfig &cfg, const DevParticles &P, int n,
                       bool all_particles, cudaStream_t stream);
// Resident CTAs of the walk kernel on the current device (queried outside graph capture).
int nbody_walk_ctas();
// The kernels launch_nbody_build launches for n particles.
inline int nbody_build_kernels(int depth, int n, bool exact) {
    if (!exact) {  // reset, bounds, paths, keys, one sort, ranges, leaf sums, the levels above
        const int wide = depth - 5 > 0 ? depth - 5 : 0;
        return 6 + (n > 1 ? 5 * ((2 * depth + 1 + 7) / 8) : 0) + 1 + wide + 1;
    }
    int k = 4;  // reset, bounds, paths, centers
    for (int d = 0; d <= depth; ++d) k += 2 + (n > 1 ? 5 * ((2 * d + 1 + 7) / 8) : 0);
    return k;
}

// split: 0 one pass; 1 / 2 its G2P and fields halves (ParticleKernelArgs::split)
void launch_particle_pass(const StepLaunch &L, const LoadFlagsHost &lf, int mode_g2p,
                          int project_in, int emit_p2g, int split = 0);
void launch_density_pass(const StepLaunch &L, const LoadFlagsHost &lf);
// Sum of the force fields' accelerations per particle, out[reference index] (n-body tree built).
void launch_field_accelerations(const StepLaunch &L, const LoadFlagsHost &lf, float2 *out);
void launch_grid_update(const StepLaunch &L);
void launch_step_begin(const StepLaunch &L);
void launch_substep_begin(const StepLaunch &L, int use_cond, unsigned long long handle,
                          int kernels_per_substep);
void launch_prime_setup(const StepLaunch &L);
void launch_region_state(const DevParticles &P, int n, float cx, float cy, float r2, void *acc,
                         cudaStream_t stream, int zones = 0);
size_t region_acc_bytes();
void region_acc_finalize(const void *acc, emerge_body_state *out);
void launch_gather_aos(const DevParticles &P, int n, emerge_particle *out, cudaStream_t stream);
// *dst_mapped = *src by a one-thread kernel (dst: pinned host memory's device address).
void launch_copy_word_to_host(const uint32_t *src, uint32_t *dst_mapped, cudaStream_t stream);
void launch_scatter_aos(const DevParticles &P, int n, const emerge_particle *in, cudaStream_t stream);
void launch_check_aos(const emerge_particle *in, int n, uint32_t *flags, cudaStream_t stream);
void launch_append_aos(const DevParticles &P, int n_old, int n_new, const emerge_particle *in,
                       cudaStream_t stream);
void launch_reinit(const DevParticles &P, int n, const MatP *mats, int n_mats, cudaStream_t stream);
void launch_mass_scatter(const DevParticles &P, int n, const GridView &g, int filter, float lox,
                         float loy, float hix, float hiy, cudaStream_t stream, int zones = 0);
void launch_mass_gather(const DevParticles &P, int lo, int hi, const GridView &g, int write_initial,
                        cudaStream_t stream, int zones = 0);
// sleep partition (step_kernels.cu): wake after P2G, zone bits from the reference index,
// index remaps after the host's replay of wake / sleep swaps and after add_body
void launch_wake(const StepLaunch &L, int substep_offset);
void launch_zone_bits(const DevParticles &P, int n, uint32_t active, cudaStream_t stream);
void launch_remap_index(const DevParticles &P, int n, const uint32_t *new_of_old, cudaStream_t stream);
void launch_insert_index(const DevParticles &P, int n_old, int n_new, uint32_t old_active, cudaStream_t stream);

// batched scenes (step_kernels.cu: grid update and controller; fast_kernels.cu: passes)
void launch_grid_update_batch(const BatchView &b, int n_tiles, cudaStream_t stream);
void launch_step_begin_batch(const BatchView &b, StepState *batch_st, cudaStream_t stream);
void launch_substep_begin_batch(const BatchView &b, StepState *batch_st, int use_cond,
                                unsigned long long handle, int kernels_per_substep, cudaStream_t stream);
void launch_prime_setup_batch(const BatchView &b, cudaStream_t stream);
// particle pass (mode_g2p, emit_p2g as launch_particle_pass) and density pass over all
// CTAs of a batch; lf: union of the scenes' load flags, model_mask: union of their models
// chunks: 256-particle chunks per CTA (1, 2 or 4)
void launch_particle_pass_batch(const DevParticles &P, const BatchView &b, int n_blocks,
                                const LoadFlagsHost &lf, unsigned model_mask, int mode_g2p,
                                int emit_p2g, int aggregate, int chunks, cudaStream_t stream);
void launch_density_pass_batch(const DevParticles &P, const BatchView &b, int n_blocks,
                               const LoadFlagsHost &lf, unsigned model_mask, int aggregate,
                               int chunks, cudaStream_t stream);

// det_kernels.cu (reference-order mode)
void launch_project(const StepLaunch &L);
// write_keys = 0 keeps the keys and values of an earlier call at the same positions (already
// sorted); fmask (optional): each record's fields (bit 0 grip, 1 solid, 2 fluid); points
// (optional): each record's (x, y, contact label) for the contact point cloud
void launch_det_records(const StepLaunch &L, int mode, uint32_t invalid_key, uint32_t *keys,
                        uint32_t *vals, float4 *payload, int filter = 0, float lox = 0.f,
                        float loy = 0.f, float hix = 0.f, float hiy = 0.f, int write_keys = 1,
                        uint8_t *fmask = nullptr, float4 *points = nullptr);
// one field's per-cell sums over the sorted records of its particles (fmask & fbit)
void launch_segsum_field(const uint32_t *keys, const uint32_t *vals, const float4 *payload,
                         const uint8_t *fmask, uint32_t fbit, int n_rec, uint32_t invalid_key,
                         const GridView &g, float4 *target, uint32_t *any, cudaStream_t stream);
// range (optional): each cell's record range
void launch_segsum(const uint32_t *keys, const uint32_t *vals, const float4 *payload, int n_rec,
                   uint32_t invalid_key, const GridView &g, int mass_only, cudaStream_t stream,
                   int2 *range = nullptr);
// multi-field contact and mixture coupling after the grid update (multifield.cu)
void launch_contact_resolve(const StepLaunch &L, const uint32_t *vals, const float4 *points);
void launch_mixture_resolve(const StepLaunch &L);
// fast pipeline: contact from the particle pass's base-cell lists (multifield_fast.cu), and
// the per-substep clear
void launch_contact_resolve_lists(const StepLaunch &L);
void launch_multi_clear(const StepLaunch &L);

// sort.cu
// Scratch for a stable LSD radix sort of up to `capacity` (key, value) pairs.
struct SortScratch {
    size_t capacity = 0;
    uint32_t *keys[2] = {nullptr, nullptr};
    uint32_t *vals[2] = {nullptr, nullptr};
    uint32_t *hist = nullptr;      // 256 * blocks
    uint32_t *partials = nullptr;  // scan partials
    size_t hist_capacity = 0;
};
size_t sort_scratch_bytes(size_t n);
// Carves the scratch arrays out of one device allocation of sort_scratch_bytes(n).
void sort_scratch_bind(SortScratch &s, void *base, size_t n);
// Keys of the particle positions: key_mode 0 = tile key, 1 = block_index key.
void launch_sort_keys(const float2 *x, int n, int res, int key_mode, uint32_t *keys, uint32_t *vals,
                      cudaStream_t stream);
int sort_key_bits(int res, int key_mode);
// Sorts (keys[0], vals[0]) stably by key; result lands in (keys[r], vals[r]), r returned.
int radix_sort_pairs(SortScratch &s, int n, int key_bits, cudaStream_t stream);
// Batched scenes: keys (scene << 20 | spatial key) of the compact particle list and the
// permutation back into each scene's slot range.  `shape`, the order the sort gives each
// scene's particles (what patch of grid a CTA's chunk covers): 0 8 x 8-cell tiles in Morton
// order, cells row by row inside; 1 the same tiles, cells in Morton order inside; 2 16 x 16
// blocks in Morton order, each as four 16 x 4 strips; 3 the same blocks as four 4 x 16 strips.
int batch_sort_key_bits(int n_scenes);
void launch_batch_sort_keys(const SceneDesc *scenes, const int *compact_start, int n_scenes,
                            const DevParticles &P, int total, uint32_t *keys, uint32_t *vals, int shape,
                            cudaStream_t stream);
void launch_permute_batch(const DevParticles &src, const DevParticles &dst, const uint32_t *keys,
                          const uint32_t *vals, const SceneDesc *scenes, const int *compact_start, int total,
                          cudaStream_t stream);
// dst[j] = src[perm[j]] for every particle array.
void launch_permute(const DevParticles &src, const DevParticles &dst, const uint32_t *perm, int n,
                    cudaStream_t stream);

}  // namespace emerge
