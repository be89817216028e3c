// device_state.cuh -- device-side layout of one simulation.
//
// Particles live in HBM as structure-of-arrays in "slot" order: slots are a
// permutation of the reference's particle indices chosen by the tile sort, so
// that a CTA's chunk of consecutive slots covers a compact patch of grid.
// slot_to_index maps a slot back to the reference index for readback/upload.
//
// The grid is dense, G x G cells, stored in 8x8-cell tiles (64 consecutive
// cells per tile, tiles x-major) so that one particle's 3x3 stencil touches
// one to four tiles.  Three per-cell arrays:
//   acc_a  float4 {mass, Ax, Ay, 0}   A = sum w*m*(v + C*d)    (P2G, dt-free part)
//   acc_s  float2 {Sx, Sy}            S = sum w*(-4*V)*(tau*d) (P2G stress part)
//   grid_v float2 velocity after the grid update (read by G2P)
// The reference scatters w*(m*(v+C*d) + coeff*(tau*d)) with coeff = -4*V*dt
// (transfer/p2g.rs:202-213); the device keeps the dt-free stress sum separate
// so that the P2G of substep k+1 can run in the same pass as the G2P of
// substep k, before dt(k+1) is known; the grid update forms A + dt*S.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "closure.cuh"
#include "physics.cuh"

namespace emerge {

constexpr int TILE = 8;               // cells per tile side
constexpr int TILE_CELLS = TILE * TILE;
constexpr int MAX_MATERIALS = 64;     // MAX_MATERIAL_SLOTS (materials/registry.rs:6)
constexpr int MAX_BOUNDARIES = 8;

struct DevParticles {
    float2 *x, *v;
    float4 *c, *f;
    float *mass, *v0, *vol, *rho;
    uint32_t *mat;
    float *jp, *h, *q, *lvs;
    float *temperature, *activation;
    float2 *act_dir;
    uint32_t *pinned;
    // cold fields: only moved by sort/upload/readback
    uint32_t *user_tag, *muscle, *contact, *sleeping;
    float *scalar;
    uint32_t *slot_to_index;
    float *rho_dp;  // density-pass result of the pending substep (0 = not written)
};

// Device-resident substep controller.  CFL data for substep k lives in
// slot (k & 1); see k_substep_begin for the protocol.
struct StepState {
    float remaining;
    float sub_dt;
    uint32_t substeps;          // substeps taken in the current step
    uint32_t cont;              // 1 while the current step has another substep to run
    uint32_t parity;            // slot the next k_substep_begin reads
    uint32_t acc_slot;          // slot the running particle pass accumulates into
    uint32_t max_speed_bits[2]; // bits of a non-negative float (ordered as uint)
    uint32_t min_mdt_bits[2];   // bits of min over finite positive material dt (+inf init)
    unsigned long long vel_clamp;          // last_vel_clamp_count of the current step
    unsigned long long jproj;              // last_j_projection_count of the current step
    unsigned long long jproj_pending[2];   // projections counted for substep slot
    unsigned long long proj_changed[2];    // particles whose projection changed their state, per slot
    float last_step_dt;
    float dropped;
    unsigned long long total_substeps;     // lifetime
    unsigned long long total_steps;        // lifetime
    unsigned long long window_fallback;    // particle-pass blocks that used global reductions
    unsigned long long window_blocks;      // particle-pass blocks in total
    unsigned long long graph_kernels;      // kernels executed inside step graphs
    uint32_t error_flags;
    uint32_t upload_flags;      // k_check_aos: bit 0 contact_group != 0, bit 1 pinned
    uint32_t active;            // batches: the scene takes part in the running substep
    uint32_t contact_active;    // Grid::has_contact_activity of the running substep
    uint32_t n_iface;           // fast pipeline: contact cells holding both fields this substep
    uint32_t cl_queued[2][CL_NMODELS];  // learned closure: particles queued per slot and model
};

struct GridView {
    int res;        // G
    int tpd;        // tiles per dimension
    float4 *acc_a;
    float2 *acc_s;
    float2 *grid_v;
    uint8_t *tile_flag;
    float2 *grid_vpre;  // ASFLIP pre-force velocities (allocated when asflip_blend > 0)
    // multi-field contact and two-phase mixture (allocated when a scene uses them):
    // per-cell sums {m, px, py, touched} of the grip particles and of each mixture phase,
    // the resolved velocities G2P reads, the total mass kept past the grid update, each
    // cell's range in the cell-sorted scatter records, and the pressure solve's scratch
    float4 *acc_grip, *acc_sol, *acc_flu;
    float2 *grip_v, *rest_v, *sol_v, *flu_v;
    float *grid_m;
    int2 *rec_range;
    float *mx_as, *mx_af, *mx_k, *mx_rhs, *mx_p[2];
    uint8_t *mx_sig;
    // fast pipeline: the fields' P2G sums in the dt-free split ({m, Ax, Ay, w}, {Sx, Sy};
    // grip, solid, fluid), turned into acc_grip / acc_sol / acc_flu by the grid update; the
    // contact point cloud as per-base-cell lists (heads indexed x * res + y, one set per
    // substep parity) of nodes {x, y, label, next} indexed by particle slot; the contact
    // cells holding both fields (flat indices, StepState::n_iface of them)
    float4 *fa[3];
    float2 *fs[3];
    int *chead[2];
    float4 *cpts;
    int *iface;
};

// StepState::error_flags bits
constexpr uint32_t ERR_CONTACT_LIST = 1u;  // a contact point-list walk was cut short
constexpr uint32_t ERR_CLOSURE_WAIT = 2u;  // a closure tile's tensor-core wait gave up (kernel returned)
constexpr uint32_t ERR_NBODY_SKIPPED = 4u; // an n-body node seen as far had no center of mass

__host__ __device__ __forceinline__ int cell_index(int x, int y, int tpd) {
    return (((x >> 3) * tpd + (y >> 3)) << 6) | ((x & 7) << 3) | (y & 7);
}
__host__ __device__ __forceinline__ bool in_domain(int x, int y, int res) {
    return x >= 0 && y >= 0 && x < res && y < res;
}

// Threads (particles) per CTA of the particle and density passes.
constexpr int PARTICLE_THREADS = 256;

// One scene of a batch (device memory).  Its particles occupy slots [p0, p0 + n) of the
// batch's particle arrays (p0 a multiple of the particle-pass CTA size), its particle-pass
// CTAs are block0 .. block0 + ceil(n / CTA) - 1, its grid tiles tile0 .. tile0 + tpd^2 - 1.
struct SceneDesc {
    DevConfig cfg;
    GridView g;
    StepState *st;
    const emerge_material_params *mats;
    int n_mats;
    int p0;
    int n;
    int block0;
    int tile0;
    int density_mode;
};

// Scene lookup tables of a batch, passed to the batched kernels.
struct BatchView {
    const SceneDesc *scenes;
    const uint16_t *block_scene;  // particle-pass CTA -> scene
    const uint16_t *tile_scene;   // global grid tile -> scene
    int n_scenes;
    int check_active;             // skip scenes whose frame has ended
    int n_chunks;                 // 256-particle chunks (rows of block_scene)
};

// Host-side handles of the step kernels (implemented in step_kernels.cu).
struct StepLaunch {
    DevParticles P;
    int n;
    const MatP *mats;
    int n_mats;
    DevConfig cfg;
    StepState *st;
    GridView g;
    int density_mode;   // any registered material needs the density pass
    int use_window;     // warp-aggregated P2G reductions
    unsigned model_mask;  // bit m set: ConstitutiveModel m is registered
    int fast;           // fast path (stencil-offset sums with FMA); 0 in the reference-order mode
    ClosureArgs cl;     // learned closure switches and buffers (fast path only)
    cudaStream_t stream;
};

}  // namespace emerge
