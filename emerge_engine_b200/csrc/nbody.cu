// nbody.cu -- NBodyGravityField's Barnes-Hut quadtree (forces/fields/n_body.rs:63-283),
// rebuilt on the device once per substep, between the G2P half and the fields half of the
// particle pass (the reference's prepare() after G2P, step.rs:221-226).
//
// The reference inserts the particles of positive mass one at a time in index order into a
// pointer quadtree.  Its shape does not depend on that order: a node below max_depth is
// split exactly when more than max_bodies_per_node bodies fall into it.  What depends on the
// order is the arithmetic: each node folds its center of mass body by body in insertion
// order (MassProps::add, n_body.rs:96-107), and a leaf sums its bodies in the order it
// holds them.  The device builds the tree in data-parallel steps:
//   1. bounds   the bodies' bounding box (the root box, n_body.rs:228-247) and that of every
//               particle (where the field is evaluated), by warp reductions and atomics;
//   2. paths    each body's quadrant path from the root (2 bits per level, the boxes'
//               centers computed as the reference's insertion computes them), stored at
//               its reference index;
//   3. levels   for every level d, a stable radix sort of the path prefixes of length d
//               taken in reference index order: the level's body order, in which every
//               level-d node is one run with its bodies in insertion order; particles
//               without mass sort behind every body.  The run boundaries give each slot's
//               range;
//   4. centers  each node's total mass and center of mass, one warp per node, folded over
//               its run in its level's order with the reference's operations.  A node that
//               no particle can see as far (its width over the largest distance to any
//               particle is at least theta) is never asked for its center and is not
//               folded: typically the root and its four children, whose folds are longest.
// The fast pipeline needs neither the insertion order nor the serial folds: it sorts once by
// the full path (every node is then one run of that single order at every level), the
// deepest level's nodes sum Σm, Σm x and Σm y over their bodies (a warp each), and every
// node above adds its four children's sums (one launch per level of more than 256 nodes,
// one CTA for the rest), so no chain is longer than a node's four children.
// In the reference-order mode every box center and fold uses the reference's operations in
// the same order with IEEE rounding, so the tree -- and the field's accelerations -- match
// the reference bit for bit; the fast pipeline's tree has the same nodes, ranges and box
// centers, and centers of mass that differ from the reference's in the last bits only.
#include <algorithm>

#include "device_state.cuh"
#include "kernels.h"

namespace emerge {

namespace {

constexpr int NB_THREADS = 256;
constexpr float EMPTY_TREE_HALF_SIZE = 1000.0f;  // n_body.rs:38
constexpr float AABB_PADDING_RATIO = 0.1f;       // n_body.rs:42
constexpr float AABB_PADDING_MIN = 1.0f;         // n_body.rs:46

// Order-preserving map of a float to uint (for atomicMin / atomicMax) and back.
__device__ __forceinline__ uint32_t ord_bits(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_float(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ uint32_t warp_min_u(uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ uint32_t warp_max_u(uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void k_nb_reset(NBodyBounds *b) {
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2; ++k) {
            b->lo[k] = 0xffffffffu;
            b->hi[k] = 0u;
            b->all_lo[k] = 0xffffffffu;
            b->all_hi[k] = 0u;
        }
        b->n_bodies = 0u;
        b->walk_next = 0u;
    }
}

// Step 1.  A NaN coordinate is left out of its minimum and maximum, as f32::min / max do.
__global__ void k_nb_bounds(const float2 *x, const float *mass, int n, NBodyBounds *b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float2 p = make_float2(0.0f, 0.0f);
    float m = 0.0f;
    if (i < n) {
        p = x[i];
        m = mass[i];
    }
    const bool body = i < n && m > 0.0f;
    const uint32_t ox = ord_bits(p.x), oy = ord_bits(p.y);
    const bool fx = i < n && p.x == p.x, fy = i < n && p.y == p.y;
    const uint32_t lo_x = warp_min_u(fx && body ? ox : 0xffffffffu), hi_x = warp_max_u(fx && body ? ox : 0u);
    const uint32_t lo_y = warp_min_u(fy && body ? oy : 0xffffffffu), hi_y = warp_max_u(fy && body ? oy : 0u);
    const uint32_t alo_x = warp_min_u(fx ? ox : 0xffffffffu), ahi_x = warp_max_u(fx ? ox : 0u);
    const uint32_t alo_y = warp_min_u(fy ? oy : 0xffffffffu), ahi_y = warp_max_u(fy ? oy : 0u);
    const uint32_t nb = __popc(__ballot_sync(0xffffffffu, body));
    // the CTA's warps combine in shared memory and one thread per CTA issues the atomics
    // (every warp issuing them made the 9 words a point of contention)
    constexpr int W = NB_THREADS / 32;
    __shared__ uint32_t sv[9][W];
    const int w = static_cast<int>(threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0) {
        sv[0][w] = lo_x;
        sv[1][w] = hi_x;
        sv[2][w] = lo_y;
        sv[3][w] = hi_y;
        sv[4][w] = nb;
        sv[5][w] = alo_x;
        sv[6][w] = ahi_x;
        sv[7][w] = alo_y;
        sv[8][w] = ahi_y;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t v[9] = {sv[0][0], sv[1][0], sv[2][0], sv[3][0], sv[4][0], sv[5][0], sv[6][0], sv[7][0], sv[8][0]};
        for (int k = 1; k < W; ++k) {
            v[0] = min(v[0], sv[0][k]);
            v[1] = max(v[1], sv[1][k]);
            v[2] = min(v[2], sv[2][k]);
            v[3] = max(v[3], sv[3][k]);
            v[4] += sv[4][k];
            v[5] = min(v[5], sv[5][k]);
            v[6] = max(v[6], sv[6][k]);
            v[7] = min(v[7], sv[7][k]);
            v[8] = max(v[8], sv[8][k]);
        }
        if (v[4]) {
            atomicMin(&b->lo[0], v[0]);
            atomicMax(&b->hi[0], v[1]);
            atomicMin(&b->lo[1], v[2]);
            atomicMax(&b->hi[1], v[3]);
            atomicAdd(&b->n_bodies, v[4]);
        }
        atomicMin(&b->all_lo[0], v[5]);
        atomicMax(&b->all_hi[0], v[6]);
        atomicMin(&b->all_lo[1], v[7]);
        atomicMax(&b->all_hi[1], v[8]);
    }
}

// Quadtree::build's root box (n_body.rs:217-256): the bodies' box padded by 10 % of its
// width plus height and one cell, then squared about its center.
__device__ __forceinline__ float4 nb_root(const NBodyBounds &b) {
    if (b.n_bodies == 0u) return make_float4(0.0f, 0.0f, EMPTY_TREE_HALF_SIZE, 0.0f);
    float min_x = b.lo[0] == 0xffffffffu ? 3.40282347e38f : ord_float(b.lo[0]);
    float min_y = b.lo[1] == 0xffffffffu ? 3.40282347e38f : ord_float(b.lo[1]);
    float max_x = b.hi[0] == 0u ? -3.40282347e38f : ord_float(b.hi[0]);
    float max_y = b.hi[1] == 0u ? -3.40282347e38f : ord_float(b.hi[1]);
    const float pad = __fadd_rn(__fmul_rn(__fadd_rn(__fsub_rn(max_x, min_x), __fsub_rn(max_y, min_y)),
                                          AABB_PADDING_RATIO),
                                AABB_PADDING_MIN);
    min_x = __fsub_rn(min_x, pad);
    min_y = __fsub_rn(min_y, pad);
    max_x = __fadd_rn(max_x, pad);
    max_y = __fadd_rn(max_y, pad);
    const float cx = __fmul_rn(__fadd_rn(min_x, max_x), 0.5f);
    const float cy = __fmul_rn(__fadd_rn(min_y, max_y), 0.5f);
    const float half = __fmul_rn(fmaxf(__fsub_rn(max_x, min_x), __fsub_rn(max_y, min_y)), 0.5f);
    return make_float4(cx, cy, half, 0.0f);
}

// One level down (Aabb2::quadrant_of / quadrant_aabb, n_body.rs:74-91): quadrant bit 0 =
// right (x >= center.x), bit 1 = bottom (y < center.y); the child's center moves by a
// quarter of the parent's size.
__device__ __forceinline__ uint32_t nb_descend(float2 p, float2 &c, float &half) {
    const uint32_t q = (p.x >= c.x ? 1u : 0u) | (p.y < c.y ? 2u : 0u);
    half = __fmul_rn(half, 0.5f);
    c.x = (q & 1u) ? __fadd_rn(c.x, half) : __fsub_rn(c.x, half);
    c.y = (q & 2u) ? __fsub_rn(c.y, half) : __fadd_rn(c.y, half);
    return q;
}

// Step 2.  path[ref] = {quadrant path of D levels, or 1 << 2D without mass; particle slot}.
__global__ void k_nb_paths(const float2 *x, const float *mass, const uint32_t *slot_to_index, int n,
                           const NBodyBounds *b, int depth, float4 *root_out, float4 *bdata, uint2 *path) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float4 rt = nb_root(*b);
    if (i == 0) root_out[0] = rt;
    if (i >= n) return;
    const uint32_t ref = slot_to_index[i];
    const float2 p = x[i];
    const float m = mass[i];
    bdata[i] = make_float4(p.x, p.y, m, __uint_as_float(ref));
    if (ref >= static_cast<uint32_t>(n)) return;
    uint32_t key = 1u << (2 * depth);
    if (m > 0.0f) {
        float2 c = make_float2(rt.x, rt.y);
        float half = rt.z;
        key = 0u;
        for (int d = 0; d < depth; ++d) key = (key << 2) | nb_descend(p, c, half);
    }
    path[ref] = make_uint2(key, static_cast<uint32_t>(i));
}

// Step 3, before the sort of level d: keys in reference index order.
__global__ void k_nb_level_keys(const uint2 *path, int n, int depth, int d, uint32_t *keys, uint32_t *vals) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint2 pv = path[r];
    keys[r] = (pv.x >> (2 * depth)) != 0u ? (1u << (2 * d)) : (pv.x >> (2 * (depth - d)));
    vals[r] = pv.y;
}

// Step 3, after the sort: the level's order and its slots' runs (range zeroed before).
__global__ void k_nb_level_ranges(const uint32_t *keys, const uint32_t *vals, int n, const NBodyBounds *b, int d,
                                  uint32_t *order, uint2 *range) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = static_cast<int>(b->n_bodies);
    if (j >= nb || j >= n) return;
    const uint32_t key = keys[j], v = vals[j];
    const bool ok = (key >> (2 * d)) == 0u && v < static_cast<uint32_t>(n);  // a body's key
    order[j] = ok ? v : 0u;  // every entry of the level's body range names a valid slot
    if (!ok) return;
    const int s = nbody_level_offset(d) + static_cast<int>(key);
    if (j == 0 || keys[j - 1] != key) range[s].x = static_cast<uint32_t>(j);
    if (j + 1 == nb || keys[j + 1] != key) range[s].y = static_cast<uint32_t>(j + 1);
}

// Step 4.  One warp per node; com.w = 1 marks a folded node (an empty one included: it is
// never far).  The fold is serial in insertion order; the warp's lanes load the next 32
// bodies of the node's run together (and the 32 after them while these are folded), and
// every lane runs the same fold on the values broadcast from the lane that loaded them.
__global__ void k_nb_centers(const uint2 *range, const float4 *bdata, const uint32_t *order, size_t stride,
                             const float4 *root, const NBodyBounds *b, int depth, float theta_max, float4 *com) {
    const int s = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= nbody_slots(depth)) return;  // warp-uniform
    int d = 0;
    while (s >= nbody_level_offset(d + 1)) ++d;
    const uint32_t pre = static_cast<uint32_t>(s - nbody_level_offset(d));
    const uint2 rg = range[s];
    if (rg.y <= rg.x) {
        if (lane == 0) com[s] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        return;
    }
    // the node's box, as the traversal computes it
    const float4 rt = root[0];
    float2 c = make_float2(rt.x, rt.y);
    float half = rt.z;
    for (int l = 0; l < d; ++l) {
        const uint32_t q = (pre >> (2 * (d - 1 - l))) & 3u;
        half = __fmul_rn(half, 0.5f);
        c.x = (q & 1u) ? __fadd_rn(c.x, half) : __fsub_rn(c.x, half);
        c.y = (q & 2u) ? __fsub_rn(c.y, half) : __fadd_rn(c.y, half);
    }
    // far for some particle only if the farthest particle is beyond width / theta (with a
    // relative margin far above the rounding of the traversal's distance and quotient)
    if (b->all_lo[0] != 0xffffffffu && b->all_lo[1] != 0xffffffffu) {
        const double ax = ord_float(b->all_lo[0]), bx = ord_float(b->all_hi[0]);
        const double ay = ord_float(b->all_lo[1]), by = ord_float(b->all_hi[1]);
        const double dx = fmax(fabs(ax - c.x), fabs(bx - c.x)), dy = fmax(fabs(ay - c.y), fabs(by - c.y));
        const double dmax = sqrt(dx * dx + dy * dy);
        if (dmax * static_cast<double>(theta_max) <= 2.0 * static_cast<double>(half) * (1.0 - 1e-4)) {
            if (lane == 0) com[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            return;
        }
    }
    const uint32_t *ord = order + static_cast<size_t>(d) * stride;
    float tm = 0.0f, cx = 0.0f, cy = 0.0f;
    float4 next = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (rg.x + lane < rg.y) next = bdata[ord[rg.x + lane]];
    for (uint32_t j0 = rg.x; j0 < rg.y; j0 += 32u) {
        const float4 q = next;
        if (j0 + 32u + lane < rg.y) next = bdata[ord[j0 + 32u + lane]];
        const int cnt = static_cast<int>(min(32u, rg.y - j0));
        for (int k = 0; k < cnt; ++k) {
            const float qx = __shfl_sync(0xffffffffu, q.x, k), qy = __shfl_sync(0xffffffffu, q.y, k);
            const float qm = __shfl_sync(0xffffffffu, q.z, k);
            const float nt = __fadd_rn(tm, qm);
            if (nt > 0.0f) {
                cx = __fdiv_rn(__fadd_rn(__fmul_rn(cx, tm), __fmul_rn(qx, qm)), nt);
                cy = __fdiv_rn(__fadd_rn(__fmul_rn(cy, tm), __fmul_rn(qy, qm)), nt);
                tm = nt;
            }
        }
    }
    if (lane == 0) com[s] = make_float4(cx, cy, tm, 1.0f);
}

// Fast pipeline, step 3: the ranges of every level from one sort by the full path (a
// level-d node's bodies are one run of that order at every level, in path order rather than
// insertion order).  `order` is shared by all levels.
__global__ void k_nb_ranges_all(const uint32_t *keys, const uint32_t *vals, int n, const NBodyBounds *b, int depth,
                                uint32_t *order, uint2 *range) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = static_cast<int>(b->n_bodies);
    if (j >= nb || j >= n) return;
    const uint32_t key = keys[j], v = vals[j];
    const bool ok = (key >> (2 * depth)) == 0u && v < static_cast<uint32_t>(n);  // a body's key
    order[j] = ok ? v : 0u;
    if (!ok) return;
    const uint32_t kp = j > 0 ? keys[j - 1] : 0xffffffffu, kn = j + 1 < nb ? keys[j + 1] : 0xffffffffu;
    for (int d = 0; d <= depth; ++d) {
        const int sh = 2 * (depth - d);
        const uint32_t kd = key >> sh;
        const int s = nbody_level_offset(d) + static_cast<int>(kd);
        if (j == 0 || (kp >> sh) != kd) range[s].x = static_cast<uint32_t>(j);
        if (j + 1 == nb || (kn >> sh) != kd) range[s].y = static_cast<uint32_t>(j + 1);
    }
}

// Fast pipeline, step 4, bottom up.  The deepest level's nodes (one warp each) sum their
// bodies' m, m x and m y into com as raw sums {Σm x, Σm y, Σm, 1}.
__global__ void k_nb_sums_leaf(const uint2 *range, const float4 *bdata, const uint32_t *order, int depth,
                               float4 *com) {
    const long long wid = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int count = 1 << (2 * depth);
    if (wid >= count) return;  // warp-uniform
    const int s = nbody_level_offset(depth) + static_cast<int>(wid);
    const uint2 rg = range[s];
    float sm = 0.0f, sx = 0.0f, sy = 0.0f;
    for (uint32_t j = rg.x + lane; j < rg.y; j += 32u) {
        const float4 q = bdata[order[j]];
        sm += q.z;
        sx = __fmaf_rn(q.z, q.x, sx);
        sy = __fmaf_rn(q.z, q.y, sy);
    }
    if (rg.y - rg.x > 1u)
        for (int o = 16; o > 0; o >>= 1) {
            sm += __shfl_xor_sync(0xffffffffu, sm, o);
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
    if (lane == 0) com[s] = make_float4(sx, sy, sm, 1.0f);
}

__device__ __forceinline__ float4 nb_finish(float4 r) {
    return r.z > 0.0f ? make_float4(__fdiv_rn(r.x, r.z), __fdiv_rn(r.y, r.z), r.z, 1.0f)
                      : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
}

// Levels d_from down to d_to: each node sums its four children's raw sums and turns the
// children's into their centers of mass (it is their only reader).  A launch covering more
// than one level is a single CTA (the barrier orders the levels); finish_root finishes slot 0.
__global__ void k_nb_sums_up(float4 *com, int d_from, int d_to, int finish_root) {
    for (int d = d_from; d >= d_to; --d) {
        const int count = 1 << (2 * d), base = nbody_level_offset(d), cbase = nbody_level_offset(d + 1);
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
            float4 t = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int cs = cbase + 4 * p + q;
                const float4 c = com[cs];
                t.x += c.x;
                t.y += c.y;
                t.z += c.z;
                com[cs] = nb_finish(c);
            }
            com[base + p] = t;
        }
        __syncthreads();
    }
    if (finish_root && blockIdx.x == 0 && threadIdx.x == 0) com[0] = nb_finish(com[0]);
}

// The tree walk of every particle (nbody_acceleration) at its stored position, one warp per
// 32 consecutive particles (tile-sort neighbours, which share most of their walk), the warps
// taking the next 32 from a counter as they finish: walks differ in length by orders of
// magnitude between a clump's core and its outskirts, and a fixed grid would wait for its
// slowest CTAs.
__global__ void __launch_bounds__(NB_THREADS) k_nb_walk(NBodyView nb, const emerge_force_field *fields,
                                                        int n_fields, const float2 *x,
                                                        const uint32_t *slot_to_index, const uint32_t *sleeping,
                                                        int zones, int n, NBodyBounds *b, float2 *accel) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        uint32_t base = 0u;
        if (lane == 0) base = atomicAdd(&b->walk_next, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= static_cast<uint32_t>(n)) return;  // warp-uniform
        const int i = static_cast<int>(base) + lane;
        bool want = i < n;
        if (want && zones) want = (sleeping[i] & ZB_OUT) == 0u;
        if (want) {
            const float2 pos = x[i];
            const uint32_t self = slot_to_index[i];
            int kn = 0;
            for (int k = 0; k < n_fields; ++k) {
                const emerge_force_field f = fields[k];
                if (f.kind != EMERGE_FIELD_NBODY_GRAVITY) continue;
                accel[static_cast<size_t>(kn) * nb.accel_stride + i] = nbody_acceleration(nb, f, pos, self);
                ++kn;
            }
        }
    }
}

}  // namespace

// Resident walk CTAs per SM the grid is sized for (0: as many as fit).
#ifndef EMERGE_NB_WALK_CTAS_PER_SM
#define EMERGE_NB_WALK_CTAS_PER_SM 0
#endif

int nbody_walk_ctas() {
    int sms = 148, per_sm = 1, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nb_walk, NB_THREADS, 0) != cudaSuccess) per_sm = 1;
    if (EMERGE_NB_WALK_CTAS_PER_SM > 0) per_sm = std::min(per_sm, EMERGE_NB_WALK_CTAS_PER_SM);
    return sms * std::max(per_sm, 1);
}

void launch_nbody_walk(const NBodyTreeHost &t, const DevConfig &cfg, const DevParticles &P, int n,
                       bool all_particles, cudaStream_t stream) {
    if (n <= 0) return;
    const int warps = (n + 31) / 32;
    const int grid = std::max(1, std::min((warps + NB_THREADS / 32 - 1) / (NB_THREADS / 32), std::max(t.walk_ctas, 1)));
    k_nb_walk<<<grid, NB_THREADS, 0, stream>>>(cfg.nbody, cfg.fields, cfg.n_fields, P.x, P.slot_to_index,
                                               P.sleeping, all_particles ? 0 : cfg.zones, n, t.bounds, t.accel);
}

void launch_nbody_build(const NBodyTreeHost &t, const DevParticles &P, int n, SortScratch &sort, bool exact,
                        cudaStream_t stream) {
    const int slots = nbody_slots(t.depth);
    const int gb = n > 0 ? (n + NB_THREADS - 1) / NB_THREADS : 1;
    k_nb_reset<<<1, 32, 0, stream>>>(t.bounds);
    k_nb_bounds<<<gb, NB_THREADS, 0, stream>>>(P.x, P.mass, n, t.bounds);
    k_nb_paths<<<gb, NB_THREADS, 0, stream>>>(P.x, P.mass, P.slot_to_index, n, t.bounds, t.depth, t.root, t.bdata,
                                              t.path);
    cudaMemsetAsync(t.range, 0, static_cast<size_t>(slots) * sizeof(uint2), stream);
    if (!exact) {
        // one sort by the full path; every node's center of mass from its children's sums
        k_nb_level_keys<<<gb, NB_THREADS, 0, stream>>>(t.path, n, t.depth, t.depth, sort.keys[0], sort.vals[0]);
        const int r = radix_sort_pairs(sort, n, 2 * t.depth + 1, stream);
        k_nb_ranges_all<<<gb, NB_THREADS, 0, stream>>>(sort.keys[r], sort.vals[r], n, t.bounds, t.depth, t.order,
                                                       t.range);
        const long long lthreads = (1ll << (2 * t.depth)) * 32;  // one warp per deepest node
        k_nb_sums_leaf<<<static_cast<int>((lthreads + NB_THREADS - 1) / NB_THREADS), NB_THREADS, 0, stream>>>(
            t.range, t.bdata, t.order, t.depth, t.com);
        int d = t.depth - 1;
        for (; d >= 0 && (1 << (2 * d)) > NB_THREADS; --d)  // one launch per wide level
            k_nb_sums_up<<<((1 << (2 * d)) + NB_THREADS - 1) / NB_THREADS, NB_THREADS, 0, stream>>>(t.com, d, d, 0);
        k_nb_sums_up<<<1, NB_THREADS, 0, stream>>>(t.com, d, 0, 1);  // the narrow levels and the root
        return;
    }
    for (int d = 0; d <= t.depth; ++d) {
        k_nb_level_keys<<<gb, NB_THREADS, 0, stream>>>(t.path, n, t.depth, d, sort.keys[0], sort.vals[0]);
        const int r = radix_sort_pairs(sort, n, 2 * d + 1, stream);
        k_nb_level_ranges<<<gb, NB_THREADS, 0, stream>>>(sort.keys[r], sort.vals[r], n, t.bounds, d,
                                                         t.order + static_cast<size_t>(d) * t.stride, t.range);
    }
    const long long threads = static_cast<long long>(slots) * 32;  // one warp per node
    k_nb_centers<<<static_cast<int>((threads + NB_THREADS - 1) / NB_THREADS), NB_THREADS, 0, stream>>>(
        t.range, t.bdata, t.order, t.stride, t.root, t.bounds, t.depth, t.theta_max, t.com);
}

}  // namespace emerge
