// particle_pass.cuh -- the per-particle passes of the fused substep.
//
// Included by two translation units: step_kernels.cu instantiates the particle pass
// with the reference's cell-by-cell expression order and IEEE arithmetic (compiled with
// -fmad=false: the reference-order mode), fast_kernels.cu instantiates the fast path
// (stencil-offset sums, compiled with contraction into FMA and approximate division and
// square root).  Both share every formula below; only the compilation differs.
#pragma once

#include <cfloat>
#include <climits>

#include "closure.cuh"
#include "device_state.cuh"
#include "kernels.h"

namespace emerge {

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ void red_add_v4(float4 *p, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c),
                 "f"(d)
                 : "memory");
}
__device__ __forceinline__ void red_add_v2(float2 *p, float a, float b) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}

__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_min(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_imin(int v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_imax(int v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ void count_warp(unsigned long long *ctr, bool pred) {
    unsigned ballot = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(ctr, (unsigned long long)__popc(ballot));
}

// ---------------------------------------------------------------- particle I/O
struct LoadFlags {
    int temperature;  // some material reads particle temperature
    int activation;   // some material has a non-zero activation scale
    int pinned;       // some particle is pinned
};

__device__ __forceinline__ PState load_state(const DevParticles &P, int i, const LoadFlags &lf) {
    PState p;
    p.x = P.x[i];
    p.v = P.v[i];
    p.c = m_from4(P.c[i]);
    p.f = m_from4(P.f[i]);
    p.mass = P.mass[i];
    p.v0 = P.v0[i];
    p.vol = P.vol[i];
    p.rho = P.rho[i];
    p.mat = P.mat[i];
    p.jp = P.jp[i];
    p.h = P.h[i];
    p.q = P.q[i];
    p.lvs = P.lvs[i];
    p.temperature = lf.temperature ? P.temperature[i] : 0.0f;
    p.activation = lf.activation ? P.activation[i] : 0.0f;
    p.act_dir = lf.activation ? P.act_dir[i] : v2(0.0f, 0.0f);
    p.pinned = lf.pinned ? P.pinned[i] : 0u;
    return p;
}

__device__ __forceinline__ bool neq(float a, float b) { return __float_as_uint(a) != __float_as_uint(b); }
__device__ __forceinline__ bool neq2(float2 a, float2 b) { return neq(a.x, b.x) || neq(a.y, b.y); }
__device__ __forceinline__ bool neqm(M2 a, M2 b) { return neq2(a.xa, b.xa) || neq2(a.ya, b.ya); }

// Writes back the fields that differ (bitwise) from what was loaded.
__device__ __forceinline__ void store_changed(const DevParticles &P, int i, const PState &o,
                                              const PState &p) {
    if (neq2(p.x, o.x)) P.x[i] = p.x;
    if (neq2(p.v, o.v)) P.v[i] = p.v;
    if (neqm(p.c, o.c)) P.c[i] = m_to4(p.c);
    if (neqm(p.f, o.f)) P.f[i] = m_to4(p.f);
    if (neq(p.mass, o.mass)) P.mass[i] = p.mass;
    if (neq(p.v0, o.v0)) P.v0[i] = p.v0;
    if (neq(p.vol, o.vol)) P.vol[i] = p.vol;
    if (neq(p.rho, o.rho)) P.rho[i] = p.rho;
    if (neq(p.jp, o.jp)) P.jp[i] = p.jp;
    if (neq(p.h, o.h)) P.h[i] = p.h;
    if (neq(p.q, o.q)) P.q[i] = p.q;
    if (neq(p.lvs, o.lvs)) P.lvs[i] = p.lvs;
}

// Fields the particle pass may leave unchanged (x, v and C always change in G2P):
// kept to skip stores of bitwise-equal values.
struct Saved {
    M2 f;
    float mass, v0, vol, rho, jp, h, q, lvs;
};
__device__ __forceinline__ Saved save_fields(const PState &p) {
    Saved o;
    o.f = p.f;
    o.mass = p.mass;
    o.v0 = p.v0;
    o.vol = p.vol;
    o.rho = p.rho;
    o.jp = p.jp;
    o.h = p.h;
    o.q = p.q;
    o.lvs = p.lvs;
    return o;
}
__device__ __forceinline__ void store_fields(const DevParticles &P, int i, const Saved &o,
                                             const PState &p) {
    P.x[i] = p.x;
    P.v[i] = p.v;
    P.c[i] = m_to4(p.c);
    if (neqm(p.f, o.f)) P.f[i] = m_to4(p.f);
    if (neq(p.mass, o.mass)) P.mass[i] = p.mass;
    if (neq(p.v0, o.v0)) P.v0[i] = p.v0;
    if (neq(p.vol, o.vol)) P.vol[i] = p.vol;
    if (neq(p.rho, o.rho)) P.rho[i] = p.rho;
    if (neq(p.jp, o.jp)) P.jp[i] = p.jp;
    if (neq(p.h, o.h)) P.h[i] = p.h;
    if (neq(p.q, o.q)) P.q[i] = p.q;
    if (neq(p.lvs, o.lvs)) P.lvs[i] = p.lvs;
}

// Tiled cell index split into an x part and a y part (cell_index = X(x) + Y(y)).
__device__ __forceinline__ int cell_x_part(int x, int tpd) { return (((x >> 3) * tpd) << 6) + ((x & 7) << 3); }
__device__ __forceinline__ int cell_y_part(int y) { return ((y >> 3) << 6) + (y & 7); }

// True when the whole 3 x 3 stencil around base cell (bx, by) lies in the domain
// (bx and by in [1, res - 2]); unsigned arithmetic keeps saturated bases false.
__device__ __forceinline__ bool stencil_inside(int bx, int by, int res) {
    return static_cast<unsigned>(bx) - 1u < static_cast<unsigned>(res - 2) &&
           static_cast<unsigned>(by) - 1u < static_cast<unsigned>(res - 2);
}

// Stencil-offset form used by the fast path.  With e = (bx - x) + 0.5, the offset of
// the centre cell, the offset of cell (bx + gx - 1, by + gy - 1) is
// d = e + (gx - 1, gy - 1), so sums over the 3 x 3 stencil factor into per-row sums.
__device__ __forceinline__ float2 centre_offset(const QW &w, float2 x) {
    return v2((static_cast<float>(w.bx) - x.x) + 0.5f, (static_cast<float>(w.by) - x.y) + 0.5f);
}

// Grid velocities (grid_v, or another float2 grid field) of the 3 x 3 stencil; cells
// outside the domain read as zero.
template <bool CHECK>
__device__ __forceinline__ void load_stencil_v(const GridView &g, const QW &w, float2 (&nv)[3][3],
                                               const float2 *field = nullptr) {
    const float2 *base = field ? field : g.grid_v;
    int yp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) yp[k] = cell_y_part(w.by + k - 1);
#pragma unroll
    for (int gx = 0; gx < 3; ++gx) {
        const float2 *row = base + cell_x_part(w.bx + gx - 1, g.tpd);
#pragma unroll
        for (int gy = 0; gy < 3; ++gy) {
            if (CHECK && !in_domain(w.bx + gx - 1, w.by + gy - 1, g.res))
                nv[gx][gy] = v2(0.0f, 0.0f);
            else
                nv[gx][gy] = row[yp[gy]];
        }
    }
}

// ASFLIP's PIC gather of the pre-force grid velocities with the G2P weights
// (transfer/g2p.rs:284-290); cells outside the domain read as zero.
template <bool FAST>
__device__ __forceinline__ float2 gather_pre_force(const GridView &g, const QW &w, bool inside) {
    float2 old_v = v2(0.0f, 0.0f);
    if constexpr (FAST) {
        float2 nv[3][3];
        if (inside)
            load_stencil_v<false>(g, w, nv, g.grid_vpre);
        else
            load_stencil_v<true>(g, w, nv, g.grid_vpre);
#pragma unroll
        for (int gx = 0; gx < 3; ++gx) {
            float2 r;
            r.x = __fmaf_rn(w.wy[0], nv[gx][0].x, __fmaf_rn(w.wy[1], nv[gx][1].x, w.wy[2] * nv[gx][2].x));
            r.y = __fmaf_rn(w.wy[0], nv[gx][0].y, __fmaf_rn(w.wy[1], nv[gx][1].y, w.wy[2] * nv[gx][2].y));
            old_v.x = __fmaf_rn(w.wx[gx], r.x, old_v.x);
            old_v.y = __fmaf_rn(w.wx[gx], r.y, old_v.y);
        }
    } else {
#pragma unroll
        for (int gx = 0; gx < 3; ++gx)
#pragma unroll
            for (int gy = 0; gy < 3; ++gy) {
                const float weight = w.wx[gx] * w.wy[gy];
                const int cx = w.bx + gx - 1, cy = w.by + gy - 1;
                const float2 pre = (inside || in_domain(cx, cy, g.res)) ? g.grid_vpre[cell_index(cx, cy, g.tpd)]
                                                                        : v2(0.0f, 0.0f);
                old_v = vadd(old_v, vmuls(pre, weight));
            }
    }
    return old_v;
}

// The grid velocity a particle of the multi-field scenes reads at a node (g2p.rs:219-238).
// sel: 1 / 2 a rest / grip particle while contact is active, 3 / 4 a solid / fluid mixture
// particle; nodes outside the field keep the total velocity.
__device__ __forceinline__ float2 field_node_v(const GridView &g, int ci, int sel, float2 v) {
    if (sel <= 2) return g.acc_grip[ci].w > 0.0f ? (sel == 2 ? g.grip_v[ci] : g.rest_v[ci]) : v;
    const bool mixture = g.acc_sol[ci].w > 0.0f || g.acc_flu[ci].w > 0.0f;
    return mixture ? (sel == 3 ? g.sol_v[ci] : g.flu_v[ci]) : v;
}

// G2P phase 1 for one particle (transfer/g2p.rs:217-326; ASFLIP and the multi-field node
// velocities compiled in with EXTRAS).  Returns 1 if the speed clamp fired.
// FAST = false: the reference's cell-by-cell expression order (bit-level parity).
// FAST = true: the same sums in stencil-offset form with fused multiply-adds:
//   v' = sum w v_i,  B = v' (x) e + [sum (gx-1) w v_i, sum (gy-1) w v_i].
template <bool FAST, bool EXTRAS = false>
__device__ __forceinline__ int g2p_particle(const GridView &g, const DevConfig &cfg, float dt,
                                            PState &p, int sel = 0) {
    QW w = quadratic_weights(p.x);
    const bool inside = stencil_inside(w.bx, w.by, g.res);
    // ASFLIP's FLIP residual (g2p.rs:281-290), gathered first so that only the residual is
    // live across the G2P sums
    float2 diff_vel = v2(0.0f, 0.0f);
    if constexpr (EXTRAS)
        if (cfg.asflip > 0.0f) diff_vel = vsub(p.v, gather_pre_force<FAST>(g, w, inside));
    float2 new_v = v2(0.0f, 0.0f);
    M2 b = mzero();
    if constexpr (FAST) {
        float2 nv[3][3];
        if (inside)
            load_stencil_v<false>(g, w, nv);
        else
            load_stencil_v<true>(g, w, nv);
        if constexpr (EXTRAS) {
            if (sel != 0) {
#pragma unroll
                for (int gx = 0; gx < 3; ++gx)
#pragma unroll
                    for (int gy = 0; gy < 3; ++gy) {
                        const int cx = w.bx + gx - 1, cy = w.by + gy - 1;
                        if (inside || in_domain(cx, cy, g.res))
                            nv[gx][gy] = field_node_v(g, cell_index(cx, cy, g.tpd), sel, nv[gx][gy]);
                    }
            }
        }
        float2 sx = v2(0.0f, 0.0f), sy = v2(0.0f, 0.0f);
#pragma unroll
        for (int gx = 0; gx < 3; ++gx) {
            // row sums over gy: R = sum wy v, Ry = sum (gy-1) wy v
            float2 r, ry;
            r.x = __fmaf_rn(w.wy[0], nv[gx][0].x, __fmaf_rn(w.wy[1], nv[gx][1].x, w.wy[2] * nv[gx][2].x));
            r.y = __fmaf_rn(w.wy[0], nv[gx][0].y, __fmaf_rn(w.wy[1], nv[gx][1].y, w.wy[2] * nv[gx][2].y));
            ry.x = __fmaf_rn(w.wy[2], nv[gx][2].x, -(w.wy[0] * nv[gx][0].x));
            ry.y = __fmaf_rn(w.wy[2], nv[gx][2].y, -(w.wy[0] * nv[gx][0].y));
            const float wx = w.wx[gx];
            new_v.x = __fmaf_rn(wx, r.x, new_v.x);
            new_v.y = __fmaf_rn(wx, r.y, new_v.y);
            sy.x = __fmaf_rn(wx, ry.x, sy.x);
            sy.y = __fmaf_rn(wx, ry.y, sy.y);
            if (gx == 0) {
                sx.x = __fmaf_rn(-wx, r.x, sx.x);
                sx.y = __fmaf_rn(-wx, r.y, sx.y);
            } else if (gx == 2) {
                sx.x = __fmaf_rn(wx, r.x, sx.x);
                sx.y = __fmaf_rn(wx, r.y, sx.y);
            }
        }
        const float2 e = centre_offset(w, p.x);
        b.xa = v2(__fmaf_rn(new_v.x, e.x, sx.x), __fmaf_rn(new_v.y, e.x, sx.y));
        b.ya = v2(__fmaf_rn(new_v.x, e.y, sy.x), __fmaf_rn(new_v.y, e.y, sy.y));
    } else {
        int xp[3], yp[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            xp[k] = cell_x_part(w.bx + k - 1, g.tpd);
            yp[k] = cell_y_part(w.by + k - 1);
        }
#pragma unroll
        for (int gx = 0; gx < 3; ++gx) {
#pragma unroll
            for (int gy = 0; gy < 3; ++gy) {
                float weight = w.wx[gx] * w.wy[gy];
                int cx = w.bx + gx - 1, cy = w.by + gy - 1;
                float2 dist = vadd(vsub(v2(static_cast<float>(cx), static_cast<float>(cy)), p.x),
                                   splat(0.5f));
                float2 node_v = v2(0.0f, 0.0f);
                if (inside || in_domain(cx, cy, g.res)) {
                    node_v = g.grid_v[xp[gx] + yp[gy]];
                    if constexpr (EXTRAS)
                        if (sel != 0) node_v = field_node_v(g, xp[gx] + yp[gy], sel, node_v);
                }
                float2 wv = vmuls(node_v, weight);
                M2 term = m2(vmuls(wv, dist.x), vmuls(wv, dist.y));
                b = madd(b, term);
                new_v = vadd(new_v, wv);
            }
        }
    }
    if (p.pinned != 0) {
        p.v = v2(0.0f, 0.0f);
        p.c = mzero();
        return 0;
    }
    float2 v_store = new_v, v_pos = new_v;
    if constexpr (EXTRAS) {
        if (cfg.asflip > 0.0f) {  // g2p.rs:281-296
            const float trace_b = b.xa.x + b.ya.y;
            const float gamma = trace_b < 0.0f ? 0.0f : 1.0f;
            v_store = vadd(new_v, svmul(cfg.asflip, diff_vel));
            v_pos = vadd(new_v, svmul(gamma * cfg.asflip, diff_vel));
        }
    }
    const float vel_limit = cfg.cell / dt;
    int clamped = 0;
    float spd = vlen(v_store);
    if (spd > vel_limit) {
        float scale = vel_limit / spd;
        v_store = vmuls(v_store, scale);
        v_pos = vmuls(v_pos, scale);
        clamped = 1;
    }
    float2 new_pos = vadd(p.x, vmuls(v_pos, dt));
    for (int k = 0; k < cfg.n_bound; ++k) new_pos = clamp_position(cfg.bound_t[k], new_pos, g.res);
    p.v = v_store;
    p.c = mscale(mscale(b, KERNEL_D_INVERSE), cfg.apic_blend);
    p.x = new_pos;
    return clamped;
}

inline int blocks_for(int n, int per) { return (n + per - 1) / per; }

// Instantiated model sets; a scene uses the smallest one covering its materials.
constexpr unsigned MASK_FLUID = (1u << M_FALLBACK) | (1u << M_FLUID);
constexpr unsigned MASK_SOLID = (1u << M_FALLBACK) | (1u << M_NEOHOOKEAN);
constexpr unsigned MASK_SOLID_FLUID = MASK_FLUID | MASK_SOLID;
constexpr unsigned MASK_GRANULAR =
    (1u << M_FALLBACK) | (1u << M_DRUCKER_PRAGER) | (1u << M_SNOW) | (1u << M_NACC);
// The same sets with the extras (force fields, ASFLIP, sleep zones, multi-field) compiled in.
constexpr unsigned EXTRAS = 1u << M_EXTRAS_BIT;
constexpr unsigned MASK_FLUID_X = MASK_FLUID | EXTRAS;
constexpr unsigned MASK_SOLID_X = MASK_SOLID | EXTRAS;
constexpr unsigned MASK_SOLID_FLUID_X = MASK_SOLID_FLUID | EXTRAS;
constexpr unsigned MASK_GRANULAR_X = MASK_GRANULAR | EXTRAS;
constexpr unsigned ALL_MODELS_X = ALL_MODELS | EXTRAS;
// The model set without the extras bit.
__host__ __device__ constexpr unsigned core_mask(unsigned m) { return m & ~EXTRAS; }

// ---------------------------------------------------------------- scatter engine
// P2G scatter of one particle per thread with vector red.global reductions (native
// in L2 on sm_100).  The contribution to cell (bx + gx - 1, by + gy - 1) is
//   mass      w m
//   momentum  w m (v + C d)        = w (qa + (gx-1) m C.x_axis + (gy-1) m C.y_axis)
//   stress    w s tau d            = w (qs + (gx-1) s tau.x_axis + (gy-1) s tau.y_axis)
// with d = e + (gx - 1, gy - 1), qa = m (v + C e), qs = s tau e (stencil-offset form),
// so a cell costs one weight product and a scale of a per-row vector.
// Optional warp aggregation: lanes whose particles share a base cell (contiguous
// after the tile sort) sum their contributions with a segmented shuffle reduction
// and the segment's first lane issues one reduction per cell.  Tile flags for the
// grid update are set once per particle (its stencil spans at most 2 x 2 tiles).
constexpr int THREADS = PARTICLE_THREADS;

struct Payload {
    float2 x;
    float m;      // mass channel weight
    float2 v;
    M2 c;
    M2 tau;
    float s;      // -4 * stress_volume (dt-free stress coefficient)
    bool do_ma;   // scatter mass + affine momentum
    bool do_s;    // scatter stress impulse
    uint32_t fields;  // multi-field sums it also adds to: bit 0 grip, 1 solid, 2 fluid
    bool excl;        // ... and to that (single) field only, not to the total (DevConfig::mf_excl)
};

// Which channels a scatter call carries: mass + momentum, stress, or per-particle flags.
enum ScatterChannels { SC_MA = 0, SC_S = 1, SC_BOTH = 2 };

// Per-particle scatter plan: weights, mass, and (momentum.xy, stress.xy) as a row base
// plus x/y steps.
struct ScatterPlan {
    QW w;
    float m;
    float4 q, sx, sy;
};

template <int SC>
__device__ __forceinline__ ScatterPlan make_plan(const Payload &p) {
    ScatterPlan r;
    r.w = quadratic_weights(p.x);
    const float2 e = centre_offset(r.w, p.x);
    r.m = 0.0f;
    r.q = r.sx = r.sy = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (SC != SC_S && (SC == SC_MA || p.do_ma)) {
        r.m = p.m;
        const float2 mx = svmul(p.m, p.c.xa), my = svmul(p.m, p.c.ya);
        r.q.x = __fmaf_rn(mx.x, e.x, __fmaf_rn(my.x, e.y, p.m * p.v.x));
        r.q.y = __fmaf_rn(mx.y, e.x, __fmaf_rn(my.y, e.y, p.m * p.v.y));
        r.sx.x = mx.x; r.sx.y = mx.y;
        r.sy.x = my.x; r.sy.y = my.y;
    }
    if (SC != SC_MA && (SC == SC_S || p.do_s)) {
        const float2 tx = svmul(p.s, p.tau.xa), ty = svmul(p.s, p.tau.ya);
        r.q.z = __fmaf_rn(tx.x, e.x, ty.x * e.y);
        r.q.w = __fmaf_rn(tx.y, e.x, ty.y * e.y);
        r.sx.z = tx.x; r.sx.w = tx.y;
        r.sy.z = ty.x; r.sy.w = ty.y;
    }
    return r;
}

__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 f4sub(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
// value of the plan's vector at stencil step k - 1 (k = 0, 1, 2)
__device__ __forceinline__ float4 f4step(float4 base, float4 step, int k) {
    return k == 0 ? f4sub(base, step) : (k == 2 ? f4add(base, step) : base);
}

// Adds the values of lanes [lane, seg_end) into `lane` (suffix sums within segments);
// `span` (warp-uniform) bounds the segment lengths.
__device__ __forceinline__ float seg_sum(float v, int lane, int seg_end, int span) {
    for (int off = 1; off < span; off <<= 1) {
        float y = __shfl_down_sync(0xffffffffu, v, off);
        if (lane + off < seg_end) v += y;
    }
    return v;
}

__device__ __forceinline__ void mark_tiles(const GridView &g, int bx, int by) {
    const int tx0 = max(bx - 1, 0) >> 3, tx1 = min(bx + 1, g.res - 1) >> 3;
    const int ty0 = max(by - 1, 0) >> 3, ty1 = min(by + 1, g.res - 1) >> 3;
    if (bx < -1 || by < -1 || bx > g.res || by > g.res) return;  // stencil misses the grid
    g.tile_flag[tx0 * g.tpd + ty0] = 1;
    if (tx1 != tx0) g.tile_flag[tx1 * g.tpd + ty0] = 1;
    if (ty1 != ty0) {
        g.tile_flag[tx0 * g.tpd + ty1] = 1;
        if (tx1 != tx0) g.tile_flag[tx1 * g.tpd + ty1] = 1;
    }
}

// One lane's 3 x 3 reductions (no aggregation) into the accumulators A (mass + momentum)
// and S (stress), and the same values into up to two more pairs (the multi-field sums; null
// when unused): one pass over the stencil, so the extra targets cost reductions only.
// CHECK skips cells outside the domain.
template <int SC, bool CHECK>
__device__ __forceinline__ void scatter_cells_to(const GridView &g, const ScatterPlan &pl,
                                                 bool do_ma, bool do_s, float4 *A, float2 *S,
                                                 float4 *A2 = nullptr, float2 *S2 = nullptr,
                                                 float4 *A3 = nullptr, float2 *S3 = nullptr) {
    const QW &w = pl.w;
    int yp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) yp[k] = cell_y_part(w.by + k - 1);
#pragma unroll
    for (int gx = 0; gx < 3; ++gx) {
        const int xp = cell_x_part(w.bx + gx - 1, g.tpd);
        const float4 r = f4step(pl.q, pl.sx, gx);
        const float wm = w.wx[gx] * pl.m;
#pragma unroll
        for (int gy = 0; gy < 3; ++gy) {
            if (CHECK && !in_domain(w.bx + gx - 1, w.by + gy - 1, g.res)) continue;
            const float4 t = f4step(r, pl.sy, gy);
            const float wt = w.wx[gx] * w.wy[gy];
            const int ci = xp + yp[gy];
            // the fourth lane counts scatters: a cell with w > 0 is in the reference's dirty set
            if (SC == SC_MA || (SC == SC_BOTH && do_ma)) {
                const float m = wm * w.wy[gy], ax = wt * t.x, ay = wt * t.y;
                red_add_v4(&A[ci], m, ax, ay, 1.0f);
                if (A2) red_add_v4(&A2[ci], m, ax, ay, 1.0f);
                if (A3) red_add_v4(&A3[ci], m, ax, ay, 1.0f);
            }
            if (SC == SC_S || (SC == SC_BOTH && do_s)) {
                const float sx = wt * t.z, sy = wt * t.w;
                red_add_v2(&S[ci], sx, sy);
                if (S2) red_add_v2(&S2[ci], sx, sy);
                if (S3) red_add_v2(&S3[ci], sx, sy);
            }
        }
    }
}

template <int SC, bool CHECK>
__device__ __forceinline__ void scatter_cells(const GridView &g, const ScatterPlan &pl,
                                              bool do_ma, bool do_s) {
    scatter_cells_to<SC, CHECK>(g, pl, do_ma, do_s, g.acc_a, g.acc_s);
}

// Warp-aggregated variant: every lane of the warp takes part (inactive lanes add zero).
// `target`, the same for every active lane: 0 the total, k + 1 multi-field sum k.
template <int SC>
__device__ __forceinline__ void scatter_cells_aggregated(const GridView &g, const ScatterPlan &pl,
                                                         bool active, bool do_ma, bool do_s,
                                                         unsigned target) {
    const int lane = threadIdx.x & 31;
    const QW &w = pl.w;
    const bool any_ma = SC != SC_S && __ballot_sync(0xffffffffu, active && do_ma) != 0u;
    const bool any_s = SC != SC_MA && __ballot_sync(0xffffffffu, active && do_s) != 0u;
    const int kx = active ? w.bx : INT_MIN, ky = active ? w.by : lane;
    const int px = __shfl_up_sync(0xffffffffu, kx, 1);
    const int py = __shfl_up_sync(0xffffffffu, ky, 1);
    const int head = (lane == 0 || !active || px != kx || py != ky) ? 1 : 0;
    const unsigned heads = __ballot_sync(0xffffffffu, head != 0);
    const unsigned after = heads & ~((2u << lane) - 1u);
    const int seg_end = after ? __ffs(after) - 1 : 32;
    // longest run of lanes sharing a base cell; 1 means nothing to combine
    const int span = static_cast<int>(
        __reduce_max_sync(0xffffffffu, head ? static_cast<unsigned>(seg_end - lane) : 0u));
    if (span <= 1) {
        if (!active) return;
        if (target)
            scatter_cells_to<SC, true>(g, pl, do_ma, do_s, g.fa[target - 1], g.fs[target - 1]);
        else
            scatter_cells_to<SC, true>(g, pl, do_ma, do_s, g.acc_a, g.acc_s);
        return;
    }
    int yp[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 3; ++k) yp[k] = cell_y_part(w.by + k - 1);
#pragma unroll
    for (int gx = 0; gx < 3; ++gx) {
        const int xp = cell_x_part(w.bx + gx - 1, g.tpd);
        const float4 r = f4step(pl.q, pl.sx, gx);
#pragma unroll
        for (int gy = 0; gy < 3; ++gy) {
            const float4 t = f4step(r, pl.sy, gy);
            const float wt = active ? w.wx[gx] * w.wy[gy] : 0.0f;
            float mc = wt * pl.m, ax = wt * t.x, ay = wt * t.y, sx = wt * t.z, sy = wt * t.w;
            if (any_ma) {
                mc = seg_sum(mc, lane, seg_end, span);
                ax = seg_sum(ax, lane, seg_end, span);
                ay = seg_sum(ay, lane, seg_end, span);
            }
            if (any_s) {
                sx = seg_sum(sx, lane, seg_end, span);
                sy = seg_sum(sy, lane, seg_end, span);
            }
            const int cx = w.bx + gx - 1, cy = w.by + gy - 1;
            if (head && active && in_domain(cx, cy, g.res)) {
                const int ci = xp + yp[gy];
                // the fourth lane counts the segment's scatters, one per particle
                float4 *A = g.acc_a;
                float2 *S = g.acc_s;
                if (target) {
                    A = g.fa[target - 1];
                    S = g.fs[target - 1];
                }
                if (any_ma) red_add_v4(&A[ci], mc, ax, ay, static_cast<float>(seg_end - lane));
                if (any_s) red_add_v2(&S[ci], sx, sy);
            }
        }
    }
}

// Lane-pair aggregation into the total: lanes 2m and 2m + 1 whose particles share a base
// cell (neighbours in tile-sort order, so usually in one cell) add their contributions with
// one shuffle per value and the even lane issues the reduction; where all four lanes of an
// aligned quad share it, a second shuffle folds the two pairs together.  A reduction in L2
// costs about the same however many lanes of a warp target one cell, so halving (quartering)
// the lanes that issue them halves (quarters) the scatter's L2 work, for 5 shuffles per cell.
// Every lane of the warp calls this (inactive lanes add nothing).
template <int SC>
__device__ __forceinline__ void scatter_cells_pairs(const GridView &g, const ScatterPlan &pl, bool active,
                                                    bool do_ma, bool do_s) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const QW &w = pl.w;
    // a unique key per inactive lane; active keys are the base cell (packed, any int range)
    const long long key = active ? (static_cast<long long>(w.bx) << 32) | static_cast<uint32_t>(w.by)
                                 : -1ll - lane;
    const bool pair = __shfl_xor_sync(full, key, 1) == key;
    const bool quad = pair && __shfl_xor_sync(full, pair ? key : -100ll - lane, 2) == key;
    const bool any_pair = __any_sync(full, pair), any_quad = __any_sync(full, quad);
    const bool issue = active && (!pair || ((lane & 1) == 0 && (!quad || (lane & 2) == 0)));
    // channels issued by this lane's group: mass + momentum if any member scatters them,
    // stress likewise (a fluid particle in the density mode pairs with a solid one)
    const bool ma_self = SC == SC_MA || (SC == SC_BOTH && active && do_ma);
    const bool s_self = SC == SC_S || (SC == SC_BOTH && active && do_s);
    int flags = (ma_self ? 1 : 0) | (s_self ? 2 : 0) | (ma_self ? 4 : 0);  // bit 2+: mass-scatter count
    if (SC == SC_BOTH) {
        if (any_pair) {
            const int o = __shfl_xor_sync(full, flags, 1);
            if (pair) flags = ((flags | o) & 3) | (((flags >> 2) + (o >> 2)) << 2);
        }
        if (any_quad) {
            const int o = __shfl_xor_sync(full, flags, 2);
            if (quad) flags = ((flags | o) & 3) | (((flags >> 2) + (o >> 2)) << 2);
        }
    } else {
        flags = SC == SC_MA ? (1 | ((quad ? 4 : (pair ? 2 : 1)) << 2)) : 2;
    }
    const bool do_a = SC != SC_S && (flags & 1), do_st = SC != SC_MA && (flags & 2);
    const float count = static_cast<float>(flags >> 2);
    const bool inside = stencil_inside(w.bx, w.by, g.res);
    int yp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) yp[k] = cell_y_part(w.by + k - 1);
#pragma unroll
    for (int gx = 0; gx < 3; ++gx) {
        const int xp = cell_x_part(w.bx + gx - 1, g.tpd);
        const float4 r = f4step(pl.q, pl.sx, gx);
        const float wm = w.wx[gx] * pl.m;
#pragma unroll
        for (int gy = 0; gy < 3; ++gy) {
            const float4 t = f4step(r, pl.sy, gy);
            const float wt = active ? w.wx[gx] * w.wy[gy] : 0.0f;
            float m = active ? wm * w.wy[gy] : 0.0f, ax = wt * t.x, ay = wt * t.y, sx = wt * t.z, sy = wt * t.w;
            if (any_pair) {
                float o0 = 0.0f, o1 = 0.0f, o2 = 0.0f, o3 = 0.0f, o4 = 0.0f;
                if (SC != SC_S) {
                    o0 = __shfl_xor_sync(full, m, 1);
                    o1 = __shfl_xor_sync(full, ax, 1);
                    o2 = __shfl_xor_sync(full, ay, 1);
                }
                if (SC != SC_MA) {
                    o3 = __shfl_xor_sync(full, sx, 1);
                    o4 = __shfl_xor_sync(full, sy, 1);
                }
                if (pair) { m += o0; ax += o1; ay += o2; sx += o3; sy += o4; }
            }
            if (any_quad) {
                float o0 = 0.0f, o1 = 0.0f, o2 = 0.0f, o3 = 0.0f, o4 = 0.0f;
                if (SC != SC_S) {
                    o0 = __shfl_xor_sync(full, m, 2);
                    o1 = __shfl_xor_sync(full, ax, 2);
                    o2 = __shfl_xor_sync(full, ay, 2);
                }
                if (SC != SC_MA) {
                    o3 = __shfl_xor_sync(full, sx, 2);
                    o4 = __shfl_xor_sync(full, sy, 2);
                }
                if (quad) { m += o0; ax += o1; ay += o2; sx += o3; sy += o4; }
            }
            if (!issue) continue;
            if (!inside && !in_domain(w.bx + gx - 1, w.by + gy - 1, g.res)) continue;
            const int ci = xp + yp[gy];
            if (do_a) red_add_v4(&g.acc_a[ci], m, ax, ay, count);
            if (do_st) red_add_v2(&g.acc_s[ci], sx, sy);
        }
    }
}

template <int SC>
__device__ __forceinline__ void scatter_particle(const GridView &g, const Payload &p, bool valid,
                                                 int aggregate) {
    const bool active = valid && (p.do_ma || p.do_s);
    ScatterPlan pl{};
    if (active) pl = make_plan<SC>(p);
    if (aggregate == 3) {  // lane pairs / quads into the total (no multi-field sums)
        scatter_cells_pairs<SC>(g, pl, active, p.do_ma, p.do_s);
        if (active) mark_tiles(g, pl.w.bx, pl.w.by);
        return;
    }
    // Exclusive field sums: a field particle's contributions go to its field's sums only, and
    // the grid update adds them to the total.  target: 0 the total, k + 1 field k.
    float4 *A = g.acc_a;
    float2 *S = g.acc_s;
    unsigned target = 0u;
    if (p.excl) {
        const int k = __ffs(p.fields) - 1;
        A = g.fa[k];
        S = g.fs[k];
        target = static_cast<unsigned>(k) + 1u;
    }
    // aggregate 2 (exclusive field sums): the warp aggregates when its active lanes share one
    // target, a warp that mixes them scatters lane by lane
    bool agg = aggregate != 0;
    if (aggregate == 2)
        agg = __reduce_min_sync(0xffffffffu, active ? target : 4u) >=
              __reduce_max_sync(0xffffffffu, active ? target : 0u);
    if (agg) {
        scatter_cells_aggregated<SC>(g, pl, active, p.do_ma, p.do_s, target);
        if (!active) return;
        // the multi-field sums of the fast pipeline (p2g.rs:60-66): the same contributions
        if (!p.excl)
            for (uint32_t f = p.fields; f != 0u; f &= f - 1u) {
                const int k = __ffs(f) - 1;
                scatter_cells_to<SC, true>(g, pl, p.do_ma, p.do_s, g.fa[k], g.fs[k]);
            }
    } else {
        if (!active) return;
        // up to two multi-field sums (grip, and a mixture phase) take the same contributions
        float4 *A2 = nullptr, *A3 = nullptr;
        float2 *S2 = nullptr, *S3 = nullptr;
        if (p.fields && !p.excl) {
            const int k2 = __ffs(p.fields) - 1;
            A2 = g.fa[k2];
            S2 = g.fs[k2];
            const uint32_t rest = p.fields & (p.fields - 1u);
            if (rest) {
                const int k3 = __ffs(rest) - 1;
                A3 = g.fa[k3];
                S3 = g.fs[k3];
            }
        }
        const QW &w = pl.w;
        if (stencil_inside(w.bx, w.by, g.res))
            scatter_cells_to<SC, false>(g, pl, p.do_ma, p.do_s, A, S, A2, S2, A3, S3);
        else
            scatter_cells_to<SC, true>(g, pl, p.do_ma, p.do_s, A, S, A2, S2, A3, S3);
    }
    mark_tiles(g, pl.w.bx, pl.w.by);
}

// The multi-field sums a particle adds to on the fast pipeline: the grip field for a
// contact group (contact.rs:41-72), its material's phase field (mixture.rs:20-58).
__device__ __forceinline__ uint32_t multi_fields(const DevConfig &cfg, const DevParticles &P, int i,
                                                 uint32_t mat, int n_mats) {
    uint32_t f = 0u;
    if ((cfg.mf_fields & 1) && P.contact[i] != 0u) f |= 1u;
    if (cfg.mf_fields & 2) {
        const uint32_t ph = cfg.mat_phase[mat < static_cast<uint32_t>(n_mats) ? mat : 0u];
        f |= ph == 1u ? 2u : (ph == 2u ? 4u : 0u);
    }
    return f;
}

// The contact point cloud on the fast pipeline (p2g.rs:54-74): every particle that scatters
// is pushed onto its base cell's list; the cells of its stencil find it in the lists of
// their 3 x 3 neighbourhood.
__device__ __forceinline__ void push_contact_point(const GridView &g, float2 x, bool grip, int i,
                                                   uint32_t slot) {
    const QW w = quadratic_weights(x);
    if (!in_domain(w.bx, w.by, g.res)) return;
    const int prev = atomicExch(&g.chead[slot][w.bx * g.res + w.by], i);
    g.cpts[i] = make_float4(x.x, x.y, grip ? 1.0f : -1.0f, __int_as_float(prev));
}

// ---------------------------------------------------------------- k_particle
struct ParticleKernelArgs {
    DevParticles P;
    int n;
    const MatP *mats;
    int n_mats;
    DevConfig cfg;
    StepState *st;
    GridView g;
    LoadFlags lf;
    int mode_g2p;       // 0: prime pass (no G2P), 1: G2P(k) + P2G(k+1)
    int density_mode;   // fluid stress deferred to k_density; G2P reads rho_dp
    int aggregate;      // warp-aggregated P2G reductions (2: in warps whose lanes share a target)
    int project_in;     // recompute the projection of substep k before G2P (fused pipeline)
    int emit_p2g;       // project for substep k+1 and scatter its P2G (fused pipeline)
    int split;          // 0: one pass; 1: G2P half (no fields, sleep scoring, CFL or P2G);
                        // 2: fields half (fields, sleep scoring, CFL, projection, P2G of the
                        // state the G2P half stored) -- the passes NBodyGravityField's tree
                        // build runs between
    ClosureArgs cl;     // learned closure (kernels instantiated with CLOSURE only)
    BatchView batch;    // batched scenes (kernels instantiated with BATCH only)
};

// Scene of this CTA in a batch (nullptr for single-scene kernels); false when the scene
// does not take part in the running substep (the whole CTA returns).
template <bool BATCH, class Args>
__device__ __forceinline__ bool batch_scene(const Args &a, const SceneDesc *&sd, int blk) {
    sd = nullptr;
    if constexpr (BATCH) {
        sd = &a.batch.scenes[a.batch.block_scene[blk]];
        if (a.batch.check_active && !sd->st->active) return false;
    }
    return true;
}

// ---------------------------------------------------------------- learned closure
// Per-lane state carried across the warp-level network evaluation.
struct ClosureWork {
    M2 u, vt;
    float2 sigma;      // Drucker-Prager: trial singular values; NACC: singular values of F
    float x[CL_IN];    // raw network inputs
    int kind;          // 0: update complete; 1: Drucker-Prager network; 2: NACC network
    int judge;         // also run the plain mapping and compare stresses
    int smooth;        // on a smooth plastic branch (network or plain fallback)
    float scale;       // Drucker-Prager: trial deviatoric norm (unit of the network's strains)
};

__device__ __forceinline__ uint32_t closure_hash(int i, const StepState *st) {
    return (static_cast<uint32_t>(i) * 2654435761u) ^ (static_cast<uint32_t>(st->total_substeps) * 40503u);
}

__device__ __forceinline__ void closure_log(const ClosureArgs &cl, int model, const float (&x)[CL_IN],
                                            float t0, float t1, float t2) {
    const unsigned long long k = atomicAdd(&cl.stats->logged[model], 1ull);
    if (k >= cl.log_cap) return;
    float *dx = cl.log_x[model] + k * CL_IN;
#pragma unroll
    for (int j = 0; j < CL_IN; ++j) dx[j] = x[j];
    float *dt = cl.log_t[model] + k * CL_OUT;
    dt[0] = t0;
    dt[1] = t1;
    dt[2] = t2;
}

__device__ __forceinline__ bool closure_in_hull(const ClosureNet &net, const float (&x)[CL_IN]) {
    bool in = net.ready != 0;
#pragma unroll
    for (int j = 0; j < CL_IN; ++j) {
        const float xn = (x[j] - net.in_shift[j]) * net.in_scale[j];
        in = in && xn >= net.hull_lo[j] && xn <= net.hull_hi[j];
    }
    return in;
}

// NACC tail of update_particle (nacc.rs:255-269) after the projection.
__device__ __forceinline__ void nacc_apply(PState &p, M2 nf, float alpha) {
    p.f = nf;
    p.lvs = alpha;
    float j = fmaxf(mdet(nf), MIN_J);
    float vol = p.v0 * j;
    p.vol = vol;
    p.rho = vol > MIN_J ? p.mass / vol : p.rho;
}

// Phase 1 of the closure update: trial state, exact branch decisions, logging; particles
// on a smooth plastic branch inside the training box are left for the network.
template <unsigned MASK>
__device__ __forceinline__ void closure_prepare(const MatP &m, PState &p, float dt, bool pr,
                                                const ClosureArgs &cl, uint32_t hash,
                                                ClosureWork &w) {
    w.kind = 0;
    w.judge = 0;
    w.smooth = 0;
    const bool dp = HAS_MODEL(MASK, M_DRUCKER_PRAGER) && m.model == M_DRUCKER_PRAGER;
    const bool nacc = HAS_MODEL(MASK, M_NACC) && m.model == M_NACC;
    if (dp) {
        const M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        svd2(f_trial, w.u, w.sigma, w.vt);
        const DpTrial t = dp_trial(m, w.sigma, p.lvs, p.q, pr);
        if (t.dev_norm == 0.0f || t.trace > 0.0f) {  // tip: exact
            dp_finish(m, p, w.u, w.sigma, w.vt, true, v2(1.0f, 1.0f), t.dev_norm, pr);
            return;
        }
        if (t.gamma <= 0.0f) {  // elastic: exact
            dp_finish(m, p, w.u, w.sigma, w.vt, false, v2(0.0f, 0.0f), 0.0f, pr);
            return;
        }
        // scale-invariant form: strains in units of the trial deviatoric norm s, so the
        // network sees O(1) inputs and its error is relative to the plastic correction
        w.smooth = 1;
        const float inv_s = 1.0f / t.dev_norm;
        w.x[0] = t.eps.x * inv_s;
        w.x[1] = t.eps.y * inv_s;
        w.x[2] = t.alpha;
        w.x[3] = t.ratio;
        w.x[4] = t.cohesion * inv_s;
        w.x[5] = em_log(t.dev_norm, pr);
        w.scale = t.dev_norm;
        float2 h;
        float dq;
        if (cl.log && hash % cl.log_stride == 0u) {
            dp_smooth(t, h, dq);
            closure_log(cl, 0, w.x, h.x * inv_s, h.y * inv_s, dq * inv_s);
        }
        if (cl.infer && closure_in_hull(cl.nets[0], w.x)) {
            w.kind = 1;
            w.judge = (hash >> 7) % cl.judge_stride == 0u;
            return;
        }
        dp_smooth(t, h, dq);
        dp_finish(m, p, w.u, w.sigma, w.vt, true, v2(em_exp(h.x, pr), em_exp(h.y, pr)), dq, pr);
        return;
    }
    if (nacc) {
        svd2(p.f, w.u, w.sigma, w.vt);
        const NaccTrial t = nacc_trial(m, w.sigma, p.lvs, pr);
        if (t.branch != 3) {  // caps and elastic: exact (nacc.rs:129-170)
            update_particle<MASK>(m, p, dt, pr);
            return;
        }
        const float kappa = nacc_kappa(m);
        w.smooth = 1;
        w.x[0] = em_log(fmaxf(w.sigma.x, LOG_CLAMP), pr);
        w.x[1] = em_log(fmaxf(w.sigma.y, LOG_CLAMP), pr);
        w.x[2] = t.p0 / kappa;
        w.x[3] = m.mu / kappa;
        w.x[4] = m.compression_limit;
        w.x[5] = m.stretch_limit;
        float2 sv_new;
        float a_new;
        if (cl.log && hash % cl.log_stride == 0u) {
            nacc_smooth(m, t, p.lvs, sv_new, a_new, pr);
            closure_log(cl, 1, w.x, em_log(sv_new.x, pr) - w.x[0], em_log(sv_new.y, pr) - w.x[1], a_new - p.lvs);
        }
        if (cl.infer && closure_in_hull(cl.nets[1], w.x)) {
            w.kind = 2;
            w.judge = (hash >> 7) % cl.judge_stride == 0u;
            return;
        }
        nacc_smooth(m, t, p.lvs, sv_new, a_new, pr);
        nacc_apply(p, reconstruct(w.u, sv_new, w.vt), a_new);
        return;
    }
    update_particle<MASK>(m, p, dt, pr);
}

// The update of the deferred mode: the constitutive update of the particle pass, except that
// a Drucker-Prager or NACC particle on the smooth plastic branch whose network is installed
// is left unupdated and returned as 1 (Drucker-Prager) or 2 (NACC) for the tile kernel.  The
// branch decision reuses the trial SVD the update needs anyway (sand.rs:156-194,
// nacc.rs:129-223); every other particle is updated exactly as update_particle does.
template <unsigned MASK>
__device__ __forceinline__ int closure_defer_update(const MatP &m, PState &p, float dt, bool pr,
                                                    const ClosureArgs &cl) {
    if (HAS_MODEL(MASK, M_DRUCKER_PRAGER) && m.model == M_DRUCKER_PRAGER && cl.nets[0].ready) {
        const M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        M2 u, vt;
        float2 sigma;
        svd2(f_trial, u, sigma, vt);
        // dp_project's decisions in its order: the tip before the friction angle
        const float2 sg = vmax2(vabs2(sigma), splat(LOG_CLAMP));
        const float2 eps = v2(em_log(sg.x, pr) + p.lvs * 0.5f, em_log(sg.y, pr) + p.lvs * 0.5f);
        const float trace = eps.x + eps.y;
        const float dev_norm = evlen(vsub(eps, splat(trace * 0.5f)));
        if (dev_norm == 0.0f || trace > 0.0f) {
            dp_finish(m, p, u, sigma, vt, true, v2(1.0f, 1.0f), dev_norm, pr);
            return 0;
        }
        const float gamma = dev_norm + ediv(m.lambda + m.mu, m.mu) * trace * dp_alpha(m, p.q, pr) -
                            ediv(m.stretch_limit, 2.0f * m.mu);
        if (gamma <= 0.0f) {
            dp_finish(m, p, u, sigma, vt, false, v2(0.0f, 0.0f), 0.0f, pr);
            return 0;
        }
        return 1;
    }
    if (HAS_MODEL(MASK, M_NACC) && m.model == M_NACC && cl.nets[1].ready) {
        M2 u, vt;
        float2 sv;
        svd2(p.f, u, sv, vt);
        const NaccTrial t = nacc_trial(m, sv, p.lvs, pr);
        if (t.branch == 3) return 2;
        M2 nf;
        float na;
        nacc_project_t(m, p.f, u, vt, t, p.lvs, nf, na, pr);
        nacc_apply(p, nf, na);
        return 0;
    }
    update_particle<MASK>(m, p, dt, pr);
    return 0;
}

// Phase 2 (all 32 lanes): network evaluation for the lanes that asked for it.
template <unsigned MASK>
__device__ __forceinline__ void closure_evaluate(const ClosureArgs &cl, const ClosureWork &w,
                                                 float (&y)[CL_OUT]) {
#pragma unroll
    for (int net = 0; net < CL_NMODELS; ++net) {
        if (net == 0 && !HAS_MODEL(MASK, M_DRUCKER_PRAGER)) continue;
        if (net == 1 && !HAS_MODEL(MASK, M_NACC)) continue;
        const bool want = w.kind == net + 1;
        if (!__any_sync(0xffffffffu, want)) continue;
        const ClosureNet &nn = cl.nets[net];
        float xn[CL_IN], yn[CL_OUT];
#pragma unroll
        for (int j = 0; j < CL_IN; ++j) xn[j] = want ? (w.x[j] - nn.in_shift[j]) * nn.in_scale[j] : 0.0f;
        closure_warp_infer(nn, want, xn, yn);
        if (want) {
#pragma unroll
            for (int j = 0; j < CL_OUT; ++j) y[j] = yn[j] * nn.out_scale[j] + nn.out_shift[j];
        }
    }
}

// Phase 3: finish the update from the network's outputs; judge sampled particles against
// the plain mapping (relative error of the principal Kirchhoff stress).
template <unsigned MASK>
__device__ __forceinline__ void closure_finish(const MatP &m, PState &p, bool pr, const ClosureWork &w,
                                               const float (&y)[CL_OUT], float &err) {
    err = -1.0f;
    if (w.kind == 1) {
        const float2 proj = v2(em_exp(y[0] * w.scale, pr), em_exp(y[1] * w.scale, pr));
        const float dq = fmaxf(y[2] * w.scale, 0.0f);
        if (w.judge) {
            const DpTrial t = dp_trial(m, w.sigma, p.lvs, p.q, pr);
            float2 h;
            float dq_ref;
            dp_smooth(t, h, dq_ref);
            const float2 s_ref = dp_principal_stress(m, v2(em_exp(h.x, pr), em_exp(h.y, pr)));
            const float2 s_net = dp_principal_stress(m, proj);
            err = vlen(vsub(s_net, s_ref)) / fmaxf(vlen(s_ref), 1e-6f * m.mu);
        }
        dp_finish(m, p, w.u, w.sigma, w.vt, true, proj, dq, pr);
    } else if (w.kind == 2) {  // outputs: the plastic correction of ln(sv)
        const float2 sv_new = v2(em_exp(y[0] + w.x[0], pr), em_exp(y[1] + w.x[1], pr));
        const float a_new = m.hardening_exponent > 0.0f ? p.lvs + y[2] : p.lvs;
        if (w.judge) {
            const NaccTrial t = nacc_trial(m, w.sigma, p.lvs, pr);
            float2 sv_ref;
            float a_ref;
            nacc_smooth(m, t, p.lvs, sv_ref, a_ref, pr);
            const float2 s_ref = nacc_principal_stress(m, sv_ref);
            const float2 s_net = nacc_principal_stress(m, sv_new);
            err = vlen(vsub(s_net, s_ref)) / fmaxf(vlen(s_ref), 1e-6f * m.mu);
        }
        nacc_apply(p, reconstruct(w.u, sv_new, w.vt), a_new);
    }
}

__device__ __forceinline__ void closure_count(const ClosureArgs &cl, int smooth, int net, int fallback,
                                              float err) {
    const unsigned full = 0xffffffffu;
    const int n_smooth = __reduce_add_sync(full, smooth);
    const int n_net = __reduce_add_sync(full, net);
    const int n_fb = __reduce_add_sync(full, fallback);
    const int n_judged = __reduce_add_sync(full, err >= 0.0f ? 1 : 0);
    float e = err >= 0.0f ? err : 0.0f;
    float e_sum = e, e_max = e;
    for (int o = 16; o > 0; o >>= 1) {
        e_sum += __shfl_xor_sync(full, e_sum, o);
        e_max = fmaxf(e_max, __shfl_xor_sync(full, e_max, o));
    }
    if ((threadIdx.x & 31) == 0 && n_smooth) {
        ClosureStats *s = cl.stats;
        atomicAdd(&s->smooth, static_cast<unsigned long long>(n_smooth));
        if (n_net) atomicAdd(&s->net, static_cast<unsigned long long>(n_net));
        if (n_fb) atomicAdd(&s->hull_fallback, static_cast<unsigned long long>(n_fb));
        if (n_judged) {
            atomicAdd(&s->judged, static_cast<unsigned long long>(n_judged));
            atomicAdd(&s->err_sum, static_cast<double>(e_sum));
            atomicMax(&s->err_max_bits, __float_as_uint(e_max));
        }
    }
    if (err >= 0.0f) atomicAdd(&cl.stats->err_hist[closure_err_bin(err)], 1ull);
}

// Body of the particle pass (one particle per thread); the kernels that run it are
// instantiated in step_kernels.cu (reference-order arithmetic) and fast_kernels.cu.
// Appends the slot of each lane with `want` to queue `model` of the learned closure (one
// atomic per warp).  Every lane of the warp calls this.
__device__ __forceinline__ void closure_enqueue(const ClosureArgs &cl, StepState *st, uint32_t slot,
                                                int model, bool want, int i) {
    const unsigned ballot = __ballot_sync(0xffffffffu, want);
    if (!ballot) return;
    const int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
    uint32_t base = 0u;
    if (lane == leader) base = atomicAdd(&st->cl_queued[slot][model], static_cast<uint32_t>(__popc(ballot)));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) cl.queue[model][base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<uint32_t>(i);
}

// CLOSURE: 0 none; 1 the learned closure evaluated inside the pass (warp-level MMA); 2 the
// particles the network maps are queued for the tile kernel (closure_tiles.cu), which
// finishes their update, CFL bound, projection and P2G.
// blk: the 256-particle chunk this CTA works on (blockIdx.x; batched CTAs may take several
// chunks in turn, see k_particle_batch).
template <unsigned MASK, bool FAST, int CLOSURE = 0, bool BATCH = false>
__device__ __forceinline__ void particle_pass(const ParticleKernelArgs &a, int blk = blockIdx.x) {
    __shared__ MatP s_mats[MAX_MATERIALS];
    __shared__ uint32_t s_max_speed, s_min_mdt, s_warps_done;
    const SceneDesc *sd;
    if (!batch_scene<BATCH>(a, sd, blk)) return;
    // this CTA's scene: the kernel arguments, or the batch's scene table
    const DevConfig &cfg = [&]() -> const DevConfig & { if constexpr (BATCH) return sd->cfg; else return a.cfg; }();
    const GridView &g = [&]() -> const GridView & { if constexpr (BATCH) return sd->g; else return a.g; }();
    const MatP *mats = BATCH ? sd->mats : a.mats;
    const int n_mats = BATCH ? sd->n_mats : a.n_mats;
    const int density_mode = BATCH ? sd->density_mode : a.density_mode;
    StepState *st = BATCH ? sd->st : a.st;
    const int i = BATCH ? sd->p0 + (blk - sd->block0) * THREADS + static_cast<int>(threadIdx.x)
                        : blk * THREADS + static_cast<int>(threadIdx.x);
    const bool in_range = BATCH ? i < sd->p0 + sd->n : i < a.n;
    // sleep partition: particles outside the active zone take no part in the substep
    uint32_t zb = 0u;
    if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT))
        if (cfg.zones && in_range) zb = a.P.sleeping[i];
    const bool valid = in_range && (zb & ZB_OUT) == 0u;
    for (int k = threadIdx.x; k < n_mats; k += THREADS) s_mats[k] = mats[k];
    if (threadIdx.x == 0) {
        s_max_speed = 0u;            // bits of 0.0f
        s_min_mdt = 0x7f800000u;     // bits of +inf
        s_warps_done = 0u;
    }
    const bool pr = cfg.precise_math != 0;
    // The particle's state loads and the controller reads are issued together before the
    // barrier that publishes the materials, so their latencies overlap.
    const uint32_t acc_slot = st->acc_slot;
    const float dt = st->sub_dt;
    PState p;
    if (valid) p = load_state(a.P, i, a.lf);
    __syncthreads();
    Payload pl;
    pl.do_ma = false;
    pl.do_s = false;
    pl.fields = 0u;
    pl.excl = false;
    float max_speed = 0.0f;
    float min_mdt = INFINITY;
    int clamped = 0, projected = 0, proj_changed = 0;
    const MatP *mp = &s_mats[0];
    Saved o;
    ClosureWork w;
    if constexpr (CLOSURE) {
        w.kind = 0;
        w.smooth = 0;
        w.judge = 0;
    }
    if (valid) {
        mp = &s_mats[p.mat < static_cast<uint32_t>(n_mats) ? p.mat : 0u];
        if (a.mode_g2p) {
            o = save_fields(p);
            // the stored state is the unprojected post-G2P state S''(k): recompute its
            // projection S'(k) (counted when it was first computed).  A particle woken after
            // this substep's P2G was neither projected nor given a density this substep.
            const bool woken = (zb & ZB_WOKEN) != 0u;
            if (a.project_in && cfg.project && !woken) project_state(cfg, p);
            if (density_mode && a.project_in && !woken) {
                float d = a.P.rho_dp[i];
                if (d > F32_EPS) {
                    p.rho = d;
                    p.vol = p.mass / d;
                }
            }
            int sel = 0;  // multi-field node velocities (g2p.rs:219-238)
            if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT)) {
                if (cfg.multi) {
                    if (st->contact_active) {
                        sel = a.P.contact[i] != 0u ? 2 : 1;
                    } else {
                        const uint32_t ph = cfg.mat_phase[p.mat < static_cast<uint32_t>(n_mats) ? p.mat : 0u];
                        sel = ph == 1u ? 3 : (ph == 2u ? 4 : 0);
                    }
                }
            }
            clamped = g2p_particle<FAST, HAS_MODEL(MASK, M_EXTRAS_BIT)>(g, cfg, dt, p, sel);
            if constexpr (CLOSURE == 2)
                w.kind = closure_defer_update<MASK>(*mp, p, dt, pr, a.cl);
            else if constexpr (CLOSURE == 1)
                closure_prepare<MASK>(*mp, p, dt, pr, a.cl, closure_hash(i, st), w);
            else
                update_particle<MASK>(*mp, p, dt, pr);
        }
        if (a.split == 2) o = save_fields(p);
    }
    bool deferred = false;  // CLOSURE == 2: queued for the tile kernel
    if constexpr (CLOSURE == 1) {
        // learned closure: the network runs for the whole warp (warp-synchronous MMA)
        float y[CL_OUT] = {0.0f, 0.0f, 0.0f};
        float err = -1.0f;
        if (a.mode_g2p) {
            closure_evaluate<MASK>(a.cl, w, y);
            if (valid) closure_finish<MASK>(*mp, p, pr, w, y, err);
            closure_count(a.cl, w.smooth, w.kind != 0 ? 1 : 0, (w.smooth && w.kind == 0 && a.cl.infer) ? 1 : 0, err);
        }
    } else if constexpr (CLOSURE == 2) {
        if (a.mode_g2p) {  // the tile kernel counts the queued particles' statistics
            deferred = valid && w.kind != 0;
            closure_enqueue(a.cl, st, acc_slot, 0, deferred && w.kind == 1, i);
            closure_enqueue(a.cl, st, acc_slot, 1, deferred && w.kind == 2, i);
        }
    }
    bool asleep = false;  // sleep scoring at the end of this substep (step.rs:299-315)
    if (valid) {
        if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT)) {
            if (a.split == 0 ? a.mode_g2p != 0 : a.split == 2) {
                apply_force_fields(cfg, p, dt, i);
                if (cfg.sleep_thr > 0.0f && (zb & ZB_FLAG) == 0u) {
                    const float act = a.lf.activation ? p.activation : a.P.activation[i];
                    asleep = act == 0.0f && vlen2(p.v) < cfg.sleep_thr * cfg.sleep_thr;
                }
            }
        }
        if (a.mode_g2p || a.split == 2) store_fields(a.P, i, o, p);
        if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT)) {
            if (asleep) {
                a.P.sleeping[i] = ZB_FLAG | ZB_OUT;
                zone_log(cfg, 2u * static_cast<uint32_t>(st->total_substeps) + 1u, a.P.slot_to_index[i]);
            } else if (zb & ZB_WOKEN) {
                a.P.sleeping[i] = zb & ~ZB_WOKEN;
            }
        }
    }
    if (valid && !asleep && a.split != 1) {
        const MatP &m = *mp;
        // CFL contribution for the next substep (step.rs:447-466); a queued particle's
        // material bound depends on its update, which the tile kernel finishes
        float sp = vlen(p.v);
        if (cfg.affine_cfl) sp += affine_cfl(p.c, cfg.cell);
        max_speed = sp;
        if (!deferred) {
            float mdt = timestep_bound<MASK>(m, p.rho, p.h, cfg.cell, cfg.mat_cfl, cfg.visc_cfl, pr);
            if (isfinite(mdt) && mdt > 0.0f) min_mdt = mdt;
        }
        if (a.emit_p2g && !deferred) {
            // projection of the next substep (step.rs:67-73) and its P2G payload
            if (cfg.project) {
                bool ch = false;
                projected = project_state(cfg, p, &ch) ? 1 : 0;
                proj_changed = ch ? 1 : 0;
            }
            pl.x = p.x;
            pl.m = p.mass;
            pl.v = p.v;
            pl.c = p.c;
            pl.do_ma = true;
            if (!(density_mode && m.model == M_FLUID)) {
                pl.tau = combined_kirchhoff_stress<MASK>(m, p, pr);
                pl.s = -stress_volume(m, p) * KERNEL_D_INVERSE;
                pl.do_s = true;
            }
            if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT)) {
                if (cfg.mf_fast) {
                    pl.fields = multi_fields(cfg, a.P, i, p.mat, n_mats);
                    pl.excl = cfg.mf_excl && pl.fields != 0u;
                    if (cfg.mf_fields & 1) push_contact_point(g, p.x, (pl.fields & 1u) != 0u, i, acc_slot);
                }
            }
        }
    }
    count_warp(&st->vel_clamp, clamped != 0);
    count_warp(&st->jproj_pending[acc_slot], projected != 0);
    count_warp(&st->proj_changed[acc_slot], proj_changed != 0);

    // CFL reduction without a block barrier: warp reduction, shared atomics, and the
    // block's last warp to arrive publishes the block's result (one global atomic each).
    max_speed = warp_max(max_speed);
    min_mdt = warp_min(min_mdt);
    if ((threadIdx.x & 31) == 0 && a.split != 1) {
        atomicMax(&s_max_speed, __float_as_uint(max_speed));  // non-negative: ordered as uint
        atomicMin(&s_min_mdt, __float_as_uint(min_mdt));      // positive or +inf
        __threadfence_block();
        if (atomicAdd(&s_warps_done, 1u) == THREADS / 32 - 1) {
            atomicMax(&st->max_speed_bits[acc_slot], atomicOr(&s_max_speed, 0u));
            atomicMin(&st->min_mdt_bits[acc_slot], atomicOr(&s_min_mdt, 0u));
            atomicAdd(&st->window_blocks, 1ull);
        }
    }
    // aggregate mode 2 (per-warp targets) only where exclusive field sums can occur
    const int aggregate = HAS_MODEL(MASK, M_EXTRAS_BIT) || a.aggregate == 3 ? a.aggregate : (a.aggregate ? 1 : 0);
    if (core_mask(MASK) == MASK_FLUID && density_mode)
        scatter_particle<SC_MA>(g, pl, valid, aggregate);
    else
        scatter_particle<SC_BOTH>(g, pl, valid, aggregate);
}

// ---------------------------------------------------------------- k_density
// Density at a particle: sum of w m over its stencil (solver/density.rs:50-71), as
// row sums sum_gx wx (sum_gy wy m).  CHECK reads cells outside the domain as zero.
// `excl_fields`: the fields whose particles scattered into their field only
// (DevConfig::mf_excl); their masses are part of the cell's total.
template <bool CHECK>
__device__ __forceinline__ float gather_density(const GridView &g, const QW &w, int excl_fields) {
    int yp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) yp[k] = cell_y_part(w.by + k - 1);
    float density = 0.0f;
#pragma unroll
    for (int gx = 0; gx < 3; ++gx) {
        const int xp = cell_x_part(w.bx + gx - 1, g.tpd);
        const float4 *row = g.acc_a + xp;
        float mk[3];
#pragma unroll
        for (int gy = 0; gy < 3; ++gy) {
            const bool out = CHECK && !in_domain(w.bx + gx - 1, w.by + gy - 1, g.res);
            mk[gy] = out ? 0.0f : row[yp[gy]].x;
            if (excl_fields && !out) {
                if (excl_fields & 1) mk[gy] += g.fa[0][xp + yp[gy]].x;
                if (excl_fields & 2) mk[gy] += g.fa[1][xp + yp[gy]].x + g.fa[2][xp + yp[gy]].x;
            }
        }
        const float r = __fmaf_rn(w.wy[0], mk[0], __fmaf_rn(w.wy[1], mk[1], w.wy[2] * mk[2]));
        density = __fmaf_rn(w.wx[gx], r, density);
    }
    return density;
}

struct DensityKernelArgs {
    DevParticles P;
    int n;
    const MatP *mats;
    int n_mats;
    DevConfig cfg;
    StepState *st;
    GridView g;
    LoadFlags lf;
    int aggregate;
    BatchView batch;    // batched scenes (kernels instantiated with BATCH only)
};

// estimate_particle_volumes gather (solver/density.rs:50-71) at the projected
// positions, stored as rho_dp, plus the stress scatter of fluid particles.
template <unsigned MASK, bool BATCH = false>
__device__ __forceinline__ void density_pass(const DensityKernelArgs &a, int blk = blockIdx.x) {
    __shared__ MatP s_mats[MAX_MATERIALS];
    const SceneDesc *sd;
    if (!batch_scene<BATCH>(a, sd, blk)) return;
    if (BATCH && !sd->density_mode) return;  // no material of the scene needs the pass
    const DevConfig &cfg = [&]() -> const DevConfig & { if constexpr (BATCH) return sd->cfg; else return a.cfg; }();
    const GridView &g = [&]() -> const GridView & { if constexpr (BATCH) return sd->g; else return a.g; }();
    const MatP *mats = BATCH ? sd->mats : a.mats;
    const int n_mats = BATCH ? sd->n_mats : a.n_mats;
    StepState *st = BATCH ? sd->st : a.st;
    const int i = BATCH ? sd->p0 + (blk - sd->block0) * THREADS + static_cast<int>(threadIdx.x)
                        : blk * THREADS + static_cast<int>(threadIdx.x);
    bool valid = BATCH ? i < sd->p0 + sd->n : i < a.n;
    if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT))
        if (cfg.zones && valid) valid = (a.P.sleeping[i] & ZB_OUT) == 0u;
    for (int k = threadIdx.x; k < n_mats; k += THREADS) s_mats[k] = mats[k];
    const bool pr = cfg.precise_math != 0;
    // Positions at the projected state S'(k): the stored state itself unless the particle
    // pass's projection changed some particle, in which case the full state is loaded and
    // projected again.  Otherwise only what the density gather and the fluid stress read
    // is loaded.
    const uint32_t acc_slot = st->acc_slot;
    const unsigned long long changed0 = st->proj_changed[0], changed1 = st->proj_changed[1];
    PState p;
    if (valid) {
        p.x = a.P.x[i];
        p.mat = a.P.mat[i];
        // the fluid stress's own fields, issued with the position so their latency overlaps
        // the density gather (in a fluid-only scene every particle is a fluid or fallback)
        if constexpr (core_mask(MASK) == MASK_FLUID) {
            p.c = m_from4(a.P.c[i]);
            p.mass = a.P.mass[i];
        }
    }
    __syncthreads();
    const bool reproject = cfg.project && (acc_slot ? changed1 : changed0) != 0ull;
    Payload pl;
    pl.do_ma = false;
    pl.do_s = false;
    pl.fields = 0u;
    pl.excl = false;
    if (valid) {
        if (reproject) {
            p = load_state(a.P, i, a.lf);
            project_state(cfg, p);
        }
        const QW w = quadratic_weights(p.x);
        const bool inside = stencil_inside(w.bx, w.by, g.res);
        // (an if statement: a ?: reading cfg here stops this nvcc's front end)
        int excl = 0;
        if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT))
            if (cfg.mf_excl) excl = cfg.mf_fields;
        const float density = inside ? gather_density<false>(g, w, excl) : gather_density<true>(g, w, excl);
        a.P.rho_dp[i] = density;
        const MatP &m = s_mats[p.mat < static_cast<uint32_t>(n_mats) ? p.mat : 0u];
        if (m.model == M_FLUID) {
            if (!reproject) {  // the fields the fluid stress reads (fluid.rs:135-195)
                if constexpr (core_mask(MASK) != MASK_FLUID) {
                    p.c = m_from4(a.P.c[i]);
                    p.mass = a.P.mass[i];
                }
                p.f = m.surface_tension_coeff != 0.0f ? m_from4(a.P.f[i]) : mident();
                p.temperature = a.lf.temperature ? a.P.temperature[i] : 0.0f;
                p.activation = 0.0f;  // no active stress for fluids
                if (!(density > F32_EPS)) {
                    p.rho = a.P.rho[i];
                    p.vol = a.P.vol[i];
                }
            }
            if (density > F32_EPS) {
                p.rho = density;
                p.vol = p.mass / density;
            }
            pl.x = p.x;
            pl.m = 0.0f;
            pl.tau = combined_kirchhoff_stress<MASK>(m, p, pr);
            pl.s = -stress_volume(m, p) * KERNEL_D_INVERSE;
            pl.do_s = true;
            if constexpr (HAS_MODEL(MASK, M_EXTRAS_BIT)) {
                if (cfg.mf_fast) {
                    pl.fields = multi_fields(cfg, a.P, i, p.mat, n_mats);
                    pl.excl = cfg.mf_excl && pl.fields != 0u;
                }
            }
        }
    }
    scatter_particle<SC_S>(g, pl, valid,
                           HAS_MODEL(MASK, M_EXTRAS_BIT) || a.aggregate == 3 ? a.aggregate : (a.aggregate ? 1 : 0));
}

// Launchers of the fast path's kernels (fast_kernels.cu).
void launch_particle_pass_fast(const ParticleKernelArgs &a, unsigned model_mask, cudaStream_t stream);
void launch_density_pass_fast(const DensityKernelArgs &a, unsigned model_mask, cudaStream_t stream);

// Smallest instantiated model set that covers the registered models.
inline unsigned covering_mask(unsigned m) {
    const unsigned masks[10] = {MASK_FLUID,   MASK_SOLID,   MASK_SOLID_FLUID,   MASK_GRANULAR,   ALL_MODELS,
                                MASK_FLUID_X, MASK_SOLID_X, MASK_SOLID_FLUID_X, MASK_GRANULAR_X, ALL_MODELS_X};
    for (unsigned c : masks)
        if ((m & ~c) == 0u) return c;
    return FULL_MODELS;
}

template <class Args>
inline void fill_common(Args &a, const StepLaunch &L, const LoadFlagsHost &lfh) {
    a.P = L.P;
    a.n = L.n;
    a.mats = L.mats;
    a.n_mats = L.n_mats;
    a.cfg = L.cfg;
    a.st = L.st;
    a.g = L.g;
    a.lf.temperature = lfh.temperature;
    a.lf.activation = lfh.activation;
    a.lf.pinned = lfh.pinned;
    // EMERGE_OPT_P2G_AGGREGATE: 1 warp segments (per-warp targets with exclusive field sums),
    // 2 lane pairs / quads (scenes without multi-field sums; others use the segments)
    a.aggregate = L.use_window == 0 ? 0 : (L.use_window == 2 && !L.cfg.mf_fast ? 3 : (L.cfg.mf_excl ? 2 : 1));
}

}  // namespace emerge
