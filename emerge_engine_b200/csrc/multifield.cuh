// multifield.cuh -- the contact resolve's device code (grid/contact.rs, contact_normal.rs,
// directional_grip.rs), shared by the reference-order kernels (multifield.cu, IEEE
// arithmetic) and the fast pipeline's (multifield_fast.cu, fast division and FMA).
#pragma once
#include <cfloat>

#include "particle_pass.cuh"

namespace emerge {
namespace {

constexpr int MF_THREADS = 256;

__device__ __forceinline__ float2 clamp_speed(float2 v, float vel_limit) {
    const float spd = vlen(v);
    return spd > vel_limit ? vmuls(v, vel_limit / spd) : v;
}

// glam Vec2::normalize: self * (1 / length)
__device__ __forceinline__ float2 normalize2(float2 a) { return vmuls(a, 1.0f / vlen(a)); }

// solve3x3 (grid/contact_normal.rs): Cramer's rule; false for |det| <= EPSILON.
__device__ bool solve3x3(const float m[3][3], const float rhs[3], float out[3]) {
    auto det3 = [](const float a[3][3]) {
        return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
               a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
               a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    };
    const float det = det3(m);
    if (fabsf(det) <= F32_EPS) return false;
    for (int col = 0; col < 3; ++col) {
        float mm_[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) mm_[r][c] = (c == col) ? rhs[r] : m[r][c];
        out[col] = det3(mm_) / det;
    }
    return true;
}

// A contact cell's point cloud, each point {x, y, label}.  The resolve reads it only through
// sums and a max / min; the serial sets sum in point order (reference order: the cell's
// scatter records, in particle index order), the warp set splits the points over the lanes
// of a warp.
template <class D>
struct SerialPoints {
    static constexpr bool kSymmetric = false;  // the fit sums all nine matrix entries in order
    __device__ __forceinline__ bool writer() const { return true; }
    template <int N, class F>
    __device__ __forceinline__ void sum(float (&acc)[N], F f) const {
        static_cast<const D *>(this)->for_each([&](const float4 &q) { f(q, acc); });
    }
    template <class F>
    __device__ __forceinline__ void max_min(float &mx, float &mn, F f) const {
        static_cast<const D *>(this)->for_each([&](const float4 &q) { f(q, mx, mn); });
    }
};
struct RecordPoints : SerialPoints<RecordPoints> {
    const uint32_t *vals;
    const float4 *points;
    int lo, hi;
    __device__ RecordPoints(const uint32_t *v, const float4 *p, int l, int h) : vals(v), points(p), lo(l), hi(h) {}
    template <class F>
    __device__ __forceinline__ void for_each(F f) const {
        for (int j = lo; j < hi; ++j) f(points[vals[j]]);
    }
};
// Fast pipeline: the particles on the lists of the 3 x 3 base cells around the cell.  Every
// particle is pushed once per pass onto lists cleared before the pass, so a walk ends; it is
// still bounded (n_max nodes, the particle count), and a walk cut short sets an error bit.
struct ListPoints : SerialPoints<ListPoints> {
    const int *head;
    const float4 *nodes;
    int res, cx, cy, n_max;
    uint32_t *err;
    __device__ ListPoints(const int *h, const float4 *nd, int r, int x, int y, int nm, uint32_t *e)
        : head(h), nodes(nd), res(r), cx(x), cy(y), n_max(nm), err(e) {}
    template <class F>
    __device__ __forceinline__ void for_each(F f) const {
        int visited = 0;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy) {
                const int bx = cx + dx, by = cy + dy;
                if (!in_domain(bx, by, res)) continue;
                for (int j = head[bx * res + by]; j >= 0;) {
                    if (j >= n_max || ++visited > n_max) {
                        atomicOr(err, ERR_CONTACT_LIST);
                        return;
                    }
                    const float4 q = nodes[j];
                    f(q);
                    j = __float_as_int(q.w);
                }
            }
    }
};
// Fast pipeline: the cell's points in shared memory, split over the 32 lanes of a warp.  The
// reductions end with lane 0's result broadcast, so every lane holds the same bits and the
// fit's decisions are warp-uniform.
__device__ __forceinline__ float warp_sum_all(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}
struct WarpPoints {
    static constexpr bool kSymmetric = true;  // the fit sums the six distinct matrix entries
    const float4 *p;
    int n, lane;
    __device__ __forceinline__ bool writer() const { return lane == 0; }
    template <int N, class F>
    __device__ __forceinline__ void sum(float (&acc)[N], F f) const {
        float part[N];
#pragma unroll
        for (int k = 0; k < N; ++k) part[k] = 0.0f;
        for (int j = lane; j < n; j += 32) f(p[j], part);
#pragma unroll
        for (int k = 0; k < N; ++k) acc[k] += warp_sum_all(part[k]);
    }
    template <class F>
    __device__ __forceinline__ void max_min(float &mx, float &mn, F f) const {
        float a = -INFINITY, b = INFINITY;
        for (int j = lane; j < n; j += 32) f(p[j], a, b);
        for (int o = 16; o > 0; o >>= 1) {
            a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fminf(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        mx = fmaxf(mx, __shfl_sync(0xffffffffu, a, 0));
        mn = fminf(mn, __shfl_sync(0xffffffffu, b, 0));
    }
};

// fit_contact_normal_lr (grid/contact_normal.rs): logistic regression of the contact labels
// on position relative to the node, up to 15 Newton steps with a small ridge penalty.
template <class PTS>
__device__ bool fit_contact_normal(const PTS &pts, float2 node, float cell, bool pr, float2 &out) {
    float labels[2] = {0.0f, 0.0f};  // grip and rest points
    pts.sum(labels, [](const float4 &q, float (&a)[2]) {
        if (q.z > 0.0f) a[0] += 1.0f;
        if (q.z < 0.0f) a[1] += 1.0f;
    });
    if (!(labels[0] > 0.0f) || !(labels[1] > 0.0f)) return false;
    const float dx2 = cell * cell;
    const float penalty[3] = {1.0e-7f * dx2, 1.0e-7f * dx2, 0.0f};
    float beta[3] = {0.0f, 0.0f, 0.0f};
    bool have_prev = false;
    float2 prev = v2(0.0f, 0.0f);
    for (int it = 0; it < 15; ++it) {
        // one point's logistic term: its weights and residual at the current beta
        auto term = [&](const float4 &pt, float xp[3], float &sigma_sq, float &resid) {
            const float2 rel = vsub(v2(pt.x, pt.y), node);
            xp[0] = rel.x;
            xp[1] = rel.y;
            xp[2] = 1.0f;
            const float z = fclampf(xp[0] * beta[0] + xp[1] * beta[1] + xp[2] * beta[2], -40.0f, 40.0f);
            const float ez = em_exp(-z, pr);
            const float denom = 1.0f + ez;
            const float f = 2.0f / denom - 1.0f;
            const float sigma = 2.0f * ez / (denom * denom);
            sigma_sq = sigma * sigma;
            resid = sigma * (pt.z - f);
        };
        float m[3][3], rhs[3];
        if constexpr (PTS::kSymmetric) {
            float acc[9];  // m00 m01 m02 m11 m12 m22, then the right-hand side
#pragma unroll
            for (int k = 0; k < 9; ++k) acc[k] = 0.0f;
            pts.sum(acc, [&](const float4 &pt, float (&a)[9]) {
                float xp[3], sq, r;
                term(pt, xp, sq, r);
                a[0] += sq * xp[0] * xp[0];
                a[1] += sq * xp[0] * xp[1];
                a[2] += sq * xp[0] * xp[2];
                a[3] += sq * xp[1] * xp[1];
                a[4] += sq * xp[1] * xp[2];
                a[5] += sq * xp[2] * xp[2];
#pragma unroll
                for (int k = 0; k < 3; ++k) a[6 + k] += r * xp[k];
            });
            m[0][0] = acc[0];
            m[0][1] = m[1][0] = acc[1];
            m[0][2] = m[2][0] = acc[2];
            m[1][1] = acc[3];
            m[1][2] = m[2][1] = acc[4];
            m[2][2] = acc[5];
            for (int k = 0; k < 3; ++k) rhs[k] = acc[6 + k];
        } else {
            float acc[12];  // the 3 x 3 normal matrix (row major), then the right-hand side
#pragma unroll
            for (int k = 0; k < 12; ++k) acc[k] = 0.0f;
            pts.sum(acc, [&](const float4 &pt, float (&a)[12]) {
                float xp[3], sq, r;
                term(pt, xp, sq, r);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
#pragma unroll
                    for (int l = 0; l < 3; ++l) a[k * 3 + l] += sq * xp[k] * xp[l];
                    a[9 + k] += r * xp[k];
                }
            });
            for (int k = 0; k < 3; ++k) {
                for (int l = 0; l < 3; ++l) m[k][l] = acc[k * 3 + l];
                rhs[k] = acc[9 + k];
            }
        }
        for (int k = 0; k < 3; ++k) {
            m[k][k] += penalty[k];
            rhs[k] -= penalty[k] * beta[k];
        }
        float delta[3];
        if (!solve3x3(m, rhs, delta)) break;
        if (!isfinite(delta[0]) || !isfinite(delta[1]) || !isfinite(delta[2])) break;
        for (int k = 0; k < 3; ++k) beta[k] += delta[k];
        const float2 raw = v2(beta[0], beta[1]);
        if (vlen2(raw) <= F32_EPS || !vfinite(raw)) continue;
        const float2 n = normalize2(raw);
        if (have_prev && 1.0f - vdot(n, prev) < 1.0e-5f) {
            prev = n;
            break;
        }
        prev = n;
        have_prev = true;
    }
    if (!have_prev) return false;
    float means[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // grip sum, grip count, rest sum, rest count
    pts.sum(means, [&](const float4 &pt, float (&a)[4]) {
        if (pt.z > 0.0f) {
            a[0] += vdot(vsub(v2(pt.x, pt.y), node), prev);
            a[1] += 1.0f;
        }
        if (pt.z < 0.0f) {
            a[2] += vdot(vsub(v2(pt.x, pt.y), node), prev);
            a[3] += 1.0f;
        }
    });
    const float grip_mean = means[0] / (means[1] > 0.0f ? means[1] : 1.0f);
    const float rest_mean = means[2] / (means[3] > 0.0f ? means[3] : 1.0f);
    out = grip_mean < rest_mean ? v2(-prev.x, -prev.y) : prev;
    return true;
}

// apply_coulomb_wall (forces/boundary/mod.rs:60-76)
__device__ __forceinline__ void coulomb_wall(float2 &v, float2 n, float mu) {
    const float v_n = vdot(v, n);
    if (v_n >= 0.0f) return;
    const float normal_speed = fabsf(v_n);
    const float2 v_t = vsub(v, svmul(v_n, n));
    const float v_t_len = vlen(v_t);
    const float friction_impulse = mu * normal_speed;
    v = v_t_len > friction_impulse ? vmuls(v_t, (v_t_len - friction_impulse) / v_t_len) : v2(0.0f, 0.0f);
}

__device__ __forceinline__ float grip_mass_at(const GridView &g, int x, int y) {
    if (!in_domain(x, y, g.res)) return 0.0f;
    const float4 gr = g.acc_grip[cell_index(x, y, g.tpd)];
    return gr.w > 0.0f ? gr.x : 0.0f;
}

// Grid::resolve_contact (grid/contact.rs:254-391) for the grip cell (x, y) whose point
// cloud is `pts` (the writer of the set stores the result).
template <class PTS>
__device__ void contact_resolve_cell(const GridView &g, const DevConfig &cfg, const StepState *st, int x,
                                     int y, int ci, const float4 gr, const PTS &pts) {
    const float dt = st->sub_dt;
    const float vel_limit = cfg.cell / dt;
    const bool pr = cfg.precise_math != 0;
    const float MIN_MASS_FRACTION = 1.0e-6f;
    const float total_mass = g.grid_m[ci];
    const float2 v_cm = g.grid_v[ci];  // normalised, gravity, boundaries, clamp
    const float grip_mass = gr.x;
    const float2 grip_momentum = v2(gr.y, gr.z);
    // fast pipeline: a grip-only cell (w = 1) has no rest mass (finalize_field)
    const float rest_mass = (cfg.mf_fast && gr.w < 1.5f) ? 0.0f : total_mass - grip_mass;
    if (grip_mass <= MIN_MASS_FRACTION || rest_mass <= MIN_MASS_FRACTION) {
        if (pts.writer()) {
            g.grip_v[ci] = v_cm;
            g.rest_v[ci] = v_cm;
        }
        return;
    }
    const float2 v_grip = clamp_speed(vadd(vdivs(grip_momentum, grip_mass), vmuls(cfg.gravity, dt)), vel_limit);
    const float2 node = v2(static_cast<float>(x), static_cast<float>(y));
    float2 fit;
    bool have = fit_contact_normal(pts, node, cfg.cell, pr, fit) && vfinite(fit);
    if (!have) {  // grip_mass_gradient_normal (contact.rs:128-140)
        auto m = [&](int dx, int dy) { return grip_mass_at(g, x + dx, y + dy); };
        const float gx_ = (m(1, -1) + 2.0f * m(1, 0) + m(1, 1)) - (m(-1, -1) + 2.0f * m(-1, 0) + m(-1, 1));
        const float gy_ = (m(-1, 1) + 2.0f * m(0, 1) + m(1, 1)) - (m(-1, -1) + 2.0f * m(0, -1) + m(1, -1));
        const float2 grad = v2(gx_, gy_);
        if (vlen2(grad) > F32_EPS) {
            fit = normalize2(grad);
            have = true;
        }
    }
    float2 v_rel = vsub(v_grip, v_cm);
    if (!have) {
        if (pts.writer()) {
            g.grip_v[ci] = v_grip;
            g.rest_v[ci] = clamp_speed(vdivs(vsub(vmuls(v_cm, total_mass), vmuls(v_grip, grip_mass)), rest_mass),
                                       vel_limit);
        }
        return;
    }
    const float2 n = v2(-fit.x, -fit.y);
    if (cfg.grip_on) {  // DirectionalContactGrip::resolve (directional_grip.rs)
        const float2 tangent = v2(-n.y, n.x);
        const float v_t = vdot(v_rel, tangent);
        const float easy_t = vdot(cfg.grip_dir, tangent);
        coulomb_wall(v_rel, n, v_t * easy_t >= 0.0f ? cfg.grip_mu_easy : cfg.grip_mu_resist);
    } else {
        coulomb_wall(v_rel, n, cfg.contact_friction);
    }
    float max_grip_proj = -INFINITY, min_rest_proj = INFINITY;
    pts.max_min(max_grip_proj, min_rest_proj, [&](const float4 &pt, float &mx, float &mn) {
        const float proj = vdot(v2(pt.x, pt.y), n);
        if (pt.z > 0.0f) mx = fmaxf(mx, proj);
        else if (pt.z < 0.0f) mn = fminf(mn, proj);
    });
    if (isfinite(max_grip_proj) && isfinite(min_rest_proj)) {
        const float gap = min_rest_proj - max_grip_proj;
        if (gap < 0.0f) {
            const float CORRECTION_RATE = 2.0f;
            const float max_correction_speed = 0.5f * cfg.cell;
            const float correction_speed = fminf(CORRECTION_RATE * (-gap), max_correction_speed);
            const float v_n = vdot(v_rel, n);
            const float target_vn = -correction_speed;
            if (v_n > target_vn) v_rel = vadd(v_rel, vmuls(n, target_vn - v_n));
        }
    }
    if (!pts.writer()) return;
    const float2 v_grip_new = clamp_speed(vadd(v_cm, v_rel), vel_limit);
    const float2 total_momentum = vmuls(v_cm, total_mass);
    g.grip_v[ci] = v_grip_new;
    g.rest_v[ci] = clamp_speed(vdivs(vsub(total_momentum, vmuls(v_grip_new, grip_mass)), rest_mass), vel_limit);
}

inline int grid_blocks(const GridView &g) {
    return static_cast<int>((static_cast<long long>(g.res) * g.res + MF_THREADS - 1) / MF_THREADS);
}

}  // namespace
}  // namespace emerge
