// multifield.cu -- multi-field contact (Bardenhagen) and two-phase mixture coupling on the
// grid, after the grid update of a substep (spacetime/solver/step.rs:166-197).
//
// Compiled like the reference-order translation unit (-fmad=false, IEEE division and square
// root): scenes that use these fields run the reference-order pipeline, whose cell-sorted
// scatter records also give each contact cell its point cloud in particle index order.
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

// fit_contact_normal_lr (grid/contact_normal.rs): logistic regression of the contact labels
// on position relative to the node, up to 15 Newton steps with a small ridge penalty; the
// points are the cell's scatter records [lo, hi) in particle index order.
__device__ bool fit_contact_normal(const uint32_t *vals, const float4 *points, int lo, int hi,
                                   float2 node, float cell, bool pr, float2 &out) {
    bool has_grip = false, has_rest = false;
    for (int j = lo; j < hi; ++j) {
        const float c = points[vals[j]].z;
        has_grip = has_grip || c > 0.0f;
        has_rest = has_rest || c < 0.0f;
    }
    if (!has_grip || !has_rest) return false;
    const float dx2 = cell * cell;
    const float penalty[3] = {1.0e-7f * dx2, 1.0e-7f * dx2, 0.0f};
    float beta[3] = {0.0f, 0.0f, 0.0f};
    bool have_prev = false;
    float2 prev = v2(0.0f, 0.0f);
    for (int it = 0; it < 15; ++it) {
        float m[3][3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
        float rhs[3] = {0.0f, 0.0f, 0.0f};
        for (int j = lo; j < hi; ++j) {
            const float4 pt = points[vals[j]];
            const float2 rel = vsub(v2(pt.x, pt.y), node);
            const float xp[3] = {rel.x, rel.y, 1.0f};
            const float z = fclampf(xp[0] * beta[0] + xp[1] * beta[1] + xp[2] * beta[2], -40.0f, 40.0f);
            const float ez = em_exp(-z, pr);
            const float denom = 1.0f + ez;
            const float f = 2.0f / denom - 1.0f;
            const float sigma = 2.0f * ez / (denom * denom);
            const float sigma_sq = sigma * sigma;
            for (int k = 0; k < 3; ++k) {
                for (int l = 0; l < 3; ++l) m[k][l] += sigma_sq * xp[k] * xp[l];
                rhs[k] += sigma * (pt.z - f) * xp[k];
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
    float gs = 0.0f, rs = 0.0f;
    int gc = 0, rc = 0;
    for (int j = lo; j < hi; ++j) {
        const float4 pt = points[vals[j]];
        if (pt.z > 0.0f) {
            gs += vdot(vsub(v2(pt.x, pt.y), node), prev);
            gc += 1;
        }
    }
    for (int j = lo; j < hi; ++j) {
        const float4 pt = points[vals[j]];
        if (pt.z < 0.0f) {
            rs += vdot(vsub(v2(pt.x, pt.y), node), prev);
            rc += 1;
        }
    }
    const float grip_mean = gs / static_cast<float>(gc > 0 ? gc : 1);
    const float rest_mean = rs / static_cast<float>(rc > 0 ? rc : 1);
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

// Grid::resolve_contact (grid/contact.rs:254-391) for every grip cell.
__global__ void k_contact_resolve(GridView g, DevConfig cfg, const StepState *st, const uint32_t *vals,
                                  const float4 *points) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    const float4 gr = g.acc_grip[ci];
    if (!(gr.w > 0.0f)) return;  // not in the grip field
    const float dt = st->sub_dt;
    const float vel_limit = cfg.cell / dt;
    const bool pr = cfg.precise_math != 0;
    const float MIN_MASS_FRACTION = 1.0e-6f;
    const float total_mass = g.grid_m[ci];
    const float2 v_cm = g.grid_v[ci];  // normalised, gravity, boundaries, clamp
    const float grip_mass = gr.x;
    const float2 grip_momentum = v2(gr.y, gr.z);
    const float rest_mass = total_mass - grip_mass;
    if (grip_mass <= MIN_MASS_FRACTION || rest_mass <= MIN_MASS_FRACTION) {
        g.grip_v[ci] = v_cm;
        g.rest_v[ci] = v_cm;
        return;
    }
    const float2 v_grip = clamp_speed(vadd(vdivs(grip_momentum, grip_mass), vmuls(cfg.gravity, dt)), vel_limit);
    const float2 node = v2(static_cast<float>(x), static_cast<float>(y));
    const int2 rr = g.rec_range[ci];
    float2 fit;
    bool have = fit_contact_normal(vals, points, rr.x, rr.y, node, cfg.cell, pr, fit) && vfinite(fit);
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
        g.grip_v[ci] = v_grip;
        g.rest_v[ci] = clamp_speed(vdivs(vsub(vmuls(v_cm, total_mass), vmuls(v_grip, grip_mass)), rest_mass),
                                   vel_limit);
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
    for (int j = rr.x; j < rr.y; ++j) {
        const float4 pt = points[vals[j]];
        const float proj = vdot(v2(pt.x, pt.y), n);
        if (pt.z > 0.0f) max_grip_proj = fmaxf(max_grip_proj, proj);
        else if (pt.z < 0.0f) min_rest_proj = fminf(min_rest_proj, proj);
    }
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
    const float2 v_grip_new = clamp_speed(vadd(v_cm, v_rel), vel_limit);
    const float2 total_momentum = vmuls(v_cm, total_mass);
    g.grip_v[ci] = v_grip_new;
    g.rest_v[ci] = clamp_speed(vdivs(vsub(total_momentum, vmuls(v_grip_new, grip_mass)), rest_mass), vel_limit);
}

__device__ __forceinline__ bool mixture_cell(const GridView &g, int ci) {
    return g.acc_sol[ci].w > 0.0f || g.acc_flu[ci].w > 0.0f;
}

// resolve_mixture_coupling (grid/mixture.rs:87-132): implicit Darcy drag per node.
__global__ void k_mix_drag(GridView g, DevConfig cfg, const StepState *st) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int ci = cell_index(static_cast<int>(k / g.res), static_cast<int>(k % g.res), g.tpd);
    if (!mixture_cell(g, ci)) return;
    const float2 total = g.grid_v[ci];
    const float4 s = g.acc_sol[ci], f = g.acc_flu[ci];
    const float m_s = s.w > 0.0f ? s.x : 0.0f, m_f = f.w > 0.0f ? f.x : 0.0f;
    if (cfg.mix_drag <= 0.0f || m_s <= 1.0e-6f || m_f <= 1.0e-6f) {
        g.sol_v[ci] = total;
        g.flu_v[ci] = total;
        return;
    }
    const float dt = st->sub_dt;
    const float2 v_s = vadd(vdivs(v2(s.y, s.z), m_s), vmuls(cfg.gravity, dt));
    const float2 v_f = vadd(vdivs(v2(f.y, f.z), m_f), vmuls(cfg.gravity, dt));
    const float a = dt * cfg.mix_drag / m_s;
    const float b = dt * cfg.mix_drag / m_f;
    const float det = 1.0f + a + b;
    g.sol_v[ci] = vdivs(vadd(svmul(1.0f + b, v_s), svmul(a, v_f)), det);
    g.flu_v[ci] = vdivs(vadd(svmul(b, v_s), svmul(1.0f + a, v_f)), det);
}

__device__ __forceinline__ float2 mix_v_or_zero(const GridView &g, const float2 *field, int x, int y) {
    if (!in_domain(x, y, g.res)) return v2(0.0f, 0.0f);
    const int ci = cell_index(x, y, g.tpd);
    return mixture_cell(g, ci) ? field[ci] : v2(0.0f, 0.0f);
}
__device__ __forceinline__ float cell_or_zero(const GridView &g, const float *field, int x, int y) {
    return in_domain(x, y, g.res) ? field[cell_index(x, y, g.tpd)] : 0.0f;  // zero outside the mixture
}

// project_mixture_incompressibility set-up (mixture.rs:150-209): volume fraction, phase
// mobilities, divergence residual of the drag-resolved velocities.
__global__ void k_mix_setup(GridView g, DevConfig cfg) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    if (!mixture_cell(g, ci)) return;
    const float MIN_MASS = 1.0e-6f;
    const float h = fmaxf(cfg.cell, 1.0e-6f);
    const float4 s = g.acc_sol[ci], f = g.acc_flu[ci];
    const float m_s = fmaxf(s.w > 0.0f ? s.x : 0.0f, 0.0f), m_f = fmaxf(f.w > 0.0f ? f.x : 0.0f, 0.0f);
    const float n = m_s + m_f > MIN_MASS ? m_f / (m_s + m_f) : 0.0f;
    const float a_s = 1.0f / fmaxf(m_s, MIN_MASS);
    const float a_f = 1.0f / fmaxf(m_f, MIN_MASS);
    const float kk = (1.0f - n) * a_s + n * a_f;
    const float total_mass = fmaxf(m_s + m_f, MIN_MASS);
    const bool solid_sig = m_s / total_mass > 0.01f, fluid_sig = m_f / total_mass > 0.01f;
    const float vs_r = mix_v_or_zero(g, g.sol_v, x + 1, y).x, vs_l = mix_v_or_zero(g, g.sol_v, x - 1, y).x;
    const float vs_u = mix_v_or_zero(g, g.sol_v, x, y + 1).y, vs_d = mix_v_or_zero(g, g.sol_v, x, y - 1).y;
    const float div_vs = (vs_r - vs_l) / (2.0f * h) + (vs_u - vs_d) / (2.0f * h);
    const float vf_r = mix_v_or_zero(g, g.flu_v, x + 1, y).x, vf_l = mix_v_or_zero(g, g.flu_v, x - 1, y).x;
    const float vf_u = mix_v_or_zero(g, g.flu_v, x, y + 1).y, vf_d = mix_v_or_zero(g, g.flu_v, x, y - 1).y;
    const float div_vf = (vf_r - vf_l) / (2.0f * h) + (vf_u - vf_d) / (2.0f * h);
    g.mx_as[ci] = a_s;
    g.mx_af[ci] = a_f;
    g.mx_k[ci] = kk;
    g.mx_rhs[ci] = (1.0f - n) * div_vs + n * div_vf;
    g.mx_sig[ci] = static_cast<uint8_t>((solid_sig ? 1 : 0) | (fluid_sig ? 2 : 0));
}

__device__ __forceinline__ float face_k(float ki, float kj) {
    return ki + kj > 1.0e-12f ? 2.0f * ki * kj / (ki + kj) : 0.0f;
}

// One Jacobi sweep of the mixture pressure (mixture.rs:226-249): src -> dst.
__global__ void k_mix_jacobi(GridView g, DevConfig cfg, const float *src, float *dst) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    if (!mixture_cell(g, ci)) return;
    const float h = fmaxf(cfg.cell, 1.0e-6f);
    const float k_i = g.mx_k[ci];
    const float k_r = face_k(k_i, cell_or_zero(g, g.mx_k, x + 1, y));
    const float k_l = face_k(k_i, cell_or_zero(g, g.mx_k, x - 1, y));
    const float k_u = face_k(k_i, cell_or_zero(g, g.mx_k, x, y + 1));
    const float k_d = face_k(k_i, cell_or_zero(g, g.mx_k, x, y - 1));
    const float k_sum = fmaxf(k_r + k_l + k_u + k_d, 1.0e-9f);
    const float p_r = cell_or_zero(g, src, x + 1, y), p_l = cell_or_zero(g, src, x - 1, y);
    const float p_u = cell_or_zero(g, src, x, y + 1), p_d = cell_or_zero(g, src, x, y - 1);
    const float weighted = k_r * p_r + k_l * p_l + k_u * p_u + k_d * p_d;
    dst[ci] = (weighted - h * h * g.mx_rhs[ci]) / k_sum;
}

// Pressure-gradient correction of the significant phases (mixture.rs:251-274).
__global__ void k_mix_correct(GridView g, DevConfig cfg, const float *p) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    if (!mixture_cell(g, ci)) return;
    const float h = fmaxf(cfg.cell, 1.0e-6f);
    const float p_r = cell_or_zero(g, p, x + 1, y), p_l = cell_or_zero(g, p, x - 1, y);
    const float p_u = cell_or_zero(g, p, x, y + 1), p_d = cell_or_zero(g, p, x, y - 1);
    const float2 grad_p = v2((p_r - p_l) / (2.0f * h), (p_u - p_d) / (2.0f * h));
    const uint8_t sig = g.mx_sig[ci];
    if (sig & 1) g.sol_v[ci] = vsub(g.sol_v[ci], svmul(g.mx_as[ci], grad_p));
    if (sig & 2) g.flu_v[ci] = vsub(g.flu_v[ci], svmul(g.mx_af[ci], grad_p));
}

int grid_blocks(const GridView &g) {
    return static_cast<int>((static_cast<long long>(g.res) * g.res + MF_THREADS - 1) / MF_THREADS);
}

}  // namespace

void launch_contact_resolve(const StepLaunch &L, const uint32_t *vals, const float4 *points) {
    k_contact_resolve<<<grid_blocks(L.g), MF_THREADS, 0, L.stream>>>(L.g, L.cfg, L.st, vals, points);
}

// The mixture pressure arrays hold zero outside the mixture cells (cleared before each
// substep's scatter), which is the reference's value for cells without a pressure entry.
void launch_mixture_resolve(const StepLaunch &L) {
    const int blocks = grid_blocks(L.g);
    k_mix_drag<<<blocks, MF_THREADS, 0, L.stream>>>(L.g, L.cfg, L.st);
    if (L.cfg.mix_drag <= 0.0f || L.cfg.mix_iters <= 0) return;
    k_mix_setup<<<blocks, MF_THREADS, 0, L.stream>>>(L.g, L.cfg);
    int cur = 0;
    for (int it = 0; it < L.cfg.mix_iters; ++it) {
        k_mix_jacobi<<<blocks, MF_THREADS, 0, L.stream>>>(L.g, L.cfg, L.g.mx_p[cur], L.g.mx_p[cur ^ 1]);
        cur ^= 1;
    }
    k_mix_correct<<<blocks, MF_THREADS, 0, L.stream>>>(L.g, L.cfg, L.g.mx_p[cur]);
}

}  // namespace emerge
