// multifield.cu -- multi-field contact (Bardenhagen) and two-phase mixture coupling on the
// grid, after the grid update of a substep (spacetime/solver/step.rs:166-197).
//
// Compiled like the reference-order translation unit (-fmad=false, IEEE division and square
// root): the reference-order contact resolve, whose cell-sorted scatter records give each
// contact cell its point cloud in particle index order, the mixture kernels and the fast
// pipeline's per-substep clear.  The fast pipeline's contact kernels are in
// multifield_fast.cu.
#include "multifield.cuh"

namespace emerge {

namespace {

// Reference order: the points are the cell's sorted scatter records.
__global__ void k_contact_resolve(GridView g, DevConfig cfg, const StepState *st, const uint32_t *vals,
                                  const float4 *points) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    const float4 gr = g.acc_grip[ci];
    if (!(gr.w > 0.0f)) return;  // not in the grip field
    const int2 rr = g.rec_range[ci];
    contact_resolve_cell(g, cfg, st, x, y, ci, gr, RecordPoints(vals, points, rr.x, rr.y));
}

// Start of a fast-pipeline substep (Grid::clear, grid/mod.rs:163-176): the finished field
// sums, the pressure scratch, the interface count, and the point lists the coming particle
// pass fills.
__global__ void k_multi_clear(GridView g, DevConfig cfg, StepState *st) {
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k == 0) st->n_iface = 0u;
    if (k >= static_cast<long long>(g.res) * g.res) return;
    const int x = static_cast<int>(k / g.res), y = static_cast<int>(k % g.res);
    const int ci = cell_index(x, y, g.tpd);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (cfg.mf_fields & 1) {
        g.acc_grip[ci] = zero;
        g.chead[st->acc_slot][k] = -1;
    }
    if (cfg.mf_fields & 2) {
        g.acc_sol[ci] = zero;
        g.acc_flu[ci] = zero;
        if (cfg.mix_drag > 0.0f && cfg.mix_iters > 0) {
            g.mx_k[ci] = 0.0f;
            g.mx_p[0][ci] = 0.0f;
            g.mx_p[1][ci] = 0.0f;
        }
    }
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

}  // namespace

void launch_contact_resolve(const StepLaunch &L, const uint32_t *vals, const float4 *points) {
    k_contact_resolve<<<grid_blocks(L.g), MF_THREADS, 0, L.stream>>>(L.g, L.cfg, L.st, vals, points);
}

void launch_multi_clear(const StepLaunch &L) {
    k_multi_clear<<<grid_blocks(L.g), MF_THREADS, 0, L.stream>>>(L.g, L.cfg, L.st);
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
