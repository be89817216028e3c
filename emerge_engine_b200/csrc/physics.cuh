// physics.cuh -- per-particle MLS-MPM math on the device.
//
// Each function restates one reference item (path:line inside the reference
// crate M1thieu/emerge-engine) in f32, in the reference's expression order.
// Translation units including this header are compiled with -fmad=false so
// a*b+c is never contracted into an FMA (the Rust reference never contracts),
// and with IEEE division/sqrt (nvcc defaults).  exp/log/sin/sinh/pow go through
// em_* below: either CUDA's single-precision functions (fast path) or a double
// evaluation rounded once to f32 (precise path, on in the reference-order mode),
// which agrees with glibc's f32 results in nearly all cases.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/emerge_cuda.h"

namespace emerge {

constexpr float F32_EPS = 1.1920929e-7f;     // f32::EPSILON
constexpr float KERNEL_D_INVERSE = 4.0f;     // spacetime/solver/config.rs:22
constexpr float MIN_J = 1e-6f;               // matter/materials/utils.rs:11
constexpr float LOG_CLAMP = 1e-10f;          // matter/materials/utils.rs:6

enum Model : uint32_t {
    M_FALLBACK = 0, M_FLUID = 1, M_NEOHOOKEAN = 2, M_COROTATED = 3, M_SNOW = 4,
    M_DRUCKER_PRAGER = 5, M_VON_MISES = 6, M_RANKINE = 7, M_DP_MUI = 8,
    M_VISCOELASTIC = 9, M_NACC = 10, M_GRANULAR_FLUID = 11
};

struct M2 { float2 xa, ya; };  // glam Mat2: columns x_axis, y_axis

#define EM_HD __host__ __device__ __forceinline__

EM_HD float2 v2(float x, float y) { return make_float2(x, y); }
EM_HD float2 vadd(float2 a, float2 b) { return v2(a.x + b.x, a.y + b.y); }
EM_HD float2 vsub(float2 a, float2 b) { return v2(a.x - b.x, a.y - b.y); }
EM_HD float2 vmulv(float2 a, float2 b) { return v2(a.x * b.x, a.y * b.y); }
EM_HD float2 vmuls(float2 a, float s) { return v2(a.x * s, a.y * s); }
EM_HD float2 svmul(float s, float2 a) { return v2(s * a.x, s * a.y); }
EM_HD float2 vdivs(float2 a, float s) { return v2(a.x / s, a.y / s); }
EM_HD float2 splat(float s) { return v2(s, s); }
EM_HD float vdot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
EM_HD float vlen(float2 a) { return sqrtf(vdot(a, a)); }
EM_HD float vlen2(float2 a) { return vdot(a, a); }
EM_HD bool vfinite(float2 a) { return isfinite(a.x) && isfinite(a.y); }
EM_HD float2 vabs2(float2 a) { return v2(fabsf(a.x), fabsf(a.y)); }
EM_HD float2 vmax2(float2 a, float2 b) { return v2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
EM_HD float2 vmin2(float2 a, float2 b) { return v2(fminf(a.x, b.x), fminf(a.y, b.y)); }
// glam Vec2::clamp: self.max(min).min(max)
EM_HD float2 vclamp2(float2 a, float2 lo, float2 hi) { return vmin2(vmax2(a, lo), hi); }
// f32::clamp keeps NaN
EM_HD float fclampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
// IEEE-rounded square root and division whatever the translation unit's -prec-sqrt /
// -prec-div flags.  The fast path is compiled with approximate (2-ulp) division and square
// root; the SVD, the polar decomposition and the return mappings use these instead, because
// their yield decisions amplify a last-bit difference over tens of substeps (measured on the
// 160k-particle granular scene over one frame: per-particle velocity error against the
// oracle, median 3.3e-5 with the approximate operations there and 2.2e-7 with these).  In
// the reference-order translation units (IEEE flags) they are the plain operators.
#ifdef __CUDA_ARCH__
EM_HD float esqrt(float x) { return __fsqrt_rn(x); }
EM_HD float ediv(float a, float b) { return __fdiv_rn(a, b); }
#else
EM_HD float esqrt(float x) { return sqrtf(x); }
EM_HD float ediv(float a, float b) { return a / b; }
#endif
EM_HD float evlen(float2 a) { return esqrt(vdot(a, a)); }
EM_HD float2 evdivs(float2 a, float s) { return v2(ediv(a.x, s), ediv(a.y, s)); }

// glam normalize_or_zero
EM_HD float2 normalize_or_zero(float2 a) {
    float rcp = ediv(1.0f, evlen(a));
    if (isfinite(rcp) && rcp > 0.0f) return vmuls(a, rcp);
    return v2(0.0f, 0.0f);
}

EM_HD M2 m2(float2 a, float2 b) { M2 r; r.xa = a; r.ya = b; return r; }
EM_HD M2 mident() { return m2(v2(1.0f, 0.0f), v2(0.0f, 1.0f)); }
EM_HD M2 mzero() { return m2(v2(0.0f, 0.0f), v2(0.0f, 0.0f)); }
EM_HD M2 mdiag(float2 d) { return m2(v2(d.x, 0.0f), v2(0.0f, d.y)); }
EM_HD M2 madd(M2 a, M2 b) { return m2(vadd(a.xa, b.xa), vadd(a.ya, b.ya)); }
EM_HD M2 msub(M2 a, M2 b) { return m2(vsub(a.xa, b.xa), vsub(a.ya, b.ya)); }
EM_HD M2 mscale(M2 a, float s) { return m2(vmuls(a.xa, s), vmuls(a.ya, s)); }
EM_HD M2 smscale(float s, M2 a) { return m2(svmul(s, a.xa), svmul(s, a.ya)); }
EM_HD float2 mv(M2 a, float2 v) { return vadd(vmuls(a.xa, v.x), vmuls(a.ya, v.y)); }
EM_HD M2 mm(M2 a, M2 b) { return m2(mv(a, b.xa), mv(a, b.ya)); }
EM_HD M2 mtrans(M2 a) { return m2(v2(a.xa.x, a.ya.x), v2(a.xa.y, a.ya.y)); }
EM_HD float mdet(M2 a) { return a.xa.x * a.ya.y - a.ya.x * a.xa.y; }
EM_HD bool mfinite(M2 a) { return vfinite(a.xa) && vfinite(a.ya); }
EM_HD M2 m_from4(float4 f) { return m2(v2(f.x, f.y), v2(f.z, f.w)); }
EM_HD float4 m_to4(M2 a) { return make_float4(a.xa.x, a.xa.y, a.ya.x, a.ya.y); }

// Rust `f32 as i32` (saturating, NaN -> 0); cvt.rzi.s32.f32 has the same semantics.
EM_HD int f2i(float f) { return static_cast<int>(f); }

// Transcendentals.  `pr` (precise) evaluates in double and rounds once to f32: the
// correctly rounded result in all but vanishingly rare cases, which is what glibc's
// f32 functions (called by the Rust reference) return in nearly all cases.  With
// `pr` false the single-precision CUDA functions are used.
EM_HD float em_exp(float x, bool pr) { return pr ? static_cast<float>(exp(static_cast<double>(x))) : expf(x); }
EM_HD float em_log(float x, bool pr) { return pr ? static_cast<float>(log(static_cast<double>(x))) : logf(x); }
EM_HD float em_sin(float x, bool pr) { return pr ? static_cast<float>(sin(static_cast<double>(x))) : sinf(x); }
EM_HD float em_sinh(float x, bool pr) { return pr ? static_cast<float>(sinh(static_cast<double>(x))) : sinhf(x); }
EM_HD float em_pow(float x, float y, bool pr) {
    if (pr) return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
#if defined(EMERGE_FAST_TU)
    // Fast path only: small integer exponents (the Tait equation of state's gamma = 7) by
    // binary exponentiation, a few multiplies instead of a log/exp evaluation.
    if (y == floorf(y) && fabsf(y) <= 16.0f) {
        int e = static_cast<int>(fabsf(y));
        float r = 1.0f, b = x;
        while (e) {
            if (e & 1) r *= b;
            b *= b;
            e >>= 1;
        }
        return y < 0.0f ? 1.0f / r : r;
    }
#endif
    return powf(x, y);
}

// axis_weights (spacetime/grid/kernel.rs:20-25)
EM_HD void axis_weights(float d, float w[3]) {
    float a = 0.5f - d;
    float b = 0.5f + d;
    w[0] = 0.5f * (a * a);
    w[1] = 0.75f - d * d;
    w[2] = 0.5f * (b * b);
}

// quadratic_weights (spacetime/grid/kernel.rs:10-18)
struct QW { int bx, by; float wx[3], wy[3]; };
EM_HD QW quadratic_weights(float2 p) {
    QW q;
    q.bx = f2i(floorf(p.x));
    q.by = f2i(floorf(p.y));
    float dx = (p.x - static_cast<float>(q.bx)) - 0.5f;
    float dy = (p.y - static_cast<float>(q.by)) - 0.5f;
    axis_weights(dx, q.wx);
    axis_weights(dy, q.wy);
    return q;
}

// ---------------------------------------------------------------- svd / polar
EM_HD float2 orthogonal_complement(float2 v) {  // materials/svd.rs:81-85
    float2 perp = v2(-v.y, v.x);
    float len = evlen(perp);
    if (len > 1e-10f) return evdivs(perp, len);
    return v2(1.0f, 0.0f);
}

// svd2 (matter/materials/svd.rs:14-76): F = U diag(sigma) Vt, det U = det V = +1,
// reflection carried by a negative sigma.y.
EM_HD void svd2(M2 f, M2 &u_out, float2 &sigma_out, M2 &vt_out) {
    float f00 = f.xa.x, f10 = f.xa.y, f01 = f.ya.x, f11 = f.ya.y;
    float c00 = f00 * f00 + f10 * f10;
    float c01 = f00 * f01 + f10 * f11;
    float c11 = f01 * f01 + f11 * f11;
    float mean = (c00 + c11) * 0.5f;
    float half_diff = (c00 - c11) * 0.5f;
    float disc = esqrt(half_diff * half_diff + c01 * c01);
    float lambda1 = mean + disc;
    float lambda2 = mean - disc;
    float2 v1;
    if (fabsf(c01) > 1e-10f * fmaxf(c00 + c11, 1e-30f)) {
        float2 raw = v2(c01, lambda1 - c00);
        v1 = evdivs(raw, evlen(raw));
    } else {
        v1 = (c00 >= c11) ? v2(1.0f, 0.0f) : v2(0.0f, 1.0f);
    }
    float2 vv2 = v2(-v1.y, v1.x);
    M2 vt = mtrans(m2(v1, vv2));
    float2 sigma = v2(esqrt(fmaxf(lambda1, 0.0f)), esqrt(fmaxf(lambda2, 0.0f)));
    float2 fv1 = mv(f, v1);
    float2 fv2 = mv(f, vv2);
    float2 u1 = (sigma.x > 1e-10f) ? evdivs(fv1, sigma.x) : orthogonal_complement(fv2);
    float2 u2 = (sigma.y > 1e-10f) ? evdivs(fv2, sigma.y) : orthogonal_complement(u1);
    M2 u = m2(u1, u2);
    if (mdet(u) < 0.0f) {
        u.ya = v2(-u.ya.x, -u.ya.y);
        sigma.y = -sigma.y;
    }
    u_out = u;
    sigma_out = sigma;
    vt_out = vt;
}

// polar_decomposition_2d (matter/materials/utils.rs:129-138)
EM_HD M2 polar(M2 f) {
    float x = f.xa.x + f.ya.y;
    float y = f.xa.y - f.ya.x;
    float norm = esqrt(x * x + y * y);
    if (norm > F32_EPS) return m2(evdivs(v2(x, y), norm), evdivs(v2(-y, x), norm));
    return mident();
}

// elastic_wave_dt (matter/materials/utils.rs:145-163)
EM_HD float elastic_wave_dt(float lambda, float mu, float hardening, float density,
                            float min_density, float cell_width, float material_cfl) {
    float rho = fmaxf(density, min_density);
    float modulus = fmaxf((lambda + 2.0f * mu) * hardening, 0.0f);
    if (modulus <= F32_EPS) return INFINITY;
    float c = sqrtf(modulus / rho);
    if (c <= F32_EPS) return INFINITY;
    return material_cfl * cell_width / c;
}

// ---------------------------------------------------------------- material view
// Device view of one MaterialParams slot.  The fields each model reads follow
// that model's params() packing (elastic.rs:275-288, fluid.rs:209-226,
// sand.rs:321-343, snow.rs:178-191, nacc.rs:300-314).  Constructor-only fields
// that params() does not carry are fixed at the reference constructors' values:
// NeoHookean min_density 1e-6 (elastic.rs:55), Fluid min_density/min_volume 1e-6
// (fluid.rs:60-61), DP volume_correction 1.0 (sand.rs:89), NACC min_density 1e-6
// (nacc.rs:71) and hardening_enabled = hardening_factor > 0 (nacc.rs:70).
typedef emerge_material_params MatP;

EM_HD float nacc_kappa(const MatP &m) { return m.lambda + m.mu; }  // inverse of nacc.rs:304

// DruckerPragerMaterial::alpha (sand.rs:135-141); dp_h0..3 = phi0, h1, h2, phi_r
EM_HD float dp_alpha(const MatP &m, float q, bool pr) {
    float phi = m.dp_h0 + (m.dp_h1 * q - m.dp_h3) * em_exp(-m.dp_h2 * q, pr);
    float s = em_sin(phi, pr);
    return ediv(sqrtf(2.0f / 3.0f) * (2.0f * s), 3.0f - s);
}

// DruckerPragerMaterial::project (sand.rs:156-194); cohesion in stretch_limit (sand.rs:335)
EM_HD bool dp_project(const MatP &m, float2 sigma_in, float lvs, float q, float2 &out,
                      float &dq, bool pr) {
    float2 sigma = vmax2(vabs2(sigma_in), splat(LOG_CLAMP));
    float2 eps = v2(em_log(sigma.x, pr) + lvs * 0.5f, em_log(sigma.y, pr) + lvs * 0.5f);
    float trace = eps.x + eps.y;
    float2 dev = vsub(eps, splat(trace * 0.5f));
    float dev_norm = evlen(dev);
    if (dev_norm == 0.0f || trace > 0.0f) {
        out = v2(1.0f, 1.0f);
        dq = dev_norm;
        return true;
    }
    float ratio = ediv(m.lambda + m.mu, m.mu);
    float alpha = dp_alpha(m, q, pr);
    float cohesion_term = ediv(m.stretch_limit, 2.0f * m.mu);
    float gamma = dev_norm + ratio * trace * alpha - cohesion_term;
    if (gamma <= 0.0f) return false;
    float2 h = vsub(eps, svmul(gamma, evdivs(dev, dev_norm)));
    out = v2(em_exp(h.x, pr), em_exp(h.y, pr));
    dq = gamma;
    return true;
}

EM_HD M2 reconstruct(M2 u, float2 s, M2 vt) { return mm(mm(u, mdiag(s)), vt); }

// hencky_strains (matter/materials/utils.rs:58-61)
EM_HD float2 hencky(float2 sigma, bool pr) {
    float2 s = vmax2(vabs2(sigma), splat(LOG_CLAMP));
    return v2(em_log(s.x, pr), em_log(s.y, pr));
}

// stress_to_hencky (matter/materials/utils.rs:76-83)
EM_HD float2 stress_to_hencky(float2 tau, float lambda, float mu) {
    float det = 4.0f * mu * (mu + lambda);
    float a = 2.0f * mu + lambda;
    return v2((a * tau.x - lambda * tau.y) / det, (a * tau.y - lambda * tau.x) / det);
}

// Corotated linear-elastic stress 2 mu (F - R) F^T + lambda (J - 1) J I with moduli already
// scaled (corotated.rs:61-77, von_mises.rs:94-102, rankine.rs, sand_mui.rs kirchhoff_stress).
EM_HD M2 corotated_stress(M2 f, float mu, float lambda) {
    float j = mdet(f);
    if (j <= MIN_J) return mzero();
    M2 r = polar(f);
    return madd(mm(smscale(2.0f * mu, msub(f, r)), mtrans(f)),
                smscale(lambda * (j - 1.0f) * j, mident()));
}

// Bingham fluid (bingham.rs): MaterialParams carries the yield stress in compression_limit
// (bingham.rs params()), so a Fluid slot with compression_limit > 0 is a Bingham fluid.
// critical_shear_rate is the constructor's 1e-4 (bingham.rs new()).
EM_HD bool is_bingham(const MatP &m) { return m.model == M_FLUID && m.compression_limit > 0.0f; }

// NaccMaterial::project (nacc.rs:129-223).  params(): hardening_exponent = xi,
// compression_limit = beta, stretch_limit = M (nacc.rs:309-311).
// NaccMaterial::project's trial quantities (nacc.rs:129-170), in its expression order, and
// the branch they select: 0 elastic, 1 the tension cap (p_tr > p0), 2 the compression cap
// (p_tr < -beta p0), 3 the ellipse (the smooth plastic branch).
struct NaccTrial {
    float2 sv, sv_sq, s_tr;
    float sv_sq_trace, p0, j_e_tr, p_tr, y0, y1, y;
    int branch;
};
EM_HD NaccTrial nacc_trial(const MatP &m, float2 sv, float alpha, bool pr) {
    NaccTrial t;
    const float kappa = nacc_kappa(m);
    const float xi = m.hardening_exponent, beta = m.compression_limit, mm_ = m.stretch_limit;
    t.sv = sv;
    t.sv_sq = vmulv(sv, sv);
    t.sv_sq_trace = t.sv_sq.x + t.sv_sq.y;
    t.p0 = kappa * (1.0e-5f + em_sinh(xi * fmaxf(-alpha, 0.0f), pr));
    t.j_e_tr = fmaxf(sv.x * sv.y, 1.0e-6f);
    t.s_tr = svmul(m.mu * ediv(1.0f, t.j_e_tr), vsub(t.sv_sq, splat(t.sv_sq_trace * 0.5f)));
    const float psi_kappa = kappa * 0.5f * (t.j_e_tr - ediv(1.0f, t.j_e_tr));
    t.p_tr = -psi_kappa * t.j_e_tr;
    t.y0 = (1.0f + 2.0f * beta) * 2.0f;
    t.y1 = mm_ * mm_ * (t.p_tr + beta * t.p0) * (t.p_tr - t.p0);
    const float s_norm_sq = t.s_tr.x * t.s_tr.x + t.s_tr.y * t.s_tr.y;
    t.y = t.y0 * s_norm_sq + t.y1;
    if (t.p_tr > t.p0) t.branch = 1;
    else if (t.p_tr < -beta * t.p0) t.branch = 2;
    else if (t.y < 1.0e-4f) t.branch = 0;
    else t.branch = 3;
    return t;
}

// The projection from F's SVD (u, sv, vt) and its trial quantities (nacc.rs:171-223).
EM_HD void nacc_project_t(const MatP &m, M2 f, M2 u, M2 vt, const NaccTrial &t, float alpha, M2 &f_out,
                          float &alpha_out, bool pr) {
    const float kappa = nacc_kappa(m);
    const float xi = m.hardening_exponent, beta = m.compression_limit, mm_ = m.stretch_limit;
    const bool hard = xi > 0.0f;
    const float p0 = t.p0, p_tr = t.p_tr, j_e_tr = t.j_e_tr;
    if (t.branch == 1) {
        float j_n1 = sqrtf(fmaxf(-2.0f * p0 / kappa + 1.0f, 1.0e-8f));
        float sv_new = em_pow(j_n1, 0.5f, pr);
        if (hard) alpha += em_log(j_e_tr / j_n1, pr);
        f_out = reconstruct(u, splat(sv_new), vt);
        alpha_out = alpha;
        return;
    }
    if (t.branch == 2) {
        float j_n1 = sqrtf(fmaxf(2.0f * beta * p0 / kappa + 1.0f, 1.0e-8f));
        float sv_new = em_pow(j_n1, 0.5f, pr);
        if (hard) alpha += em_log(j_e_tr / j_n1, pr);
        f_out = reconstruct(u, splat(sv_new), vt);
        alpha_out = alpha;
        return;
    }
    if (t.branch == 0) {
        f_out = f;
        alpha_out = alpha;
        return;
    }
    const float2 s_tr = t.s_tr;
    if (hard && p0 > 1.0e-4f && p_tr < p0 - 1.0e-4f && p_tr > -beta * p0 + 1.0e-4f) {
        float p_c = (1.0f - beta) * p0 * 0.5f;
        float q_tr = sqrtf(2.0f) * vlen(s_tr);
        float2 dir = normalize_or_zero(v2(p_c - p_tr, -q_tr));
        float c = mm_ * mm_ * (p_c + beta * p0) * (p_c - p0);
        float b = mm_ * mm_ * dir.x * (2.0f * p_c - p0 + beta * p0);
        float a = mm_ * mm_ * dir.x * dir.x + (1.0f + 2.0f * beta) * dir.y * dir.y;
        float discr = sqrtf(fmaxf(b * b - 4.0f * a * c, 0.0f));
        float l1 = (-b + discr) / (2.0f * a);
        float l2 = (-b - discr) / (2.0f * a);
        float p1 = p_c + l1 * dir.x;
        float p2 = p_c + l2 * dir.x;
        float p_x = ((p_tr - p_c) * (p1 - p_c) > 0.0f) ? p1 : p2;
        float j_e_x = sqrtf(fmaxf(fabsf(-2.0f * p_x / kappa + 1.0f), 1.0e-8f));
        if (j_e_x > 1.0e-4f) alpha += em_log(j_e_tr / j_e_x, pr);
    }
    float scale = esqrt(fmaxf(ediv(-t.y1, fmaxf(t.y0, 1.0e-10f)), 0.0f)) * ediv(j_e_tr, m.mu);
    float2 b_n1 = vadd(svmul(scale, normalize_or_zero(s_tr)), splat(t.sv_sq_trace / 2.0f));
    float2 sv_new = v2(esqrt(fmaxf(b_n1.x, 1.0e-8f)), esqrt(fmaxf(b_n1.y, 1.0e-8f)));
    f_out = reconstruct(u, sv_new, vt);
    alpha_out = alpha;
}

// The projection given F's SVD (u, sv, vt), as computed by svd2.
EM_HD void nacc_project_sv(const MatP &m, M2 f, M2 u, float2 sv, M2 vt, float alpha, M2 &f_out,
                           float &alpha_out, bool pr) {
    nacc_project_t(m, f, u, vt, nacc_trial(m, sv, alpha, pr), alpha, f_out, alpha_out, pr);
}

EM_HD void nacc_project(const MatP &m, M2 f, float alpha, M2 &f_out, float &alpha_out, bool pr) {
    M2 u, vt;
    float2 sv;
    svd2(f, u, sv, vt);
    nacc_project_sv(m, f, u, sv, vt, alpha, f_out, alpha_out, pr);
}

// Kernels are specialised on the set of models present in a scene: MASK bit m set
// means ConstitutiveModel m is compiled in; other models' code is left out.
#define HAS_MODEL(mask, model) ((((mask) >> (model)) & 1u) != 0u)
constexpr unsigned ALL_MODELS = (1u << M_FALLBACK) | (1u << M_FLUID) | (1u << M_NEOHOOKEAN) |
                                (1u << M_SNOW) | (1u << M_DRUCKER_PRAGER) | (1u << M_NACC);
// Mask bits 12 and 13 are not ConstitutiveModel ids.  Bit 12 marks a scene with a Bingham
// fluid (a Fluid slot with compression_limit > 0); bit 13 a scene with force fields or
// ASFLIP.  Kernels instantiated without them leave those branches out.
constexpr uint32_t M_BINGHAM_BIT = 12;
constexpr uint32_t M_EXTRAS_BIT = 13;
// Every ConstitutiveModel id (materials/mod.rs:53-66) and both extra bits.  Kernels for
// scenes whose models all lie in ALL_MODELS keep the smaller instantiation.
constexpr unsigned FULL_MODELS = 0x3FFFu;

// Model-mask bits of one material slot.
EM_HD unsigned model_bits(const MatP &m) {
    return (1u << m.model) | (is_bingham(m) ? (1u << M_BINGHAM_BIT) : 0u);
}

// ---------------------------------------------------------------- particle view
// Registers of one particle while a kernel works on it.
struct PState {
    float2 x, v;
    M2 c, f;
    float mass, v0, vol, rho;
    uint32_t mat;
    float jp, h, q, lvs;
    float temperature, activation;
    float2 act_dir;
    uint32_t pinned;
};

// MaterialModel::kirchhoff_stress per model.
template <unsigned MASK = FULL_MODELS>
EM_HD M2 kirchhoff_stress(const MatP &m, const PState &p, bool pr) {
    const M2 f = p.f;
    switch (m.model) {
    case M_NEOHOOKEAN: {
        if constexpr (HAS_MODEL(MASK, M_NEOHOOKEAN)) {  // elastic.rs:180-255; damage rate in cohesion_coeff (elastic.rs:284)
        float j = mdet(f);
        if (j <= MIN_J) return mzero();
        float t_scale = 1.0f + m.thermal_expansion * p.temperature;
        float damage_scale = em_exp(-m.cohesion_coeff * p.q, pr);
        float mu = m.mu * t_scale * damage_scale;
        float lambda = m.lambda * t_scale * damage_scale;
        M2 b = mm(f, mtrans(f));
        float tr_b = b.xa.x + b.ya.y;
        M2 dev_b = msub(b, mdiag(splat(tr_b * 0.5f)));
        float k = lambda + mu;
        M2 dev_stress = smscale(mu / j, dev_b);
        M2 vol_stress = smscale(k * em_log(j, pr), mident());
        M2 viscous = mzero();
        if (m.dynamic_viscosity > 0.0f) {  // viscosity in dynamic_viscosity (elastic.rs:285)
            M2 sym = madd(p.c, mtrans(p.c));
            M2 d = mscale(sym, 0.5f);
            float d_trace = d.xa.x + d.ya.y;
            M2 d_dev = msub(d, mdiag(splat(d_trace * 0.5f)));
            viscous = smscale(m.dynamic_viscosity, d_dev);
        }
        return madd(madd(dev_stress, vol_stress), viscous);
    }
        return mzero();
    }
    case M_FLUID: {
        if constexpr (HAS_MODEL(MASK, M_FLUID)) {  // fluid.rs:135-191 (min_density 1e-6, fluid.rs:60)
        float density = fminf(fmaxf(p.rho, 1.0e-6f), m.rest_density * 2.0f);
        float pressure = fmaxf(
            m.eos_stiffness * (em_pow(density / m.rest_density, m.eos_power, pr) - 1.0f),
            m.pressure_floor);
        M2 stress = mdiag(splat(-pressure));
        if (HAS_MODEL(MASK, M_BINGHAM_BIT) && is_bingham(m)) {  // bingham.rs kirchhoff_stress
            M2 d = mscale(madd(p.c, mtrans(p.c)), 0.5f);
            float trace = d.xa.x + d.ya.y;
            M2 d_dev = msub(d, mdiag(splat(trace * 0.5f)));
            float dxx = d_dev.xa.x, dyy = d_dev.ya.y, dxy = d_dev.xa.y;
            float d_sq = dxx * dxx + dyy * dyy + 2.0f * dxy * dxy;
            float shear_rate = sqrtf(2.0f * d_sq);
            if (!(shear_rate < 1.0e-4f))
                stress = madd(stress, mscale(d_dev, m.compression_limit / shear_rate + m.dynamic_viscosity));
            if (m.surface_tension_coeff != 0.0f) {
                float j = f.xa.x * f.ya.y - f.xa.y * f.ya.x;
                stress = madd(stress, mdiag(splat(m.surface_tension_coeff * j)));
            }
            return stress;
        }
        float eff_visc = m.dynamic_viscosity;
        if (m.thermal_viscosity_coeff > 0.0f)
            eff_visc = m.dynamic_viscosity * em_exp(-m.thermal_viscosity_coeff * p.temperature, pr);
        M2 sym = madd(p.c, mtrans(p.c));
        float div_v = sym.xa.x + sym.ya.y;
        M2 strain_dev = msub(sym, mdiag(splat(div_v * 0.5f)));
        stress = madd(stress, smscale(eff_visc, strain_dev));
        if (m.bulk_viscosity > 0.0f)
            stress = madd(stress, mdiag(splat(m.bulk_viscosity * div_v * 0.5f)));
        if (m.surface_tension_coeff != 0.0f) {
            float j = f.xa.x * f.ya.y - f.xa.y * f.ya.x;
            stress = madd(stress, mdiag(splat(m.surface_tension_coeff * j)));
        }
        return stress;
    }
        return mzero();
    }
    case M_DRUCKER_PRAGER: {
        if constexpr (HAS_MODEL(MASK, M_DRUCKER_PRAGER)) {  // sand.rs:220-231
        float j = mdet(f);
        if (j <= MIN_J) return mzero();
        M2 r = polar(f);
        M2 a = mm(smscale(2.0f * m.mu, msub(f, r)), mtrans(f));
        M2 b = smscale(m.lambda * (j - 1.0f) * j, mident());
        return madd(a, b);
    }
        return mzero();
    }
    case M_SNOW: {
        if constexpr (HAS_MODEL(MASK, M_SNOW)) {  // snow.rs:109-136
        float j = mdet(f);
        if (j <= MIN_J) return mzero();
        M2 r = polar(f);
        float mu_eff = m.mu * p.h;
        float lambda_eff = m.lambda * p.h;
        M2 tau = madd(mm(smscale(2.0f * mu_eff, msub(f, r)), mtrans(f)),
                      smscale(lambda_eff * (j - 1.0f) * j, mident()));
        if (m.cohesion_coeff > 0.0f && p.jp < 1.0f && j > 1.0f)
            tau = madd(tau, smscale(m.cohesion_coeff * p.jp * (j - 1.0f) * j, mident()));
        return tau;
    }
        return mzero();
    }
    case M_NACC: {
        if constexpr (HAS_MODEL(MASK, M_NACC)) {  // nacc.rs:236-249
        float j = fmaxf(mdet(f), MIN_J);
        M2 b = mm(f, mtrans(f));
        float tr_b = b.xa.x + b.ya.y;
        M2 dev_b = msub(b, mdiag(splat(tr_b * 0.5f)));
        M2 dev_stress = smscale(m.mu / j, dev_b);
        M2 vol_stress = smscale(nacc_kappa(m) * 0.5f * (j * j - 1.0f), mident());
        return madd(dev_stress, vol_stress);
    }
        return mzero();
    }
    case M_COROTATED: {
        if constexpr (HAS_MODEL(MASK, M_COROTATED)) {  // corotated.rs:61-77
            float t_scale = 1.0f + m.thermal_expansion * p.temperature;
            return corotated_stress(f, m.mu * p.h * t_scale, m.lambda * p.h * t_scale);
        }
        return mzero();
    }
    case M_VON_MISES:
        if constexpr (HAS_MODEL(MASK, M_VON_MISES)) return corotated_stress(f, m.mu, m.lambda);
        return mzero();
    case M_RANKINE:
        if constexpr (HAS_MODEL(MASK, M_RANKINE)) return corotated_stress(f, m.mu, m.lambda);
        return mzero();
    case M_DP_MUI:
        if constexpr (HAS_MODEL(MASK, M_DP_MUI)) return corotated_stress(f, m.mu, m.lambda);
        return mzero();
    case M_VISCOELASTIC: {
        if constexpr (HAS_MODEL(MASK, M_VISCOELASTIC)) {  // viscoelastic.rs kirchhoff_stress
        // params(): viscosity in dynamic_viscosity, j_min in volume_ratio_min
        float j = fminf(fmaxf(f.xa.x * f.ya.y - f.xa.y * f.ya.x, m.volume_ratio_min),
                        1.0f / m.volume_ratio_min);
        float t_scale = 1.0f + m.thermal_expansion * p.temperature;
        float mu = m.mu * t_scale;
        float lambda = m.lambda * t_scale;
        M2 b = mm(f, mtrans(f));
        M2 elastic = madd(smscale(mu, msub(b, mident())), mdiag(splat(lambda * em_log(j, pr))));
        M2 d = mscale(madd(p.c, mtrans(p.c)), 0.5f);
        float trace = d.xa.x + d.ya.y;
        M2 d_dev = msub(d, mdiag(splat(trace * 0.5f)));
        return madd(elastic, smscale(m.dynamic_viscosity * t_scale, d_dev));
    }
        return mzero();
    }
    case M_GRANULAR_FLUID: {
        if constexpr (HAS_MODEL(MASK, M_GRANULAR_FLUID)) {  // granular_fluid.rs kirchhoff_stress
        float j = fmaxf(mdet(f), MIN_J);
        float density = fmaxf(m.rest_density / j, 1.0e-6f);
        float ratio = fmaxf(density / fmaxf(m.rest_density, 1.0e-6f), 1.0e-6f);
        float pressure = fmaxf(m.eos_stiffness * (em_pow(ratio, m.eos_power, pr) - 1.0f),
                               m.pressure_floor);
        M2 r = polar(f);
        M2 coro = mm(smscale(2.0f * (m.mu * p.h), msub(f, r)), mtrans(f));
        float tr = coro.xa.x + coro.ya.y;
        M2 dev_coro = msub(coro, mdiag(splat(tr * 0.5f)));
        M2 lam_vol = smscale(m.lambda * p.h * (j - 1.0f) * j, mident());
        return madd(madd(mdiag(splat(-pressure)), dev_coro), lam_vol);
    }
        return mzero();
    }
    default:  // FallbackMaterial: zero stress (materials/mod.rs:362-366)
        return mzero();
    }
}

// MaterialModel::activation_scale: NeoHookean (elastic.rs:271-273), Corotated and
// Viscoelastic report active_stress_coeff; every other model 0 (materials/mod.rs:181-183).
EM_HD float activation_scale(const MatP &m) {
    return (m.model == M_NEOHOOKEAN || m.model == M_COROTATED || m.model == M_VISCOELASTIC)
               ? m.active_stress_coeff
               : 0.0f;
}

// combined_kirchhoff_stress (spacetime/transfer.rs:77-104): Viscoelastic's active stress
// is isotropic, every other model's follows the fibre direction.
template <unsigned MASK = FULL_MODELS>
EM_HD M2 combined_kirchhoff_stress(const MatP &m, const PState &p, bool pr) {
    M2 tau = kirchhoff_stress<MASK>(m, p, pr);
    float coeff = activation_scale(m);
    if (p.activation <= 0.0f || coeff <= 0.0f) return tau;
    M2 tau_active;
    float2 n = p.act_dir;
    float len_sq = vdot(n, n);
    if (m.model == M_VISCOELASTIC) {
        tau_active = mdiag(splat(p.activation * coeff));
    } else if (len_sq > F32_EPS) {
        float2 n0 = vdivs(n, sqrtf(len_sq));
        M2 n_outer = m2(vmuls(n0, n0.x), vmuls(n0, n0.y));
        M2 a_mat = mscale(n_outer, p.activation * coeff);
        tau_active = mm(mm(p.f, a_mat), mtrans(p.f));
    } else {
        tau_active = mdiag(splat(p.activation * coeff));
    }
    return madd(tau, tau_active);
}

// MaterialModel::stress_volume: Fluid and Bingham use max(volume, 1e-6) (fluid.rs:193-195,
// bingham.rs min_volume), GranularFluid max(volume, 1e-6) (granular_fluid.rs), every other
// model the initial volume (materials/mod.rs:114).
EM_HD float stress_volume(const MatP &m, const PState &p) {
    if (m.model == M_FLUID || m.model == M_GRANULAR_FLUID) return fmaxf(p.vol, 1.0e-6f);
    return p.v0;
}

// MaterialModel::timestep_bound
template <unsigned MASK = FULL_MODELS>
EM_HD float timestep_bound(const MatP &m, float density, float h, float cell, float mat_cfl,
                           float visc_cfl, bool pr) {
    switch (m.model) {
    case M_NEOHOOKEAN: {
        if constexpr (HAS_MODEL(MASK, M_NEOHOOKEAN)) {  // elastic.rs:290-327
        float elastic_dt = elastic_wave_dt(m.lambda, m.mu, 1.0f, density, 1.0e-6f, cell, mat_cfl);
        float viscous_dt = INFINITY;
        if (m.dynamic_viscosity > 0.0f) {
            float d = fmaxf(density, 1.0e-6f);
            float kinematic = m.dynamic_viscosity / d;
            if (kinematic > F32_EPS) viscous_dt = visc_cfl * cell * cell / kinematic;
        }
        return fminf(elastic_dt, viscous_dt);
    }
        return INFINITY;
    }
    case M_FLUID: {
        if constexpr (HAS_MODEL(MASK, M_FLUID)) {  // fluid.rs:228-259
        const float MIN_DENSITY_RATIO = 1.0e-6f;
        float d = fmaxf(density, 1.0e-6f);
        float ratio = fmaxf(d / fmaxf(m.rest_density, 1.0e-6f), MIN_DENSITY_RATIO);
        float dt_bound = INFINITY;
        float c2 = m.eos_stiffness * m.eos_power * em_pow(ratio, m.eos_power - 1.0f, pr) /
                   fmaxf(m.rest_density, 1.0e-6f);
        if (isfinite(c2) && c2 > F32_EPS) dt_bound = fminf(dt_bound, mat_cfl * cell / sqrtf(c2));
        if (m.dynamic_viscosity > 0.0f) {
            float kin = m.dynamic_viscosity / d;
            if (kin > F32_EPS) dt_bound = fminf(dt_bound, visc_cfl * cell * cell / kin);
        }
        return dt_bound;
    }
        return INFINITY;
    }
    case M_DRUCKER_PRAGER:  // sand.rs:345-362
        if constexpr (HAS_MODEL(MASK, M_DRUCKER_PRAGER))
            return elastic_wave_dt(m.lambda, m.mu, 1.0f, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_SNOW:  // snow.rs:193-211
        if constexpr (HAS_MODEL(MASK, M_SNOW))
            return elastic_wave_dt(m.lambda, m.mu, h, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_NACC: {
        if constexpr (HAS_MODEL(MASK, M_NACC)) {  // nacc.rs:279-298: lambda = kappa - mu = params().lambda
        return elastic_wave_dt(m.lambda, m.mu, h, density, 1.0e-6f, cell, mat_cfl);
    }
        return INFINITY;
    }
    case M_COROTATED:  // corotated.rs timestep_bound
        if constexpr (HAS_MODEL(MASK, M_COROTATED))
            return elastic_wave_dt(m.lambda, m.mu, h, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_GRANULAR_FLUID:  // granular_fluid.rs timestep_bound
        if constexpr (HAS_MODEL(MASK, M_GRANULAR_FLUID))
            return elastic_wave_dt(m.lambda, m.mu, h, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_VON_MISES:  // von_mises.rs:154-171
        if constexpr (HAS_MODEL(MASK, M_VON_MISES))
            return elastic_wave_dt(m.lambda, m.mu, 1.0f, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_RANKINE:  // rankine.rs timestep_bound
        if constexpr (HAS_MODEL(MASK, M_RANKINE))
            return elastic_wave_dt(m.lambda, m.mu, 1.0f, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_DP_MUI:  // sand_mui.rs timestep_bound
        if constexpr (HAS_MODEL(MASK, M_DP_MUI))
            return elastic_wave_dt(m.lambda, m.mu, 1.0f, density, MIN_J, cell, mat_cfl);
        return INFINITY;
    case M_VISCOELASTIC: {
        if constexpr (HAS_MODEL(MASK, M_VISCOELASTIC)) {  // viscoelastic.rs timestep_bound
        float elastic_dt = elastic_wave_dt(m.lambda, m.mu, 1.0f, density, 1.0e-6f, cell, mat_cfl);
        float viscous_dt = INFINITY;
        if (m.dynamic_viscosity > 0.0f) {
            float d = fmaxf(density, 1.0e-6f);
            float kinematic = m.dynamic_viscosity / d;
            if (kinematic > F32_EPS) viscous_dt = visc_cfl * cell * cell / kinematic;
        }
        return fminf(elastic_dt, viscous_dt);
    }
        return INFINITY;
    }
    default:
        return INFINITY;
    }
}

EM_HD void sync_volume_density(PState &p) {
    float j = fmaxf(mdet(p.f), MIN_J);
    float v = fmaxf(p.v0 * j, 1.0e-6f);
    p.vol = v;
    p.rho = ediv(p.mass, v);
}

// DP update after the return map decision (sand.rs:258-318).
EM_HD void dp_finish(const MatP &m, PState &p, M2 u, float2 sigma, M2 vt, bool projected,
                     float2 proj, float dq, bool pr) {
    float2 new_sigma = sigma;
    if (projected) {
        float2 sigma_abs = vmax2(vabs2(sigma), splat(LOG_CLAMP));
        float prev_det = sigma_abs.x * sigma_abs.y;
        float new_det = proj.x * proj.y;
        float diff = new_det - prev_det;
        float corrected = diff > 0.0f ? new_det : prev_det + diff * 1.0f;  // volume_correction 1.0
        p.lvs += em_log(prev_det, pr) - em_log(corrected, pr);
        float q_max = 5.0f / fmaxf(m.dp_h2, 1e-6f);
        p.q = fminf(p.q + dq, q_max);
        if (m.compression_limit > 0.0f) p.lvs += em_sin(m.compression_limit, pr) * dq;  // dilatancy
        new_sigma = proj;
    }
    new_sigma = vabs2(new_sigma);
    float j_new = new_sigma.x * new_sigma.y;
    if (j_new < m.volume_ratio_min)
        new_sigma = vmuls(new_sigma, esqrt(ediv(m.volume_ratio_min, fmaxf(j_new, 1e-6f))));
    p.f = mm(mm(u, mdiag(new_sigma)), vt);
    sync_volume_density(p);
}

// MaterialModel::update_particle
template <unsigned MASK = FULL_MODELS>
EM_HD void update_particle(const MatP &m, PState &p, float dt, bool pr) {
    switch (m.model) {
    case M_NEOHOOKEAN: {
        if constexpr (HAS_MODEL(MASK, M_NEOHOOKEAN)) {  // elastic.rs:262-269
        M2 fp_new = madd(mident(), smscale(dt, p.c));
        p.f = mm(fp_new, p.f);
        sync_volume_density(p);
        break;
    }
        break;
    }
    case M_FLUID: {
        if constexpr (HAS_MODEL(MASK, M_FLUID)) {  // fluid.rs:197-207; settling_damping in dp_h0 (fluid.rs:223)
        float j = fclampf(mdet(p.f), 0.5f, 2.0f);
        float s = sqrtf(j);
        p.f = m2(v2(s, 0.0f), v2(0.0f, s));
        if (m.dp_h0 > 0.0f) {
            float k = 1.0f - fminf(m.dp_h0 * dt, 0.5f);
            p.v.x *= k;
            p.v.y *= k;
        }
        break;
    }
        break;
    }
    case M_DRUCKER_PRAGER: {
        if constexpr (HAS_MODEL(MASK, M_DRUCKER_PRAGER)) {  // sand.rs:248-319
        M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        M2 u, vt;
        float2 sigma;
        svd2(f_trial, u, sigma, vt);
        float2 proj;
        float dq = 0.0f;
        bool projected = dp_project(m, sigma, p.lvs, p.q, proj, dq, pr);
        dp_finish(m, p, u, sigma, vt, projected, proj, dq, pr);
        break;
    }
        break;
    }
    case M_SNOW: {
        if constexpr (HAS_MODEL(MASK, M_SNOW)) {  // snow.rs:142-176
        M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        M2 u, vt;
        float2 sigma;
        svd2(f_trial, u, sigma, vt);
        float lo = 1.0f - m.compression_limit, hi = 1.0f + m.stretch_limit;
        float2 sigma_c = v2(fclampf(sigma.x, lo, hi), fclampf(sigma.y, lo, hi));
        float jp_new = ediv(p.jp * (sigma.x * sigma.y), sigma_c.x * sigma_c.y);
        p.jp = fclampf(jp_new, m.volume_ratio_min, m.volume_ratio_max);
        p.h = fclampf(em_exp(m.hardening_exponent * (1.0f - p.jp), pr), 0.1f, 7.0f);
        p.f = mm(mm(u, mdiag(sigma_c)), vt);
        sync_volume_density(p);
        break;
    }
        break;
    }
    case M_NACC: {
        if constexpr (HAS_MODEL(MASK, M_NACC)) {  // nacc.rs:255-269 (no F advance on the CPU path)
        M2 nf;
        float na;
        nacc_project(m, p.f, p.lvs, nf, na, pr);
        p.f = nf;
        p.lvs = na;
        float j = fmaxf(mdet(nf), MIN_J);
        float vol = p.v0 * j;
        p.vol = vol;
        p.rho = vol > MIN_J ? p.mass / vol : p.rho;
        break;
    }
        break;
    }
    case M_COROTATED:       // corotated.rs update_particle
    case M_VISCOELASTIC: {  // viscoelastic.rs update_particle
        if constexpr (HAS_MODEL(MASK, M_COROTATED) || HAS_MODEL(MASK, M_VISCOELASTIC)) {
        M2 fp_new = madd(mident(), smscale(dt, p.c));
        p.f = mm(fp_new, p.f);
        sync_volume_density(p);
    }
        break;
    }
    case M_VON_MISES: {
        if constexpr (HAS_MODEL(MASK, M_VON_MISES)) {  // von_mises.rs:108-141
        // params(): yield_stress in hardening_exponent, H in hardening_modulus
        M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        M2 u, vt;
        float2 sigma;
        svd2(f_trial, u, sigma, vt);
        float2 eps = hencky(sigma, pr);
        float tr = eps.x + eps.y;
        float2 dev = vsub(eps, splat(tr * 0.5f));
        float dev_norm = vlen(dev);
        float kappa = p.q;
        float effective_yield = m.hardening_exponent + m.hardening_modulus * kappa;
        float elastic_dev = 2.0f * m.mu * dev_norm;
        float2 sigma_new = sigma;
        if (elastic_dev > effective_yield && dev_norm > LOG_CLAMP) {
            float denom = 2.0f * m.mu + m.hardening_modulus;
            float gamma = denom > F32_EPS ? (elastic_dev - effective_yield) / denom : 0.0f;
            p.q = kappa + gamma;
            float2 eps_proj = vadd(vmuls(dev, effective_yield / elastic_dev), splat(tr * 0.5f));
            sigma_new = v2(em_exp(eps_proj.x, pr), em_exp(eps_proj.y, pr));
        }
        p.f = reconstruct(u, sigma_new, vt);
        sync_volume_density(p);
    }
        break;
    }
    case M_RANKINE: {
        if constexpr (HAS_MODEL(MASK, M_RANKINE)) {  // rankine.rs update_particle
        // params(): tensile_strength in hardening_exponent, softening_rate in hardening_modulus
        M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        M2 u, vt;
        float2 sigma;
        svd2(f_trial, u, sigma, vt);
        float2 eps = hencky(sigma, pr);
        float a = 2.0f * m.mu + m.lambda;
        float2 tau = v2(a * eps.x + m.lambda * eps.y, m.lambda * eps.x + a * eps.y);
        float damage = p.q;
        float ts = m.hardening_exponent, rate = m.hardening_modulus;
        float t_eff = fmaxf(ts * em_exp(-rate * damage, pr), ts * 0.05f);  // utils.rs:28
        bool t1 = tau.x > t_eff, t2 = tau.y > t_eff;
        float2 sigma_new = sigma;
        if (t1 || t2) {
            float2 tau_proj = (t1 && t2) ? splat(t_eff) : (t1 ? v2(t_eff, tau.y) : v2(tau.x, t_eff));
            float2 eps_proj = stress_to_hencky(tau_proj, m.lambda, m.mu);
            float2 eps_trial = stress_to_hencky(tau, m.lambda, m.mu);
            // rankine_damage_saturation_point (utils.rs:43-49)
            float sat = rate <= 0.0f ? INFINITY : -em_log(0.05f, pr) / rate;
            p.q = fminf(damage + vlen(vsub(eps_trial, eps_proj)), sat);
            sigma_new = v2(em_exp(eps_proj.x, pr), em_exp(eps_proj.y, pr));
        }
        p.f = reconstruct(u, sigma_new, vt);
        sync_volume_density(p);
    }
        break;
    }
    case M_DP_MUI: {
        if constexpr (HAS_MODEL(MASK, M_DP_MUI)) {  // sand_mui.rs update_particle
        // params(): mu_static, mu_dynamic, inertial_q in dp_h0, dp_h1, dp_h2
        const float SQRT_2 = 1.41421356237f;
        const float mu_s = m.dp_h0, mu_d = m.dp_h1, i0 = m.dp_h2;
        M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        M2 u, vt;
        float2 sigma;
        svd2(f_trial, u, sigma, vt);
        float2 eps = hencky(sigma, pr);
        float tr = eps.x + eps.y;
        float p_trial = -(m.lambda + m.mu) * tr;
        float2 dev = vsub(eps, splat(tr * 0.5f));
        float dev_norm = vlen(dev);
        float2 sigma_new;
        float q_new = mu_s;
        if (p_trial <= 0.0f) {
            sigma_new = v2(1.0f, 1.0f);
        } else if (SQRT_2 * m.mu * dev_norm <= mu_s * p_trial || dev_norm < F32_EPS) {
            sigma_new = sigma;
        } else {
            float delta_q = SQRT_2 * m.mu * dev_norm - mu_s * p_trial;
            float sqrt_p = sqrtf(p_trial);
            float a = m.mu * dt;
            float b = p_trial * (mu_d - mu_s) + a * i0 * sqrt_p - delta_q;
            float c = -delta_q * i0 * sqrt_p;
            float gamma_dot = fmaxf((-b + sqrtf(b * b - 4.0f * a * c)) / (2.0f * a), 0.0f);
            if (gamma_dot > F32_EPS) q_new = mu_s + (mu_d - mu_s) / (i0 * sqrt_p / gamma_dot + 1.0f);
            float delta_gamma = gamma_dot * dt;
            float2 n_hat = vdivs(dev, dev_norm);
            float2 eps_new = vsub(eps, vmuls(n_hat, delta_gamma / SQRT_2));
            sigma_new = v2(em_exp(eps_new.x, pr), em_exp(eps_new.y, pr));
        }
        p.f = reconstruct(u, sigma_new, vt);
        p.q = q_new;
        sync_volume_density(p);
    }
        break;
    }
    case M_GRANULAR_FLUID: {
        if constexpr (HAS_MODEL(MASK, M_GRANULAR_FLUID)) {  // granular_fluid.rs update_particle
        M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        if (m.compression_limit > 0.0f || m.stretch_limit > 0.0f) {
            M2 u, vt;
            float2 sigma;
            svd2(f_trial, u, sigma, vt);
            float lo = 1.0f - m.compression_limit, hi = 1.0f + m.stretch_limit;
            float2 sigma_c = v2(fclampf(sigma.x, lo, hi), fclampf(sigma.y, lo, hi));
            float jp_new = p.jp * (sigma.x * sigma.y) / fmaxf(sigma_c.x * sigma_c.y, 1.0e-10f);
            p.jp = fclampf(jp_new, m.volume_ratio_min, m.volume_ratio_max);
            p.h = fclampf(em_exp(m.hardening_exponent * (1.0f - p.jp), pr), 0.1f, 7.0f);
            p.f = mm(mm(u, mdiag(sigma_c)), vt);
        } else {
            p.f = f_trial;
        }
        sync_volume_density(p);
    }
        break;
    }
    default:
        break;
    }
}

// MaterialModel::init_particle
EM_HD void init_particle(const MatP &m, emerge_particle &p) {
    switch (m.model) {
    case M_DRUCKER_PRAGER:  // sand.rs:237-246
        p.friction_hardening = m.dp_h1 > 0.0f ? m.dp_h3 / m.dp_h1 : 0.0f;
        break;
    case M_SNOW:  // snow.rs:104-107
        p.plastic_volume_ratio = 1.0f;
        p.hardening_scale = 1.0f;
        break;
    case M_NACC:  // nacc.rs:271-273
        p.log_volume_strain = 0.0f;
        break;
    case M_COROTATED:       // corotated.rs init_particle
    case M_GRANULAR_FLUID:  // granular_fluid.rs init_particle
        p.hardening_scale = 1.0f;
        p.plastic_volume_ratio = 1.0f;
        break;
    case M_DP_MUI:  // sand_mui.rs init_particle: mu_static in dp_h0
        p.friction_hardening = m.dp_h0;
        break;
    default:
        break;
    }
}

// ---------------------------------------------------------------- solver pieces
// NBodyGravityField's Barnes-Hut quadtree (forces/fields/n_body.rs:63-283), rebuilt on the
// device every substep (nbody.cu).  The tree is stored as the complete quadtree of `depth`
// levels: the node of level d whose quadrant path from the root is `pre` (2 bits per level,
// quadrant 0 first) is slot (4^d - 1) / 3 + pre.  A node exists when its parent holds more
// than max_bodies bodies; it is a leaf when it holds at most max_bodies or sits at level
// `depth` -- the tree the reference's one-at-a-time insertion builds, which does not depend
// on the insertion order.  Level d keeps its own order of the bodies, sorted by the level's
// path prefix and, within a node, by reference index (the insertion order): the bodies of a
// level-d slot are the run [first, end) of that order, so a leaf sums its bodies, and a node
// folds its center of mass, in the reference's order.
constexpr int NBODY_MAX_DEPTH = 10;
struct NBodyView {
    int depth;             // max_depth (0..NBODY_MAX_DEPTH)
    int max_bodies;        // max_bodies_per_node
    const float4 *root;    // {center.x, center.y, half size, 0} of the root box
    const float4 *bdata;   // per particle slot: x, y, mass, reference index (as bits)
    const uint32_t *order; // level d's body order (particle slots) at order + d * stride
    size_t stride;
    const uint2 *range;    // per tree slot: [first, end) into its level's order
    const float4 *com;     // per tree slot: center of mass x, y, total mass; w = 1 if computed
    uint32_t *error;       // StepState::error_flags (a far node without its center of mass)
    int fast;              // pulls by the approximate reciprocal square root (fast pipeline)
    const float2 *accel;   // the walk's result per NBody field k and particle slot i, at
                           // accel[k * accel_stride + i] (written before the fields half)
    size_t accel_stride;
};

__host__ __device__ __forceinline__ int nbody_level_offset(int d) { return ((1 << (2 * d)) - 1) / 3; }
__host__ __device__ __forceinline__ int nbody_slots(int depth) { return nbody_level_offset(depth + 1); }

struct DevConfig {
    int res;                 // grid_res
    float cell;              // grid_cell_size
    float dt;                // frame dt
    int adaptive;
    int affine_cfl;
    float cfl, mat_cfl, visc_cfl, min_dt;
    int project;
    float min_density, min_volume, min_j;
    float2 gravity;
    int thickness;           // config.boundary_thickness
    float default_v0;
    float particle_mass;
    int max_substeps;
    float apic_blend, j_max;
    int precise_math;        // evaluate exp/log/sin/sinh/pow in double, round once
    int n_bound;             // slip boundaries in order
    int bound_t[8];
    float asflip;            // asflip_blend (transfer/g2p.rs:263-296)
    int n_fields;            // force fields, application order
    const emerge_force_field *fields;
    const float *field_data;
    float sleep_thr;         // sleep_threshold (step.rs:299-315); 0 = no sleep scoring
    int zones;               // the sleep partition is in use: zone bits live in `sleeping`
    unsigned long long *zone_log;  // wake / sleep events: (key << 32) | reference index
    uint32_t *zone_log_count;
    uint32_t zone_log_cap;
    int multi;               // multi-field contact / mixture fields in use
    float contact_friction;  // SimConfig::contact_friction
    int grip_on;             // DirectionalContactGrip set
    float grip_mu_easy, grip_mu_resist;
    float2 grip_dir;
    float mix_drag;          // SimConfig::mixture_drag_coefficient
    int mix_iters;           // SimConfig::mixture_pressure_iterations
    const uint32_t *mat_phase;  // MixturePhase per material slot: 0 none, 1 solid, 2 fluid
    int mf_fast;             // multi-field scene on the fast (fused, unordered-sum) pipeline
    int mf_fields;           // fields in use: bit 0 grip (contact), bit 1 solid + fluid (mixture)
    int mf_excl;             // fast pipeline, one kind of field: a field particle scatters into
                             // its field only, and the grid update adds the fields to the total
    NBodyView nbody;         // NBodyGravityField's tree (body == nullptr: no such field)
};

// Bits of DevParticles::sleeping while the sleep partition is in use: bit 0 is
// Particle::sleeping, bit 1 marks a particle outside the active zone (reference index at or
// above active_count), bit 2 a particle woken during the running substep.
constexpr uint32_t ZB_FLAG = 1u, ZB_OUT = 2u, ZB_WOKEN = 4u;

// Records a wake (key = 2 substep) or sleep (key = 2 substep + 1) event of the particle with
// reference index `index`; the host replays the index swaps in the reference's order.
__device__ __forceinline__ void zone_log(const DevConfig &cfg, uint32_t key, uint32_t index) {
    const uint32_t k = atomicAdd(cfg.zone_log_count, 1u);
    if (k < cfg.zone_log_cap) cfg.zone_log[k] = (static_cast<unsigned long long>(key) << 32) | index;
}

// smooth_cutoff (spacetime/solver/cutoff.rs:17-26)
EM_HD float smooth_cutoff(float r, float r_on, float r_cut) {
    if (r >= r_cut) return 0.0f;
    if (r <= r_on) return 1.0f;
    float x = (r - r_on) / (r_cut - r_on);
    return 1.0f - 3.0f * x * x + 2.0f * x * x * x;
}

// Field::acceleration of one built-in force field at a particle (forces/fields/: gravity.rs,
// buoyancy.rs, drag.rs, confinement.rs, coulomb.rs, em.rs, chemotaxis.rs).  Material charge
// maps are tables by material id; ids past the table have no charge.
EM_HD float2 field_acceleration(const emerge_force_field &f, const float *data, const PState &p) {
    const float *pr = f.params;
    const float2 x = p.x;
    switch (f.kind) {
    case EMERGE_FIELD_GRAVITY_WELL: {
        float2 acc = v2(0.0f, 0.0f);
        const float eps2 = pr[1] * pr[1];
        for (uint32_t k = 0; k < f.count; ++k) {
            const float *src = data + f.data_offset + 3 * k;
            const float2 r_vec = vsub(v2(src[0], src[1]), x);  // toward the source
            const float r2 = vlen2(r_vec);
            const float r = sqrtf(r2);
            if (r >= pr[2] || r < F32_EPS) continue;
            const float norm_s = r2 + eps2;
            const float force_scale = pr[0] * src[2] / (norm_s * sqrtf(norm_s));
            if (!isfinite(force_scale)) continue;
            acc = vadd(acc, vmuls(vmuls(r_vec, force_scale), smooth_cutoff(r, pr[3], pr[2])));
        }
        return acc;
    }
    case EMERGE_FIELD_BUOYANCY:
        return vmuls(v2(-pr[1], -pr[2]), pr[0] / fmaxf(p.rho, pr[3]));
    case EMERGE_FIELD_LINEAR_DRAG:
        if (f.material_mask != EMERGE_FIELD_ALL_MATERIALS && (f.material_mask & (1u << (p.mat & 31u))) == 0u)
            return v2(0.0f, 0.0f);
        return svmul(pr[2], vsub(v2(pr[0], pr[1]), p.v));
    case EMERGE_FIELD_RADIAL_CONFINEMENT: {
        const float2 r_vec = vsub(x, v2(pr[0], pr[1]));
        const float dist = vlen(r_vec);
        const float overshoot = dist - pr[2];
        if (overshoot <= 0.0f || dist < F32_EPS) return v2(0.0f, 0.0f);
        return vmuls(v2(-r_vec.x, -r_vec.y), pr[3] * overshoot / dist);
    }
    case EMERGE_FIELD_AABB_CONFINEMENT: {
        float2 acc = v2(0.0f, 0.0f);
        if (x.x < pr[0]) acc.x += pr[4] * (pr[0] - x.x);
        else if (x.x > pr[2]) acc.x -= pr[4] * (x.x - pr[2]);
        if (x.y < pr[1]) acc.y += pr[4] * (pr[1] - x.y);
        else if (x.y > pr[3]) acc.y -= pr[4] * (x.y - pr[3]);
        return acc;
    }
    case EMERGE_FIELD_COULOMB: {
        const float q_p = p.mat < f.n_charges ? data[f.data_offset + 3 * f.count + p.mat] : 0.0f;
        if (!(fabsf(q_p) > F32_EPS)) return v2(0.0f, 0.0f);
        float2 acc = v2(0.0f, 0.0f);
        const float eps2 = pr[1] * pr[1];
        const float inv_mass = p.mass > F32_EPS ? 1.0f / p.mass : 0.0f;
        for (uint32_t k = 0; k < f.count; ++k) {
            const float *src = data + f.data_offset + 3 * k;
            const float2 r_vec = vsub(x, v2(src[0], src[1]));  // away from the source
            const float r2 = vlen2(r_vec);
            const float r = sqrtf(r2);
            if (r >= pr[2] || r < F32_EPS) continue;
            const float norm_s = r2 + eps2;
            const float force_scale = pr[0] * src[2] * q_p / (norm_s * sqrtf(norm_s));
            if (!isfinite(force_scale)) continue;
            acc = vadd(acc, vmuls(r_vec, force_scale * smooth_cutoff(r, pr[3], pr[2]) * inv_mass));
        }
        return acc;
    }
    case EMERGE_FIELD_UNIFORM_ELECTRIC: {
        const float q = p.mat < f.n_charges ? data[f.data_offset + p.mat] : 0.0f;
        if (!(fabsf(q) > F32_EPS)) return v2(0.0f, 0.0f);
        const float inv_mass = p.mass > F32_EPS ? 1.0f / p.mass : 0.0f;
        return vmuls(v2(pr[0], pr[1]), q * inv_mass);
    }
    case EMERGE_FIELD_CHEMOTAXIS: {
        if (f.material_filter != EMERGE_FIELD_ALL_MATERIALS && p.mat != f.material_filter)
            return v2(0.0f, 0.0f);
        const int res = static_cast<int>(f.count);
        const int ix = f2i(floorf(x.x)), iy = f2i(floorf(x.y));
        const float *phi = data + f.data_offset;
        auto at = [&](int xi, int yi) -> float {
            if (xi < 0 || yi < 0 || xi >= res || yi >= res) return 0.0f;
            return phi[static_cast<size_t>(xi) * res + yi];
        };
        const float2 grad = v2((at(ix + 1, iy) - at(ix - 1, iy)) * 0.5f, (at(ix, iy + 1) - at(ix, iy - 1)) * 0.5f);
        return svmul(pr[0], grad);
    }
    default:
        return v2(0.0f, 0.0f);
    }
}

// Plummer-softened pull of mass m at offset r (n_body.rs:180-189, 199-207): zero when the
// scale is not finite.
EM_HD float2 nbody_pull(float2 r, float m, float g, float eps2) {
    const float ns = vdot(r, r) + eps2;
    const float scale = ediv(g * m, ns * esqrt(ns));
    return isfinite(scale) ? vmuls(r, scale) : v2(0.0f, 0.0f);
}

// The same pull on the fast pipeline: g m / ns^1.5 as g m (1/sqrt ns)^3 with the hardware's
// approximate reciprocal square root (a few ulp, where the division and square root above
// are correctly rounded); ns = 0 gives an infinite scale and no pull, as above.
__device__ __forceinline__ float2 nbody_pull_fast(float2 r, float m, float g, float eps2) {
    const float ns = vdot(r, r) + eps2;
    const float inv = rsqrtf(ns);
    const float scale = (g * m) * (inv * inv * inv);
    return isfinite(scale) ? vmuls(r, scale) : v2(0.0f, 0.0f);
}

// The reference's far test of a node holding bodies (n_body.rs:184-187): with dist = |pos -
// center| correctly rounded, the node is far when !(dist < softening) and (2 half) / dist,
// correctly rounded, is below theta.  Both comparisons are first made from s = |pos -
// center|^2 (the same rounded value the distance's square root takes) and the hardware's
// approximate 1/sqrt(s), whose error (a few ulp, ~1e-6 at most) is far inside the 1e-5
// relative margins below: outside the margins the outcome is certain, and the correctly
// rounded square root and division run only inside them (or for non-finite inputs, whose
// comparisons are all false).
__device__ __forceinline__ bool nbody_far(float2 dv, float half, float soft, float theta) {
    const float s = vdot(dv, dv);
    const float s2 = soft * soft;
    if (s < s2 * 0.99999f) return false;  // dist < soft for certain
    const float q = (half * 2.0f) * rsqrtf(s);
    if (s > s2 * 1.00001f) {              // dist >= soft for certain
        if (q < theta * 0.99999f) return true;
        if (q > theta * 1.00001f) return false;
    }
    const float dist = esqrt(s);
    return !(dist < soft) && ediv(half * 2.0f, dist) < theta;
}

// NBodyGravityField::acceleration (n_body.rs:178-208, 347-360) of the particle with reference
// index `self` at `pos`.  A node is far when the particle is at least the softening length
// from its box center, it holds mass, and its width over that distance is below theta; far
// nodes pull with their center of mass, leaves with each body but the particle itself and
// those closer than the softening length, and an internal node sums its four children in
// quadrant order (the reference's recursion).
//
// The lanes that call it together walk the tree together, depth first: the warp opens a node
// when any lane needs it opened, so neighbouring particles (tile-sorted) share one walk and a
// leaf's bodies are read once for all of them.  Each lane keeps the reference's arithmetic:
// a lane that stops at a node (far for it, or a leaf) adds that node's value to its parent's
// accumulator at once -- where its own recursion would -- and sits out the node's subtree
// (`skip`); a lane that opens a node accumulates its children into the node's own level and
// adds the total when the walk leaves the node.  So every lane makes the additions of its
// own recursion, in the same order, whatever its neighbours need.  The fast pipeline adds
// every value into one running sum instead (the same terms, another order).
__device__ __forceinline__ float2 nbody_acceleration(const NBodyView &nb, const emerge_force_field &f, float2 pos,
                                                     uint32_t self) {
    const float g = f.params[0], soft = f.params[1], theta = f.params[2];
    const float eps2 = soft * soft;
    if (!nb.bdata) return v2(0.0f, 0.0f);
    const unsigned mask = __activemask();
    const bool full = mask == 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const float4 rt = nb.root[0];
    float2 ctr[NBODY_MAX_DEPTH + 1];
    float2 acc[NBODY_MAX_DEPTH + 1];
    float2 result = v2(0.0f, 0.0f);
    uint32_t opened = 0u;  // bit d: this lane opened the path's node at depth d
    int skip = -1;         // depth of the node whose subtree this lane sits out (-1: none)
    int d = 0;             // the walk's position (the same in every lane)
    uint32_t pre = 0u;
    int base = 0;          // nbody_level_offset(d), kept as the walk moves
    float2 c = v2(rt.x, rt.y);
    float half = rt.z;
    for (;;) {
        // first visit of node (d, pre): box center c, half size `half`
        const int slot = base + static_cast<int>(pre);
        const uint2 rg = nb.range[slot];
        // the center of mass is loaded with the range (one wait instead of two in a row),
        // whether or not the node turns out far
        const float4 cm = nb.com[slot];
        const bool leaf = d >= nb.depth || rg.y - rg.x <= static_cast<uint32_t>(nb.max_bodies);
        const bool part = skip < 0;
        bool need_open = false, need_leaf = false;
        float2 r = v2(0.0f, 0.0f);
        if (part) {
            const bool far = rg.y > rg.x && nbody_far(vsub(pos, c), half, soft, theta);
            if (far) {
                if (cm.w == 0.0f) atomicOr(nb.error, 4u);  // ERR_NBODY_SKIPPED (device_state.cuh)
                const float2 rv = vsub(v2(cm.x, cm.y), pos);
                r = nb.fast ? nbody_pull_fast(rv, cm.z, g, eps2) : nbody_pull(rv, cm.z, g, eps2);
            } else if (leaf) {
                need_leaf = true;
            } else {
                need_open = true;
            }
        }
        if (leaf) {
            // the leaf's bodies in order, summed by the lanes that stop here: for a large leaf
            // (only the deepest level holds more than max_bodies_per_node) a full warp loads
            // the next 32 (one per lane) and passes each to every lane; otherwise the lanes
            // load them one by one
            const uint32_t *ord = nb.order + static_cast<size_t>(d) * nb.stride;
            if (full && rg.y - rg.x > 8u) {
                if (__any_sync(0xffffffffu, need_leaf)) {
                    for (uint32_t j0 = rg.x; j0 < rg.y; j0 += 32u) {
                        float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        if (j0 + lane < rg.y) q = nb.bdata[ord[j0 + lane]];
                        const int cnt = static_cast<int>(min(32u, rg.y - j0));
                        for (int k = 0; k < cnt; ++k) {
                            const float bx = __shfl_sync(0xffffffffu, q.x, k);
                            const float by = __shfl_sync(0xffffffffu, q.y, k);
                            const float bm = __shfl_sync(0xffffffffu, q.z, k);
                            const float bw = __shfl_sync(0xffffffffu, q.w, k);
                            if (!need_leaf || __float_as_uint(bw) == self) continue;
                            const float2 rv = vsub(v2(bx, by), pos);
                            if (vdot(rv, rv) < eps2) continue;
                            r = vadd(r, nb.fast ? nbody_pull_fast(rv, bm, g, eps2) : nbody_pull(rv, bm, g, eps2));
                        }
                    }
                }
            } else if (need_leaf) {
                for (uint32_t j = rg.x; j < rg.y; ++j) {
                    const float4 bd = nb.bdata[ord[j]];
                    if (__float_as_uint(bd.w) == self) continue;
                    const float2 rv = vsub(v2(bd.x, bd.y), pos);
                    if (vdot(rv, rv) < eps2) continue;
                    r = vadd(r, nb.fast ? nbody_pull_fast(rv, bd.z, g, eps2) : nbody_pull(rv, bd.z, g, eps2));
                }
            }
        }
        if (part && !need_open) {  // this lane's value of the node: to its parent now
            if (nb.fast) result = vadd(result, r);  // fast pipeline: one running sum
            else if (d == 0) result = r;
            else acc[d - 1] = vadd(acc[d - 1], r);
        }
        if (__any_sync(mask, need_open)) {  // the walk descends into quadrant 0 (left, top)
            if (part && !need_open) skip = d;
            if (need_open && !nb.fast) {
                acc[d] = v2(0.0f, 0.0f);
                opened |= 1u << d;
            }
            ctr[d] = c;
            half *= 0.5f;
            c = v2(c.x - half, c.y + half);
            ++d;
            base = 4 * base + 1;
            pre <<= 2;
            continue;
        }
        // the walk leaves node (d, pre): finish it, move to its next sibling or leave its parent
        for (;;) {
            if (opened & (1u << d)) {  // this lane opened it: its children's total goes up
                opened &= ~(1u << d);
                if (d == 0) result = acc[0];
                else acc[d - 1] = vadd(acc[d - 1], acc[d]);
            }
            if (skip == d) skip = -1;
            if (d == 0) return result;
            const uint32_t q = pre & 3u;
            pre >>= 2;
            --d;
            if (q < 3u) {
                const uint32_t nq = q + 1u;
                const float quarter = half;  // the children's half size
                c = v2((nq & 1u) ? ctr[d].x + quarter : ctr[d].x - quarter,
                       (nq & 2u) ? ctr[d].y - quarter : ctr[d].y + quarter);
                ++d;
                pre = (pre << 2) | nq;
                break;
            }
            base = (base - 1) >> 2;
            half *= 2.0f;
        }
    }
}

// Sum of the force fields' accelerations at a particle, in application order (step.rs:
// 232-236).  `slot`: the particle's slot; an NBodyGravityField's value is the tree walk's
// (k_nb_walk, run for every particle before this sum is formed).
EM_HD float2 force_field_sum(const DevConfig &cfg, const PState &p, int slot) {
    float2 dv = v2(0.0f, 0.0f);
    int kn = 0;  // NBody fields met so far
    for (int k = 0; k < cfg.n_fields; ++k) {
        const emerge_force_field &f = cfg.fields[k];
        if (f.kind == EMERGE_FIELD_NBODY_GRAVITY) {
            if (cfg.nbody.accel)
                dv = vadd(dv, cfg.nbody.accel[static_cast<size_t>(kn) * cfg.nbody.accel_stride + slot]);
            ++kn;
            continue;
        }
        dv = vadd(dv, field_acceleration(f, cfg.field_data, p));
    }
    return dv;
}

// Force fields after G2P (step.rs:212-259): v += dt * sum of the accelerations, then the
// G2P speed clamp again; pinned particles are skipped.
EM_HD void apply_force_fields(const DevConfig &cfg, PState &p, float dt, int slot) {
    if (cfg.n_fields <= 0 || p.pinned != 0) return;
    const float2 dv = force_field_sum(cfg, p, slot);
    p.v = vadd(p.v, svmul(dt, dv));
    const float vel_limit = cfg.cell / dt;
    const float spd = vlen(p.v);
    if (spd > vel_limit) p.v = vmuls(p.v, vel_limit / spd);
}

// affine_cfl_speed_contribution (step.rs:481-488)
EM_HD float affine_cfl(M2 c, float cell) {
    const float STENCIL_CORNER_DISTANCE = 1.5f * 1.41421356f;
    float grad_norm = sqrtf(vlen2(c.xa) + vlen2(c.ya));
    return grad_norm * STENCIL_CORNER_DISTANCE * cell;
}

// cfl_bound (step.rs:472-479)
EM_HD float cfl_bound(const DevConfig &c, float max_speed, float min_mat_dt, float max_dt) {
    float dt = max_dt;
    if (max_speed > F32_EPS) dt = fminf(dt, c.cfl * c.cell / max_speed);
    dt = fminf(dt, min_mat_dt);
    return fclampf(dt, fminf(c.min_dt, max_dt), max_dt);
}

EM_HD int sat_sub(int a, int b) { return a > b ? a - b : 0; }

// project_particle_state_to_admissible (step.rs:347-429); returns true if corrected.
// `changed` (optional) is set when the projection altered any field, the position clamp
// and the density floor included: a state with changed == false is its own projection.
EM_HD bool project_state(const DevConfig &c, PState &q, bool *changed = nullptr) {
    bool projected = false;
    bool clamped = false;
    float mn = static_cast<float>(sat_sub(c.thickness, 1));
    float mx = static_cast<float>(sat_sub(c.res, c.thickness));
    float2 center = splat((mn + mx) * 0.5f);
    if (!vfinite(q.x)) {
        q.x = center;
        projected = true;
    } else {
        const float2 xc = vclamp2(q.x, splat(mn), splat(mx));
        clamped = xc.x != q.x.x || xc.y != q.x.y;
        q.x = xc;
    }
    if (!vfinite(q.v)) {
        q.v = v2(0.0f, 0.0f);
        projected = true;
    }
    if (!mfinite(q.c)) {
        q.c = mzero();
        projected = true;
    }
    if (!mfinite(q.f) || mdet(q.f) <= c.min_j) {
        q.f = mident();
        projected = true;
    } else {
        float j = mdet(q.f);
        if (j > c.j_max) {
            q.f = mscale(q.f, sqrtf(c.j_max / j));
            projected = true;
        }
    }
    if (!isfinite(q.jp) || q.jp <= 0.0f) { q.jp = 1.0f; projected = true; }
    if (!isfinite(q.h) || q.h <= 0.0f) { q.h = 1.0f; projected = true; }
    if (!isfinite(q.q)) { q.q = 0.0f; projected = true; }
    if (!isfinite(q.lvs)) { q.lvs = 0.0f; projected = true; }
    if (!isfinite(q.mass) || q.mass <= 0.0f) { q.mass = c.particle_mass; projected = true; }
    if (!isfinite(q.v0) || q.v0 <= 0.0f) {
        q.v0 = fmaxf(c.default_v0, c.min_volume);
        projected = true;
    }
    if (!isfinite(q.vol) || q.vol <= 0.0f) {
        q.vol = fmaxf(q.v0, c.min_volume);
        projected = true;
    }
    if (!isfinite(q.rho) || q.rho <= 0.0f) {
        q.rho = fmaxf(q.mass / q.vol, c.min_density);
        projected = true;
    } else {
        clamped = clamped || q.rho < c.min_density;
        q.rho = fmaxf(q.rho, c.min_density);
    }
    if (changed) *changed = projected || clamped;
    return projected;
}

// apply_slip_wall_velocity (forces/boundary/mod.rs:78-101) for cell (x, y)
EM_HD void slip_velocity(int thickness, int x, int y, int res, float2 &v) {
    int hi = res - (thickness + 1);
    if (x < thickness) v.x = fmaxf(v.x, 0.0f);
    if (x > hi) v.x = fminf(v.x, 0.0f);
    if (y < thickness) v.y = fmaxf(v.y, 0.0f);
    if (y > hi) v.y = fminf(v.y, 0.0f);
}

// clamp_position_inside_grid (forces/boundary/mod.rs:103-111)
EM_HD float2 clamp_position(int thickness, float2 pos, int res) {
    float mn = static_cast<float>(sat_sub(thickness, 1));
    float mx = static_cast<float>(sat_sub(res, thickness));
    return vclamp2(pos, splat(mn), splat(mx));
}

}  // namespace emerge
