// emerge_oracle.cpp -- CPU oracle: a C++17 restatement of the reference
// emerge-engine MLS-MPM step (Rust crate M1thieu/emerge-engine 0.1.0).
//
// TEST INFRASTRUCTURE.  Used only by tests/, the smoke check and bench.py's
// CPU-baseline leg, as the parity checker and the timed CPU baseline.  The
// product CUDA library never links this file.
//
// Every function cites the reference file:line it restates.  Arithmetic is
// f32 throughout, evaluated in the reference's expression order, compiled
// with -ffp-contract=off (Rust does not contract a*b+c into FMA).  glam's
// Mat2/Vec2 operations are restated from their definitions (column-major
// Mat2; determinant = x_axis.x*y_axis.y - y_axis.x*x_axis.y; length =
// sqrt(dot)); glam 0.30's source is not present here, so bit-level identity
// with the Rust build is not claimed.  Transcendentals (expf, logf, sinf,
// sinhf, powf, sqrtf) call glibc's libm, which is what Rust's f32 methods
// call on Linux.
//
// The sparse FxHash grid of the reference (grid/mod.rs:112-139) is restated
// as a dense column-major array (index x*res+y) plus a dirty list in
// first-touch order: per-cell summation order (particle index order) is the
// same, and every per-cell grid operation is order-independent, so results
// are unchanged; only the constant factor of the baseline differs (a dense
// array is faster than a hash map, so the CPU baseline timed from this file
// is an upper bound on the reference's own CPU throughput).

#include "emerge_oracle.h"

#include <algorithm>
#include <functional>
#include <unordered_map>
#include <utility>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <utility>
#include <vector>

#include <thread>

namespace {

int g_threads = 0;  // 0 = std::thread::hardware_concurrency()

// Static-partition parallel for over [0, n): stands in for rayon's par_iter in
// G2P phase 1 (per-particle work with no cross-particle dependency).
template <class Fn>
void parallel_for(long n, Fn fn) {
    int t = g_threads > 0 ? g_threads : static_cast<int>(std::thread::hardware_concurrency());
    if (t < 1) t = 1;
    if (n < 4096 || t == 1) {
        fn(0L, n);
        return;
    }
    std::vector<std::thread> pool;
    long chunk = (n + t - 1) / t;
    for (int k = 0; k < t; ++k) {
        long lo = k * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([=] { fn(lo, hi); });
    }
    for (auto &th : pool) th.join();
}

constexpr float F32_EPS = 1.1920929e-7f;         // f32::EPSILON
constexpr float KERNEL_D_INVERSE = 4.0f;         // config.rs:22
constexpr float MIN_J = 1e-6f;                   // materials/utils.rs:11
constexpr float LOG_CLAMP = 1e-10f;              // materials/utils.rs:6
constexpr size_t MAX_MATERIAL_SLOTS = 64;        // registry.rs:6

// ---------------------------------------------------------------- glam restated
struct V2 { float x, y; };
struct M2 { V2 xa, ya; };  // x_axis, y_axis (columns)

inline V2 v2(float x, float y) { return V2{x, y}; }
inline V2 add(V2 a, V2 b) { return v2(a.x + b.x, a.y + b.y); }
inline V2 sub(V2 a, V2 b) { return v2(a.x - b.x, a.y - b.y); }
inline V2 mul(V2 a, V2 b) { return v2(a.x * b.x, a.y * b.y); }
inline V2 muls(V2 a, float s) { return v2(a.x * s, a.y * s); }
inline V2 smul(float s, V2 a) { return v2(s * a.x, s * a.y); }
inline V2 divs(V2 a, float s) { return v2(a.x / s, a.y / s); }
inline V2 splat(float s) { return v2(s, s); }
inline float dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline float length(V2 a) { return std::sqrt(dot(a, a)); }
inline float length_sq(V2 a) { return dot(a, a); }
inline bool finite2(V2 a) { return std::isfinite(a.x) && std::isfinite(a.y); }
inline V2 vabs(V2 a) { return v2(std::fabs(a.x), std::fabs(a.y)); }
// f32::max / f32::min semantics (a NaN operand yields the other operand).
inline float fmax_(float a, float b) { return std::fmax(a, b); }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline V2 vmax(V2 a, V2 b) { return v2(fmax_(a.x, b.x), fmax_(a.y, b.y)); }
inline V2 vmin(V2 a, V2 b) { return v2(fmin_(a.x, b.x), fmin_(a.y, b.y)); }
// glam Vec2::clamp = self.max(min).min(max)
inline V2 vclamp(V2 a, V2 lo, V2 hi) { return vmin(vmax(a, lo), hi); }
// f32::clamp: NaN stays NaN
inline float fclamp(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// Transcendentals.  By default the C library's f32 functions, which is what the Rust
// reference's f32::exp / ln / powf / sin / sinh call on Linux.  Those are not always
// correctly rounded (glibc's logf differs from the correctly rounded result in the last
// bit for a few percent of arguments near 1); with oracle_set_correctly_rounded(1) each
// is instead evaluated in double and rounded once, which isolates the algorithm from the
// library's last-bit behaviour.
int g_correctly_rounded = 0;
inline float m_exp(float x) { return g_correctly_rounded ? float(std::exp(double(x))) : std::exp(x); }
inline float m_log(float x) { return g_correctly_rounded ? float(std::log(double(x))) : std::log(x); }
inline float m_sin(float x) { return g_correctly_rounded ? float(std::sin(double(x))) : std::sin(x); }
inline float m_sinh(float x) { return g_correctly_rounded ? float(std::sinh(double(x))) : std::sinh(x); }
inline float m_pow(float x, float y) {
    return g_correctly_rounded ? float(std::pow(double(x), double(y))) : std::pow(x, y);
}
// glam normalize_or_zero: self * (1 / length) when finite and > 0
inline V2 normalize_or_zero(V2 a) {
    float rcp = 1.0f / length(a);
    if (std::isfinite(rcp) && rcp > 0.0f) return muls(a, rcp);
    return v2(0.0f, 0.0f);
}

inline M2 m2(V2 a, V2 b) { return M2{a, b}; }
inline M2 ident() { return m2(v2(1, 0), v2(0, 1)); }
inline M2 zero2() { return m2(v2(0, 0), v2(0, 0)); }
inline M2 diag(V2 d) { return m2(v2(d.x, 0.0f), v2(0.0f, d.y)); }
inline M2 madd(M2 a, M2 b) { return m2(add(a.xa, b.xa), add(a.ya, b.ya)); }
inline M2 msub(M2 a, M2 b) { return m2(sub(a.xa, b.xa), sub(a.ya, b.ya)); }
inline M2 mscale(M2 a, float s) { return m2(muls(a.xa, s), muls(a.ya, s)); }
inline M2 smscale(float s, M2 a) { return m2(smul(s, a.xa), smul(s, a.ya)); }
inline V2 mv(M2 a, V2 v) { return add(muls(a.xa, v.x), muls(a.ya, v.y)); }
inline M2 mm(M2 a, M2 b) { return m2(mv(a, b.xa), mv(a, b.ya)); }
inline M2 transpose(M2 a) { return m2(v2(a.xa.x, a.ya.x), v2(a.xa.y, a.ya.y)); }
inline float det(M2 a) { return a.xa.x * a.ya.y - a.ya.x * a.xa.y; }
inline bool finite_m(M2 a) { return finite2(a.xa) && finite2(a.ya); }

inline M2 load_m(const float *f) { return m2(v2(f[0], f[1]), v2(f[2], f[3])); }
inline void store_m(float *f, M2 a) { f[0] = a.xa.x; f[1] = a.xa.y; f[2] = a.ya.x; f[3] = a.ya.y; }
inline V2 load_v(const float *f) { return v2(f[0], f[1]); }
inline void store_v(float *f, V2 a) { f[0] = a.x; f[1] = a.y; }

struct IV2 { int32_t x, y; };

// Rust `f32 as i32`: saturating, NaN -> 0.
inline int32_t f2i_sat(float f) {
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return std::numeric_limits<int32_t>::max();
    if (f <= -2147483648.0f) return std::numeric_limits<int32_t>::min();
    return static_cast<int32_t>(f);
}

// ---------------------------------------------------------------- grid/kernel.rs
// axis_weights (grid/kernel.rs:20-25); powi(2) lowers to x*x.
inline void axis_weights(float d, float w[3]) {
    float a = 0.5f - d;
    float b = 0.5f + d;
    w[0] = 0.5f * (a * a);
    w[1] = 0.75f - d * d;
    w[2] = 0.5f * (b * b);
}

struct QW { IV2 base; float wx[3], wy[3]; };
// quadratic_weights (grid/kernel.rs:10-18)
inline QW quadratic_weights(V2 p) {
    QW q;
    q.base.x = f2i_sat(std::floor(p.x));
    q.base.y = f2i_sat(std::floor(p.y));
    float dx = (p.x - static_cast<float>(q.base.x)) - 0.5f;
    float dy = (p.y - static_cast<float>(q.base.y)) - 0.5f;
    axis_weights(dx, q.wx);
    axis_weights(dy, q.wy);
    return q;
}

// ---------------------------------------------------------------- materials
// svd2 (materials/svd.rs:14-76) + orthogonal_complement (:81-85)
inline V2 orthogonal_complement(V2 v) {
    V2 perp = v2(-v.y, v.x);
    float len = length(perp);
    if (len > 1e-10f) return divs(perp, len);
    return v2(1.0f, 0.0f);
}

void svd2(M2 f, M2 &u_out, V2 &sigma_out, M2 &vt_out) {
    float f00 = f.xa.x, f10 = f.xa.y, f01 = f.ya.x, f11 = f.ya.y;
    float c00 = f00 * f00 + f10 * f10;
    float c01 = f00 * f01 + f10 * f11;
    float c11 = f01 * f01 + f11 * f11;
    float mean = (c00 + c11) * 0.5f;
    float half_diff = (c00 - c11) * 0.5f;
    float disc = std::sqrt(half_diff * half_diff + c01 * c01);
    float lambda1 = mean + disc;
    float lambda2 = mean - disc;
    V2 v1;
    if (std::fabs(c01) > 1e-10f * fmax_(c00 + c11, 1e-30f)) {
        V2 raw = v2(c01, lambda1 - c00);
        v1 = divs(raw, length(raw));
    } else {
        v1 = (c00 >= c11) ? v2(1.0f, 0.0f) : v2(0.0f, 1.0f);
    }
    V2 vv2 = v2(-v1.y, v1.x);
    M2 v_sorted = m2(v1, vv2);
    M2 vt = transpose(v_sorted);
    V2 sigma = v2(std::sqrt(fmax_(lambda1, 0.0f)), std::sqrt(fmax_(lambda2, 0.0f)));
    V2 fv1 = mv(f, v1);
    V2 fv2 = mv(f, vv2);
    V2 u1 = (sigma.x > 1e-10f) ? divs(fv1, sigma.x) : orthogonal_complement(fv2);
    V2 u2 = (sigma.y > 1e-10f) ? divs(fv2, sigma.y) : orthogonal_complement(u1);
    M2 u = m2(u1, u2);
    if (det(u) < 0.0f) {
        u.ya = v2(-u.ya.x, -u.ya.y);
        sigma.y = -sigma.y;
    }
    u_out = u;
    sigma_out = sigma;
    vt_out = vt;
}

// polar_decomposition_2d (materials/utils.rs:129-138)
M2 polar(M2 f) {
    float x = f.xa.x + f.ya.y;
    float y = f.xa.y - f.ya.x;
    float norm = std::sqrt(x * x + y * y);
    if (norm > F32_EPS) return m2(divs(v2(x, y), norm), divs(v2(-y, x), norm));
    return ident();
}

// elastic_wave_dt (materials/utils.rs:145-163)
float elastic_wave_dt(float lambda, float mu, float hardening, float density,
                      float min_density, float cell_width, float material_cfl) {
    float rho = fmax_(density, min_density);
    float modulus = fmax_((lambda + 2.0f * mu) * hardening, 0.0f);
    if (modulus <= F32_EPS) return INFINITY;
    float c = std::sqrt(modulus / rho);
    if (c <= F32_EPS) return INFINITY;
    return material_cfl * cell_width / c;
}

enum Model : uint32_t {
    FALLBACK = 0, FLUID = 1, NEOHOOKEAN = 2, COROTATED = 3, SNOW = 4,
    DRUCKER_PRAGER = 5, VON_MISES = 6, RANKINE = 7, DP_MUI = 8,
    VISCOELASTIC = 9, NACC = 10, GRANULAR_FLUID = 11
};

using Mat = oracle_material;
using P = oracle_particle;

// DruckerPragerMaterial::alpha (sand.rs:135-141)
float dp_alpha(const Mat &m, float q) {
    float phi = m.friction_angle +
                (m.hardening_peak * q - m.friction_residual) * m_exp(-m.hardening_decay * q);
    float s = m_sin(phi);
    return std::sqrt(2.0f / 3.0f) * (2.0f * s) / (3.0f - s);
}

// DruckerPragerMaterial::project (sand.rs:156-194)
bool dp_project(const Mat &m, V2 sigma_in, float lvs, float q, V2 &out, float &dq) {
    V2 sigma = vmax(vabs(sigma_in), splat(LOG_CLAMP));
    V2 eps = v2(m_log(sigma.x) + lvs * 0.5f, m_log(sigma.y) + lvs * 0.5f);
    float trace = eps.x + eps.y;
    V2 dev = sub(eps, splat(trace * 0.5f));
    float dev_norm = length(dev);
    if (dev_norm == 0.0f || trace > 0.0f) {
        out = v2(1.0f, 1.0f);
        dq = dev_norm;
        return true;
    }
    float ratio = (m.lambda + m.mu) / m.mu;
    float alpha = dp_alpha(m, q);
    float cohesion_term = m.cohesion / (2.0f * m.mu);
    float gamma = dev_norm + ratio * trace * alpha - cohesion_term;
    if (gamma <= 0.0f) return false;
    V2 h = sub(eps, smul(gamma, divs(dev, dev_norm)));
    out = v2(m_exp(h.x), m_exp(h.y));
    dq = gamma;
    return true;
}

inline M2 reconstruct(M2 u, V2 s, M2 vt) { return mm(mm(u, diag(s)), vt); }

// NaccMaterial::project (nacc.rs:129-223)
void nacc_project(const Mat &m, M2 f, float alpha, M2 &f_out, float &alpha_out) {
    float xi = m.hardening_factor;
    float beta = m.nacc_cohesion;
    float mm_ = m.friction;
    M2 u, vt;
    V2 sigma;
    svd2(f, u, sigma, vt);
    V2 sv = sigma;
    V2 sv_sq = mul(sv, sv);
    float sv_sq_trace = sv_sq.x + sv_sq.y;
    float p0 = m.kappa * (1.0e-5f + m_sinh(xi * fmax_(-alpha, 0.0f)));
    float j_e_tr = fmax_(sv.x * sv.y, 1.0e-6f);
    V2 s_tr = smul(m.mu * (1.0f / j_e_tr), sub(sv_sq, splat(sv_sq_trace * 0.5f)));
    float psi_kappa = m.kappa * 0.5f * (j_e_tr - 1.0f / j_e_tr);
    float p_tr = -psi_kappa * j_e_tr;
    bool hard = m.hardening_enabled != 0;
    if (p_tr > p0) {
        float j_n1 = std::sqrt(fmax_(-2.0f * p0 / m.kappa + 1.0f, 1.0e-8f));
        float sv_new = m_pow(j_n1, 0.5f);
        if (hard) alpha += m_log(j_e_tr / j_n1);
        f_out = reconstruct(u, splat(sv_new), vt);
        alpha_out = alpha;
        return;
    }
    if (p_tr < -beta * p0) {
        float j_n1 = std::sqrt(fmax_(2.0f * beta * p0 / m.kappa + 1.0f, 1.0e-8f));
        float sv_new = m_pow(j_n1, 0.5f);
        if (hard) alpha += m_log(j_e_tr / j_n1);
        f_out = reconstruct(u, splat(sv_new), vt);
        alpha_out = alpha;
        return;
    }
    float y0 = (1.0f + 2.0f * beta) * 2.0f;
    float y1 = mm_ * mm_ * (p_tr + beta * p0) * (p_tr - p0);
    float s_norm_sq = s_tr.x * s_tr.x + s_tr.y * s_tr.y;
    float y = y0 * s_norm_sq + y1;
    if (y < 1.0e-4f) {
        f_out = f;
        alpha_out = alpha;
        return;
    }
    if (hard && p0 > 1.0e-4f && p_tr < p0 - 1.0e-4f && p_tr > -beta * p0 + 1.0e-4f) {
        float p_c = (1.0f - beta) * p0 * 0.5f;
        float q_tr = std::sqrt(2.0f) * length(s_tr);
        V2 dir = normalize_or_zero(v2(p_c - p_tr, -q_tr));
        float c = mm_ * mm_ * (p_c + beta * p0) * (p_c - p0);
        float b = mm_ * mm_ * dir.x * (2.0f * p_c - p0 + beta * p0);
        float a = mm_ * mm_ * dir.x * dir.x + (1.0f + 2.0f * beta) * dir.y * dir.y;
        float discr = std::sqrt(fmax_(b * b - 4.0f * a * c, 0.0f));
        float l1 = (-b + discr) / (2.0f * a);
        float l2 = (-b - discr) / (2.0f * a);
        float p1 = p_c + l1 * dir.x;
        float p2 = p_c + l2 * dir.x;
        float p_x = ((p_tr - p_c) * (p1 - p_c) > 0.0f) ? p1 : p2;
        float j_e_x = std::sqrt(fmax_(std::fabs(-2.0f * p_x / m.kappa + 1.0f), 1.0e-8f));
        if (j_e_x > 1.0e-4f) alpha += m_log(j_e_tr / j_e_x);
    }
    float scale = std::sqrt(fmax_(-y1 / fmax_(y0, 1.0e-10f), 0.0f)) * (j_e_tr / m.mu);
    V2 b_n1 = add(smul(scale, normalize_or_zero(s_tr)), splat(sv_sq_trace / 2.0f));
    V2 sv_new = v2(std::sqrt(fmax_(b_n1.x, 1.0e-8f)), std::sqrt(fmax_(b_n1.y, 1.0e-8f)));
    f_out = reconstruct(u, sv_new, vt);
    alpha_out = alpha;
}

// MaterialModel::kirchhoff_stress per model.
M2 kirchhoff_stress(const Mat &m, const P &p) {
    M2 f = load_m(p.f);
    switch (m.model) {
    case NEOHOOKEAN: {  // elastic.rs:180-255
        float j = det(f);
        if (j <= MIN_J) return zero2();
        float t_scale = 1.0f + m.thermal_expansion * p.temperature;
        float damage_scale = m_exp(-m.damage_softening_rate * p.friction_hardening);
        float mu = m.mu * t_scale * damage_scale;
        float lambda = m.lambda * t_scale * damage_scale;
        M2 b = mm(f, transpose(f));
        float tr_b = b.xa.x + b.ya.y;
        M2 dev_b = msub(b, diag(splat(tr_b * 0.5f)));
        float k = lambda + mu;
        M2 dev_stress = smscale(mu / j, dev_b);
        M2 vol_stress = smscale(k * m_log(j), ident());
        M2 viscous = zero2();
        if (m.viscosity > 0.0f) {
            M2 c = load_m(p.c);
            M2 sym = madd(c, transpose(c));
            M2 d = mscale(sym, 0.5f);
            float d_trace = d.xa.x + d.ya.y;
            M2 d_dev = msub(d, diag(splat(d_trace * 0.5f)));
            viscous = smscale(m.viscosity, d_dev);
        }
        return madd(madd(dev_stress, vol_stress), viscous);
    }
    case FLUID: {  // fluid.rs:135-191
        float density = fmin_(fmax_(p.density, m.fluid_min_density), m.rest_density * 2.0f);
        float pressure = fmax_(
            m.eos_stiffness * (m_pow(density / m.rest_density, m.eos_power) - 1.0f),
            m.pressure_floor);
        M2 stress = diag(splat(-pressure));
        float eff_visc = m.dynamic_viscosity;
        if (m.thermal_viscosity_coeff > 0.0f)
            eff_visc = m.dynamic_viscosity * m_exp(-m.thermal_viscosity_coeff * p.temperature);
        M2 c = load_m(p.c);
        M2 sym = madd(c, transpose(c));
        float div_v = sym.xa.x + sym.ya.y;
        M2 strain_dev = msub(sym, diag(splat(div_v * 0.5f)));
        stress = madd(stress, smscale(eff_visc, strain_dev));
        if (m.bulk_viscosity > 0.0f)
            stress = madd(stress, diag(splat(m.bulk_viscosity * div_v * 0.5f)));
        if (m.surface_tension_coeff != 0.0f) {
            float j = f.xa.x * f.ya.y - f.xa.y * f.ya.x;
            stress = madd(stress, diag(splat(m.surface_tension_coeff * j)));
        }
        return stress;
    }
    case DRUCKER_PRAGER: {  // sand.rs:220-231
        float j = det(f);
        if (j <= MIN_J) return zero2();
        M2 r = polar(f);
        M2 f_t = transpose(f);
        M2 a = mm(smscale(2.0f * m.mu, msub(f, r)), f_t);
        M2 b = smscale(m.lambda * (j - 1.0f) * j, ident());
        return madd(a, b);
    }
    case SNOW: {  // snow.rs:109-136
        float j = det(f);
        if (j <= MIN_J) return zero2();
        M2 r = polar(f);
        float h = p.hardening_scale;
        float mu_eff = m.mu * h;
        float lambda_eff = m.lambda * h;
        M2 f_t = transpose(f);
        M2 tau = madd(mm(smscale(2.0f * mu_eff, msub(f, r)), f_t),
                      smscale(lambda_eff * (j - 1.0f) * j, ident()));
        if (m.cohesion_coeff > 0.0f && p.plastic_volume_ratio < 1.0f && j > 1.0f)
            tau = madd(tau, smscale(m.cohesion_coeff * p.plastic_volume_ratio * (j - 1.0f) * j,
                                    ident()));
        return tau;
    }
    case NACC: {  // nacc.rs:236-249
        float j = fmax_(det(f), MIN_J);
        M2 b = mm(f, transpose(f));
        float tr_b = b.xa.x + b.ya.y;
        M2 dev_b = msub(b, diag(splat(tr_b * 0.5f)));
        M2 dev_stress = smscale(m.mu / j, dev_b);
        M2 vol_stress = smscale(m.kappa * 0.5f * (j * j - 1.0f), ident());
        return madd(dev_stress, vol_stress);
    }
    case COROTATED: {  // corotated.rs:61-77
        float j = det(f);
        if (j <= MIN_J) return zero2();
        M2 r = polar(f);
        float h = p.hardening_scale;
        float t_scale = 1.0f + m.thermal_expansion * p.temperature;
        float mu_eff = m.mu * h * t_scale;
        float lambda_eff = m.lambda * h * t_scale;
        return madd(mm(smscale(2.0f * mu_eff, msub(f, r)), transpose(f)),
                    smscale(lambda_eff * (j - 1.0f) * j, ident()));
    }
    case VON_MISES:    // von_mises.rs:96-104
    case RANKINE:      // rankine.rs kirchhoff_stress
    case DP_MUI: {     // sand_mui.rs kirchhoff_stress
        float j = det(f);
        if (j <= MIN_J) return zero2();
        M2 r = polar(f);
        return madd(mm(smscale(2.0f * m.mu, msub(f, r)), transpose(f)),
                    smscale(m.lambda * (j - 1.0f) * j, ident()));
    }
    case VISCOELASTIC: {  // viscoelastic.rs kirchhoff_stress
        float j = fmin_(fmax_(f.xa.x * f.ya.y - f.xa.y * f.ya.x, m.j_min), 1.0f / m.j_min);
        float t_scale = 1.0f + m.thermal_expansion * p.temperature;
        float mu = m.mu * t_scale;
        float lambda = m.lambda * t_scale;
        M2 b = mm(f, transpose(f));
        M2 elastic = madd(smscale(mu, msub(b, ident())), diag(splat(lambda * m_log(j))));
        M2 c = load_m(p.c);
        M2 d = mscale(madd(c, transpose(c)), 0.5f);
        float trace = d.xa.x + d.ya.y;
        M2 d_dev = msub(d, diag(splat(trace * 0.5f)));
        return madd(elastic, smscale(m.viscosity * t_scale, d_dev));
    }
    case GRANULAR_FLUID: {  // granular_fluid.rs kirchhoff_stress
        float j = fmax_(det(f), MIN_J);
        float density = fmax_(m.rest_density / j, 1.0e-6f);
        float ratio = fmax_(density / fmax_(m.rest_density, 1.0e-6f), 1.0e-6f);
        float pressure = fmax_(m.eos_stiffness * (m_pow(ratio, m.eos_power) - 1.0f),
                               m.pressure_floor);
        float h = p.hardening_scale;
        M2 r = polar(f);
        float mu_eff = m.mu * h;
        M2 coro = mm(smscale(2.0f * mu_eff, msub(f, r)), transpose(f));
        float tr = coro.xa.x + coro.ya.y;
        M2 dev_coro = msub(coro, diag(splat(tr * 0.5f)));
        M2 lam_vol = smscale(m.lambda * h * (j - 1.0f) * j, ident());
        return madd(madd(diag(splat(-pressure)), dev_coro), lam_vol);
    }
    default:  // FallbackMaterial (materials/mod.rs:362-366): zero stress
        return zero2();
    }
}

// BinghamFluidMaterial::kirchhoff_stress (bingham.rs): Tait pressure plus the
// Bingham deviatoric stress with apparent viscosity yield / shear_rate + viscosity.
M2 bingham_kirchhoff(const Mat &m, const P &p) {
    float density = fmin_(fmax_(p.density, m.fluid_min_density), m.rest_density * 2.0f);
    float pressure = fmax_(
        m.eos_stiffness * (m_pow(density / m.rest_density, m.eos_power) - 1.0f), m.pressure_floor);
    M2 hydrostatic = diag(splat(-pressure));
    M2 c = load_m(p.c);
    M2 d = mscale(madd(c, transpose(c)), 0.5f);
    float trace = d.xa.x + d.ya.y;
    M2 d_dev = msub(d, diag(splat(trace * 0.5f)));
    float dxx = d_dev.xa.x, dyy = d_dev.ya.y, dxy = d_dev.xa.y;
    float d_sq = dxx * dxx + dyy * dyy + 2.0f * dxy * dxy;
    float shear_rate = std::sqrt(2.0f * d_sq);
    M2 deviatoric = zero2();
    if (!(shear_rate < m.critical_shear_rate)) {
        float eta_app = m.bingham_yield_stress / shear_rate + m.dynamic_viscosity;
        deviatoric = mscale(d_dev, eta_app);
    }
    M2 surface = zero2();
    if (m.surface_tension_coeff != 0.0f) {
        M2 f = load_m(p.f);
        float j = f.xa.x * f.ya.y - f.xa.y * f.ya.x;
        surface = diag(splat(m.surface_tension_coeff * j));
    }
    return madd(madd(hydrostatic, deviatoric), surface);
}

// MaterialModel::activation_scale (mod.rs:181-183): NeoHookean, Corotated and
// Viscoelastic override it.
inline float activation_scale(const Mat &m) {
    return (m.model == NEOHOOKEAN || m.model == COROTATED || m.model == VISCOELASTIC)
               ? m.active_stress_coeff
               : 0.0f;
}

// combined_kirchhoff_stress (spacetime/transfer.rs:77-104)
M2 combined_kirchhoff_stress(const Mat &m, const P &p) {
    M2 tau = (m.model == FLUID && m.bingham) ? bingham_kirchhoff(m, p) : kirchhoff_stress(m, p);
    float coeff = activation_scale(m);
    if (p.activation <= 0.0f || coeff <= 0.0f) return tau;
    bool isotropic = m.model == VISCOELASTIC;
    M2 tau_active;
    if (isotropic) {
        tau_active = diag(splat(p.activation * coeff));
    } else {
        V2 n = load_v(p.activation_dir);
        float len_sq = dot(n, n);
        if (len_sq > F32_EPS) {
            V2 n0 = divs(n, std::sqrt(len_sq));
            M2 n_outer = m2(muls(n0, n0.x), muls(n0, n0.y));
            M2 a_mat = mscale(n_outer, p.activation * coeff);
            M2 f = load_m(p.f);
            tau_active = mm(mm(f, a_mat), transpose(f));
        } else {
            tau_active = diag(splat(p.activation * coeff));
        }
    }
    return madd(tau, tau_active);
}

// MaterialModel::stress_volume
inline float stress_volume(const Mat &m, const P &p) {
    if (m.model == FLUID) return fmax_(p.volume, m.fluid_min_volume);  // fluid.rs:193-195, bingham.rs
    if (m.model == GRANULAR_FLUID) return fmax_(p.volume, 1.0e-6f);     // granular_fluid.rs
    return p.initial_volume;  // mod.rs:114 default and every other in-scope model
}

// MaterialModel::timestep_bound
float timestep_bound(const Mat &m, float density, float h, float cell, float mat_cfl,
                     float visc_cfl) {
    switch (m.model) {
    case NEOHOOKEAN: {  // elastic.rs:290-327
        float elastic_dt = elastic_wave_dt(m.lambda, m.mu, 1.0f, density, m.min_density, cell,
                                           mat_cfl);
        float viscous_dt = INFINITY;
        if (m.viscosity > 0.0f) {
            float d = fmax_(density, 1.0e-6f);
            float kinematic = m.viscosity / d;
            if (kinematic > F32_EPS) viscous_dt = visc_cfl * cell * cell / kinematic;
        }
        return fmin_(elastic_dt, viscous_dt);
    }
    case FLUID: {  // fluid.rs:228-259
        const float MIN_DENSITY_RATIO = 1.0e-6f;
        float d = fmax_(density, m.fluid_min_density);
        float ratio = fmax_(d / fmax_(m.rest_density, m.fluid_min_density), MIN_DENSITY_RATIO);
        float dt_bound = INFINITY;
        float c2 = m.eos_stiffness * m.eos_power * m_pow(ratio, m.eos_power - 1.0f) /
                   fmax_(m.rest_density, m.fluid_min_density);
        if (std::isfinite(c2) && c2 > F32_EPS)
            dt_bound = fmin_(dt_bound, mat_cfl * cell / std::sqrt(c2));
        if (m.dynamic_viscosity > 0.0f) {
            float kin = m.dynamic_viscosity / d;
            if (kin > F32_EPS) dt_bound = fmin_(dt_bound, visc_cfl * cell * cell / kin);
        }
        return dt_bound;
    }
    case DRUCKER_PRAGER:  // sand.rs:345-362
        return elastic_wave_dt(m.lambda, m.mu, 1.0f, density, MIN_J, cell, mat_cfl);
    case SNOW:  // snow.rs:193-211
        return elastic_wave_dt(m.lambda, m.mu, h, density, MIN_J, cell, mat_cfl);
    case NACC: {  // nacc.rs:279-298
        float lambda = m.kappa - m.mu;
        return elastic_wave_dt(lambda, m.mu, h, density, m.nacc_min_density, cell, mat_cfl);
    }
    case COROTATED:       // corotated.rs timestep_bound
    case GRANULAR_FLUID:  // granular_fluid.rs timestep_bound
        return elastic_wave_dt(m.lambda, m.mu, h, density, MIN_J, cell, mat_cfl);
    case VON_MISES:  // von_mises.rs, rankine.rs, sand_mui.rs timestep_bound
    case RANKINE:
    case DP_MUI:
        return elastic_wave_dt(m.lambda, m.mu, 1.0f, density, MIN_J, cell, mat_cfl);
    case VISCOELASTIC: {  // viscoelastic.rs timestep_bound
        float elastic_dt = elastic_wave_dt(m.lambda, m.mu, 1.0f, density, 1.0e-6f, cell, mat_cfl);
        float viscous_dt = INFINITY;
        if (m.viscosity > 0.0f) {
            float d = fmax_(density, 1.0e-6f);
            float kinematic = m.viscosity / d;
            if (kinematic > F32_EPS) viscous_dt = visc_cfl * cell * cell / kinematic;
        }
        return fmin_(elastic_dt, viscous_dt);
    }
    default:
        return INFINITY;
    }
}

// MaterialModel::init_particle
void init_particle(const Mat &m, P &p) {
    switch (m.model) {
    case DRUCKER_PRAGER:  // sand.rs:237-246
        p.friction_hardening = m.hardening_peak > 0.0f ? m.friction_residual / m.hardening_peak
                                                       : 0.0f;
        break;
    case SNOW:  // snow.rs:104-107
        p.plastic_volume_ratio = 1.0f;
        p.hardening_scale = 1.0f;
        break;
    case NACC:  // nacc.rs:271-273
        p.log_volume_strain = 0.0f;
        break;
    case COROTATED:  // corotated.rs init_particle
        p.hardening_scale = 1.0f;
        p.plastic_volume_ratio = 1.0f;
        break;
    case GRANULAR_FLUID:  // granular_fluid.rs init_particle
        p.plastic_volume_ratio = 1.0f;
        p.hardening_scale = 1.0f;
        break;
    case DP_MUI:  // sand_mui.rs init_particle
        p.friction_hardening = m.mu_static;
        break;
    default:
        break;
    }
}

// Hencky strains of singular values (utils.rs hencky_strains).
inline V2 hencky(V2 sigma) {
    V2 s = vmax(vabs(sigma), splat(LOG_CLAMP));
    return v2(m_log(s.x), m_log(s.y));
}

// stress_to_hencky (utils.rs): principal Kirchhoff stress -> Hencky strain.
inline V2 stress_to_hencky(V2 tau, float lambda, float mu) {
    float d = 4.0f * mu * (mu + lambda);
    float a = 2.0f * mu + lambda;
    return v2((a * tau.x - lambda * tau.y) / d, (a * tau.y - lambda * tau.x) / d);
}

// rankine_damage_saturation_point (utils.rs)
inline float rankine_saturation(float softening_rate) {
    if (softening_rate <= 0.0f) return INFINITY;
    return -m_log(0.05f) / softening_rate;
}

// Shared tail of the elastoplastic updates: volume/density from J.
inline void sync_volume_density(P &p, M2 f) {
    float j = fmax_(det(f), MIN_J);
    float v = fmax_(p.initial_volume * j, 1.0e-6f);
    p.volume = v;
    p.density = p.mass / v;
}

// MaterialModel::update_particle
void update_particle(const Mat &m, P &p, float dt) {
    switch (m.model) {
    case NEOHOOKEAN: {  // elastic.rs:262-269
        M2 fp_new = madd(ident(), smscale(dt, load_m(p.c)));
        M2 f = mm(fp_new, load_m(p.f));
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case FLUID: {  // fluid.rs:197-207
        float j = fclamp(det(load_m(p.f)), 0.5f, 2.0f);
        float s = std::sqrt(j);
        store_m(p.f, m2(v2(s, 0.0f), v2(0.0f, s)));
        if (m.settling_damping > 0.0f) {
            float k = 1.0f - fmin_(m.settling_damping * dt, 0.5f);
            p.v[0] *= k;
            p.v[1] *= k;
        }
        break;
    }
    case DRUCKER_PRAGER: {  // sand.rs:248-319
        M2 f_trial = mm(madd(ident(), smscale(dt, load_m(p.c))), load_m(p.f));
        M2 u, vt;
        V2 sigma;
        svd2(f_trial, u, sigma, vt);
        V2 new_sigma = sigma;
        V2 proj;
        float dq;
        if (dp_project(m, sigma, p.log_volume_strain, p.friction_hardening, proj, dq)) {
            V2 sigma_abs = vmax(vabs(sigma), splat(LOG_CLAMP));
            float prev_det = sigma_abs.x * sigma_abs.y;
            float new_det = proj.x * proj.y;
            float diff = new_det - prev_det;
            float corrected = diff > 0.0f ? new_det : prev_det + diff * m.volume_correction;
            p.log_volume_strain += m_log(prev_det) - m_log(corrected);
            float q_max = 5.0f / fmax_(m.hardening_decay, 1e-6f);
            p.friction_hardening = fmin_(p.friction_hardening + dq, q_max);
            if (m.dilatancy_angle > 0.0f) p.log_volume_strain += m_sin(m.dilatancy_angle) * dq;
            new_sigma = proj;
        }
        new_sigma = vabs(new_sigma);
        float j_new = new_sigma.x * new_sigma.y;
        if (j_new < m.min_volume_jacobian)
            new_sigma = muls(new_sigma, std::sqrt(m.min_volume_jacobian / fmax_(j_new, 1e-6f)));
        M2 f = mm(mm(u, diag(new_sigma)), vt);
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case SNOW: {  // snow.rs:142-176
        M2 f_trial = mm(madd(ident(), smscale(dt, load_m(p.c))), load_m(p.f));
        M2 u, vt;
        V2 sigma;
        svd2(f_trial, u, sigma, vt);
        float lo = 1.0f - m.compression_limit, hi = 1.0f + m.stretch_limit;
        V2 sigma_c = v2(fclamp(sigma.x, lo, hi), fclamp(sigma.y, lo, hi));
        float jp_new = p.plastic_volume_ratio * (sigma.x * sigma.y) / (sigma_c.x * sigma_c.y);
        p.plastic_volume_ratio = fclamp(jp_new, m.min_plastic_jacobian, m.max_plastic_jacobian);
        p.hardening_scale =
            fclamp(m_exp(m.hardening_exponent * (1.0f - p.plastic_volume_ratio)), 0.1f, 7.0f);
        M2 f = mm(mm(u, diag(sigma_c)), vt);
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case COROTATED:      // corotated.rs update_particle
    case VISCOELASTIC: {  // viscoelastic.rs update_particle
        M2 fp_new = madd(ident(), smscale(dt, load_m(p.c)));
        M2 f = mm(fp_new, load_m(p.f));
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case VON_MISES: {  // von_mises.rs update_particle
        M2 f_trial = mm(madd(ident(), smscale(dt, load_m(p.c))), load_m(p.f));
        M2 u, vt;
        V2 sigma;
        svd2(f_trial, u, sigma, vt);
        V2 eps = hencky(sigma);
        float tr = eps.x + eps.y;
        V2 dev = sub(eps, splat(tr * 0.5f));
        float dev_norm = length(dev);
        float kappa = p.friction_hardening;
        float effective_yield = m.yield_stress + m.hardening_modulus * kappa;
        float elastic_dev = 2.0f * m.mu * dev_norm;
        V2 sigma_new = sigma;
        if (elastic_dev > effective_yield && dev_norm > LOG_CLAMP) {
            float denom = 2.0f * m.mu + m.hardening_modulus;
            float gamma = denom > F32_EPS ? (elastic_dev - effective_yield) / denom : 0.0f;
            p.friction_hardening = kappa + gamma;
            V2 eps_proj = add(muls(dev, effective_yield / elastic_dev), splat(tr * 0.5f));
            sigma_new = v2(m_exp(eps_proj.x), m_exp(eps_proj.y));
        }
        M2 f = reconstruct(u, sigma_new, vt);
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case RANKINE: {  // rankine.rs update_particle
        M2 f_trial = mm(madd(ident(), smscale(dt, load_m(p.c))), load_m(p.f));
        M2 u, vt;
        V2 sigma;
        svd2(f_trial, u, sigma, vt);
        V2 eps = hencky(sigma);
        float a = 2.0f * m.mu + m.lambda;
        V2 tau = v2(a * eps.x + m.lambda * eps.y, m.lambda * eps.x + a * eps.y);
        float damage = p.friction_hardening;
        float ts = m.tensile_strength;
        float t_eff = fmax_(ts * m_exp(-m.softening_rate * damage), ts * 0.05f);
        bool t1 = tau.x > t_eff, t2 = tau.y > t_eff;
        V2 sigma_new = sigma;
        if (t1 || t2) {
            V2 tau_proj = (t1 && t2) ? splat(t_eff) : (t1 ? v2(t_eff, tau.y) : v2(tau.x, t_eff));
            V2 eps_proj = stress_to_hencky(tau_proj, m.lambda, m.mu);
            V2 eps_trial = stress_to_hencky(tau, m.lambda, m.mu);
            p.friction_hardening = fmin_(damage + length(sub(eps_trial, eps_proj)),
                                         rankine_saturation(m.softening_rate));
            sigma_new = v2(m_exp(eps_proj.x), m_exp(eps_proj.y));
        }
        M2 f = reconstruct(u, sigma_new, vt);
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case DP_MUI: {  // sand_mui.rs update_particle
        const float SQRT_2 = 1.41421356237f;  // std::f32::consts::SQRT_2
        M2 f_trial = mm(madd(ident(), smscale(dt, load_m(p.c))), load_m(p.f));
        M2 u, vt;
        V2 sigma;
        svd2(f_trial, u, sigma, vt);
        V2 eps = hencky(sigma);
        float tr = eps.x + eps.y;
        float k_2d = m.lambda + m.mu;
        float p_trial = -k_2d * tr;
        if (p_trial <= 0.0f) {
            M2 f = reconstruct(u, v2(1.0f, 1.0f), vt);
            store_m(p.f, f);
            p.friction_hardening = m.mu_static;
            sync_volume_density(p, f);
            break;
        }
        V2 dev = sub(eps, splat(tr * 0.5f));
        float dev_norm = length(dev);
        float q_trial = SQRT_2 * m.mu * dev_norm;
        float q_yield = m.mu_static * p_trial;
        if (q_trial <= q_yield || dev_norm < F32_EPS) {
            M2 f = reconstruct(u, sigma, vt);
            store_m(p.f, f);
            p.friction_hardening = m.mu_static;
            sync_volume_density(p, f);
            break;
        }
        float delta_q = q_trial - q_yield;
        float sqrt_p = std::sqrt(p_trial);
        float a = m.mu * dt;
        float b = p_trial * (m.mu_dynamic - m.mu_static) + a * m.inertial_q * sqrt_p - delta_q;
        float c = -delta_q * m.inertial_q * sqrt_p;
        float gamma_dot = fmax_((-b + std::sqrt(b * b - 4.0f * a * c)) / (2.0f * a), 0.0f);
        float mu_i = gamma_dot > F32_EPS
                         ? m.mu_static + (m.mu_dynamic - m.mu_static) /
                                             (m.inertial_q * sqrt_p / gamma_dot + 1.0f)
                         : m.mu_static;
        float delta_gamma = gamma_dot * dt;
        V2 n_hat = v2(dev.x / dev_norm, dev.y / dev_norm);
        V2 eps_new = sub(eps, muls(n_hat, delta_gamma / SQRT_2));
        M2 f = reconstruct(u, v2(m_exp(eps_new.x), m_exp(eps_new.y)), vt);
        store_m(p.f, f);
        p.friction_hardening = mu_i;
        sync_volume_density(p, f);
        break;
    }
    case GRANULAR_FLUID: {  // granular_fluid.rs update_particle
        M2 f_trial = mm(madd(ident(), smscale(dt, load_m(p.c))), load_m(p.f));
        M2 f = f_trial;
        if (m.compression_limit > 0.0f || m.stretch_limit > 0.0f) {
            M2 u, vt;
            V2 sigma;
            svd2(f_trial, u, sigma, vt);
            float lo = 1.0f - m.compression_limit, hi = 1.0f + m.stretch_limit;
            V2 sigma_c = v2(fclamp(sigma.x, lo, hi), fclamp(sigma.y, lo, hi));
            float jp_new = p.plastic_volume_ratio * (sigma.x * sigma.y) /
                           fmax_(sigma_c.x * sigma_c.y, 1.0e-10f);
            p.plastic_volume_ratio = fclamp(jp_new, m.min_plastic_jacobian, m.max_plastic_jacobian);
            p.hardening_scale =
                fclamp(m_exp(m.hardening_exponent * (1.0f - p.plastic_volume_ratio)), 0.1f, 7.0f);
            f = mm(mm(u, diag(sigma_c)), vt);
        }
        store_m(p.f, f);
        sync_volume_density(p, f);
        break;
    }
    case NACC: {  // nacc.rs:255-269
        M2 nf;
        float na;
        nacc_project(m, load_m(p.f), p.log_volume_strain, nf, na);
        store_m(p.f, nf);
        p.log_volume_strain = na;
        float j = fmax_(det(nf), MIN_J);
        float vol = p.initial_volume * j;
        p.volume = vol;
        p.density = vol > MIN_J ? p.mass / vol : p.density;
        break;
    }
    default:
        break;
    }
}

inline bool needs_density_recompute(const Mat &m) { return m.model == FLUID; }

// ---------------------------------------------------------------- boundary
// apply_slip_wall_velocity (forces/boundary/mod.rs:78-101)
inline void slip_velocity(size_t thickness, size_t cell_index, size_t res, V2 &v) {
    size_t hi = res - (thickness + 1);
    size_t x = cell_index / res;
    size_t y = cell_index % res;
    if (x < thickness) v.x = fmax_(v.x, 0.0f);
    if (x > hi) v.x = fmin_(v.x, 0.0f);
    if (y < thickness) v.y = fmax_(v.y, 0.0f);
    if (y > hi) v.y = fmin_(v.y, 0.0f);
}

inline size_t sat_sub(size_t a, size_t b) { return a > b ? a - b : 0; }

// clamp_position_inside_grid (forces/boundary/mod.rs:103-111)
inline V2 clamp_position(size_t thickness, V2 pos, size_t res) {
    float mn = static_cast<float>(sat_sub(thickness, 1));
    float mx = static_cast<float>(sat_sub(res, thickness));
    return vclamp(pos, splat(mn), splat(mx));
}

// ---------------------------------------------------------------- grid/mod.rs
struct Grid {
    size_t res = 0;
    std::vector<float> mass;
    std::vector<V2> mom;
    std::vector<uint8_t> touched;
    std::vector<uint32_t> dirty;  // first-touch order (mod.rs:127)
    std::vector<V2> pre;          // ASFLIP pre-force snapshot, valid at touched cells
    // multi-field contact (grid/contact.rs:10-124): grip field, point cloud, resolution
    std::vector<float> grip_mass;
    std::vector<V2> grip_mom, grip_v, rest_v;
    std::vector<uint8_t> contact_touched;
    std::vector<uint32_t> contact_dirty;
    std::unordered_map<uint32_t, std::vector<std::pair<V2, float>>> points;
    // two-phase mixture (grid/mixture.rs:7-85)
    std::vector<float> solid_mass, fluid_mass;
    std::vector<V2> solid_mom, fluid_mom, solid_v, fluid_v;
    std::vector<uint8_t> mixture_touched;
    std::vector<uint32_t> mixture_dirty;

    void init(size_t r) {
        res = r;
        mass.assign(r * r, 0.0f);
        mom.assign(r * r, v2(0, 0));
        touched.assign(r * r, 0);
        pre.assign(r * r, v2(0, 0));
        dirty.clear();
        grip_mass.assign(r * r, 0.0f);
        grip_mom.assign(r * r, v2(0, 0));
        grip_v.assign(r * r, v2(0, 0));
        rest_v.assign(r * r, v2(0, 0));
        contact_touched.assign(r * r, 0);
        contact_dirty.clear();
        points.clear();
        solid_mass.assign(r * r, 0.0f);
        fluid_mass.assign(r * r, 0.0f);
        solid_mom.assign(r * r, v2(0, 0));
        fluid_mom.assign(r * r, v2(0, 0));
        solid_v.assign(r * r, v2(0, 0));
        fluid_v.assign(r * r, v2(0, 0));
        mixture_touched.assign(r * r, 0);
        mixture_dirty.clear();
    }
    bool has_contact_activity() const { return !contact_dirty.empty(); }
    // add_grip_mass_momentum (contact.rs:41-72)
    void add_grip(IV2 c, float m, V2 p) {
        uint32_t idx;
        if (!flat_index(c, idx)) return;
        if (contact_touched[idx]) {
            grip_mass[idx] += m;
            grip_mom[idx] = ::add(grip_mom[idx], p);
        } else {
            contact_touched[idx] = 1;
            contact_dirty.push_back(idx);
            grip_mass[idx] = m;
            grip_mom[idx] = p;
            grip_v[idx] = rest_v[idx] = v2(0, 0);
        }
    }
    // add_contact_point (contact.rs:74-85): only at cells of the grip field
    void add_point(IV2 c, V2 x, float label) {
        uint32_t idx;
        if (!flat_index(c, idx) || !contact_touched[idx]) return;
        points[idx].push_back({x, label});
    }
    // add_mixture_mass_momentum (mixture.rs:20-58); phase 1 solid, 2 fluid
    void add_mixture(IV2 c, uint32_t phase, float m, V2 p) {
        uint32_t idx;
        if (!flat_index(c, idx)) return;
        if (!mixture_touched[idx]) {
            mixture_touched[idx] = 1;
            mixture_dirty.push_back(idx);
            solid_mass[idx] = fluid_mass[idx] = 0.0f;
            solid_mom[idx] = fluid_mom[idx] = v2(0, 0);
            solid_v[idx] = fluid_v[idx] = v2(0, 0);
            if (phase == 1) {
                solid_mass[idx] = m;
                solid_mom[idx] = p;
            } else {
                fluid_mass[idx] = m;
                fluid_mom[idx] = p;
            }
            return;
        }
        if (phase == 1) {
            solid_mass[idx] += m;
            solid_mom[idx] = ::add(solid_mom[idx], p);
        } else {
            fluid_mass[idx] += m;
            fluid_mom[idx] = ::add(fluid_mom[idx], p);
        }
    }
    // cell_is_active (grid/mod.rs:231-241): the cell is in the dirty set
    bool cell_is_active(IV2 c) const {
        uint32_t idx;
        return flat_index(c, idx) && touched[idx];
    }
    // snapshot_velocities / pre_force_velocity_at (grid/mod.rs:300-317): the snapshot's
    // keys are the dirty cells, which stay touched until the next clear.
    V2 pre_force_velocity_at(IV2 c) const {
        uint32_t idx;
        if (!flat_index(c, idx) || !touched[idx]) return v2(0, 0);
        return pre[idx];
    }
    // Grid::clear (mod.rs:163-176)
    void clear() {
        for (uint32_t idx : dirty) {
            mass[idx] = 0.0f;
            mom[idx] = v2(0, 0);
            touched[idx] = 0;
        }
        dirty.clear();
        for (uint32_t idx : contact_dirty) contact_touched[idx] = 0;
        contact_dirty.clear();
        points.clear();
        for (uint32_t idx : mixture_dirty) mixture_touched[idx] = 0;
        mixture_dirty.clear();
    }
    // flat_index (mod.rs:89-99)
    bool flat_index(IV2 c, uint32_t &idx) const {
        if (c.x < 0 || c.y < 0) return false;
        size_t x = static_cast<size_t>(c.x), y = static_cast<size_t>(c.y);
        if (x >= res || y >= res) return false;
        idx = static_cast<uint32_t>(x * res + y);
        return true;
    }
    // add_mass_momentum / accumulate (mod.rs:190-212)
    void add(IV2 c, float m, V2 p) {
        uint32_t idx;
        if (!flat_index(c, idx)) return;
        if (touched[idx]) {
            mass[idx] += m;
            mom[idx] = add2(mom[idx], p);
        } else {
            touched[idx] = 1;
            dirty.push_back(idx);
            mass[idx] = m;
            mom[idx] = p;
        }
    }
    static V2 add2(V2 a, V2 b) { return ::add(a, b); }
    // velocity_at (mod.rs:215-227): zero for out-of-domain and untouched cells.
    V2 velocity_at(IV2 c) const {
        uint32_t idx;
        if (!flat_index(c, idx)) return v2(0, 0);
        return touched[idx] ? mom[idx] : v2(0, 0);
    }
    float mass_at(IV2 c) const {
        uint32_t idx;
        if (!flat_index(c, idx)) return 0.0f;
        return touched[idx] ? mass[idx] : 0.0f;
    }
};

}  // namespace

// ---------------------------------------------------------------- Simulation
struct oracle_sim {
    oracle_config cfg{};
    std::vector<P> p;
    size_t active_count = 0;
    uint32_t next_tag = 1;
    std::vector<Mat> materials;
    std::vector<size_t> boundaries;  // slip thicknesses, in application order
    Grid grid;
    std::vector<oracle_force_field> fields;  // force_fields, application order
    std::vector<float> field_data;
    // DirectionalContactGrip (grid/directional_grip.rs), if set (lifecycle.rs:125-131)
    int grip_on = 0;
    float grip_mu_easy = 0.0f, grip_mu_resist = 0.0f;
    V2 grip_dir = {0.0f, 0.0f};
    float last_step_dt = 0.0f;
    size_t last_substeps = 0;
    size_t last_vel_clamp_count = 0;
    size_t last_j_projection_count = 0;
    float last_sim_time_dropped = 0.0f;
    double timing[7] = {0, 0, 0, 0, 0, 0, 0};

    // MaterialRegistry::get (registry.rs:66-76): unknown ids fall back to slot 0.
    const Mat &mat(uint32_t id) const {
        return id < materials.size() ? materials[id] : materials[0];
    }
    bool any_needs_density() const {
        for (const Mat &m : materials)
            if (needs_density_recompute(m)) return true;
        return false;
    }
};

namespace {

using clk = std::chrono::steady_clock;
inline double us_since(clk::time_point t) {
    return std::chrono::duration<double, std::micro>(clk::now() - t).count();
}

// SimConfig::validate (config.rs:247-299)
bool validate_config(const oracle_config &c) {
    if (c.grid_res < 4) return false;
    if (!(c.grid_cell_size > 0.0f)) return false;
    if (!(c.dt > 0.0f)) return false;
    if (!(c.cfl_coefficient > 0.0f)) return false;
    if (!(c.material_cfl_coefficient > 0.0f)) return false;
    if (!(c.viscous_timestep_coefficient > 0.0f)) return false;
    if (!(c.min_dt > 0.0f)) return false;
    if (!(c.min_dt <= c.dt)) return false;
    if (!(c.projection_min_density > 0.0f)) return false;
    if (!(c.projection_min_volume > 0.0f)) return false;
    if (!(c.projection_min_deformation_j > 0.0f)) return false;
    if (!(c.particle_mass > 0.0f)) return false;
    if (!(c.contact_friction >= 0.0f)) return false;
    if (c.max_substeps_per_step == 0) return false;
    if (!(c.default_initial_volume > 0.0f)) return false;
    if (!(c.j_max > 1.0f)) return false;
    if (!(c.apic_blend >= 0.0f && c.apic_blend <= 1.0f)) return false;
    if (!(c.boundary_thickness > 0 && c.boundary_thickness < c.grid_res - 1)) return false;
    return true;
}

// SpawnRegion::fits_in_sim (config.rs:472-482) + validate_for_sim (:485-505)
bool spawn_fits(const oracle_spawn &s, const oracle_config &c) {
    if (!(s.spacing > 0.0f) || s.box_size[0] <= 0 || s.box_size[1] <= 0) return false;
    V2 half = muls(v2(static_cast<float>(s.box_size[0]), static_cast<float>(s.box_size[1])), 0.5f);
    V2 mn = sub(v2(s.box_center[0], s.box_center[1]), half);
    V2 mx = add(v2(s.box_center[0], s.box_center[1]), half);
    float dmin = static_cast<float>(c.boundary_thickness);
    float dmax = static_cast<float>(sat_sub(c.grid_res, c.boundary_thickness));
    return mn.x >= dmin && mn.y >= dmin && mx.x <= dmax && mx.y <= dmax;
}

// LcgRng (spacetime/solver/mod.rs:154-175)
struct Lcg {
    uint32_t state;
    uint32_t next_u32() {
        state = state * 1664525u + 1013904223u;
        return state;
    }
    float next_f32() { return static_cast<float>(next_u32()) / 4294967296.0f; }
};

// initialize_particles (spacetime/solver/mod.rs:88-151)
std::vector<P> initialize_particles(const oracle_config &c, const oracle_spawn &s, Lcg &rng) {
    float mass = s.has_mass_override ? s.mass_override : c.particle_mass;
    std::vector<P> out;
    V2 half = muls(v2(static_cast<float>(s.box_size[0]), static_cast<float>(s.box_size[1])), 0.5f);
    V2 center = v2(s.box_center[0], s.box_center[1]);
    V2 mn = sub(center, half);
    V2 mx = add(center, half);
    float i = mn.x;
    while (i < mx.x) {
        float j = mn.y;
        while (j < mx.y) {
            V2 pos = v2(i, j);
            bool inside = true;
            if (s.shape == 1) inside = length(sub(pos, center)) <= s.disk_radius;
            if (inside) {
                float jitter_mag = s.position_jitter * s.spacing;
                float jx = (rng.next_f32() - 0.5f) * 2.0f * jitter_mag;
                float jy = (rng.next_f32() - 0.5f) * 2.0f * jitter_mag;
                V2 jittered = add(pos, v2(jx, jy));
                float rx = rng.next_f32();
                float ry = rng.next_f32();
                V2 vel = muls(sub(v2(rx, ry), splat(0.5f)), s.initial_velocity_scale);
                P q;
                std::memset(&q, 0, sizeof(q));
                store_v(q.x, jittered);
                store_v(q.v, vel);
                std::memcpy(q.f, s.initial_deformation_gradient, sizeof(q.f));
                q.mass = mass;
                q.initial_volume = c.default_initial_volume;
                q.volume = c.default_initial_volume;
                q.density = mass / c.default_initial_volume;
                q.material_id = s.material_id;
                q.plastic_volume_ratio = 1.0f;
                q.hardening_scale = 1.0f;
                out.push_back(q);
            }
            j += s.spacing;
        }
        i += s.spacing;
    }
    return out;
}

// scatter_particle_mass (transfer/p2g.rs:230-243) over [0, count)
void scatter_particle_mass(oracle_sim &s, size_t count) {
    for (size_t i = 0; i < count; ++i) {
        V2 x = load_v(s.p[i].x);
        float mass = s.p[i].mass;
        QW w = quadratic_weights(x);
        for (int gx = 0; gx < 3; ++gx)
            for (int gy = 0; gy < 3; ++gy) {
                float weight = w.wx[gx] * w.wy[gy];
                IV2 cell{w.base.x + gx - 1, w.base.y + gy - 1};
                s.grid.add(cell, weight * mass, v2(0, 0));
            }
    }
}

// Density gather shared by estimate_particle_volumes / _local (density.rs:50-71,122-143)
void gather_density(oracle_sim &s, size_t lo, size_t hi, bool write_initial) {
    for (size_t i = lo; i < hi; ++i) {
        P &q = s.p[i];
        V2 x = load_v(q.x);
        float mass = q.mass;
        QW w = quadratic_weights(x);
        float density = 0.0f;
        for (int gx = 0; gx < 3; ++gx)
            for (int gy = 0; gy < 3; ++gy) {
                float weight = w.wx[gx] * w.wy[gy];
                IV2 cell{w.base.x + gx - 1, w.base.y + gy - 1};
                density += s.grid.mass_at(cell) * weight;
            }
        if (density > F32_EPS) {
            q.density = density;
            q.volume = mass / density;
            if (write_initial) q.initial_volume = q.volume;
        }
    }
}

// estimate_particle_volumes (density.rs:41-72)
void estimate_particle_volumes(oracle_sim &s, size_t count, bool write_initial) {
    s.grid.clear();
    scatter_particle_mass(s, count);
    gather_density(s, 0, count, write_initial);
}

// estimate_particle_volumes_local (density.rs:81-144)
void estimate_particle_volumes_local(oracle_sim &s, size_t active, size_t new_start,
                                     bool write_initial) {
    if (new_start >= active) return;
    V2 lo = splat(std::numeric_limits<float>::max());
    V2 hi = splat(std::numeric_limits<float>::lowest());
    for (size_t i = new_start; i < active; ++i) {
        lo = vmin(lo, load_v(s.p[i].x));
        hi = vmax(hi, load_v(s.p[i].x));
    }
    const float MARGIN = 3.0f;
    lo = sub(lo, splat(MARGIN));
    hi = add(hi, splat(MARGIN));
    s.grid.clear();
    for (size_t i = 0; i < active; ++i) {
        V2 x = load_v(s.p[i].x);
        if (x.x < lo.x || x.y < lo.y || x.x > hi.x || x.y > hi.y) continue;
        float mass = s.p[i].mass;
        QW w = quadratic_weights(x);
        for (int gx = 0; gx < 3; ++gx)
            for (int gy = 0; gy < 3; ++gy) {
                float weight = w.wx[gx] * w.wy[gy];
                IV2 cell{w.base.x + gx - 1, w.base.y + gy - 1};
                s.grid.add(cell, weight * mass, v2(0, 0));
            }
    }
    gather_density(s, new_start, active, write_initial);
}

// affine_cfl_speed_contribution (step.rs:481-488)
inline float affine_cfl(M2 c, float cell) {
    const float STENCIL_CORNER_DISTANCE = 1.5f * 1.41421356f;
    float grad_norm = std::sqrt(length_sq(c.xa) + length_sq(c.ya));
    return grad_norm * STENCIL_CORNER_DISTANCE * cell;
}

// cfl_bound (step.rs:472-479)
float cfl_bound(const oracle_config &c, float max_speed, float min_mat_dt, float max_dt) {
    float dt = max_dt;
    if (max_speed > F32_EPS) dt = fmin_(dt, c.cfl_coefficient * c.grid_cell_size / max_speed);
    dt = fmin_(dt, min_mat_dt);
    return fclamp(dt, fmin_(c.min_dt, max_dt), max_dt);
}

// choose_substep_dt (step.rs:434-468)
float choose_substep_dt(const oracle_sim &s, float max_dt) {
    const oracle_config &c = s.cfg;
    if (!c.adaptive_timestep) return fmin_(max_dt, c.dt);
    float max_speed = 0.0f;
    float min_mat_dt = max_dt;
    for (size_t i = 0; i < s.active_count; ++i) {
        const P &q = s.p[i];
        float sp = length(load_v(q.v));
        if (c.cfl_include_affine_speed) sp += affine_cfl(load_m(q.c), c.grid_cell_size);
        max_speed = fmax_(max_speed, sp);
        float mdt = timestep_bound(s.mat(q.material_id), q.density, q.hardening_scale,
                                   c.grid_cell_size, c.material_cfl_coefficient,
                                   c.viscous_timestep_coefficient);
        if (std::isfinite(mdt) && mdt > 0.0f) min_mat_dt = fmin_(min_mat_dt, mdt);
    }
    return cfl_bound(c, max_speed, min_mat_dt, max_dt);
}

// project_particle_state_to_admissible (step.rs:347-429)
bool project_particle(const oracle_config &c, P &q) {
    bool projected = false;
    float mn = static_cast<float>(sat_sub(c.boundary_thickness, 1));
    float mx = static_cast<float>(sat_sub(c.grid_res, c.boundary_thickness));
    V2 center = splat((mn + mx) * 0.5f);
    V2 x = load_v(q.x);
    if (!finite2(x)) {
        store_v(q.x, center);
        projected = true;
    } else {
        store_v(q.x, vclamp(x, splat(mn), splat(mx)));
    }
    if (!finite2(load_v(q.v))) {
        store_v(q.v, v2(0, 0));
        projected = true;
    }
    if (!finite_m(load_m(q.c))) {
        store_m(q.c, zero2());
        projected = true;
    }
    M2 f = load_m(q.f);
    if (!finite_m(f) || det(f) <= c.projection_min_deformation_j) {
        store_m(q.f, ident());
        projected = true;
    } else {
        float j = det(f);
        if (j > c.j_max) {
            store_m(q.f, mscale(f, std::sqrt(c.j_max / j)));
            projected = true;
        }
    }
    if (!std::isfinite(q.plastic_volume_ratio) || q.plastic_volume_ratio <= 0.0f) {
        q.plastic_volume_ratio = 1.0f;
        projected = true;
    }
    if (!std::isfinite(q.hardening_scale) || q.hardening_scale <= 0.0f) {
        q.hardening_scale = 1.0f;
        projected = true;
    }
    if (!std::isfinite(q.friction_hardening)) {
        q.friction_hardening = 0.0f;
        projected = true;
    }
    if (!std::isfinite(q.log_volume_strain)) {
        q.log_volume_strain = 0.0f;
        projected = true;
    }
    if (!std::isfinite(q.mass) || q.mass <= 0.0f) {
        q.mass = c.particle_mass;
        projected = true;
    }
    if (!std::isfinite(q.initial_volume) || q.initial_volume <= 0.0f) {
        q.initial_volume = fmax_(c.default_initial_volume, c.projection_min_volume);
        projected = true;
    }
    if (!std::isfinite(q.volume) || q.volume <= 0.0f) {
        q.volume = fmax_(q.initial_volume, c.projection_min_volume);
        projected = true;
    }
    if (!std::isfinite(q.density) || q.density <= 0.0f) {
        q.density = fmax_(q.mass / q.volume, c.projection_min_density);
        projected = true;
    } else {
        q.density = fmax_(q.density, c.projection_min_density);
    }
    return projected;
}

// scatter_particles_to_grid (transfer/p2g.rs:24-72); contact and mixture scatters are
// gated off (contact_group == 0, no mixture phase) for every supported scene.
void p2g(oracle_sim &s, float dt) {
    for (size_t i = 0; i < s.active_count; ++i) {
        const P &q = s.p[i];
        const Mat &m = s.mat(q.material_id);
        V2 x = load_v(q.x);
        float mass_i = q.mass;
        V2 v_i = load_v(q.v);
        M2 c_i = load_m(q.c);
        M2 stress = combined_kirchhoff_stress(m, q);
        float stress_coeff = -stress_volume(m, q) * KERNEL_D_INVERSE * dt;
        QW w = quadratic_weights(x);
        for (int gx = 0; gx < 3; ++gx)
            for (int gy = 0; gy < 3; ++gy) {
                float weight = w.wx[gx] * w.wy[gy];
                IV2 cell{w.base.x + gx - 1, w.base.y + gy - 1};
                V2 cell_dist = add(sub(v2(static_cast<float>(cell.x), static_cast<float>(cell.y)), x),
                                   splat(0.5f));
                V2 momentum = smul(weight, add(smul(mass_i, add(v_i, mv(c_i, cell_dist))),
                                               smul(stress_coeff, mv(stress, cell_dist))));
                s.grid.add(cell, weight * mass_i, momentum);
                if (q.contact_group != 0) s.grid.add_grip(cell, weight * mass_i, momentum);
                if (m.mixture_phase != 0) s.grid.add_mixture(cell, m.mixture_phase, weight * mass_i, momentum);
            }
    }
}

// gather_contact_point_cloud (p2g.rs:54-74): every active particle adds its position, labelled
// +1 (grip) or -1, to each stencil cell of the grip field, in index order.
void gather_contact_point_cloud(oracle_sim &s) {
    if (!s.grid.has_contact_activity()) return;
    for (size_t i = 0; i < s.active_count; ++i) {
        const P &q = s.p[i];
        V2 x = load_v(q.x);
        float label = q.contact_group != 0 ? 1.0f : -1.0f;
        QW w = quadratic_weights(x);
        for (int gx = 0; gx < 3; ++gx)
            for (int gy = 0; gy < 3; ++gy) s.grid.add_point(IV2{w.base.x + gx - 1, w.base.y + gy - 1}, x, label);
    }
}

// solve3x3 (contact_normal.rs): Cramer's rule, None for |det| <= EPSILON.
bool solve3x3(const float m[3][3], const float rhs[3], float out[3]) {
    auto det3 = [](const float a[3][3]) {
        return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
               a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
               a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    };
    float det = det3(m);
    if (std::fabs(det) <= F32_EPS) return false;
    for (int col = 0; col < 3; ++col) {
        float mm_[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) mm_[r][c] = m[r][c];
        for (int r = 0; r < 3; ++r) mm_[r][col] = rhs[r];
        out[col] = det3(mm_) / det;
    }
    return true;
}

// glam Vec2::normalize: self * (1 / length)
inline V2 normalize(V2 a) { return muls(a, 1.0f / length(a)); }

// fit_contact_normal_lr (contact_normal.rs): logistic regression of the point labels on
// position relative to the node, Newton steps with a small ridge penalty.
bool fit_contact_normal_lr(const std::vector<std::pair<V2, float>> &points, V2 node_pos, float cell, V2 &out) {
    bool has_grip = false, has_rest = false;
    for (const auto &pc : points) {
        if (pc.second > 0.0f) has_grip = true;
        if (pc.second < 0.0f) has_rest = true;
    }
    if (!has_grip || !has_rest) return false;
    const float dx2 = cell * cell;
    const float penalty[3] = {1.0e-7f * dx2, 1.0e-7f * dx2, 0.0f};
    float beta[3] = {0.0f, 0.0f, 0.0f};
    bool have_prev = false;
    V2 prev = v2(0, 0);
    for (int it = 0; it < 15; ++it) {
        float m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        float rhs[3] = {0, 0, 0};
        for (const auto &pc : points) {
            V2 rel = sub(pc.first, node_pos);
            const float xp[3] = {rel.x, rel.y, 1.0f};
            float z = fclamp(xp[0] * beta[0] + xp[1] * beta[1] + xp[2] * beta[2], -40.0f, 40.0f);
            float ez = m_exp(-z);
            float denom = 1.0f + ez;
            float f = 2.0f / denom - 1.0f;
            float sigma = 2.0f * ez / (denom * denom);
            float sigma_sq = sigma * sigma;
            for (int k = 0; k < 3; ++k) {
                for (int l = 0; l < 3; ++l) m[k][l] += sigma_sq * xp[k] * xp[l];
                rhs[k] += sigma * (pc.second - f) * xp[k];
            }
        }
        for (int k = 0; k < 3; ++k) {
            m[k][k] += penalty[k];
            rhs[k] -= penalty[k] * beta[k];
        }
        float delta[3];
        if (!solve3x3(m, rhs, delta)) break;
        if (!std::isfinite(delta[0]) || !std::isfinite(delta[1]) || !std::isfinite(delta[2])) break;
        for (int k = 0; k < 3; ++k) beta[k] += delta[k];
        V2 raw = v2(beta[0], beta[1]);
        if (length_sq(raw) <= F32_EPS || !finite2(raw)) continue;
        V2 n = normalize(raw);
        if (have_prev && 1.0f - dot(n, prev) < 1.0e-5f) {
            prev = n;
            break;
        }
        prev = n;
        have_prev = true;
    }
    if (!have_prev) return false;
    float gs = 0.0f, rs = 0.0f;
    size_t gc = 0, rc = 0;
    for (const auto &pc : points) {
        if (pc.second > 0.0f) {
            gs += dot(sub(pc.first, node_pos), prev);
            gc += 1;
        }
    }
    for (const auto &pc : points) {
        if (pc.second < 0.0f) {
            rs += dot(sub(pc.first, node_pos), prev);
            rc += 1;
        }
    }
    const float grip_mean = gs / static_cast<float>(gc > 0 ? gc : 1);
    const float rest_mean = rs / static_cast<float>(rc > 0 ? rc : 1);
    out = grip_mean < rest_mean ? v2(-prev.x, -prev.y) : prev;
    return true;
}

// apply_coulomb_wall (forces/boundary/mod.rs:60-76)
void apply_coulomb_wall(V2 &v, V2 n, float mu) {
    float v_n = dot(v, n);
    if (v_n >= 0.0f) return;
    float normal_speed = std::fabs(v_n);
    V2 v_t = sub(v, smul(v_n, n));
    float v_t_len = length(v_t);
    float friction_impulse = mu * normal_speed;
    v = v_t_len > friction_impulse ? muls(v_t, (v_t_len - friction_impulse) / v_t_len) : v2(0, 0);
}

// Grid::resolve_contact (contact.rs:254-391): per grip cell, the grip and rest velocities
// after Coulomb friction (or the directional grip) and the overlap correction.
void resolve_contact(oracle_sim &s, float dt, V2 gravity, float friction, float vel_limit, float cell) {
    Grid &g = s.grid;
    const float MIN_MASS_FRACTION = 1.0e-6f;
    auto clamp_speed = [&](V2 v) {
        float spd = length(v);
        return spd > vel_limit ? muls(v, vel_limit / spd) : v;
    };
    const size_t res = g.res;
    auto grip_mass_at = [&](int x, int y) -> float {
        uint32_t idx;
        if (!g.flat_index(IV2{x, y}, idx) || !g.contact_touched[idx]) return 0.0f;
        return g.grip_mass[idx];
    };
    for (uint32_t idx : g.contact_dirty) {
        const int cx = static_cast<int>(idx / res), cy = static_cast<int>(idx % res);
        V2 node_pos = v2(static_cast<float>(idx / res), static_cast<float>(idx % res));
        if (!g.touched[idx]) continue;
        const float total_mass = g.mass[idx];
        const V2 v_cm = g.mom[idx];  // normalised, gravity, boundaries, clamp
        const float grip_mass = g.grip_mass[idx];
        const V2 grip_momentum = g.grip_mom[idx];
        const float rest_mass = total_mass - grip_mass;
        if (grip_mass <= MIN_MASS_FRACTION || rest_mass <= MIN_MASS_FRACTION) {
            g.grip_v[idx] = v_cm;
            g.rest_v[idx] = v_cm;
            continue;
        }
        V2 v_grip = clamp_speed(add(divs(grip_momentum, grip_mass), muls(gravity, dt)));
        V2 fit;
        bool have = false;
        auto it = g.points.find(idx);
        static const std::vector<std::pair<V2, float>> none;
        if (fit_contact_normal_lr(it == g.points.end() ? none : it->second, node_pos, cell, fit) &&
            finite2(fit))
            have = true;
        if (!have) {  // grip_mass_gradient_normal (contact.rs:128-140)
            auto m = [&](int dx, int dy) { return grip_mass_at(cx + dx, cy + dy); };
            float gx_ = (m(1, -1) + 2.0f * m(1, 0) + m(1, 1)) - (m(-1, -1) + 2.0f * m(-1, 0) + m(-1, 1));
            float gy_ = (m(-1, 1) + 2.0f * m(0, 1) + m(1, 1)) - (m(-1, -1) + 2.0f * m(0, -1) + m(1, -1));
            V2 grad = v2(gx_, gy_);
            if (length_sq(grad) > F32_EPS) {
                fit = normalize(grad);
                have = true;
            }
        }
        V2 v_rel = sub(v_grip, v_cm);
        if (!have) {
            g.grip_v[idx] = v_grip;
            g.rest_v[idx] = clamp_speed(divs(sub(muls(v_cm, total_mass), muls(v_grip, grip_mass)), rest_mass));
            continue;
        }
        const V2 n = v2(-fit.x, -fit.y);
        if (s.grip_on) {  // DirectionalContactGrip::resolve (directional_grip.rs)
            V2 tangent = v2(-n.y, n.x);
            float v_t = dot(v_rel, tangent);
            float easy_t = dot(s.grip_dir, tangent);
            float mu = v_t * easy_t >= 0.0f ? s.grip_mu_easy : s.grip_mu_resist;
            apply_coulomb_wall(v_rel, n, mu);
        } else {
            apply_coulomb_wall(v_rel, n, friction);
        }
        float max_grip_proj = -INFINITY, min_rest_proj = INFINITY;
        if (it != g.points.end())
            for (const auto &pc : it->second) {
                float proj = dot(pc.first, n);
                if (pc.second > 0.0f) max_grip_proj = fmax_(max_grip_proj, proj);
                else if (pc.second < 0.0f) min_rest_proj = fmin_(min_rest_proj, proj);
            }
        if (std::isfinite(max_grip_proj) && std::isfinite(min_rest_proj)) {
            float gap = min_rest_proj - max_grip_proj;
            if (gap < 0.0f) {
                const float CORRECTION_RATE = 2.0f;
                float max_correction_speed = 0.5f * cell;
                float correction_speed = fmin_(CORRECTION_RATE * (-gap), max_correction_speed);
                float v_n = dot(v_rel, n);
                float target_vn = -correction_speed;
                if (v_n > target_vn) v_rel = add(v_rel, muls(n, target_vn - v_n));
            }
        }
        V2 v_grip_new = clamp_speed(add(v_cm, v_rel));
        V2 total_momentum = muls(v_cm, total_mass);
        g.grip_v[idx] = v_grip_new;
        g.rest_v[idx] = clamp_speed(divs(sub(total_momentum, muls(v_grip_new, grip_mass)), rest_mass));
    }
}

// Grid::resolve_mixture_coupling (mixture.rs:87-132) and project_mixture_incompressibility
// (:150-275): implicit Darcy drag between the phases per node, then Jacobi iterations of a
// mass-weighted pressure Poisson problem over the mixture nodes.
void resolve_mixture(oracle_sim &s, float dt, V2 gravity, float drag, float cell, uint32_t iterations) {
    Grid &g = s.grid;
    const size_t res = g.res;
    const float MIN_MASS_FRACTION = 1.0e-6f;
    if (drag <= 0.0f) {
        for (uint32_t idx : g.mixture_dirty) {
            if (!g.touched[idx]) continue;
            g.solid_v[idx] = g.fluid_v[idx] = g.mom[idx];
        }
        return;
    }
    for (uint32_t idx : g.mixture_dirty) {
        if (!g.touched[idx]) continue;
        const float m_s = g.solid_mass[idx], m_f = g.fluid_mass[idx];
        if (m_s <= MIN_MASS_FRACTION || m_f <= MIN_MASS_FRACTION) {
            g.solid_v[idx] = g.fluid_v[idx] = g.mom[idx];
            continue;
        }
        V2 v_s = add(divs(g.solid_mom[idx], m_s), muls(gravity, dt));
        V2 v_f = add(divs(g.fluid_mom[idx], m_f), muls(gravity, dt));
        float a = dt * drag / m_s;
        float b = dt * drag / m_f;
        float det_ = 1.0f + a + b;
        g.solid_v[idx] = divs(add(smul(1.0f + b, v_s), smul(a, v_f)), det_);
        g.fluid_v[idx] = divs(add(smul(b, v_s), smul(1.0f + a, v_f)), det_);
    }
    if (iterations == 0) return;
    const float MIN_MASS = 1.0e-6f;
    const float h = fmax_(cell, 1.0e-6f);
    auto pos_of = [&](uint32_t idx) { return IV2{static_cast<int>(idx / res), static_cast<int>(idx % res)}; };
    auto sv = [&](IV2 c) -> V2 {
        uint32_t i;
        return (g.flat_index(c, i) && g.mixture_touched[i]) ? g.solid_v[i] : v2(0, 0);
    };
    auto fv = [&](IV2 c) -> V2 {
        uint32_t i;
        return (g.flat_index(c, i) && g.mixture_touched[i]) ? g.fluid_v[i] : v2(0, 0);
    };
    std::unordered_map<uint32_t, float> alpha_s, alpha_f, mobility, rhs, pressure;
    std::unordered_map<uint32_t, std::pair<bool, bool>> significant;
    for (uint32_t idx : g.mixture_dirty) {
        IV2 pos = pos_of(idx);
        float m_s = fmax_(g.solid_mass[idx], 0.0f), m_f = fmax_(g.fluid_mass[idx], 0.0f);
        float n = m_s + m_f > MIN_MASS ? m_f / (m_s + m_f) : 0.0f;
        float a_s = 1.0f / fmax_(m_s, MIN_MASS);
        float a_f = 1.0f / fmax_(m_f, MIN_MASS);
        float k = (1.0f - n) * a_s + n * a_f;
        const float MIN_SIG = 0.01f;
        float total_mass = fmax_(m_s + m_f, MIN_MASS);
        bool solid_sig = m_s / total_mass > MIN_SIG, fluid_sig = m_f / total_mass > MIN_SIG;
        float vs_r = sv(IV2{pos.x + 1, pos.y}).x, vs_l = sv(IV2{pos.x - 1, pos.y}).x;
        float vs_u = sv(IV2{pos.x, pos.y + 1}).y, vs_d = sv(IV2{pos.x, pos.y - 1}).y;
        float div_vs = (vs_r - vs_l) / (2.0f * h) + (vs_u - vs_d) / (2.0f * h);
        float vf_r = fv(IV2{pos.x + 1, pos.y}).x, vf_l = fv(IV2{pos.x - 1, pos.y}).x;
        float vf_u = fv(IV2{pos.x, pos.y + 1}).y, vf_d = fv(IV2{pos.x, pos.y - 1}).y;
        float div_vf = (vf_r - vf_l) / (2.0f * h) + (vf_u - vf_d) / (2.0f * h);
        float residual = (1.0f - n) * div_vs + n * div_vf;
        alpha_s[idx] = a_s;
        alpha_f[idx] = a_f;
        significant[idx] = {solid_sig, fluid_sig};
        mobility[idx] = k;
        rhs[idx] = residual;
        pressure[idx] = 0.0f;
    }
    auto k_or_zero = [&](IV2 c) -> float {
        uint32_t i;
        if (!g.flat_index(c, i)) return 0.0f;
        auto it = mobility.find(i);
        return it == mobility.end() ? 0.0f : it->second;
    };
    auto p_or_zero = [&](const std::unordered_map<uint32_t, float> &p, IV2 c) -> float {
        uint32_t i;
        if (!g.flat_index(c, i)) return 0.0f;
        auto it = p.find(i);
        return it == p.end() ? 0.0f : it->second;
    };
    auto face_k = [](float ki, float kj) { return ki + kj > 1.0e-12f ? 2.0f * ki * kj / (ki + kj) : 0.0f; };
    for (uint32_t itn = 0; itn < iterations; ++itn) {
        std::unordered_map<uint32_t, float> next = pressure;
        for (uint32_t idx : g.mixture_dirty) {
            IV2 pos = pos_of(idx);
            float r = rhs[idx], k_i = mobility[idx];
            float k_r = face_k(k_i, k_or_zero(IV2{pos.x + 1, pos.y}));
            float k_l = face_k(k_i, k_or_zero(IV2{pos.x - 1, pos.y}));
            float k_u = face_k(k_i, k_or_zero(IV2{pos.x, pos.y + 1}));
            float k_d = face_k(k_i, k_or_zero(IV2{pos.x, pos.y - 1}));
            float k_sum = fmax_(k_r + k_l + k_u + k_d, 1.0e-9f);
            float p_r = p_or_zero(pressure, IV2{pos.x + 1, pos.y}), p_l = p_or_zero(pressure, IV2{pos.x - 1, pos.y});
            float p_u = p_or_zero(pressure, IV2{pos.x, pos.y + 1}), p_d = p_or_zero(pressure, IV2{pos.x, pos.y - 1});
            float weighted = k_r * p_r + k_l * p_l + k_u * p_u + k_d * p_d;
            next[idx] = (weighted - h * h * r) / k_sum;
        }
        pressure = next;
    }
    for (uint32_t idx : g.mixture_dirty) {
        IV2 pos = pos_of(idx);
        float p_r = p_or_zero(pressure, IV2{pos.x + 1, pos.y}), p_l = p_or_zero(pressure, IV2{pos.x - 1, pos.y});
        float p_u = p_or_zero(pressure, IV2{pos.x, pos.y + 1}), p_d = p_or_zero(pressure, IV2{pos.x, pos.y - 1});
        V2 grad_p = v2((p_r - p_l) / (2.0f * h), (p_u - p_d) / (2.0f * h));
        if (significant[idx].first) g.solid_v[idx] = sub(g.solid_v[idx], smul(alpha_s[idx], grad_p));
        if (significant[idx].second) g.fluid_v[idx] = sub(g.fluid_v[idx], smul(alpha_f[idx], grad_p));
    }
}

// Grid::update_velocities (grid/mod.rs:264-291) + boundaries (step.rs:150-152, 334-344)
// + grid speed clamp (step.rs:155-165)
void grid_update(oracle_sim &s, float dt) {
    Grid &g = s.grid;
    V2 grav = v2(s.cfg.gravity[0], s.cfg.gravity[1]);
    for (uint32_t idx : g.dirty)
        if (g.mass[idx] > 0.0f) g.mom[idx] = divs(g.mom[idx], g.mass[idx]);
    // ASFLIP snapshot between normalisation and gravity (step.rs:140-147)
    if (s.cfg.asflip_blend > 0.0f)
        for (uint32_t idx : g.dirty) g.pre[idx] = g.mom[idx];
    for (uint32_t idx : g.dirty)
        if (g.mass[idx] > 0.0f) g.mom[idx] = add(g.mom[idx], muls(grav, dt));
    size_t res = g.res;
    for (size_t t : s.boundaries)
        for (uint32_t idx : g.dirty)
            if (g.mass[idx] > 0.0f) slip_velocity(t, idx, res, g.mom[idx]);
    float vel_limit = s.cfg.grid_cell_size / dt;
    for (uint32_t idx : g.dirty) {
        if (g.mass[idx] > 0.0f) {
            float spd = length(g.mom[idx]);
            if (spd > vel_limit) g.mom[idx] = muls(g.mom[idx], vel_limit / spd);
        }
    }
    // multi-field contact and mixture coupling after the clamp (step.rs:166-197)
    resolve_contact(s, dt, grav, s.cfg.contact_friction, vel_limit, s.cfg.grid_cell_size);
    resolve_mixture(s, dt, grav, s.cfg.mixture_drag_coefficient, s.cfg.grid_cell_size,
                    s.cfg.mixture_pressure_iterations);
}

// gather_grid_to_particles (transfer/g2p.rs:151-343) with ASFLIP (g2p.rs:263-296);
// contact and mixture gated off (no grip or mixture particles).
// The grid velocity a particle reads at a node (g2p.rs:219-238): with contact active, the
// resolved grip velocity for grip particles and the rest velocity for the others; else a
// mixture particle's resolved phase velocity; both fall back to the total velocity at nodes
// outside their field.
V2 node_velocity(const oracle_sim &s, const P &q, IV2 cell, bool contact_active) {
    const Grid &g = s.grid;
    uint32_t idx;
    if (!g.flat_index(cell, idx)) return v2(0, 0);
    if (contact_active) {
        if (!g.contact_touched[idx]) return g.velocity_at(cell);
        return q.contact_group != 0 ? g.grip_v[idx] : g.rest_v[idx];
    }
    const uint32_t phase = s.mat(q.material_id).mixture_phase;
    if (phase != 0) {
        if (!g.mixture_touched[idx]) return g.velocity_at(cell);
        return phase == 1 ? g.solid_v[idx] : g.fluid_v[idx];
    }
    return g.velocity_at(cell);
}

size_t g2p(oracle_sim &s, float dt) {
    const bool contact_active = s.grid.has_contact_activity();
    const float vel_limit = s.cfg.grid_cell_size / dt;
    const float apic_blend = s.cfg.apic_blend;
    const float asflip_blend = s.cfg.asflip_blend;
    const size_t res = s.grid.res;
    const long n = static_cast<long>(s.active_count);
    std::vector<size_t> clamp_counts(static_cast<size_t>(n > 0 ? n : 0), 0);
    // Phase 1 (g2p.rs:189-328): independent per particle -> parallel, as rayon does.
    parallel_for(n, [&](long lo, long hi) {
        for (long ii = lo; ii < hi; ++ii) {
            P &q = s.p[static_cast<size_t>(ii)];
            V2 x = load_v(q.x);
            const V2 v_old = load_v(q.v);
            QW w = quadratic_weights(x);
            V2 new_v = v2(0, 0);
            M2 b = zero2();
            for (int gx = 0; gx < 3; ++gx)
                for (int gy = 0; gy < 3; ++gy) {
                    float weight = w.wx[gx] * w.wy[gy];
                    IV2 cell{w.base.x + gx - 1, w.base.y + gy - 1};
                    V2 dist = add(sub(v2(static_cast<float>(cell.x), static_cast<float>(cell.y)), x),
                                  splat(0.5f));
                    V2 node_v = node_velocity(s, q, cell, contact_active);
                    V2 wv = muls(node_v, weight);
                    M2 term = m2(muls(wv, dist.x), muls(wv, dist.y));
                    b = madd(b, term);
                    new_v = add(new_v, wv);
                }
            if (q.pinned != 0) {
                store_v(q.v, v2(0, 0));
                store_m(q.c, zero2());
                continue;
            }
            V2 v_store = new_v, v_pos = new_v;
            if (asflip_blend > 0.0f) {
                V2 old_v = v2(0, 0);
                for (int gx = 0; gx < 3; ++gx)
                    for (int gy = 0; gy < 3; ++gy) {
                        float weight = w.wx[gx] * w.wy[gy];
                        IV2 cell{w.base.x + gx - 1, w.base.y + gy - 1};
                        old_v = add(old_v, muls(s.grid.pre_force_velocity_at(cell), weight));
                    }
                V2 diff_vel = sub(v_old, old_v);
                float trace_b = b.xa.x + b.ya.y;
                float gamma = trace_b < 0.0f ? 0.0f : 1.0f;
                v_store = add(new_v, smul(asflip_blend, diff_vel));
                v_pos = add(new_v, smul(gamma * asflip_blend, diff_vel));
            }
            float spd = length(v_store);
            if (spd > vel_limit) {
                float scale = vel_limit / spd;
                v_store = muls(v_store, scale);
                v_pos = muls(v_pos, scale);
                clamp_counts[static_cast<size_t>(ii)] = 1;
            }
            V2 new_pos = add(x, muls(v_pos, dt));
            for (size_t t : s.boundaries) new_pos = clamp_position(t, new_pos, res);
            store_v(q.v, v_store);
            store_m(q.c, mscale(mscale(b, KERNEL_D_INVERSE), apic_blend));
            store_v(q.x, new_pos);
        }
    });
    size_t clamp_count = 0;
    for (size_t c : clamp_counts) clamp_count += c;
    // Phase 2 (g2p.rs:333-340): sequential constitutive update.
    for (size_t i = 0; i < s.active_count; ++i) update_particle(s.mat(s.p[i].material_id), s.p[i], dt);
    return clamp_count;
}

// smooth_cutoff (solver/cutoff.rs:17-26)
float smooth_cutoff(float r, float r_on, float r_cut) {
    if (r >= r_cut) return 0.0f;
    if (r <= r_on) return 1.0f;
    float x = (r - r_on) / (r_cut - r_on);
    return 1.0f - 3.0f * x * x + 2.0f * x * x * x;
}

// Charge of a material (HashMap lookup; a missing id has none).
float field_charge(const oracle_force_field &f, const float *data, uint32_t id, uint32_t skip) {
    return id < f.n_charges ? data[f.data_offset + skip + id] : 0.0f;
}

// Field::acceleration of the built-in fields (forces/fields/*.rs).
V2 field_acceleration(const oracle_force_field &f, const float *data, const P &q, uint32_t id) {
    const float *pr = f.params;
    const V2 x = load_v(q.x);
    switch (f.kind) {
    case 1: {  // GravityWellField (gravity.rs)
        V2 acc = v2(0, 0);
        float eps2 = pr[1] * pr[1];
        for (uint32_t k = 0; k < f.count; ++k) {
            const float *src = data + f.data_offset + 3 * k;
            V2 r_vec = sub(v2(src[0], src[1]), x);
            float r2 = length_sq(r_vec);
            float r = std::sqrt(r2);
            if (r >= pr[2] || r < F32_EPS) continue;
            float norm_s = r2 + eps2;
            float force_scale = pr[0] * src[2] / (norm_s * std::sqrt(norm_s));
            if (!std::isfinite(force_scale)) continue;
            float sw = smooth_cutoff(r, pr[3], pr[2]);
            acc = add(acc, muls(muls(r_vec, force_scale), sw));
        }
        return acc;
    }
    case 2: {  // BuoyancyField (buoyancy.rs)
        float rho = fmax_(q.density, pr[3]);
        return muls(v2(-pr[1], -pr[2]), pr[0] / rho);
    }
    case 3: {  // LinearDragField (drag.rs)
        if (f.material_mask != 0xFFFFFFFFu && (f.material_mask & (1u << (id & 31u))) == 0u)
            return v2(0, 0);
        return smul(pr[2], sub(v2(pr[0], pr[1]), load_v(q.v)));
    }
    case 4: {  // RadialConfinementField (confinement.rs)
        V2 r_vec = sub(x, v2(pr[0], pr[1]));
        float dist = length(r_vec);
        float overshoot = dist - pr[2];
        if (overshoot <= 0.0f || dist < F32_EPS) return v2(0, 0);
        return muls(v2(-r_vec.x, -r_vec.y), pr[3] * overshoot / dist);
    }
    case 5: {  // AabbConfinementField (confinement.rs)
        V2 acc = v2(0, 0);
        if (x.x < pr[0]) acc.x += pr[4] * (pr[0] - x.x);
        else if (x.x > pr[2]) acc.x -= pr[4] * (x.x - pr[2]);
        if (x.y < pr[1]) acc.y += pr[4] * (pr[1] - x.y);
        else if (x.y > pr[3]) acc.y -= pr[4] * (x.y - pr[3]);
        return acc;
    }
    case 6: {  // CoulombField (coulomb.rs)
        float q_p = field_charge(f, data, id, 3 * f.count);
        if (!(std::fabs(q_p) > F32_EPS)) return v2(0, 0);
        V2 acc = v2(0, 0);
        float eps2 = pr[1] * pr[1];
        float inv_mass = q.mass > F32_EPS ? 1.0f / q.mass : 0.0f;
        for (uint32_t k = 0; k < f.count; ++k) {
            const float *src = data + f.data_offset + 3 * k;
            V2 r_vec = sub(x, v2(src[0], src[1]));
            float r2 = length_sq(r_vec);
            float r = std::sqrt(r2);
            if (r >= pr[2] || r < F32_EPS) continue;
            float norm_s = r2 + eps2;
            float force_scale = pr[0] * src[2] * q_p / (norm_s * std::sqrt(norm_s));
            if (!std::isfinite(force_scale)) continue;
            float sw = smooth_cutoff(r, pr[3], pr[2]);
            acc = add(acc, muls(r_vec, force_scale * sw * inv_mass));
        }
        return acc;
    }
    case 7: {  // UniformElectricField (em.rs)
        float qc = field_charge(f, data, id, 0);
        if (!(std::fabs(qc) > F32_EPS)) return v2(0, 0);
        float inv_mass = q.mass > F32_EPS ? 1.0f / q.mass : 0.0f;
        return muls(v2(pr[0], pr[1]), qc * inv_mass);
    }
    case 8: {  // ChemotaxisField (chemotaxis.rs)
        if (f.material_filter != 0xFFFFFFFFu && id != f.material_filter) return v2(0, 0);
        const int res = static_cast<int>(f.count);
        const int ix = static_cast<int>(std::floor(x.x)), iy = static_cast<int>(std::floor(x.y));
        auto phi = [&](int xi, int yi) -> float {
            if (xi < 0 || yi < 0 || xi >= res || yi >= res) return 0.0f;
            return data[f.data_offset + static_cast<size_t>(xi) * res + yi];
        };
        V2 grad = v2((phi(ix + 1, iy) - phi(ix - 1, iy)) * 0.5f,
                     (phi(ix, iy + 1) - phi(ix, iy - 1)) * 0.5f);
        return smul(pr[0], grad);
    }
    default:
        return v2(0, 0);
    }
}

// ---- NBodyGravityField (forces/fields/n_body.rs): Barnes-Hut quadtree ----
// A pointer-free restatement of the reference's Node / Quadtree: nodes in one vector,
// children as four consecutive entries, built by inserting the bodies one at a time in
// index order (n_body.rs:143-175, 210-256) so that every node's MassProps accumulates in
// the reference's order.
struct NbNode {
    V2 center;
    float half;               // Aabb2 half size (square: both components equal)
    size_t depth;
    float mass = 0.0f;        // MassProps (n_body.rs:94-107)
    V2 com = {0.0f, 0.0f};
    std::vector<uint32_t> bodies;  // positions in the snapshot
    int64_t child = -1;       // first of the four children, -1 = none
};

struct NbTree {
    std::vector<NbNode> nodes;
    std::vector<V2> pos;          // snapshot: particles of positive mass, index order
    std::vector<float> mass;
    std::vector<uint32_t> index;  // their particle indices
    size_t max_depth = 8;
    size_t max_bodies = 4;
};

// MassProps::add (n_body.rs:96-107)
void nb_mass_add(NbNode &n, V2 p, float m) {
    const float nt = n.mass + m;
    if (nt > 0.0f) {
        n.com = divs(add(muls(n.com, n.mass), muls(p, m)), nt);
        n.mass = nt;
    }
}

// Aabb2::quadrant_of (n_body.rs:74-78): bit 0 right, bit 1 bottom.
size_t nb_quadrant(const NbNode &n, V2 p) {
    return static_cast<size_t>(p.x >= n.center.x) | (static_cast<size_t>(p.y < n.center.y) << 1);
}

// Node::insert (n_body.rs:143-175)
void nb_insert(NbTree &t, size_t node, uint32_t b) {
    nb_mass_add(t.nodes[node], t.pos[b], t.mass[b]);
    {
        NbNode &n = t.nodes[node];
        if (n.depth >= t.max_depth || (n.bodies.size() < t.max_bodies && n.child < 0)) {
            n.bodies.push_back(b);
            return;
        }
    }
    if (t.nodes[node].child < 0) {
        // quadrant_aabb (n_body.rs:80-91): the children's centers a quarter of the size away
        const V2 c = t.nodes[node].center;
        const float quarter = t.nodes[node].half * 0.5f;
        const size_t depth = t.nodes[node].depth + 1;
        const size_t first = t.nodes.size();
        for (size_t q = 0; q < 4; ++q) {
            NbNode ch;
            const float xs = (q & 1) == 0 ? -1.0f : 1.0f, ys = (q & 2) == 0 ? 1.0f : -1.0f;
            ch.center = add(c, v2(xs * quarter, ys * quarter));
            ch.half = quarter;
            ch.depth = depth;
            t.nodes.push_back(std::move(ch));
        }
        t.nodes[node].child = static_cast<int64_t>(first);
        std::vector<uint32_t> existing;
        existing.swap(t.nodes[node].bodies);
        for (uint32_t e : existing) nb_insert(t, first + nb_quadrant(t.nodes[node], t.pos[e]), e);
    }
    nb_insert(t, static_cast<size_t>(t.nodes[node].child) + nb_quadrant(t.nodes[node], t.pos[b]), b);
}

// NBodyGravityField::prepare + Quadtree::build (n_body.rs:210-256, 332-345): every particle of
// positive mass, the root box their bounding box padded and squared.
void nb_build(NbTree &t, const std::vector<P> &ps, size_t max_depth, size_t max_bodies) {
    t = NbTree{};
    t.max_depth = max_depth;
    t.max_bodies = max_bodies;
    for (size_t i = 0; i < ps.size(); ++i) {
        if (!(ps[i].mass > 0.0f)) continue;
        t.pos.push_back(load_v(ps[i].x));
        t.mass.push_back(ps[i].mass);
        t.index.push_back(static_cast<uint32_t>(i));
    }
    NbNode root;
    root.depth = 0;
    if (t.pos.empty()) {
        root.center = v2(0.0f, 0.0f);
        root.half = 1000.0f;  // EMPTY_TREE_HALF_SIZE
        t.nodes.push_back(std::move(root));
        return;
    }
    float min_x = std::numeric_limits<float>::max(), min_y = min_x;
    float max_x = std::numeric_limits<float>::lowest(), max_y = max_x;
    for (V2 p : t.pos) {
        min_x = fmin_(min_x, p.x);
        min_y = fmin_(min_y, p.y);
        max_x = fmax_(max_x, p.x);
        max_y = fmax_(max_y, p.y);
    }
    const float pad = ((max_x - min_x) + (max_y - min_y)) * 0.1f + 1.0f;  // AABB_PADDING_RATIO, _MIN
    min_x -= pad;
    min_y -= pad;
    max_x += pad;
    max_y += pad;
    root.center = v2((min_x + max_x) * 0.5f, (min_y + max_y) * 0.5f);
    root.half = fmax_(max_x - min_x, max_y - min_y) * 0.5f;
    t.nodes.push_back(std::move(root));
    for (uint32_t b = 0; b < t.pos.size(); ++b) nb_insert(t, 0, b);
}

// Plummer pull (n_body.rs:180-189, 199-207): zero when the scale is not finite.
V2 nb_pull(V2 r, float m, float g, float eps2) {
    const float ns = length_sq(r) + eps2;
    const float scale = g * m / (ns * std::sqrt(ns));
    return std::isfinite(scale) ? muls(r, scale) : v2(0.0f, 0.0f);
}

// Node::acceleration_on (n_body.rs:177-214) with is_far_enough (n_body.rs:131-141).
V2 nb_accel(const NbTree &t, size_t node, size_t self, V2 pos, float g, float soft, float theta) {
    const NbNode &n = t.nodes[node];
    const float eps2 = soft * soft;
    const float dist = length(sub(pos, n.center));
    const bool far = !(dist < soft || n.mass <= 0.0f) && (n.half * 2.0f) / dist < theta;
    if (far) return nb_pull(sub(n.com, pos), n.mass, g, eps2);
    if (n.child < 0) {
        V2 total = v2(0.0f, 0.0f);
        for (uint32_t b : n.bodies) {
            if (t.index[b] == self) continue;
            const V2 r = sub(t.pos[b], pos);
            if (length_sq(r) < eps2) continue;
            total = add(total, nb_pull(r, t.mass[b], g, eps2));
        }
        return total;
    }
    V2 total = v2(0.0f, 0.0f);
    for (size_t q = 0; q < 4; ++q)
        total = add(total, nb_accel(t, static_cast<size_t>(n.child) + q, self, pos, g, soft, theta));
    return total;
}

// Force fields (step.rs:212-259): prepare() of every field (the n-body trees), then
// v += dt * sum of accelerations, then the speed clamp.
void apply_force_fields(oracle_sim &s, float dt) {
    if (s.fields.empty()) return;
    const float *data = s.field_data.data();
    std::vector<NbTree> trees(s.fields.size());
    for (size_t k = 0; k < s.fields.size(); ++k) {
        const oracle_force_field &f = s.fields[k];
        if (f.kind == 9)
            nb_build(trees[k], s.p, static_cast<size_t>(f.params[3]), static_cast<size_t>(f.params[4]));
    }
    for (size_t i = 0; i < s.active_count; ++i) {
        P &q = s.p[i];
        if (q.pinned != 0) continue;
        V2 dv = v2(0, 0);
        for (size_t k = 0; k < s.fields.size(); ++k) {
            const oracle_force_field &f = s.fields[k];
            if (f.kind == 9)  // NBodyGravityField (n_body.rs:347-360)
                dv = add(dv, nb_accel(trees[k], 0, i, load_v(q.x), f.params[0], f.params[1], f.params[2]));
            else
                dv = add(dv, field_acceleration(f, data, q, q.material_id));
        }
        store_v(q.v, add(load_v(q.v), smul(dt, dv)));
    }
    const float vel_limit = s.cfg.grid_cell_size / dt;
    for (size_t i = 0; i < s.active_count; ++i) {
        P &q = s.p[i];
        if (q.pinned != 0) continue;
        V2 v = load_v(q.v);
        float spd = length(v);
        if (spd > vel_limit) store_v(q.v, muls(v, vel_limit / spd));
    }
}

// sleep_particle (solver/particles.rs:227-245): flag, swap with the last active particle
// (Particles::swap moves every field, particle.rs:403-429), shrink the active zone.
void sleep_particle(oracle_sim &s, size_t i) {
    if (s.p[i].sleeping || s.active_count == 0) return;
    s.p[i].sleeping = 1;
    size_t last_active = s.active_count - 1;
    if (i != last_active) std::swap(s.p[i], s.p[last_active]);
    s.active_count -= 1;
}

// wake_particle (solver/particles.rs:252-268): swap with the first sleeping particle.
void wake_particle(oracle_sim &s, size_t i) {
    if (!s.p[i].sleeping) return;
    s.p[i].sleeping = 0;
    size_t first_sleeping = s.active_count;
    if (i != first_sleeping) std::swap(s.p[i], s.p[first_sleeping]);
    s.active_count += 1;
}

// Wake after P2G (step.rs:107-131): sleeping particles whose stencil overlaps an active
// cell, woken in ascending index order.
void wake_touched(oracle_sim &s) {
    if (s.active_count >= s.p.size()) return;
    std::vector<size_t> to_wake;
    for (size_t i = s.active_count; i < s.p.size(); ++i) {
        QW w = quadratic_weights(load_v(s.p[i].x));
        bool hit = false;
        for (int gx = 0; gx < 3 && !hit; ++gx)
            for (int gy = 0; gy < 3 && !hit; ++gy)
                hit = s.grid.cell_is_active(IV2{w.base.x + gx - 1, w.base.y + gy - 1});
        if (hit) to_wake.push_back(i);
    }
    for (size_t i : to_wake) wake_particle(s, i);
}

// Sleep scoring at the end of a substep (step.rs:299-315): active particles with zero
// activation and speed below the threshold, put to sleep in descending index order.
void sleep_scoring(oracle_sim &s) {
    const float threshold = s.cfg.sleep_threshold;
    if (!(threshold > 0.0f)) return;
    const float threshold_sq = threshold * threshold;
    std::vector<size_t> to_sleep;
    for (size_t i = 0; i < s.active_count; ++i)
        if (s.p[i].activation == 0.0f && length_sq(load_v(s.p[i].v)) < threshold_sq) to_sleep.push_back(i);
    std::sort(to_sleep.begin(), to_sleep.end(), std::greater<size_t>());
    for (size_t i : to_sleep) sleep_particle(s, i);
}

// Simulation::do_substep (step.rs:62-317) restricted to the gated-on phases.
void do_substep(oracle_sim &s, float sub_dt) {
    auto t0 = clk::now();
    if (s.cfg.project_invalid_state)
        for (size_t i = 0; i < s.active_count; ++i)
            if (project_particle(s.cfg, s.p[i])) s.last_j_projection_count += 1;
    s.timing[1] += us_since(t0);
    t0 = clk::now();
    if (s.cfg.recompute_density_each_step || s.any_needs_density())
        estimate_particle_volumes(s, s.active_count, false);
    s.timing[2] += us_since(t0);
    t0 = clk::now();
    s.grid.clear();
    p2g(s, sub_dt);
    gather_contact_point_cloud(s);
    wake_touched(s);
    s.timing[3] += us_since(t0);
    t0 = clk::now();
    grid_update(s, sub_dt);
    s.timing[4] += us_since(t0);
    t0 = clk::now();
    s.last_vel_clamp_count += g2p(s, sub_dt);
    s.timing[5] += us_since(t0);
    apply_force_fields(s, sub_dt);
    sleep_scoring(s);
}

// Simulation::step (step.rs:23-60)
void step_once(oracle_sim &s) {
    auto t_start = clk::now();
    for (double &t : s.timing) t = 0.0;
    float remaining = s.cfg.dt;
    size_t substeps = 0;
    s.last_vel_clamp_count = 0;
    s.last_j_projection_count = 0;
    while (remaining > F32_EPS && substeps < s.cfg.max_substeps_per_step) {
        auto t_cfl = clk::now();
        float sub_dt = choose_substep_dt(s, remaining);
        s.timing[0] += us_since(t_cfl);
        do_substep(s, sub_dt);
        remaining -= sub_dt;
        s.last_step_dt = sub_dt;
        substeps += 1;
    }
    s.last_substeps = substeps;
    s.last_sim_time_dropped = fmax_(remaining, 0.0f);
    s.timing[6] = us_since(t_start);
}

}  // namespace

// ---------------------------------------------------------------- C API
extern "C" {

oracle_sim *oracle_create(const oracle_config *cfg) {
    if (!cfg || !validate_config(*cfg)) return nullptr;
    oracle_sim *s = new oracle_sim();
    s->cfg = *cfg;
    Mat fallback;
    std::memset(&fallback, 0, sizeof(fallback));
    fallback.model = FALLBACK;
    s->materials.push_back(fallback);
    s->boundaries.push_back(static_cast<size_t>(cfg->boundary_thickness));
    s->grid.init(static_cast<size_t>(cfg->grid_res));
    s->last_step_dt = cfg->dt;
    return s;
}

void oracle_destroy(oracle_sim *s) { delete s; }

int oracle_set_material(oracle_sim *s, uint32_t id, const oracle_material *m) {
    if (id >= MAX_MATERIAL_SLOTS) return -1;
    if (id < s->materials.size()) {
        s->materials[id] = *m;
    } else if (id == s->materials.size()) {
        s->materials.push_back(*m);
    } else {
        return -1;
    }
    if (id == 0)  // with_default_material -> reinit_all_particle_state (lifecycle.rs:328-334)
        for (P &q : s->p) init_particle(s->mat(q.material_id), q);
    return 0;
}

int oracle_add_slip_boundary(oracle_sim *s, uint64_t thickness, int clear_first) {
    if (clear_first) s->boundaries.clear();
    s->boundaries.push_back(static_cast<size_t>(thickness));
    return 0;
}

int oracle_add_body(oracle_sim *s, const oracle_spawn *spawn, uint32_t *tag_out) {
    if (!spawn_fits(*spawn, s->cfg)) return -1;
    uint32_t tag = s->next_tag++;
    size_t old_active = s->active_count;
    Lcg rng{spawn->rng_seed};
    std::vector<P> np = initialize_particles(s->cfg, *spawn, rng);
    bool registered = spawn->material_id < s->materials.size();
    for (P &q : np) {
        q.user_tag = tag;
        if (registered) init_particle(s->materials[spawn->material_id], q);
    }
    // New particles go before the sleeping zone (particles.rs:389-410): a rotation keeps
    // [active | new | sleeping].
    s->p.insert(s->p.begin() + static_cast<long>(old_active), np.begin(), np.end());
    s->active_count = old_active + np.size();
    estimate_particle_volumes_local(*s, s->active_count, old_active, true);
    if (tag_out) *tag_out = tag;
    return 0;
}

int oracle_init_with_spawn(oracle_sim *s, const oracle_spawn *spawn) {
    if (!spawn_fits(*spawn, s->cfg) || !s->p.empty()) return -1;
    Lcg rng{spawn->rng_seed};
    s->p = initialize_particles(s->cfg, *spawn, rng);
    s->active_count = s->p.size();
    if (spawn->precompute_initial_volumes) estimate_particle_volumes(*s, s->p.size(), true);
    return 0;
}

int oracle_push_particles(oracle_sim *s, const oracle_particle *p, uint64_t n) {
    s->p.insert(s->p.end(), p, p + n);
    s->active_count = s->p.size();
    return 0;
}

void oracle_step(oracle_sim *s, uint32_t n_steps) {
    for (uint32_t k = 0; k < n_steps; ++k) step_once(*s);
}

uint64_t oracle_particle_count(const oracle_sim *s) { return s->p.size(); }

uint64_t oracle_active_count(const oracle_sim *s) { return s->active_count; }

int oracle_replace_particles(oracle_sim *s, const oracle_particle *p, uint64_t n, uint64_t active_count) {
    if (active_count > n) return -1;
    s->p.assign(p, p + n);
    s->active_count = static_cast<size_t>(active_count);
    return 0;
}

// wake_tag / sleep_tag (solver/particles.rs:271-312); the tag's members are the particles
// carrying the tag.
void oracle_wake_tag(oracle_sim *s, uint32_t tag) {
    std::vector<size_t> idx;
    for (size_t i = 0; i < s->p.size(); ++i)
        if (s->p[i].user_tag == tag && s->p[i].sleeping) idx.push_back(i);
    for (size_t i : idx) wake_particle(*s, i);  // ascending
}

void oracle_sleep_tag(oracle_sim *s, uint32_t tag) {
    std::vector<size_t> idx;
    for (size_t i = 0; i < s->p.size(); ++i)
        if (s->p[i].user_tag == tag && !s->p[i].sleeping) idx.push_back(i);
    std::sort(idx.begin(), idx.end(), std::greater<size_t>());
    for (size_t i : idx) sleep_particle(*s, i);
}

void oracle_read_particles(const oracle_sim *s, oracle_particle *out) {
    std::memcpy(out, s->p.data(), s->p.size() * sizeof(P));
}

void oracle_write_particles(oracle_sim *s, const oracle_particle *in) {
    std::memcpy(s->p.data(), in, s->p.size() * sizeof(P));
}

// region_state (spacetime/solver/queries.rs:125-141): candidates in SpatialHash
// iteration order (spatial_hash.rs:47-105: cells gx outer, gy inner, each bucket in
// particle index order), exact |x-c|^2 <= r^2 filter, BodyState::accumulate/finalize
// (query.rs:123-142).
void oracle_region_state(const oracle_sim *s, float cx, float cy, float r,
                         oracle_body_state *out) {
    float inv_cell = 1.0f / s->cfg.grid_cell_size;
    auto cell_of = [&](V2 pp) {
        return std::make_pair(f2i_sat(std::floor(pp.x * inv_cell)),
                              f2i_sat(std::floor(pp.y * inv_cell)));
    };
    std::map<std::pair<int32_t, int32_t>, std::vector<size_t>> table;
    for (size_t i = 0; i < s->active_count; ++i) table[cell_of(load_v(s->p[i].x))].push_back(i);
    V2 center = v2(cx, cy);
    int32_t r_cells = f2i_sat(std::ceil(r * inv_cell));
    auto cc = cell_of(center);
    float r2 = r * r;
    uint64_t count = 0;
    V2 centroid = v2(0, 0);
    float avg_speed = 0, avg_vr = 0, max_vr = 0, avg_det = 0, avg_den = 0;
    for (int32_t gx = -r_cells; gx <= r_cells; ++gx)
        for (int32_t gy = -r_cells; gy <= r_cells; ++gy) {
            auto it = table.find(std::make_pair(cc.first + gx, cc.second + gy));
            if (it == table.end()) continue;
            for (size_t i : it->second) {
                const P &q = s->p[i];
                V2 x = load_v(q.x);
                if (length_sq(sub(x, center)) <= r2) {
                    count += 1;
                    centroid = add(centroid, x);
                    avg_speed += length(load_v(q.v));
                    avg_vr += q.plastic_volume_ratio;
                    max_vr = fmax_(max_vr, q.plastic_volume_ratio);
                    avg_det += det(load_m(q.f));
                    avg_den += q.density;
                }
            }
        }
    if (count > 0) {
        float n = static_cast<float>(count);
        centroid = divs(centroid, n);
        avg_speed /= n;
        avg_vr /= n;
        avg_det /= n;
        avg_den /= n;
    }
    std::memset(out, 0, sizeof(*out));
    out->count = count;
    out->avg_volume_ratio = avg_vr;
    out->max_volume_ratio = max_vr;
    out->avg_speed = avg_speed;
    out->avg_det_f = avg_det;
    out->avg_density = avg_den;
    out->centroid[0] = centroid.x;
    out->centroid[1] = centroid.y;
}

float oracle_effective_dt(const oracle_sim *s) { return s->last_step_dt; }
uint64_t oracle_last_substeps(const oracle_sim *s) { return s->last_substeps; }
uint64_t oracle_last_vel_clamp_count(const oracle_sim *s) { return s->last_vel_clamp_count; }
uint64_t oracle_last_j_projection_count(const oracle_sim *s) { return s->last_j_projection_count; }
void oracle_last_timing_us(const oracle_sim *s, double out[7]) {
    for (int i = 0; i < 7; ++i) out[i] = s->timing[i];
}

int oracle_set_threads(int n) {
    if (n >= 0) g_threads = n;
    return g_threads > 0 ? g_threads : static_cast<int>(std::thread::hardware_concurrency());
}

void oracle_svd2(const float f[4], float u[4], float sigma[2], float vt[4]) {
    M2 uu, vv;
    V2 ss;
    svd2(load_m(f), uu, ss, vv);
    store_m(u, uu);
    store_v(sigma, ss);
    store_m(vt, vv);
}

void oracle_polar(const float f[4], float r[4]) { store_m(r, polar(load_m(f))); }

void oracle_axis_weights(float d, float w[3]) { axis_weights(d, w); }

void oracle_kirchhoff(const oracle_material *m, const oracle_particle *p, float tau[4]) {
    store_m(tau, combined_kirchhoff_stress(*m, *p));
}

void oracle_set_correctly_rounded(int on) { g_correctly_rounded = on ? 1 : 0; }

void oracle_set_contact_grip(oracle_sim *s, int on, float mu_easy, float mu_resist, float dir_x,
                             float dir_y) {
    s->grip_on = on ? 1 : 0;
    s->grip_mu_easy = mu_easy;
    s->grip_mu_resist = mu_resist;
    V2 d = v2(dir_x, dir_y);
    s->grip_dir = normalize_or_zero(d);  // DirectionalContactGrip::new normalises
}

int oracle_fit_contact_normal(const float *points, uint32_t n, float node_x, float node_y,
                              float cell, float normal[2]) {
    std::vector<std::pair<V2, float>> pts;
    for (uint32_t k = 0; k < n; ++k) pts.push_back({v2(points[3 * k], points[3 * k + 1]), points[3 * k + 2]});
    V2 out;
    if (!fit_contact_normal_lr(pts, v2(node_x, node_y), cell, out)) return 0;
    normal[0] = out.x;
    normal[1] = out.y;
    return 1;
}

void oracle_field_acceleration(const oracle_force_field *f, const float *data,
                               const oracle_particle *p, float out[2]) {
    V2 a = field_acceleration(*f, data, *p, p->material_id);
    out[0] = a.x;
    out[1] = a.y;
}

void oracle_field_accelerations(oracle_sim *s, float *out) {
    const float *data = s->field_data.data();
    std::vector<NbTree> trees(s->fields.size());
    for (size_t k = 0; k < s->fields.size(); ++k) {
        const oracle_force_field &f = s->fields[k];
        if (f.kind == 9)
            nb_build(trees[k], s->p, static_cast<size_t>(f.params[3]), static_cast<size_t>(f.params[4]));
    }
    for (size_t i = 0; i < s->p.size(); ++i) {
        const P &q = s->p[i];
        V2 dv = v2(0, 0);
        for (size_t k = 0; k < s->fields.size(); ++k) {
            const oracle_force_field &f = s->fields[k];
            if (f.kind == 9)
                dv = add(dv, nb_accel(trees[k], 0, i, load_v(q.x), f.params[0], f.params[1], f.params[2]));
            else
                dv = add(dv, field_acceleration(f, data, q, q.material_id));
        }
        out[2 * i] = dv.x;
        out[2 * i + 1] = dv.y;
    }
}

int oracle_set_force_fields(oracle_sim *s, const oracle_force_field *fields, uint32_t n,
                            const float *data, uint64_t n_data) {
    for (uint32_t k = 0; k < n; ++k) {
        const oracle_force_field &f = fields[k];
        if (f.kind < 1 || f.kind > 9) return -1;
        if (f.kind == 9) {  // theta in (0, 1] (n_body.rs:306-311); integral depth and leaf size
            const float theta = f.params[2], depth = f.params[3], maxb = f.params[4];
            if (!(theta > 0.0f && theta <= 1.0f)) return -1;
            if (!(depth >= 0.0f && depth <= 24.0f && depth == std::floor(depth))) return -1;
            if (!(maxb >= 0.0f && maxb <= 2147483647.0f && maxb == std::floor(maxb))) return -1;
        }
        uint64_t need = 0;
        if (f.kind == 1) need = 3ull * f.count;
        if (f.kind == 6) need = 3ull * f.count + f.n_charges;
        if (f.kind == 7) need = f.n_charges;
        if (f.kind == 8) need = static_cast<uint64_t>(f.count) * f.count;
        if (static_cast<uint64_t>(f.data_offset) + need > n_data) return -1;
    }
    s->fields.assign(fields, fields + n);
    s->field_data.assign(data, data + n_data);
    return 0;
}

void oracle_update_particle(const oracle_material *m, oracle_particle *p, float dt) {
    update_particle(*m, *p, dt);
}

void oracle_init_particle(const oracle_material *m, oracle_particle *p) { init_particle(*m, *p); }

float oracle_timestep_bound(const oracle_material *m, float density, float h, float cell,
                            float mat_cfl, float visc_cfl) {
    return timestep_bound(*m, density, h, cell, mat_cfl, visc_cfl);
}

void oracle_nacc_project(const oracle_material *m, const float f[4], float alpha, float f_out[4],
                         float *alpha_out) {
    M2 nf;
    nacc_project(*m, load_m(f), alpha, nf, *alpha_out);
    store_m(f_out, nf);
}

int oracle_dp_project(const oracle_material *m, const float sigma[2], float lvs, float q,
                      float sigma_out[2], float *dq_out) {
    V2 o;
    float dq = 0.0f;
    bool r = dp_project(*m, load_v(sigma), lvs, q, o, dq);
    if (r) {
        store_v(sigma_out, o);
        *dq_out = dq;
    }
    return r ? 1 : 0;
}

void oracle_slip_velocity(uint64_t thickness, uint64_t cell_index, uint64_t res, float v[2]) {
    V2 vv = load_v(v);
    slip_velocity(static_cast<size_t>(thickness), static_cast<size_t>(cell_index),
                  static_cast<size_t>(res), vv);
    store_v(v, vv);
}

// block_index (systems/gpu/shaders/particle_sort.wgsl:94-102), NUM_BLOCKS_PER_DIM = 16.
uint32_t oracle_block_index(float px, float py, uint32_t grid_res) {
    const uint32_t NB = 16;
    uint32_t max_cell = grid_res - 1u;
    float fx = fmin_(fmax_(px, 0.0f), static_cast<float>(max_cell));
    float fy = fmin_(fmax_(py, 0.0f), static_cast<float>(max_cell));
    uint32_t cell_x = static_cast<uint32_t>(fx);
    uint32_t cell_y = static_cast<uint32_t>(fy);
    uint32_t block_size = (grid_res + NB - 1u) / NB;
    uint32_t bx = std::min(cell_x / block_size, NB - 1u);
    uint32_t by = std::min(cell_y / block_size, NB - 1u);
    return by * NB + bx;
}

void oracle_stable_argsort_u32(const uint32_t *keys, uint64_t n, uint32_t *perm_out) {
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::stable_sort(idx.begin(), idx.end(),
                     [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    std::memcpy(perm_out, idx.data(), n * sizeof(uint32_t));
}

int oracle_project_particle(const oracle_config *cfg, oracle_particle *p) {
    return project_particle(*cfg, *p) ? 1 : 0;
}

float oracle_choose_substep_dt(const oracle_sim *s, float max_dt) {
    return choose_substep_dt(*s, max_dt);
}

}  // extern "C"
