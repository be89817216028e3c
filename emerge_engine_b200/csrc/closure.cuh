// closure.cuh -- learned closure for the Drucker-Prager and NACC return mappings.
//
// A 6 -> 64 -> 64 -> 64 -> 3 SiLU MLP stands in for the smooth plastic branch of
//   DruckerPragerMaterial::project (sand.rs:156-194), in units of the trial deviatoric
//     norm s = |dev eps| (the mapping is invariant under that scaling): eps / s with
//     eps = ln|sigma| + lvs/2, alpha(q) (sand.rs:135), (lambda + mu) / mu,
//     cohesion / (2 mu s), ln s -> projected log-strain h / s (sigma' = exp(h)) and the
//     hardening increment dq / s;
//   NaccMaterial::project (nacc.rs:129-223), ellipse branch: ln(sv), p0 / kappa, mu / kappa,
//     beta, M -> the plastic correction ln(sv') - ln(sv) and the hardening increment
//     d(alpha) (predicting ln(sv') itself would ask the BF16 network to reproduce the
//     near-identity part to better than its 2^-8 resolution).
// The cheap, exact decisions stay exact: the yield test, the DP tip (trace > 0), and the
// NACC tension / compression caps and elastic test.  Only particles on the smooth plastic
// branch run the network; inputs outside the training data's box ("hull") use the plain
// mapping, and every step a sample of particles is also run through the plain mapping to
// measure the network's error in projected stress.
//
// Inference runs per warp on the tensor cores: mma.sync m16n8k16 BF16 x BF16 -> FP32,
// one 16-row tile (16 lanes' particles) at a time.  The FP32 accumulator fragments of two
// adjacent 8-column tiles are exactly the A-operand fragment of the next layer's 16-wide
// K slice, so activations never leave registers.  Weights are stored pre-swizzled in
// B-fragment order (one 8-byte load per lane per MMA).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

#include "physics.cuh"

namespace emerge {

constexpr int CL_IN = 6;       // network inputs
constexpr int CL_OUT = 3;      // network outputs
constexpr int CL_H = 64;       // hidden width
constexpr int CL_NMODELS = 2;  // 0 = DruckerPrager, 1 = NACC
// B fragments per layer: K/16 x N/8
constexpr int CL_FRAG_L1 = 1 * 8, CL_FRAG_L2 = 4 * 8, CL_FRAG_L3 = 4 * 8, CL_FRAG_L4 = 4 * 1;
constexpr int CL_FRAGS = CL_FRAG_L1 + CL_FRAG_L2 + CL_FRAG_L3 + CL_FRAG_L4;  // 76
// FP32 master parameters of one network, in this order:
//   W1[6][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][3] b4[3]   (W[k][n], row = input)
constexpr int CL_OFF_W1 = 0;
constexpr int CL_OFF_B1 = CL_OFF_W1 + CL_IN * CL_H;
constexpr int CL_OFF_W2 = CL_OFF_B1 + CL_H;
constexpr int CL_OFF_B2 = CL_OFF_W2 + CL_H * CL_H;
constexpr int CL_OFF_W3 = CL_OFF_B2 + CL_H;
constexpr int CL_OFF_B3 = CL_OFF_W3 + CL_H * CL_H;
constexpr int CL_OFF_W4 = CL_OFF_B3 + CL_H;
constexpr int CL_OFF_B4 = CL_OFF_W4 + CL_H * CL_OUT;
constexpr int CL_NPARAMS = CL_OFF_B4 + CL_OUT;  // 8963

// Weights of one network for the 5th-generation tensor cores (tcgen05.mma, kind::f16): each
// layer's W^T as a K-major BF16 operand in the no-swizzle core-matrix layout -- element
// (n, k) of an N x K operand at byte (n / 8) (K / 8) 128 + (k / 8) 128 + (n % 8) 16 + (k % 8) 2,
// i.e. 8 x 8 core matrices of 128 contiguous bytes, adjacent along K (leading byte offset
// 128) and K / 8 apart along N (stride byte offset K 16).  Layer 1 pads K from 6 to 16,
// layer 4 pads N from 3 to 16 (the smallest N of an M = 128 MMA).
constexpr int CL_TC_K1 = 16, CL_TC_N4 = 16;
constexpr int CL_TC_BYTES_L1 = CL_H * CL_TC_K1 * 2;   // 2 KB
constexpr int CL_TC_BYTES_L2 = CL_H * CL_H * 2;       // 8 KB
constexpr int CL_TC_BYTES_L4 = CL_TC_N4 * CL_H * 2;   // 2 KB
constexpr int CL_TC_OFF_L1 = 0, CL_TC_OFF_L2 = CL_TC_BYTES_L1, CL_TC_OFF_L3 = CL_TC_OFF_L2 + CL_TC_BYTES_L2,
              CL_TC_OFF_L4 = CL_TC_OFF_L3 + CL_TC_BYTES_L2, CL_TC_BYTES = CL_TC_OFF_L4 + CL_TC_BYTES_L4;  // 20 KB

__host__ __device__ __forceinline__ uint32_t km_offset(int n, int k, int kdim) {
    return static_cast<uint32_t>(((n >> 3) * (kdim >> 3) + (k >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

// Inference form of one network (device memory).
struct ClosureNet {
    uint2 frag[CL_FRAGS][32];       // BF16 pairs, m16n8k16 B-fragment order
    float bias[3 * CL_H + 8];       // b1, b2, b3, b4 (b4 padded to 8)
    alignas(16) unsigned char tc[CL_TC_BYTES];  // tcgen05 operand form (above)
    float in_shift[8], in_scale[8];  // x_n = (x - shift) * scale
    float out_shift[4], out_scale[4];  // y = y_n * scale + shift
    float hull_lo[8], hull_hi[8];   // box of the normalised training inputs
    int ready;                      // weights installed
    int pad_[3];
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low 16 bits)
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// One hidden layer on a 16-row tile: out = silu(in * W + b), 64 wide, K = 16 * KT.
// `in` holds KT A fragments (4 registers each); `out` receives 4 A fragments (K = 64).
template <int KT>
__device__ __forceinline__ void cl_hidden(const ClosureNet &net, int frag0, const float *bias,
                                          const uint32_t (&in)[KT][4], uint32_t (&out)[4][4]) {
    const int lane = threadIdx.x & 31, tig = lane & 3;
#pragma unroll
    for (int np = 0; np < 4; ++np) {  // pairs of 8-column tiles -> one 16-wide K slice
        float acc[2][4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int nt = 2 * np + h;
            const float b0 = bias[nt * 8 + 2 * tig], b1 = bias[nt * 8 + 2 * tig + 1];
            acc[h][0] = b0;
            acc[h][1] = b1;
            acc[h][2] = b0;
            acc[h][3] = b1;
#pragma unroll
            for (int kt = 0; kt < KT; ++kt) mma_bf16(acc[h], in[kt], net.frag[frag0 + kt * 8 + nt][lane]);
        }
        out[np][0] = pack_bf16(silu(acc[0][0]), silu(acc[0][1]));  // row g,   k = 2tig..
        out[np][1] = pack_bf16(silu(acc[0][2]), silu(acc[0][3]));  // row g+8
        out[np][2] = pack_bf16(silu(acc[1][0]), silu(acc[1][1]));  // row g,   k = 8+2tig..
        out[np][3] = pack_bf16(silu(acc[1][2]), silu(acc[1][3]));  // row g+8
    }
}

// Evaluates network `net` for the lanes of this warp whose `want` is set.  Must be called
// by all 32 lanes (warp-synchronous).  x: normalised inputs; y: normalised outputs.
__device__ __forceinline__ void closure_warp_infer(const ClosureNet &net, bool want,
                                                   const float (&x)[CL_IN], float (&y)[CL_OUT]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
    // features packed in pairs: (x0,x1), (x2,x3), (x4,x5)
    const uint32_t p0 = pack_bf16(x[0], x[1]), p1 = pack_bf16(x[2], x[3]), p2 = pack_bf16(x[4], x[5]);
    const unsigned any = __ballot_sync(0xffffffffu, want);
#pragma unroll
    for (int tile = 0; tile < 2; ++tile) {
        if (((any >> (16 * tile)) & 0xffffu) == 0u) continue;  // warp-uniform
        const int r0 = 16 * tile + g, r1 = r0 + 8;  // rows held by this lane's fragments
        // layer-1 A fragment: k = 2tig, 2tig+1 (features 0..5, zero beyond), k + 8 = 0
        const uint32_t a0_0 = __shfl_sync(0xffffffffu, p0, r0), a0_1 = __shfl_sync(0xffffffffu, p1, r0),
                       a0_2 = __shfl_sync(0xffffffffu, p2, r0);
        const uint32_t a1_0 = __shfl_sync(0xffffffffu, p0, r1), a1_1 = __shfl_sync(0xffffffffu, p1, r1),
                       a1_2 = __shfl_sync(0xffffffffu, p2, r1);
        uint32_t in1[1][4];
        in1[0][0] = tig == 0 ? a0_0 : (tig == 1 ? a0_1 : (tig == 2 ? a0_2 : 0u));
        in1[0][1] = tig == 0 ? a1_0 : (tig == 1 ? a1_1 : (tig == 2 ? a1_2 : 0u));
        in1[0][2] = 0u;
        in1[0][3] = 0u;
        uint32_t h1[4][4], h2[4][4];
        cl_hidden<1>(net, 0, net.bias, in1, h1);
        cl_hidden<4>(net, CL_FRAG_L1, net.bias + CL_H, h1, h2);
        cl_hidden<4>(net, CL_FRAG_L1 + CL_FRAG_L2, net.bias + 2 * CL_H, h2, h1);
        // output layer: 64 -> 8 (3 used), FP32 accumulate
        float o[4];
        const float b0 = net.bias[3 * CL_H + 2 * tig], b1 = net.bias[3 * CL_H + 2 * tig + 1];
        o[0] = b0;
        o[1] = b1;
        o[2] = b0;
        o[3] = b1;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt)
            mma_bf16(o, h1[kt], net.frag[CL_FRAG_L1 + CL_FRAG_L2 + CL_FRAG_L3 + kt][lane]);
        // gather: particle of lane L (row r = L - 16 tile) reads columns 0, 1 from lane
        // 4 (r mod 8) and column 2 from lane 4 (r mod 8) + 1; rows >= 8 use o[2], o[3]
        const int r = lane - 16 * tile;
        const bool mine = r >= 0 && r < 16;
        const int src = 4 * (r & 7);
        const float c0lo = __shfl_sync(0xffffffffu, o[0], src & 31), c1lo = __shfl_sync(0xffffffffu, o[1], src & 31);
        const float c0hi = __shfl_sync(0xffffffffu, o[2], src & 31), c1hi = __shfl_sync(0xffffffffu, o[3], src & 31);
        const float c2lo = __shfl_sync(0xffffffffu, o[0], (src + 1) & 31);
        const float c2hi = __shfl_sync(0xffffffffu, o[2], (src + 1) & 31);
        if (mine) {
            const bool hi = r >= 8;
            y[0] = hi ? c0hi : c0lo;
            y[1] = hi ? c1hi : c1lo;
            y[2] = hi ? c2hi : c2lo;
        }
    }
}

// ------------------------------------------------------------------ features
// Drucker-Prager, smooth plastic branch (sand.rs:156-194): returns true when the network
// is to be used (gamma > 0 and not the tip); `plastic`/`tip` report the exact decisions.
struct DpTrial {
    float2 eps, dev;
    float trace, dev_norm, alpha, ratio, cohesion, gamma;
};
__device__ __forceinline__ DpTrial dp_trial(const MatP &m, float2 sigma_in, float lvs, float q, bool pr) {
    DpTrial t;
    const float2 sigma = vmax2(vabs2(sigma_in), splat(LOG_CLAMP));
    t.eps = v2(em_log(sigma.x, pr) + lvs * 0.5f, em_log(sigma.y, pr) + lvs * 0.5f);
    t.trace = t.eps.x + t.eps.y;
    t.dev = vsub(t.eps, splat(t.trace * 0.5f));
    t.dev_norm = evlen(t.dev);  // the arithmetic of dp_project (physics.cuh), so both decide alike
    t.ratio = ediv(m.lambda + m.mu, m.mu);
    t.alpha = dp_alpha(m, q, pr);
    t.cohesion = ediv(m.stretch_limit, 2.0f * m.mu);
    t.gamma = t.dev_norm + t.ratio * t.trace * t.alpha - t.cohesion;
    return t;
}

// The plain mapping on the smooth plastic branches, in the reference's expression order
// (the same arithmetic as dp_project / nacc_project): targets for logging, the hull
// fallback and the judge.
__device__ __forceinline__ void dp_smooth(const DpTrial &t, float2 &h, float &dq) {
    h = vsub(t.eps, svmul(t.gamma, evdivs(t.dev, t.dev_norm)));
    dq = t.gamma;
}

__device__ __forceinline__ void nacc_smooth(const MatP &m, const NaccTrial &t, float alpha,
                                            float2 &sv_new, float &alpha_new, bool pr) {
    const float kappa = nacc_kappa(m);
    const float xi = m.hardening_exponent, beta = m.compression_limit, mm_ = m.stretch_limit;
    const bool hard = xi > 0.0f;
    const float sv_sq_trace = t.sv_sq_trace;
    const float p0 = t.p0, p_tr = t.p_tr, j_e_tr = t.j_e_tr;
    const float2 s_tr = t.s_tr;
    const float y0 = t.y0;
    const float y1 = t.y1;
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
    float scale = esqrt(fmaxf(ediv(-y1, fmaxf(y0, 1.0e-10f)), 0.0f)) * ediv(j_e_tr, m.mu);
    float2 b_n1 = vadd(svmul(scale, normalize_or_zero(s_tr)), splat(sv_sq_trace / 2.0f));
    sv_new = v2(esqrt(fmaxf(b_n1.x, 1.0e-8f)), esqrt(fmaxf(b_n1.y, 1.0e-8f)));
    alpha_new = alpha;
}

// Principal Kirchhoff stresses used to judge the network: Drucker-Prager (sand.rs:220-231,
// in principal axes 2 mu (s - 1) s + lambda (J - 1) J) and NACC (nacc.rs:236-249:
// mu / J (s^2 - tr/2) + kappa / 2 (J^2 - 1)).
__device__ __forceinline__ float2 dp_principal_stress(const MatP &m, float2 s) {
    const float j = s.x * s.y;
    const float vol = m.lambda * (j - 1.0f) * j;
    return v2(2.0f * m.mu * (s.x - 1.0f) * s.x + vol, 2.0f * m.mu * (s.y - 1.0f) * s.y + vol);
}
__device__ __forceinline__ float2 nacc_principal_stress(const MatP &m, float2 s) {
    const float j = fmaxf(s.x * s.y, MIN_J);
    const float2 sq = vmulv(s, s);
    const float half_tr = (sq.x + sq.y) * 0.5f;
    const float vol = nacc_kappa(m) * 0.5f * (j * j - 1.0f);
    return v2(m.mu / j * (sq.x - half_tr) + vol, m.mu / j * (sq.y - half_tr) + vol);
}

// Judged errors are also binned: bin b covers [10^(b/4 - 8), 10^((b+1)/4 - 8)) (a quarter
// decade from 1e-8 to 1e4), for the percentiles.
constexpr int CL_ERR_BINS = 48;
__device__ __forceinline__ int closure_err_bin(float e) {
    if (!(e > 1e-8f)) return 0;
    const int b = static_cast<int>(floorf((log10f(e) + 8.0f) * 4.0f));
    return b < 0 ? 0 : (b >= CL_ERR_BINS ? CL_ERR_BINS - 1 : b);
}

// Lifetime counters of the closure (device memory).
struct ClosureStats {
    unsigned long long smooth;        // particles on a smooth plastic branch
    unsigned long long net;           // of which evaluated by the network
    unsigned long long hull_fallback; // of which outside the training box (plain mapping)
    unsigned long long judged;        // network results also run through the plain mapping
    unsigned long long logged[CL_NMODELS];
    double err_sum;                   // sum of judged relative stress errors
    unsigned int err_max_bits;        // max judged relative stress error (float bits)
    unsigned int pad_;
    unsigned long long judge_replaced;   // judged results above the bar, replaced by the plain one
    unsigned long long err_hist[CL_ERR_BINS];
};

// Closure switches and buffers of a particle pass.
struct ClosureArgs {
    const ClosureNet *nets;   // [CL_NMODELS]
    ClosureStats *stats;
    float *log_x[CL_NMODELS]; // [cap][CL_IN]
    float *log_t[CL_NMODELS]; // [cap][CL_OUT]
    unsigned long long log_cap;
    uint32_t log_stride;      // log one smooth-branch evaluation in log_stride (hashed)
    uint32_t judge_stride;    // judge one network evaluation in judge_stride (hashed)
    int infer;                // use installed networks
    int log;                  // record (inputs, targets) of the plain mapping
    // Deferred evaluation: the particle pass queues the particles the network is to map
    // (slot indices, one queue per model, counted in StepState::cl_queued) and a tile kernel
    // evaluates them 128 at a time on tcgen05 and finishes their update and P2G.
    int defer;
    uint32_t *queue[CL_NMODELS];
    float judge_bar;          // judged results with a larger relative stress error use the plain result
};

}  // namespace emerge
