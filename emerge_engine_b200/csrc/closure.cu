// closure.cu -- training and management of the learned return-mapping closure.
//
// Data: the closure particle pass logs (inputs, targets) of the plain mapping on the
// smooth plastic branches (closure.cuh).  Training runs on the GPU with this file's own
// FP32 kernels: a layer forward (z = x W + b, a = silu(z)), the MSE loss, the backward
// passes (dA = dZ W^T, dW = x^T dZ, db = sum dZ, dZ = dA silu'(z)) and Adam.  The trained
// FP32 master weights are packed into BF16 m16n8k16 B fragments for the tensor-core
// inference inside the particle pass.  Training is off the hot path (seconds per model);
// its GEMMs are 64 wide, so plain CUDA-core kernels are used.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "closure_host.h"
#include "kernels.h"

namespace emerge {

// ------------------------------------------------------------------ device kernels
__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

// z = x W + b (x: B x K, row stride ldx; W: K x N), a = silu(z) when act.
__global__ void k_mlp_fwd(const float *x, int ldx, int K, const float *W, const float *b, int N,
                          float *z, float *a, int B, int act) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * N) return;
    const int r = idx / N, n = idx % N;
    float s = b[n];
    const float *xr = x + static_cast<size_t>(r) * ldx;
    for (int k = 0; k < K; ++k) s = fmaf(xr[k], W[k * N + n], s);
    z[idx] = s;
    if (a) a[idx] = act ? s * sigmoidf_(s) : s;
}

// MSE over B x 3 outputs: loss += sum (y - t)^2 / (B * 3), dY = 2 (y - t) / (B * 3).
__global__ void k_mlp_loss(const float *y, const float *t, int B, float *dy, double *loss) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    float e2 = 0.0f;
    if (idx < B * CL_OUT) {
        const float d = y[idx] - t[idx];
        dy[idx] = 2.0f * d / static_cast<float>(B * CL_OUT);
        e2 = d * d;
    }
    for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    if ((threadIdx.x & 31) == 0 && e2 != 0.0f) atomicAdd(loss, static_cast<double>(e2) / (B * CL_OUT));
}

// dIn = dZ W^T (dZ: B x N, W: K x N); when z_in is given, dIn *= silu'(z_in).
__global__ void k_mlp_bwd_data(const float *dz, int N, const float *W, int K, const float *z_in,
                               float *din, int B) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * K) return;
    const int r = idx / K, k = idx % K;
    const float *dzr = dz + static_cast<size_t>(r) * N;
    float s = 0.0f;
    for (int n = 0; n < N; ++n) s = fmaf(dzr[n], W[k * N + n], s);
    if (z_in) {
        const float zz = z_in[idx], sg = sigmoidf_(zz);
        s *= sg * (1.0f + zz * (1.0f - sg));
    }
    din[idx] = s;
}

// dW += x^T dZ and db += sum dZ over a chunk of rows (dW, db zeroed beforehand).
constexpr int BWD_ROWS = 512;
__global__ void k_mlp_bwd_weight(const float *x, int ldx, int K, const float *dz, int N, int B,
                                 float *dW, float *db) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;  // over (K + 1) x N, last row = bias
    if (e >= (K + 1) * N) return;
    const int k = e / N, n = e % N;
    const int r0 = blockIdx.y * BWD_ROWS, r1 = min(B, r0 + BWD_ROWS);
    float s = 0.0f;
    for (int r = r0; r < r1; ++r) {
        const float xv = k < K ? x[static_cast<size_t>(r) * ldx + k] : 1.0f;
        s = fmaf(xv, dz[static_cast<size_t>(r) * N + n], s);
    }
    atomicAdd(k < K ? &dW[k * N + n] : &db[n], s);
}

// Adam (Kingma & Ba) with bias correction; t is the 1-based step.
__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, int t, float lr, float b1,
                       float b2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.0f - powf(b1, static_cast<float>(t)));
    const float vh = vi / (1.0f - powf(b2, static_cast<float>(t)));
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

// Packs FP32 master weights into the inference form (BF16 B fragments + FP32 biases).
__global__ void k_pack_net(const float *P, ClosureNet *net) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per (fragment, lane)
    if (t < CL_FRAGS * 32) {
        const int f = t / 32, lane = t % 32, g = lane >> 2, tig = lane & 3;
        int layer, kt, nt;
        if (f < CL_FRAG_L1) { layer = 0; kt = 0; nt = f; }
        else if (f < CL_FRAG_L1 + CL_FRAG_L2) { layer = 1; kt = (f - CL_FRAG_L1) / 8; nt = (f - CL_FRAG_L1) % 8; }
        else if (f < CL_FRAG_L1 + CL_FRAG_L2 + CL_FRAG_L3) {
            layer = 2; kt = (f - CL_FRAG_L1 - CL_FRAG_L2) / 8; nt = (f - CL_FRAG_L1 - CL_FRAG_L2) % 8;
        } else { layer = 3; kt = f - CL_FRAG_L1 - CL_FRAG_L2 - CL_FRAG_L3; nt = 0; }
        const int K = layer == 0 ? CL_IN : CL_H, N = layer == 3 ? CL_OUT : CL_H;
        const float *W = P + (layer == 0 ? CL_OFF_W1 : layer == 1 ? CL_OFF_W2 : layer == 2 ? CL_OFF_W3 : CL_OFF_W4);
        const int n = nt * 8 + g;
        auto w = [&](int k) { return (k < K && n < N) ? W[k * N + n] : 0.0f; };
        const int k0 = kt * 16 + 2 * tig;
        net->frag[f][lane] = make_uint2(pack_bf16(w(k0), w(k0 + 1)), pack_bf16(w(k0 + 8), w(k0 + 9)));
    }
    if (t < 3 * CL_H + 8) {
        float b;
        if (t < CL_H) b = P[CL_OFF_B1 + t];
        else if (t < 2 * CL_H) b = P[CL_OFF_B2 + t - CL_H];
        else if (t < 3 * CL_H) b = P[CL_OFF_B3 + t - 2 * CL_H];
        else b = (t - 3 * CL_H) < CL_OUT ? P[CL_OFF_B4 + t - 3 * CL_H] : 0.0f;
        net->bias[t] = b;
    }
}

// Packs the tcgen05 operand form (closure.cuh): one thread per BF16 element of W1^T
// (64 x 16), W2^T, W3^T (64 x 64) and W4^T (16 x 64); padding is zero.
__global__ void k_pack_tc(const float *P, ClosureNet *net) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int E1 = CL_H * CL_TC_K1, E2 = CL_H * CL_H, E4 = CL_TC_N4 * CL_H;
    if (t >= E1 + 2 * E2 + E4) return;
    int layer, n, k, kdim, off;
    if (t < E1) { layer = 0; n = t / CL_TC_K1; k = t % CL_TC_K1; kdim = CL_TC_K1; off = CL_TC_OFF_L1; }
    else if (t < E1 + E2) { layer = 1; n = (t - E1) / CL_H; k = (t - E1) % CL_H; kdim = CL_H; off = CL_TC_OFF_L2; }
    else if (t < E1 + 2 * E2) { layer = 2; n = (t - E1 - E2) / CL_H; k = (t - E1 - E2) % CL_H; kdim = CL_H; off = CL_TC_OFF_L3; }
    else { layer = 3; n = (t - E1 - 2 * E2) / CL_H; k = (t - E1 - 2 * E2) % CL_H; kdim = CL_H; off = CL_TC_OFF_L4; }
    const int K = layer == 0 ? CL_IN : CL_H, N = layer == 3 ? CL_OUT : CL_H;
    const float *W = P + (layer == 0 ? CL_OFF_W1 : layer == 1 ? CL_OFF_W2 : layer == 2 ? CL_OFF_W3 : CL_OFF_W4);
    const float v = (k < K && n < N) ? W[k * N + n] : 0.0f;  // W[k][n]: row = input
    *reinterpret_cast<__nv_bfloat16 *>(net->tc + off + km_offset(n, k, kdim)) = __float2bfloat16_rn(v);
}

// Tensor-core inference of normalised inputs (test hook and validation).
__global__ void k_infer(const ClosureNet *net, const float *x, int n, float *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    float xi[CL_IN], yi[CL_OUT] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int j = 0; j < CL_IN; ++j) xi[j] = valid ? x[static_cast<size_t>(i) * CL_IN + j] : 0.0f;
    closure_warp_infer(*net, valid, xi, yi);
    if (valid)
        for (int j = 0; j < CL_OUT; ++j) y[static_cast<size_t>(i) * CL_OUT + j] = yi[j];
}

// ------------------------------------------------------------------ host helpers
namespace {

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) {
        if (p) cudaFree(p);
        p = nullptr;
        return cudaMalloc(&p, bytes);
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

inline int nblk(long long n, int t = 256) { return static_cast<int>((n + t - 1) / t); }

// Device workspace of one training / gradient evaluation at batch size B.
struct MlpWork {
    DevBuf z1, a1, z2, a2, z3, a3, y, dy, d3, d2, d1, grad;
    cudaError_t alloc(int B) {
        cudaError_t e = cudaSuccess;
        for (DevBuf *b : {&z1, &a1, &z2, &a2, &z3, &a3, &d3, &d2, &d1})
            if (e == cudaSuccess) e = b->alloc(static_cast<size_t>(B) * CL_H * sizeof(float));
        if (e == cudaSuccess) e = y.alloc(static_cast<size_t>(B) * CL_OUT * sizeof(float));
        if (e == cudaSuccess) e = dy.alloc(static_cast<size_t>(B) * CL_OUT * sizeof(float));
        if (e == cudaSuccess) e = grad.alloc(CL_NPARAMS * sizeof(float));
        return e;
    }
};

// Forward, loss and backward on one batch (x: B x 6, t: B x 3, normalised); gradient
// into w.grad; loss accumulated into *loss (device double).
void mlp_loss_grad(const float *P, const float *x, const float *t, int B, MlpWork &w, double *loss,
                   cudaStream_t s) {
    float *z1 = w.z1.as<float>(), *a1 = w.a1.as<float>(), *z2 = w.z2.as<float>(), *a2 = w.a2.as<float>();
    float *z3 = w.z3.as<float>(), *a3 = w.a3.as<float>(), *y = w.y.as<float>(), *dy = w.dy.as<float>();
    float *d3 = w.d3.as<float>(), *d2 = w.d2.as<float>(), *d1 = w.d1.as<float>(), *G = w.grad.as<float>();
    k_mlp_fwd<<<nblk((long long)B * CL_H), 256, 0, s>>>(x, CL_IN, CL_IN, P + CL_OFF_W1, P + CL_OFF_B1, CL_H, z1, a1, B, 1);
    k_mlp_fwd<<<nblk((long long)B * CL_H), 256, 0, s>>>(a1, CL_H, CL_H, P + CL_OFF_W2, P + CL_OFF_B2, CL_H, z2, a2, B, 1);
    k_mlp_fwd<<<nblk((long long)B * CL_H), 256, 0, s>>>(a2, CL_H, CL_H, P + CL_OFF_W3, P + CL_OFF_B3, CL_H, z3, a3, B, 1);
    k_mlp_fwd<<<nblk((long long)B * CL_OUT), 256, 0, s>>>(a3, CL_H, CL_H, P + CL_OFF_W4, P + CL_OFF_B4, CL_OUT, y, nullptr, B, 0);
    k_mlp_loss<<<nblk((long long)B * CL_OUT), 256, 0, s>>>(y, t, B, dy, loss);
    cudaMemsetAsync(G, 0, CL_NPARAMS * sizeof(float), s);
    const int rows = (B + BWD_ROWS - 1) / BWD_ROWS;
    // layer 4
    k_mlp_bwd_weight<<<dim3(nblk((CL_H + 1) * CL_OUT), rows), 256, 0, s>>>(a3, CL_H, CL_H, dy, CL_OUT, B, G + CL_OFF_W4, G + CL_OFF_B4);
    k_mlp_bwd_data<<<nblk((long long)B * CL_H), 256, 0, s>>>(dy, CL_OUT, P + CL_OFF_W4, CL_H, z3, d3, B);
    // layer 3
    k_mlp_bwd_weight<<<dim3(nblk((CL_H + 1) * CL_H), rows), 256, 0, s>>>(a2, CL_H, CL_H, d3, CL_H, B, G + CL_OFF_W3, G + CL_OFF_B3);
    k_mlp_bwd_data<<<nblk((long long)B * CL_H), 256, 0, s>>>(d3, CL_H, P + CL_OFF_W3, CL_H, z2, d2, B);
    // layer 2
    k_mlp_bwd_weight<<<dim3(nblk((CL_H + 1) * CL_H), rows), 256, 0, s>>>(a1, CL_H, CL_H, d2, CL_H, B, G + CL_OFF_W2, G + CL_OFF_B2);
    k_mlp_bwd_data<<<nblk((long long)B * CL_H), 256, 0, s>>>(d2, CL_H, P + CL_OFF_W2, CL_H, z1, d1, B);
    // layer 1
    k_mlp_bwd_weight<<<dim3(nblk((CL_IN + 1) * CL_H), rows), 256, 0, s>>>(x, CL_IN, CL_IN, d1, CL_H, B, G + CL_OFF_W1, G + CL_OFF_B1);
}

// Seeded initialisation: uniform(-sqrt(6 / (fan_in + fan_out)), +...) weights, zero biases.
void init_params(std::vector<float> &P, uint64_t seed) {
    std::mt19937_64 rng(seed);
    P.assign(CL_NPARAMS, 0.0f);
    auto fill = [&](int off, int K, int N) {
        const float a = std::sqrt(6.0f / static_cast<float>(K + N));
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < K * N; ++i) P[off + i] = u(rng);
    };
    fill(CL_OFF_W1, CL_IN, CL_H);
    fill(CL_OFF_W2, CL_H, CL_H);
    fill(CL_OFF_W3, CL_H, CL_H);
    fill(CL_OFF_W4, CL_H, CL_OUT);
}

// Relative error of the principal Kirchhoff stress for normalised-output pairs, scale-free
// (units of mu for Drucker-Prager, of kappa for NACC).
float stress_rel_err(int model, const float *xraw, const float *y_pred, const float *y_ref) {
    // Drucker-Prager outputs are in units of the trial deviatoric norm s = exp(x[5])
    // NACC outputs are the plastic correction ln(sv') - ln(sv) of the log singular values
    const float unit = model == 0 ? std::exp(xraw[5]) : 1.0f;
    const float off0 = model == 0 ? 0.0f : xraw[0], off1 = model == 0 ? 0.0f : xraw[1];
    auto stress = [&](const float *y, float &s0, float &s1) {
        const float a = std::exp(y[0] * unit + off0), b = std::exp(y[1] * unit + off1), j = a * b;
        if (model == 0) {  // tau / mu = 2 (s - 1) s + (lambda / mu) (J - 1) J, lambda/mu = ratio - 1
            const float lam = xraw[3] - 1.0f;
            s0 = 2.0f * (a - 1.0f) * a + lam * (j - 1.0f) * j;
            s1 = 2.0f * (b - 1.0f) * b + lam * (j - 1.0f) * j;
        } else {  // tau / kappa = (mu/kappa) / J (s^2 - tr/2) + (J^2 - 1) / 2
            const float jj = std::max(j, 1e-6f), mk = xraw[3], ht = 0.5f * (a * a + b * b);
            s0 = mk / jj * (a * a - ht) + 0.5f * (jj * jj - 1.0f);
            s1 = mk / jj * (b * b - ht) + 0.5f * (jj * jj - 1.0f);
        }
    };
    float p0, p1, r0, r1;
    stress(y_pred, p0, p1);
    stress(y_ref, r0, r1);
    const float num = std::sqrt((p0 - r0) * (p0 - r0) + (p1 - r1) * (p1 - r1));
    const float den = std::max(std::sqrt(r0 * r0 + r1 * r1), 1e-6f);
    return num / den;
}

}  // namespace

// ------------------------------------------------------------------ ClosureHost
struct ClosureHost {
    DevBuf nets, stats;
    DevBuf log_x[CL_NMODELS], log_t[CL_NMODELS];
    DevBuf params[CL_NMODELS];
    DevBuf queue;              // CL_NMODELS queues of queue_cap slot indices (deferred mode)
    size_t queue_cap = 0;
    unsigned long long log_cap = 0;
    uint32_t log_stride = 1, judge_stride = 64;
    int infer = 0, log = 0;
    int defer = 1;
    float judge_bar = 1e-3f;
    std::vector<float> norm[CL_NMODELS];  // in_shift[6] in_scale[6] out_shift[3] out_scale[3]
};

ClosureArgs closure_args(const ClosureHost *c, size_t n) {
    ClosureArgs a;
    std::memset(&a, 0, sizeof(a));
    if (!c || !c->nets.p) return a;
    // deferred evaluation needs queues for every particle (re-enable after adding particles)
    a.defer = c->infer && c->defer && c->queue.p && c->queue_cap >= n ? 1 : 0;
    for (int m = 0; m < CL_NMODELS; ++m)
        a.queue[m] = a.defer ? c->queue.as<uint32_t>() + m * c->queue_cap : nullptr;
    a.judge_bar = c->judge_bar;
    a.nets = c->nets.as<ClosureNet>();
    a.stats = c->stats.as<ClosureStats>();
    for (int m = 0; m < CL_NMODELS; ++m) {
        a.log_x[m] = c->log_x[m].as<float>();
        a.log_t[m] = c->log_t[m].as<float>();
    }
    a.log_cap = c->log ? c->log_cap : 0ull;
    a.log_stride = c->log_stride ? c->log_stride : 1u;
    a.judge_stride = c->judge_stride ? c->judge_stride : 1u;
    a.infer = c->infer;
    a.log = c->log && c->log_cap > 0;
    return a;
}

void closure_destroy(ClosureHost *c) { delete c; }

static emerge_status ensure_closure(emerge_sim *s, ClosureHost *&c) {
    if (c) return EMERGE_OK;
    c = new ClosureHost();
    if (c->nets.alloc(CL_NMODELS * sizeof(ClosureNet)) != cudaSuccess ||
        c->stats.alloc(sizeof(ClosureStats)) != cudaSuccess) {
        delete c;
        c = nullptr;
        return sim_fail(s, EMERGE_ERR_OOM, "closure: device allocation failed");
    }
    cudaMemset(c->nets.p, 0, CL_NMODELS * sizeof(ClosureNet));
    cudaMemset(c->stats.p, 0, sizeof(ClosureStats));
    return EMERGE_OK;
}

// Installs master weights + normalisation + hull for `model` into the inference form.
static emerge_status install_net(emerge_sim *s, ClosureHost *c, int model, const float *P_dev,
                                 const float *norm, const float *hull, cudaStream_t st) {
    ClosureNet *net = c->nets.as<ClosureNet>() + model;
    k_pack_net<<<nblk(CL_FRAGS * 32), 256, 0, st>>>(P_dev, net);
    k_pack_tc<<<nblk(CL_H * CL_TC_K1 + 2 * CL_H * CL_H + CL_TC_N4 * CL_H), 256, 0, st>>>(P_dev, net);
    struct Tail {
        float in_shift[8], in_scale[8], out_shift[4], out_scale[4], hull_lo[8], hull_hi[8];
        int ready, pad_[3];
    } tail;
    std::memset(&tail, 0, sizeof(tail));
    for (int j = 0; j < CL_IN; ++j) {
        tail.in_shift[j] = norm[j];
        tail.in_scale[j] = norm[CL_IN + j];
        tail.hull_lo[j] = hull[j];
        tail.hull_hi[j] = hull[CL_IN + j];
    }
    for (int j = 0; j < CL_OUT; ++j) {
        tail.out_shift[j] = norm[2 * CL_IN + j];
        tail.out_scale[j] = norm[2 * CL_IN + CL_OUT + j];
    }
    tail.ready = 1;
    static_assert(sizeof(Tail) == sizeof(ClosureNet) - offsetof(ClosureNet, in_shift), "ClosureNet tail layout");
    if (cudaMemcpyAsync(reinterpret_cast<char *>(net) + offsetof(ClosureNet, in_shift), &tail, sizeof(tail),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: install failed");
    c->norm[model].assign(norm, norm + 2 * CL_IN + 2 * CL_OUT);
    return EMERGE_OK;
}

}  // namespace emerge

using namespace emerge;

extern "C" {

emerge_status emerge_cuda_closure_log(emerge_sim *s, uint64_t capacity, uint32_t stride) {
    if (!s || (capacity && stride == 0)) return EMERGE_ERR_INVALID_ARG;
    ClosureHost *&c = sim_closure(s);
    emerge_status st = ensure_closure(s, c);
    if (st != EMERGE_OK) return st;
    if (capacity == 0) {
        c->log = 0;
    } else {
        for (int m = 0; m < CL_NMODELS; ++m)
            if (c->log_x[m].alloc(capacity * CL_IN * sizeof(float)) != cudaSuccess ||
                c->log_t[m].alloc(capacity * CL_OUT * sizeof(float)) != cudaSuccess)
                return sim_fail(s, EMERGE_ERR_OOM, "closure: log buffers");
        ClosureStats zero;
        std::memset(&zero, 0, sizeof(zero));
        if (cudaMemcpy(c->stats.p, &zero, sizeof(zero), cudaMemcpyHostToDevice) != cudaSuccess)
            return sim_fail(s, EMERGE_ERR_CUDA, "closure: stats reset");
        c->log_cap = capacity;
        c->log_stride = stride;
        c->log = 1;
    }
    sim_invalidate_graph(s);
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_enable(emerge_sim *s, int on, uint32_t judge_stride) {
    if (!s || judge_stride == 0) return EMERGE_ERR_INVALID_ARG;
    ClosureHost *&c = sim_closure(s);
    emerge_status st = ensure_closure(s, c);
    if (st != EMERGE_OK) return st;
    c->infer = on ? 1 : 0;
    c->judge_stride = judge_stride;
    const size_t cap = sim_capacity(s);
    if (on && c->defer && c->queue_cap < cap) {  // queues for the deferred mode
        c->queue_cap = 0;
        if (c->queue.alloc(CL_NMODELS * cap * sizeof(uint32_t)) != cudaSuccess)
            return sim_fail(s, EMERGE_ERR_OOM, "closure: queue allocation failed");
        c->queue_cap = cap;
    }
    sim_invalidate_graph(s);
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_set_mode(emerge_sim *s, int defer, float judge_bar) {
    if (!s || !(judge_bar >= 0.0f)) return EMERGE_ERR_INVALID_ARG;
    ClosureHost *&c = sim_closure(s);
    emerge_status st = ensure_closure(s, c);
    if (st != EMERGE_OK) return st;
    c->defer = defer ? 1 : 0;
    c->judge_bar = judge_bar;
    if (c->infer) return emerge_cuda_closure_enable(s, 1, c->judge_stride);  // (re)sizes the queues
    sim_invalidate_graph(s);
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_stats(emerge_sim *s, emerge_closure_stats *out, int reset) {
    if (!s || !out) return EMERGE_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    ClosureHost *c = sim_closure(s);
    if (!c) return EMERGE_OK;
    cudaStream_t st = sim_stream(s);
    ClosureStats h;
    if (cudaMemcpyAsync(&h, c->stats.p, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: stats read");
    out->smooth = h.smooth;
    out->net = h.net;
    out->hull_fallback = h.hull_fallback;
    out->judged = h.judged;
    for (int m = 0; m < CL_NMODELS; ++m) out->logged[m] = std::min<unsigned long long>(h.logged[m], c->log_cap);
    out->err_mean = h.judged ? h.err_sum / static_cast<double>(h.judged) : 0.0;
    uint32_t bits = h.err_max_bits;
    std::memcpy(&out->err_max, &bits, sizeof(float));
    out->judge_replaced = h.judge_replaced;
    {  // percentiles from the quarter-decade bins (upper bin edge)
        unsigned long long total = 0ull;
        for (int b = 0; b < CL_ERR_BINS; ++b) total += h.err_hist[b];
        auto pct = [&](double q) -> float {
            if (!total) return 0.0f;
            unsigned long long acc = 0ull;
            for (int b = 0; b < CL_ERR_BINS; ++b) {
                acc += h.err_hist[b];
                if (static_cast<double>(acc) >= q * static_cast<double>(total))
                    return static_cast<float>(std::pow(10.0, (b + 1) / 4.0 - 8.0));
            }
            return static_cast<float>(std::pow(10.0, CL_ERR_BINS / 4.0 - 8.0));
        };
        out->err_p50 = pct(0.5);
        out->err_p99 = pct(0.99);
    }
    if (reset) {
        ClosureStats z;
        std::memset(&z, 0, sizeof(z));
        for (int m = 0; m < CL_NMODELS; ++m) z.logged[m] = h.logged[m];
        if (cudaMemcpyAsync(c->stats.p, &z, sizeof(z), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return sim_fail(s, EMERGE_ERR_CUDA, "closure: stats reset");
    }
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_train(emerge_sim *s, int model, const emerge_closure_train_config *cfg,
                                        emerge_closure_train_report *rep) {
    if (!s || !cfg || model < 0 || model >= CL_NMODELS || cfg->batch == 0 || cfg->batch > 65536 ||
        !(cfg->val_fraction >= 0.0f && cfg->val_fraction < 1.0f))
        return EMERGE_ERR_INVALID_ARG;
    ClosureHost *c = sim_closure(s);
    if (!c || !c->log_x[model].p) return sim_fail(s, EMERGE_ERR_INVALID_ARG, "closure: nothing logged");
    const auto t_start = std::chrono::steady_clock::now();
    cudaStream_t st = sim_stream(s);
    ClosureStats hs;
    if (cudaMemcpy(&hs, c->stats.p, sizeof(hs), cudaMemcpyDeviceToHost) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: stats read");
    size_t n = std::min<unsigned long long>(hs.logged[model], c->log_cap);
    if (cfg->max_samples) n = std::min<size_t>(n, cfg->max_samples);
    if (n < 64) return sim_fail(s, EMERGE_ERR_INVALID_ARG, "closure: fewer than 64 logged samples");
    // samples to the host: normalisation, hull and the seeded split
    std::vector<float> X(n * CL_IN), T(n * CL_OUT);
    if (cudaMemcpy(X.data(), c->log_x[model].p, X.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(T.data(), c->log_t[model].p, T.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: log read");
    std::vector<float> norm(2 * CL_IN + 2 * CL_OUT), hull(2 * CL_IN);
    auto moments = [&](const std::vector<float> &A, int w, int j, float &mean, float &scale) {
        double s1 = 0, s2 = 0;
        for (size_t i = 0; i < n; ++i) {
            s1 += A[i * w + j];
            s2 += static_cast<double>(A[i * w + j]) * A[i * w + j];
        }
        const double mu = s1 / n, var = std::max(s2 / n - mu * mu, 0.0);
        mean = static_cast<float>(mu);
        scale = var > 1e-20 ? static_cast<float>(1.0 / std::sqrt(var)) : 1.0f;
    };
    for (int j = 0; j < CL_IN; ++j) moments(X, CL_IN, j, norm[j], norm[CL_IN + j]);
    for (int j = 0; j < CL_OUT; ++j) {
        float mean, scale;
        moments(T, CL_OUT, j, mean, scale);
        norm[2 * CL_IN + j] = mean;
        norm[2 * CL_IN + CL_OUT + j] = 1.0f / scale;  // y = y_n * std + mean
    }
    std::vector<uint32_t> perm(n);
    for (size_t i = 0; i < n; ++i) perm[i] = static_cast<uint32_t>(i);
    std::mt19937_64 rng(cfg->seed);
    std::shuffle(perm.begin(), perm.end(), rng);
    const size_t n_val = static_cast<size_t>(cfg->val_fraction * n);
    const size_t n_train = n - n_val;
    std::vector<float> Xn(n * CL_IN), Tn(n * CL_OUT);
    for (int j = 0; j < CL_IN; ++j) {
        hull[j] = INFINITY;
        hull[CL_IN + j] = -INFINITY;
    }
    for (size_t r = 0; r < n; ++r) {
        const size_t i = perm[r];
        for (int j = 0; j < CL_IN; ++j) {
            const float v = (X[i * CL_IN + j] - norm[j]) * norm[CL_IN + j];
            Xn[r * CL_IN + j] = v;
            if (r < n_train) {
                hull[j] = std::min(hull[j], v);
                hull[CL_IN + j] = std::max(hull[CL_IN + j], v);
            }
        }
        for (int j = 0; j < CL_OUT; ++j)
            Tn[r * CL_OUT + j] = (T[i * CL_OUT + j] - norm[2 * CL_IN + j]) / norm[2 * CL_IN + CL_OUT + j];
    }
    DevBuf dX, dT, dP, dM, dV, dLoss, dY;
    MlpWork w;
    const int B = static_cast<int>(std::min<size_t>(cfg->batch, n_train));
    if (dX.alloc(Xn.size() * sizeof(float)) != cudaSuccess || dT.alloc(Tn.size() * sizeof(float)) != cudaSuccess ||
        dP.alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess || dM.alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess ||
        dV.alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess || dLoss.alloc(sizeof(double)) != cudaSuccess ||
        dY.alloc(std::max<size_t>(n_val, 1) * CL_OUT * sizeof(float)) != cudaSuccess || w.alloc(B) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_OOM, "closure: training buffers");
    std::vector<float> P;
    init_params(P, cfg->seed ^ 0x9e3779b97f4a7c15ull);
    cudaMemcpyAsync(dX.p, Xn.data(), Xn.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dT.p, Tn.data(), Tn.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dP.p, P.data(), CL_NPARAMS * sizeof(float), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(dM.p, 0, CL_NPARAMS * sizeof(float), st);
    cudaMemsetAsync(dV.p, 0, CL_NPARAMS * sizeof(float), st);
    const size_t batches = n_train / B;
    int step = 0;
    double last_epoch_loss = 0.0;
    for (uint32_t ep = 0; ep < cfg->epochs; ++ep) {
        cudaMemsetAsync(dLoss.p, 0, sizeof(double), st);
        const size_t rot = batches > 1 ? (static_cast<size_t>(rng()) % batches) : 0;
        for (size_t bi = 0; bi < batches; ++bi) {
            const size_t b = (bi + rot) % batches;
            const float *xb = dX.as<float>() + b * B * CL_IN;
            const float *tb = dT.as<float>() + b * B * CL_OUT;
            mlp_loss_grad(dP.as<float>(), xb, tb, B, w, dLoss.as<double>(), st);
            ++step;
            const float lr = cfg->lr * (cfg->lr_decay > 0.0f ? std::pow(cfg->lr_decay, static_cast<float>(ep)) : 1.0f);
            k_adam<<<nblk(CL_NPARAMS), 256, 0, st>>>(dP.as<float>(), w.grad.as<float>(), dM.as<float>(), dV.as<float>(),
                                                    CL_NPARAMS, step, lr, cfg->beta1, cfg->beta2, cfg->eps);
        }
        double l = 0.0;
        cudaMemcpyAsync(&l, dLoss.p, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return sim_fail(s, EMERGE_ERR_CUDA, "closure: training");
        last_epoch_loss = batches ? l / static_cast<double>(batches) : 0.0;
    }
    // install, then validate with the tensor-core inference itself
    emerge_status ist = install_net(s, c, model, dP.as<float>(), norm.data(), hull.data(), st);
    if (ist != EMERGE_OK) return ist;
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->n_train = n_train;
        rep->n_val = n_val;
        rep->train_loss = static_cast<float>(last_epoch_loss);
        rep->steps = static_cast<uint32_t>(step);
    }
    if (n_val > 0 && rep) {
        const float *xv = dX.as<float>() + n_train * CL_IN;
        k_infer<<<nblk(static_cast<long long>(n_val)), 256, 0, st>>>(c->nets.as<ClosureNet>() + model, xv,
                                                                   static_cast<int>(n_val), dY.as<float>());
        std::vector<float> Y(n_val * CL_OUT);
        if (cudaMemcpyAsync(Y.data(), dY.p, Y.size() * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return sim_fail(s, EMERGE_ERR_CUDA, "closure: validation");
        std::vector<float> errs(n_val);
        double mse = 0.0, trial_sum = 0.0;
        for (size_t r = 0; r < n_val; ++r) {
            const size_t i = perm[n_train + r];
            float yp[CL_OUT], xr[CL_IN];
            for (int j = 0; j < CL_OUT; ++j) {
                const float yn = Y[r * CL_OUT + j], tn = Tn[(n_train + r) * CL_OUT + j];
                mse += static_cast<double>(yn - tn) * (yn - tn);
                yp[j] = yn * norm[2 * CL_IN + CL_OUT + j] + norm[2 * CL_IN + j];
            }
            for (int j = 0; j < CL_IN; ++j) xr[j] = X[i * CL_IN + j];
            errs[r] = stress_rel_err(model, xr, yp, &T[i * CL_OUT]);
            // the mapping skipped: the trial strains (DP: eps / s; NACC: no correction)
            const float y_trial[CL_OUT] = {model == 0 ? xr[0] : 0.0f, model == 0 ? xr[1] : 0.0f, 0.0f};
            trial_sum += stress_rel_err(model, xr, y_trial, &T[i * CL_OUT]);
        }
        std::vector<float> sorted = errs;
        std::sort(sorted.begin(), sorted.end());
        double sum = 0.0;
        for (float e : errs) sum += e;
        rep->val_loss = static_cast<float>(mse / (n_val * CL_OUT));
        rep->val_err_mean = static_cast<float>(sum / n_val);
        rep->val_err_p50 = sorted[n_val / 2];
        rep->val_err_p99 = sorted[std::min(n_val - 1, static_cast<size_t>(0.99 * n_val))];
        rep->val_err_max = sorted.back();
        rep->val_err_trial_mean = static_cast<float>(trial_sum / n_val);
    }
    if (cudaMemcpy(c->params[model].alloc(CL_NPARAMS * sizeof(float)) == cudaSuccess ? c->params[model].p : nullptr,
                   dP.p, CL_NPARAMS * sizeof(float), cudaMemcpyDeviceToDevice) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: keep params");
    if (rep)
        rep->seconds = std::chrono::duration<float>(std::chrono::steady_clock::now() - t_start).count();
    sim_invalidate_graph(s);
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_get_log(emerge_sim *s, int model, float *x, float *t, uint64_t max,
                                          uint64_t *n) {
    if (!s || !n || model < 0 || model >= CL_NMODELS || (max && (!x || !t))) return EMERGE_ERR_INVALID_ARG;
    *n = 0;
    ClosureHost *c = sim_closure(s);
    if (!c || !c->log_x[model].p) return EMERGE_OK;
    ClosureStats hs;
    if (cudaMemcpy(&hs, c->stats.p, sizeof(hs), cudaMemcpyDeviceToHost) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: stats read");
    const uint64_t k = std::min<unsigned long long>(std::min<unsigned long long>(hs.logged[model], c->log_cap), max);
    if (k && (cudaMemcpy(x, c->log_x[model].p, k * CL_IN * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
              cudaMemcpy(t, c->log_t[model].p, k * CL_OUT * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess))
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: log read");
    *n = k;
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_get_params(emerge_sim *s, int model, float *params, float *norm) {
    if (!s || !params || model < 0 || model >= CL_NMODELS) return EMERGE_ERR_INVALID_ARG;
    ClosureHost *c = sim_closure(s);
    if (!c || !c->params[model].p) return sim_fail(s, EMERGE_ERR_INVALID_ARG, "closure: no trained network");
    if (cudaMemcpy(params, c->params[model].p, CL_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: read params");
    if (norm) std::memcpy(norm, c->norm[model].data(), c->norm[model].size() * sizeof(float));
    return EMERGE_OK;
}

emerge_status emerge_cuda_closure_set_params(emerge_sim *s, int model, const float *params, const float *norm,
                                             const float *hull) {
    if (!s || !params || !norm || !hull || model < 0 || model >= CL_NMODELS) return EMERGE_ERR_INVALID_ARG;
    ClosureHost *&c = sim_closure(s);
    emerge_status st = ensure_closure(s, c);
    if (st != EMERGE_OK) return st;
    if (c->params[model].alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess)
        return sim_fail(s, EMERGE_ERR_OOM, "closure: params");
    cudaStream_t cs = sim_stream(s);
    if (cudaMemcpyAsync(c->params[model].p, params, CL_NPARAMS * sizeof(float), cudaMemcpyHostToDevice, cs) !=
        cudaSuccess)
        return sim_fail(s, EMERGE_ERR_CUDA, "closure: params upload");
    st = install_net(s, c, model, c->params[model].as<float>(), norm, hull, cs);
    sim_invalidate_graph(s);
    return st;
}

// ---- stand-alone test hooks: host arrays in and out -----------------------------------
emerge_status emerge_cuda_mlp_loss_grad(const float *params, const float *x, const float *t, uint32_t B,
                                        float *loss, float *grad) {
    if (!params || !x || !t || !loss || !grad || B == 0 || B > 65536) return EMERGE_ERR_INVALID_ARG;
    DevBuf dP, dX, dT, dL;
    MlpWork w;
    if (dP.alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess || dX.alloc(B * CL_IN * sizeof(float)) != cudaSuccess ||
        dT.alloc(B * CL_OUT * sizeof(float)) != cudaSuccess || dL.alloc(sizeof(double)) != cudaSuccess ||
        w.alloc(static_cast<int>(B)) != cudaSuccess)
        return EMERGE_ERR_OOM;
    cudaMemcpy(dP.p, params, CL_NPARAMS * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dX.p, x, B * CL_IN * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dT.p, t, B * CL_OUT * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(dL.p, 0, sizeof(double));
    mlp_loss_grad(dP.as<float>(), dX.as<float>(), dT.as<float>(), static_cast<int>(B), w, dL.as<double>(), 0);
    double l = 0.0;
    if (cudaMemcpy(&l, dL.p, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(grad, w.grad.p, CL_NPARAMS * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return EMERGE_ERR_CUDA;
    *loss = static_cast<float>(l);
    return cudaGetLastError() == cudaSuccess ? EMERGE_OK : EMERGE_ERR_CUDA;
}

emerge_status emerge_cuda_mlp_adam(float *params, float *m, float *v, const float *grad, uint32_t n, uint32_t step,
                                   float lr, float beta1, float beta2, float eps) {
    if (!params || !m || !v || !grad || n == 0 || step == 0) return EMERGE_ERR_INVALID_ARG;
    DevBuf dP, dM, dV, dG;
    if (dP.alloc(n * sizeof(float)) != cudaSuccess || dM.alloc(n * sizeof(float)) != cudaSuccess ||
        dV.alloc(n * sizeof(float)) != cudaSuccess || dG.alloc(n * sizeof(float)) != cudaSuccess)
        return EMERGE_ERR_OOM;
    cudaMemcpy(dP.p, params, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dM.p, m, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dV.p, v, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dG.p, grad, n * sizeof(float), cudaMemcpyHostToDevice);
    k_adam<<<nblk(n), 256>>>(dP.as<float>(), dG.as<float>(), dM.as<float>(), dV.as<float>(), static_cast<int>(n),
                             static_cast<int>(step), lr, beta1, beta2, eps);
    if (cudaMemcpy(params, dP.p, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(m, dM.p, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(v, dV.p, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return EMERGE_ERR_CUDA;
    return EMERGE_OK;
}

emerge_status emerge_cuda_mlp_infer_bf16(const float *params, const float *x, uint32_t n, float *y) {
    if (!params || !x || !y || n == 0) return EMERGE_ERR_INVALID_ARG;
    DevBuf dP, dNet, dX, dY;
    if (dP.alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess || dNet.alloc(sizeof(ClosureNet)) != cudaSuccess ||
        dX.alloc(static_cast<size_t>(n) * CL_IN * sizeof(float)) != cudaSuccess ||
        dY.alloc(static_cast<size_t>(n) * CL_OUT * sizeof(float)) != cudaSuccess)
        return EMERGE_ERR_OOM;
    cudaMemcpy(dP.p, params, CL_NPARAMS * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dX.p, x, static_cast<size_t>(n) * CL_IN * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(dNet.p, 0, sizeof(ClosureNet));
    k_pack_net<<<nblk(CL_FRAGS * 32), 256>>>(dP.as<float>(), dNet.as<ClosureNet>());
    k_infer<<<nblk(n), 256>>>(dNet.as<ClosureNet>(), dX.as<float>(), static_cast<int>(n), dY.as<float>());
    if (cudaMemcpy(y, dY.p, static_cast<size_t>(n) * CL_OUT * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return EMERGE_ERR_CUDA;
    return cudaGetLastError() == cudaSuccess ? EMERGE_OK : EMERGE_ERR_CUDA;
}

emerge_status emerge_cuda_mlp_infer_tc(const float *params, const float *x, uint32_t n, float *y) {
    if (!params || !x || !y || n == 0) return EMERGE_ERR_INVALID_ARG;
    DevBuf dP, dNet, dX, dY, dErr;
    if (dP.alloc(CL_NPARAMS * sizeof(float)) != cudaSuccess || dNet.alloc(sizeof(ClosureNet)) != cudaSuccess ||
        dX.alloc(static_cast<size_t>(n) * CL_IN * sizeof(float)) != cudaSuccess ||
        dY.alloc(static_cast<size_t>(n) * CL_OUT * sizeof(float)) != cudaSuccess ||
        dErr.alloc(sizeof(uint32_t)) != cudaSuccess)
        return EMERGE_ERR_OOM;
    cudaMemcpy(dP.p, params, CL_NPARAMS * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dX.p, x, static_cast<size_t>(n) * CL_IN * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(dNet.p, 0, sizeof(ClosureNet));
    cudaMemset(dErr.p, 0, sizeof(uint32_t));
    k_pack_net<<<nblk(CL_FRAGS * 32), 256>>>(dP.as<float>(), dNet.as<ClosureNet>());
    k_pack_tc<<<nblk(CL_H * CL_TC_K1 + 2 * CL_H * CL_H + CL_TC_N4 * CL_H), 256>>>(dP.as<float>(), dNet.as<ClosureNet>());
    if (launch_mlp_tiles(dNet.as<ClosureNet>(), dX.as<float>(), static_cast<int>(n), dY.as<float>(),
                         dErr.as<uint32_t>(), nullptr) != cudaSuccess)
        return EMERGE_ERR_CUDA;
    uint32_t err = 0u;
    if (cudaMemcpy(y, dY.p, static_cast<size_t>(n) * CL_OUT * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&err, dErr.p, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return EMERGE_ERR_CUDA;
    if (err) return EMERGE_ERR_TIMEOUT;
    return cudaGetLastError() == cudaSuccess ? EMERGE_OK : EMERGE_ERR_CUDA;
}

emerge_status emerge_cuda_silu_fast(const float *x, uint32_t n, float *y) {
    if (!x || !y || n == 0) return EMERGE_ERR_INVALID_ARG;
    DevBuf dX, dY;
    if (dX.alloc(static_cast<size_t>(n) * sizeof(float)) != cudaSuccess ||
        dY.alloc(static_cast<size_t>(n) * sizeof(float)) != cudaSuccess)
        return EMERGE_ERR_OOM;
    if (cudaMemcpy(dX.p, x, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        launch_silu_fast(dX.as<float>(), static_cast<int>(n), dY.as<float>(), nullptr) != cudaSuccess ||
        cudaMemcpy(y, dY.p, static_cast<size_t>(n) * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return EMERGE_ERR_CUDA;
    return EMERGE_OK;
}

}  // extern "C"
