// closure_tiles.cu -- the learned closure's network on the 5th-generation tensor cores.
//
// The particle pass (CLOSURE == 2 in particle_pass.cuh) queues every particle whose return
// mapping the network is to replace: a Drucker-Prager or NACC particle on the smooth plastic
// branch inside the training box (about 6 % of the particles of the 4M-particle granular
// scene per substep).  This kernel takes them 128 at a time:
//   1. each thread recomputes its particle's trial state and network inputs from the state
//      the particle pass stored (G2P done, update not), exactly as the pass decided them;
//   2. the four layers run as tcgen05.mma (kind::f16, BF16 operands, FP32 accumulators in
//      tensor memory): A = the tile's activations (128 x K, K-major, shared memory), B = the
//      layer's weights (shared memory, loaded once per CTA), D = 128 x N FP32 in TMEM; one
//      thread issues the MMAs, tcgen05.commit signals an mbarrier, and every thread reads
//      its row back with tcgen05.ld, adds the bias, applies SiLU and writes the next layer's
//      BF16 row into shared memory;
//   3. each thread finishes its particle like the particle pass would have: the update from
//      the network's outputs (sampled particles also through the plain mapping: the judge,
//      whose results above the bar replace the network's), CFL bound, projection for the
//      next substep, Kirchhoff stress and the P2G scatter.
// Persistent CTAs of 128 threads loop over the tiles of both queues.  Every wait on an
// mbarrier is bounded; a wait that runs out sets ERR_CLOSURE_WAIT in StepState::error_flags,
// the CTA stops issuing work, and the TMEM it holds is freed before it returns.
#define EMERGE_FAST_TU 1
#include <cstring>

#include "particle_pass.cuh"

namespace emerge {

namespace {

// Resident tile CTAs per SM (the persistent grid is this many per SM): registers bound it,
// 65,536 / (128 threads x the kernel's registers).
#ifndef EMERGE_CLOSURE_TILE_CTAS_PER_SM
#define EMERGE_CLOSURE_TILE_CTAS_PER_SM 3
#endif
constexpr int CT_M = 128;         // rows (particles) per tile = TMEM lanes = threads
constexpr int CT_TMEM_COLS = 64;  // FP32 accumulator columns (the widest layer)

// Shared memory of one CTA (dynamic, 1 KB aligned).
struct TileSmem {
    unsigned char a[CT_M * CL_H * 2];            // activations, K-major (K = 64) core matrices
    unsigned char w[CL_TC_BYTES];                // the weights of the network in use (loaded_net)
    float bias[CL_NMODELS][3 * CL_H + 8];
    float in_shift[CL_NMODELS][8], in_scale[CL_NMODELS][8];
    float out_shift[CL_NMODELS][4], out_scale[CL_NMODELS][4];
    MatP mats[MAX_MATERIALS];
    unsigned long long mbar;
    uint32_t tmem_base;
    uint32_t abort;
    uint32_t min_mdt_bits;
    int loaded_net;                              // network whose weights are in w (-1: none)
};

// Shared-memory matrix descriptor (tcgen05 "matrix descriptor"): start address, leading
// dimension byte offset (between core matrices adjacent along K), stride dimension byte
// offset (between 8-row groups), each in 16-byte units; descriptor version 1 (bits 46-47);
// base offset 0, no swizzling (layout type 0 in bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) |
           (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both operands K-major:
// D format (bits 4-5) = 1 (F32), A format (7-9) = 1 and B format (10-12) = 1 (BF16),
// N / 8 in bits 17-22, M / 16 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
    const uint32_t mask = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask), "r"(mask), "r"(mask),
          "r"(mask));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(mbar)
                 : "memory");
}

// Waits for phase `parity` of the mbarrier, giving up after about a second; true if done.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 2000000000ll) return false;
    }
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (one row per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// 16 consecutive FP32 columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// SiLU(z) = z sigma(z) = z (1 + tanh(z / 2)) / 2, with one hardware tanh (tanh.approx.f32,
// max relative error about 2^-11): the activations are rounded to BF16 (2^-9) for the next
// layer anyway.
__device__ __forceinline__ float silu_fast(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    return 0.5f * z * (1.0f + t);
}

// Test hook: y = silu_fast(x), elementwise.
__global__ void k_silu_fast(const float *x, int n, float *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = silu_fast(x[i]);
}

// Writes 8 consecutive BF16 values of row `r` starting at K index k0 (a multiple of 8) into
// the activation tile (K = 64 layout).
__device__ __forceinline__ void put_row8(unsigned char *a, int r, int k0, const float *v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4 *>(a + km_offset(r, k0, CL_H)) = q;
}

// The particle's trial state and network inputs (the same computation as closure_prepare in
// the particle pass, from the state it stored).  Returns false if the particle is no longer
// on the network's branch (it always is: the pass decided on the same values).
template <unsigned MASK>
__device__ __forceinline__ bool tile_prepare(const MatP &m, const PState &p, float dt, bool pr,
                                             int model, ClosureWork &w) {
    w.kind = 0;
    w.judge = 0;
    w.smooth = 1;
    if (model == 0) {
        const M2 f_trial = mm(madd(mident(), smscale(dt, p.c)), p.f);
        svd2(f_trial, w.u, w.sigma, w.vt);
        const DpTrial t = dp_trial(m, w.sigma, p.lvs, p.q, pr);
        if (t.dev_norm == 0.0f || t.trace > 0.0f || t.gamma <= 0.0f) return false;
        const float inv_s = 1.0f / t.dev_norm;
        w.x[0] = t.eps.x * inv_s;
        w.x[1] = t.eps.y * inv_s;
        w.x[2] = t.alpha;
        w.x[3] = t.ratio;
        w.x[4] = t.cohesion * inv_s;
        w.x[5] = em_log(t.dev_norm, pr);
        w.scale = t.dev_norm;
        w.kind = 1;
        return true;
    }
    svd2(p.f, w.u, w.sigma, w.vt);
    const NaccTrial t = nacc_trial(m, w.sigma, p.lvs, pr);
    if (t.branch != 3) return false;
    const float kappa = nacc_kappa(m);
    w.x[0] = em_log(fmaxf(w.sigma.x, LOG_CLAMP), pr);
    w.x[1] = em_log(fmaxf(w.sigma.y, LOG_CLAMP), pr);
    w.x[2] = t.p0 / kappa;
    w.x[3] = m.mu / kappa;
    w.x[4] = m.compression_limit;
    w.x[5] = m.stretch_limit;
    w.kind = 2;
    return true;
}

// Tensor-core resources of one CTA: the TMEM columns, the mbarrier and its phase.
struct TileMma {
    uint32_t tmem, mbar, a_addr, row_taddr, phase;
};

// Allocates TMEM (warp 0), initialises the mbarrier; every thread calls it (CTA barrier).
__device__ __forceinline__ TileMma tile_mma_begin(TileSmem &S) {
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        S.abort = 0u;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&S.tmem_base)),
                     "r"(CT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    TileMma t;
    t.tmem = S.tmem_base;
    t.mbar = smem_u32(&S.mbar);
    t.a_addr = smem_u32(S.a);
    t.row_taddr = t.tmem + (static_cast<uint32_t>(warp * 32) << 16);  // this warp's TMEM lanes
    t.phase = 0u;
    return t;
}

// Frees the TMEM (warp 0) after every thread is done with it; after a wait that ran out, the
// MMAs issued before are waited for (with the same bound) first.  Returns true if a wait
// ran out during the CTA's work.  Every thread calls it.
__device__ __forceinline__ bool tile_mma_end(TileSmem &S, TileMma &t) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool aborted = S.abort != 0u;
    if (threadIdx.x == 0 && aborted) {
        umma_commit(t.mbar);  // arrives once every MMA issued before it has completed
        mbar_wait(t.mbar, t.phase);
    }
    __syncthreads();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(t.tmem), "r"(CT_TMEM_COLS)
                     : "memory");
    return aborted;
}

// One MMA layer: D (TMEM columns 0..n-1) = A (K = 16 kt) x W^T, issued by thread 0; every
// thread waits for it.  False (CTA-uniform) if the wait ran out.
__device__ __forceinline__ bool tile_layer(TileSmem &S, TileMma &t, uint32_t w_addr, int kt, int n,
                                           uint32_t sbo_b) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A rows written by the threads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
        const uint32_t id = idesc_bf16(CT_M, n);
        for (int k = 0; k < kt; ++k)  // K slice k = core matrices 2k and 2k + 1 (256 bytes)
            umma_bf16(t.tmem, smem_desc(t.a_addr + 256u * k, 128u, CL_H * 16u),
                      smem_desc(w_addr + 256u * k, 128u, sbo_b), id, k > 0 ? 1u : 0u);
        umma_commit(t.mbar);
    }
    const bool ok = mbar_wait(t.mbar, t.phase);
    t.phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) atomicOr(&S.abort, 1u);
    __syncthreads();
    return S.abort == 0u;
}

// The network `net` on the CTA's 128 rows: row threadIdx.x has normalised inputs x and gets
// normalised outputs y.  Every thread calls it.  False (CTA-uniform) if a wait ran out.
__device__ __forceinline__ bool tile_mlp(TileSmem &S, TileMma &t, int net, const float (&x)[CL_IN],
                                         float (&y)[CL_OUT]) {
    const int tid = threadIdx.x;
    {
        float in[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) in[j] = j < CL_IN ? x[j] : 0.0f;
        put_row8(S.a, tid, 0, in);
        put_row8(S.a, tid, 8, in + 8);
    }
    const uint32_t wb = smem_u32(S.w);
    const float *bias = S.bias[net];
    bool ok = tile_layer(S, t, wb + CL_TC_OFF_L1, 1, CL_H, CL_TC_K1 * 16u);
#pragma unroll 1
    for (int l = 0; l < 3 && ok; ++l) {
        // this row's 64 accumulators: bias, SiLU, the next layer's BF16 row
        float v[32];
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            tmem_ld32(t.row_taddr + 32u * half, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = silu_fast(v[j] + bias[l * CL_H + 32 * half + j]);
#pragma unroll
            for (int c = 0; c < 4; ++c) put_row8(S.a, tid, 32 * half + 8 * c, v + 8 * c);
        }
        if (l < 2)
            ok = tile_layer(S, t, wb + (l == 0 ? CL_TC_OFF_L2 : CL_TC_OFF_L3), 4, CL_H, CL_H * 16u);
        else
            ok = tile_layer(S, t, wb + CL_TC_OFF_L4, 4, CL_TC_N4, CL_H * 16u);
    }
    if (!ok) return false;
    float v[16];
    tmem_ld16(t.row_taddr, v);
#pragma unroll
    for (int j = 0; j < CL_OUT; ++j) y[j] = v[j] + bias[3 * CL_H + j];
    return true;
}

// Copies network `net`'s tcgen05 weights into shared memory if they are not there yet; every
// thread calls it (CTA barrier).  The MMAs of the previous tile have completed (waited for).
__device__ __forceinline__ void tile_use_net(TileSmem &S, const ClosureNet *nets, int net) {
    if (S.loaded_net == net) return;  // CTA-uniform
    __syncthreads();
    const uint4 *src = reinterpret_cast<const uint4 *>(nets[net].tc);
    uint4 *dst = reinterpret_cast<uint4 *>(S.w);
    for (int k = threadIdx.x; k < CL_TC_BYTES / 16; k += CT_M) dst[k] = src[k];
    __syncthreads();
    if (threadIdx.x == 0) S.loaded_net = net;
    __syncthreads();
}

// Copies the networks' biases and normalisation into shared memory.
__device__ __forceinline__ void tile_load_nets(TileSmem &S, const ClosureNet *nets, int n_nets) {
    const int tid = threadIdx.x;
    if (tid == 0) S.loaded_net = -1;
    for (int net = 0; net < n_nets; ++net) {
        const ClosureNet &nn = nets[net];
        for (int k = tid; k < 3 * CL_H + 8; k += CT_M) S.bias[net][k] = nn.bias[k];
        if (tid < 8) {
            S.in_shift[net][tid] = nn.in_shift[tid];
            S.in_scale[net][tid] = nn.in_scale[tid];
        }
        if (tid < 4) {
            S.out_shift[net][tid] = nn.out_shift[tid];
            S.out_scale[net][tid] = nn.out_scale[tid];
        }
    }
}

// Stores the fields an update can change (the particle pass stored x, v and C already).
__device__ __forceinline__ void store_update(const DevParticles &P, int i, const Saved &o, const PState &p) {
    if (neqm(p.f, o.f)) P.f[i] = m_to4(p.f);
    if (neq(p.vol, o.vol)) P.vol[i] = p.vol;
    if (neq(p.rho, o.rho)) P.rho[i] = p.rho;
    if (neq(p.jp, o.jp)) P.jp[i] = p.jp;
    if (neq(p.h, o.h)) P.h[i] = p.h;
    if (neq(p.q, o.q)) P.q[i] = p.q;
    if (neq(p.lvs, o.lvs)) P.lvs[i] = p.lvs;
}

struct TileArgs {
    DevParticles P;
    const MatP *mats;
    int n_mats;
    DevConfig cfg;
    StepState *st;
    GridView g;
    LoadFlags lf;
    ClosureArgs cl;
};

template <unsigned MASK>
__global__ void __launch_bounds__(CT_M, EMERGE_CLOSURE_TILE_CTAS_PER_SM) k_closure_tiles(TileArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    const int tid = threadIdx.x;
    StepState *st = a.st;
    const uint32_t slot = st->acc_slot;
    const uint32_t n_q0 = st->cl_queued[slot][0], n_q1 = st->cl_queued[slot][1];
    const int tiles0 = static_cast<int>((n_q0 + CT_M - 1) / CT_M);
    const int tiles = tiles0 + static_cast<int>((n_q1 + CT_M - 1) / CT_M);
    if (static_cast<int>(blockIdx.x) >= tiles) return;  // CTA-uniform: nothing allocated yet

    // ---- set-up: weights, materials, mbarrier, TMEM
    tile_load_nets(S, a.cl.nets, CL_NMODELS);
    for (int k = tid; k < a.n_mats; k += CT_M) S.mats[k] = a.mats[k];
    if (tid == 0) S.min_mdt_bits = 0x7f800000u;
    TileMma t = tile_mma_begin(S);
    const bool pr = a.cfg.precise_math != 0;
    const float dt = st->sub_dt;
    const ClosureArgs &cl = a.cl;
    const GridView &g = a.g;
    const DevConfig &cfg = a.cfg;
    unsigned long long n_net = 0ull;  // per thread: network results applied

    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int model = tile < tiles0 ? 0 : 1;
        const uint32_t q = static_cast<uint32_t>((model ? tile - tiles0 : tile) * CT_M + tid);
        const bool valid = q < (model ? n_q1 : n_q0);
        const int i = valid ? static_cast<int>(cl.queue[model][q]) : 0;
        PState p;
        Saved o;
        ClosureWork w;
        w.kind = 0;
        w.smooth = 0;
        const MatP *mp = &S.mats[0];
        bool on_branch = false;
        if (valid) {
            p = load_state(a.P, i, a.lf);
            o = save_fields(p);
            mp = &S.mats[p.mat < static_cast<uint32_t>(a.n_mats) ? p.mat : 0u];
            on_branch = tile_prepare<MASK>(*mp, p, dt, pr, model, w);
        }
        // inputs outside the box of the normalised training inputs use the plain mapping
        const bool use_net = on_branch && closure_in_hull(cl.nets[model], w.x);
        float xn[CL_IN], y[CL_OUT];
#pragma unroll
        for (int j = 0; j < CL_IN; ++j)
            xn[j] = use_net ? (w.x[j] - S.in_shift[model][j]) * S.in_scale[model][j] : 0.0f;
        tile_use_net(S, a.cl.nets, model);
        if (!tile_mlp(S, t, model, xn, y)) break;  // CTA-uniform
#pragma unroll
        for (int j = 0; j < CL_OUT; ++j) y[j] = y[j] * S.out_scale[model][j] + S.out_shift[model][j];
        // ---- finish: update from the outputs (judge and fallback), CFL, projection, P2G
        Payload pl;
        pl.do_ma = false;
        pl.do_s = false;
        pl.fields = 0u;
        pl.excl = false;
        float err = -1.0f;
        int replaced = 0, projected = 0, proj_changed = 0;
        float min_mdt = INFINITY;
        if (valid) {
            const MatP &m = *mp;
            if (use_net) {
                w.judge = (closure_hash(i, st) >> 7) % cl.judge_stride == 0u;
                PState pn = p;
                closure_finish<MASK>(m, pn, pr, w, y, err);
                if (err > cl.judge_bar) {  // the judge ran the plain mapping: keep its result
                    update_particle<MASK>(m, p, dt, pr);
                    replaced = 1;
                } else {
                    p = pn;
                    n_net += 1ull;
                }
            } else {
                update_particle<MASK>(m, p, dt, pr);
            }
            store_update(a.P, i, o, p);
            const float mdt = timestep_bound<MASK>(m, p.rho, p.h, cfg.cell, cfg.mat_cfl, cfg.visc_cfl, pr);
            if (isfinite(mdt) && mdt > 0.0f) min_mdt = mdt;
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
            pl.tau = combined_kirchhoff_stress<MASK>(m, p, pr);
            pl.s = -stress_volume(m, p) * KERNEL_D_INVERSE;
            pl.do_s = true;
        }
        // statistics of the queued particles and the network's results (one atomic per warp)
        {
            const unsigned full = 0xffffffffu;
            const int n_smooth = __reduce_add_sync(full, valid && on_branch ? 1 : 0);
            const int n_hull = __reduce_add_sync(full, valid && on_branch && !use_net ? 1 : 0);
            if ((tid & 31) == 0 && n_smooth) {
                atomicAdd(&cl.stats->smooth, static_cast<unsigned long long>(n_smooth));
                if (n_hull) atomicAdd(&cl.stats->hull_fallback, static_cast<unsigned long long>(n_hull));
            }
            const int n_judged = __reduce_add_sync(full, err >= 0.0f ? 1 : 0);
            const int n_rep = __reduce_add_sync(full, replaced);
            float e_sum = err >= 0.0f ? err : 0.0f, e_max = e_sum;
            for (int off = 16; off > 0; off >>= 1) {
                e_sum += __shfl_xor_sync(full, e_sum, off);
                e_max = fmaxf(e_max, __shfl_xor_sync(full, e_max, off));
            }
            if ((tid & 31) == 0 && n_judged) {
                atomicAdd(&cl.stats->judged, static_cast<unsigned long long>(n_judged));
                atomicAdd(&cl.stats->err_sum, static_cast<double>(e_sum));
                atomicMax(&cl.stats->err_max_bits, __float_as_uint(e_max));
                if (n_rep) atomicAdd(&cl.stats->judge_replaced, static_cast<unsigned long long>(n_rep));
            }
            if (err >= 0.0f) atomicAdd(&cl.stats->err_hist[closure_err_bin(err)], 1ull);
            count_warp(&st->jproj_pending[slot], projected != 0);
            count_warp(&st->proj_changed[slot], proj_changed != 0);
            const float mw = warp_min(min_mdt);
            if ((tid & 31) == 0 && mw < INFINITY) atomicMin(&S.min_mdt_bits, __float_as_uint(mw));
        }
        scatter_particle<SC_BOTH>(g, pl, valid, 0);
    }
    if (n_net) atomicAdd(&cl.stats->net, n_net);
    // ---- tear-down: publish the CFL bound, free TMEM (also after a wait that ran out)
    const bool aborted = tile_mma_end(S, t);
    if (tid == 0) {
        if (S.min_mdt_bits != 0x7f800000u) atomicMin(&st->min_mdt_bits[slot], S.min_mdt_bits);
        if (aborted) atomicOr(&st->error_flags, ERR_CLOSURE_WAIT);
    }
}

// Test hook: the network on n normalised inputs (128 per CTA), outputs normalised.
__global__ void __launch_bounds__(CT_M, 1) k_mlp_tiles(const ClosureNet *net, const float *x, int n, float *y,
                                                     uint32_t *error) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    const int tid = threadIdx.x;
    tile_load_nets(S, net, 1);
    TileMma t = tile_mma_begin(S);
    tile_use_net(S, net, 0);
    const int tiles = (n + CT_M - 1) / CT_M;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int r = tile * CT_M + tid;
        float xi[CL_IN], yi[CL_OUT];
#pragma unroll
        for (int j = 0; j < CL_IN; ++j) xi[j] = r < n ? x[static_cast<size_t>(r) * CL_IN + j] : 0.0f;
        if (!tile_mlp(S, t, 0, xi, yi)) break;
        if (r < n)
#pragma unroll
            for (int j = 0; j < CL_OUT; ++j) y[static_cast<size_t>(r) * CL_OUT + j] = yi[j];
    }
    if (tile_mma_end(S, t) && tid == 0) atomicOr(error, 1u);
}

}  // namespace

// Test hook launcher: returns the kernel's error word (0 = every wait completed).
cudaError_t launch_mlp_tiles(const ClosureNet *net, const float *x, int n, float *y, uint32_t *error,
                             cudaStream_t stream) {
    const size_t smem = sizeof(TileSmem);
    cudaError_t e = cudaFuncSetAttribute(k_mlp_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const int tiles = (n + CT_M - 1) / CT_M;
    k_mlp_tiles<<<tiles < 296 ? tiles : 296, CT_M, smem, stream>>>(net, x, n, y, error);
    return cudaGetLastError();
}

// Launches the tile kernel after the particle pass of a substep (same stream).  Persistent
// CTAs: three per SM (the registers of 3 x 128 threads and about 45 KB of shared memory
// each), each looping over the tiles both queues hold this substep.
cudaError_t launch_silu_fast(const float *x, int n, float *y, cudaStream_t stream) {
    if (n > 0) k_silu_fast<<<(n + 255) / 256, 256, 0, stream>>>(x, n, y);
    return cudaGetLastError();
}

void launch_closure_tiles(const StepLaunch &L, const LoadFlagsHost &lfh, int sm_count) {
    if (L.n == 0 || !L.cl.defer) return;
    TileArgs a;
    std::memset(&a, 0, sizeof(a));
    a.P = L.P;
    a.mats = L.mats;
    a.n_mats = L.n_mats;
    a.cfg = L.cfg;
    a.st = L.st;
    a.g = L.g;
    a.lf.temperature = lfh.temperature;
    a.lf.activation = lfh.activation;
    a.lf.pinned = lfh.pinned;
    a.cl = L.cl;
    const size_t smem = sizeof(TileSmem);
    const int grid = EMERGE_CLOSURE_TILE_CTAS_PER_SM * (sm_count > 0 ? sm_count : 148);
    const unsigned cover = covering_mask(L.model_mask);
    if (cover == MASK_GRANULAR) {
        cudaFuncSetAttribute(k_closure_tiles<MASK_GRANULAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        k_closure_tiles<MASK_GRANULAR><<<grid, CT_M, smem, L.stream>>>(a);
    } else if (cover == ALL_MODELS) {
        cudaFuncSetAttribute(k_closure_tiles<ALL_MODELS>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        k_closure_tiles<ALL_MODELS><<<grid, CT_M, smem, L.stream>>>(a);
    } else {
        cudaFuncSetAttribute(k_closure_tiles<FULL_MODELS>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        k_closure_tiles<FULL_MODELS><<<grid, CT_M, smem, L.stream>>>(a);
    }
}

}  // namespace emerge
