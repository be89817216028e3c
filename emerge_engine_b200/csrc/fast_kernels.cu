// fast_kernels.cu -- the fast path's particle and density passes.
//
// Compiled with approximate division and square root outside the constitutive math and no
// implicit contraction (see build.py): the fused pipeline's default mode, whose results
// differ from the reference only in float rounding (summation order of the L2 reductions,
// the explicit fused multiply-adds of the stencil sums, 2-ulp division and square root).
// The reference-order mode runs the exact instantiation in step_kernels.cu.
#define EMERGE_FAST_TU 1  // em_pow: integer exponents by repeated multiplication
#include <cstring>

#include "particle_pass.cuh"

// Resident CTAs per SM the register allocation is sized for (256 threads each).
#ifndef EMERGE_PARTICLE_CTAS_PER_SM
#define EMERGE_PARTICLE_CTAS_PER_SM 4
#endif
#ifndef EMERGE_DENSITY_CTAS_PER_SM
#define EMERGE_DENSITY_CTAS_PER_SM 6
#endif

namespace emerge {

template <unsigned MASK>
__global__ void __launch_bounds__(THREADS, EMERGE_PARTICLE_CTAS_PER_SM) k_particle_fast(ParticleKernelArgs a) {
    particle_pass<MASK, true>(a);
}

// The particle pass with the learned closure (or its data logging) for scenes with
// Drucker-Prager or NACC particles; 2 CTAs per SM leave registers for the network.
#ifndef EMERGE_CLOSURE_CTAS_PER_SM
#define EMERGE_CLOSURE_CTAS_PER_SM 2
#endif
template <unsigned MASK>
__global__ void __launch_bounds__(THREADS, EMERGE_CLOSURE_CTAS_PER_SM) k_particle_closure(ParticleKernelArgs a) {
    particle_pass<MASK, true, 1>(a);
}

// The particle pass that queues the network's particles for the tile kernel (no network in
// this kernel, so it keeps the plain pass's register budget and occupancy).
template <unsigned MASK>
__global__ void __launch_bounds__(THREADS, EMERGE_PARTICLE_CTAS_PER_SM) k_particle_closure_queue(ParticleKernelArgs a) {
    particle_pass<MASK, true, 2>(a);
}

// estimate_particle_volumes gather (solver/density.rs:50-71) at the projected
// positions, stored as rho_dp, plus the stress scatter of fluid particles.
template <unsigned MASK>
__global__ void __launch_bounds__(THREADS, EMERGE_DENSITY_CTAS_PER_SM) k_density(DensityKernelArgs a) {
    density_pass<MASK>(a);
}

// Batched scenes: every chunk of 256 particles finds its scene in the batch's tables; all
// model sets.  A CTA works through K consecutive chunks (K x 256 particles per CTA, an
// autotuned choice), with a barrier between chunks so the per-chunk shared state (materials,
// CFL reduction) starts afresh.
template <unsigned MASK, int K>
__global__ void __launch_bounds__(THREADS, EMERGE_PARTICLE_CTAS_PER_SM) k_particle_batch(ParticleKernelArgs a) {
#pragma unroll 1
    for (int c = 0; c < K; ++c) {
        const int chunk = static_cast<int>(blockIdx.x) * K + c;
        if (chunk >= a.batch.n_chunks) break;  // CTA-uniform
        if (c > 0) __syncthreads();
        particle_pass<MASK, true, 0, true>(a, chunk);
    }
}
template <unsigned MASK, int K>
__global__ void __launch_bounds__(THREADS, EMERGE_DENSITY_CTAS_PER_SM) k_density_batch(DensityKernelArgs a) {
#pragma unroll 1
    for (int c = 0; c < K; ++c) {
        const int chunk = static_cast<int>(blockIdx.x) * K + c;
        if (chunk >= a.batch.n_chunks) break;
        if (c > 0) __syncthreads();
        density_pass<MASK, true>(a, chunk);
    }
}

template <int K>
void batch_particle_launch(const ParticleKernelArgs &a, unsigned model_mask, cudaStream_t stream) {
    const int grid = (a.batch.n_chunks + K - 1) / K;
    if ((model_mask & ~ALL_MODELS) == 0u)
        k_particle_batch<ALL_MODELS, K><<<grid, THREADS, 0, stream>>>(a);
    else
        k_particle_batch<FULL_MODELS, K><<<grid, THREADS, 0, stream>>>(a);
}
template <int K>
void batch_density_launch(const DensityKernelArgs &a, unsigned model_mask, cudaStream_t stream) {
    const int grid = (a.batch.n_chunks + K - 1) / K;
    if ((model_mask & ~ALL_MODELS) == 0u)
        k_density_batch<ALL_MODELS, K><<<grid, THREADS, 0, stream>>>(a);
    else
        k_density_batch<FULL_MODELS, K><<<grid, THREADS, 0, stream>>>(a);
}

void launch_particle_pass_batch(const DevParticles &P, const BatchView &b, int n_blocks,
                                const LoadFlagsHost &lf, unsigned model_mask, int mode_g2p,
                                int emit_p2g, int aggregate, int chunks, cudaStream_t stream) {
    if (n_blocks <= 0) return;
    ParticleKernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.P = P;
    a.lf.temperature = lf.temperature;
    a.lf.activation = lf.activation;
    a.lf.pinned = lf.pinned;
    a.mode_g2p = mode_g2p;
    a.project_in = mode_g2p;  // recompute the stored state's projection (where the scene projects)
    a.emit_p2g = emit_p2g;
    a.aggregate = aggregate;
    a.batch = b;
    a.batch.n_chunks = n_blocks;
    if (chunks >= 4) batch_particle_launch<4>(a, model_mask, stream);
    else if (chunks == 2) batch_particle_launch<2>(a, model_mask, stream);
    else batch_particle_launch<1>(a, model_mask, stream);
}

void launch_density_pass_batch(const DevParticles &P, const BatchView &b, int n_blocks,
                               const LoadFlagsHost &lf, unsigned model_mask, int aggregate,
                               int chunks, cudaStream_t stream) {
    if (n_blocks <= 0) return;
    DensityKernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.P = P;
    a.lf.temperature = lf.temperature;
    a.lf.activation = lf.activation;
    a.lf.pinned = lf.pinned;
    a.aggregate = aggregate;
    a.batch = b;
    a.batch.n_chunks = n_blocks;
    if (chunks >= 4) batch_density_launch<4>(a, model_mask, stream);
    else if (chunks == 2) batch_density_launch<2>(a, model_mask, stream);
    else batch_density_launch<1>(a, model_mask, stream);
}

void launch_particle_pass_fast(const ParticleKernelArgs &a, unsigned model_mask, cudaStream_t stream) {
    const int grid = blocks_for(a.n, THREADS);
    const unsigned plastic = (1u << M_DRUCKER_PRAGER) | (1u << M_NACC);
    if (a.cl.defer && a.mode_g2p && (model_mask & plastic) && !(model_mask & EXTRAS)) {
        const unsigned cover = covering_mask(model_mask);
        if (cover == MASK_GRANULAR)
            k_particle_closure_queue<MASK_GRANULAR><<<grid, THREADS, 0, stream>>>(a);
        else if (cover == ALL_MODELS)
            k_particle_closure_queue<ALL_MODELS><<<grid, THREADS, 0, stream>>>(a);
        else
            k_particle_closure_queue<FULL_MODELS><<<grid, THREADS, 0, stream>>>(a);
        return;
    }
    if ((a.cl.infer || a.cl.log) && (model_mask & plastic)) {
        const unsigned cover = (model_mask & EXTRAS) ? FULL_MODELS : covering_mask(model_mask);
        if (cover == MASK_GRANULAR)
            k_particle_closure<MASK_GRANULAR><<<grid, THREADS, 0, stream>>>(a);
        else if (cover == FULL_MODELS)
            k_particle_closure<FULL_MODELS><<<grid, THREADS, 0, stream>>>(a);
        else
            k_particle_closure<ALL_MODELS><<<grid, THREADS, 0, stream>>>(a);
        return;
    }
    switch (covering_mask(model_mask)) {
    case MASK_FLUID: k_particle_fast<MASK_FLUID><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID: k_particle_fast<MASK_SOLID><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID_FLUID: k_particle_fast<MASK_SOLID_FLUID><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_GRANULAR: k_particle_fast<MASK_GRANULAR><<<grid, THREADS, 0, stream>>>(a); break;
    case ALL_MODELS: k_particle_fast<ALL_MODELS><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_FLUID_X: k_particle_fast<MASK_FLUID_X><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID_X: k_particle_fast<MASK_SOLID_X><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID_FLUID_X: k_particle_fast<MASK_SOLID_FLUID_X><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_GRANULAR_X: k_particle_fast<MASK_GRANULAR_X><<<grid, THREADS, 0, stream>>>(a); break;
    case ALL_MODELS_X: k_particle_fast<ALL_MODELS_X><<<grid, THREADS, 0, stream>>>(a); break;
    default: k_particle_fast<FULL_MODELS><<<grid, THREADS, 0, stream>>>(a); break;
    }
}

void launch_density_pass_fast(const DensityKernelArgs &a, unsigned model_mask, cudaStream_t stream) {
    const int grid = blocks_for(a.n, THREADS);
    switch (covering_mask(model_mask)) {
    case MASK_FLUID: k_density<MASK_FLUID><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID: k_density<MASK_SOLID><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID_FLUID: k_density<MASK_SOLID_FLUID><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_GRANULAR: k_density<MASK_GRANULAR><<<grid, THREADS, 0, stream>>>(a); break;
    case ALL_MODELS: k_density<ALL_MODELS><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_FLUID_X: k_density<MASK_FLUID_X><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID_X: k_density<MASK_SOLID_X><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_SOLID_FLUID_X: k_density<MASK_SOLID_FLUID_X><<<grid, THREADS, 0, stream>>>(a); break;
    case MASK_GRANULAR_X: k_density<MASK_GRANULAR_X><<<grid, THREADS, 0, stream>>>(a); break;
    case ALL_MODELS_X: k_density<ALL_MODELS_X><<<grid, THREADS, 0, stream>>>(a); break;
    default: k_density<FULL_MODELS><<<grid, THREADS, 0, stream>>>(a); break;
    }
}

}  // namespace emerge
