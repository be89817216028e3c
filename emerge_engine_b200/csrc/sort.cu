// sort.cu -- stable device LSD radix sort of particle keys.
//
// The reference GPU path sorts particles by a coarse block key with a counting
// sort whose scatter is atomic and therefore unordered within a block
// (systems/gpu/shaders/particle_sort.wgsl:124-245).  Here the sort is a stable
// least-significant-digit radix sort (8-bit digits): per pass a per-CTA digit
// histogram, one exclusive scan over [digit][cta], and a stable scatter that
// ranks equal digits with __match_any_sync inside a warp and running per-digit
// counters across warps and rounds.  Ties keep their input order, so the
// resulting permutation is deterministic: it equals std::stable_sort of the keys.
#include "device_state.cuh"
#include "kernels.h"

namespace emerge {

constexpr int SORT_THREADS = 256;
constexpr int SORT_ROUNDS = 8;
constexpr int SORT_ITEMS = SORT_THREADS * SORT_ROUNDS;  // items per CTA per pass
constexpr int RADIX = 256;
constexpr int SCAN_CHUNK = 1024;

static inline int sort_blocks(int n) { return (n + SORT_ITEMS - 1) / SORT_ITEMS; }

size_t sort_scratch_bytes(size_t n) {
    size_t nb = (n + SORT_ITEMS - 1) / SORT_ITEMS;
    size_t hist = RADIX * (nb > 0 ? nb : 1);
    size_t partials = (hist + SCAN_CHUNK - 1) / SCAN_CHUNK + 1;
    return (4 * n + hist + partials) * sizeof(uint32_t) + 8 * 256;
}

void sort_scratch_bind(SortScratch &s, void *base, size_t n) {
    auto align = [](uintptr_t p) { return (p + 255) & ~static_cast<uintptr_t>(255); };
    uintptr_t p = align(reinterpret_cast<uintptr_t>(base));
    s.capacity = n;
    for (int k = 0; k < 2; ++k) {
        s.keys[k] = reinterpret_cast<uint32_t *>(p);
        p = align(p + n * sizeof(uint32_t));
        s.vals[k] = reinterpret_cast<uint32_t *>(p);
        p = align(p + n * sizeof(uint32_t));
    }
    size_t nb = (n + SORT_ITEMS - 1) / SORT_ITEMS;
    s.hist_capacity = RADIX * (nb > 0 ? nb : 1);
    s.hist = reinterpret_cast<uint32_t *>(p);
    p = align(p + s.hist_capacity * sizeof(uint32_t));
    s.partials = reinterpret_cast<uint32_t *>(p);
}

__device__ __forceinline__ uint32_t morton2(uint32_t x, uint32_t y) {
    uint32_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((x >> b) & 1u) << (2 * b) | ((y >> b) & 1u) << (2 * b + 1);
    return r;
}

// key_mode 0: (Morton(tile_x, tile_y) << 6) | (cell_x & 7) << 3 | (cell_y & 7)
// key_mode 1: block_index (particle_sort.wgsl:94-102), NUM_BLOCKS_PER_DIM = 16
__global__ void k_sort_keys(const float2 *x, int n, int res, int key_mode, uint32_t *keys,
                            uint32_t *vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 p = x[i];
    uint32_t key;
    if (key_mode == 1) {
        const uint32_t NB = 16u;
        uint32_t max_cell = static_cast<uint32_t>(res) - 1u;
        uint32_t cx = static_cast<uint32_t>(fminf(fmaxf(p.x, 0.0f), static_cast<float>(max_cell)));
        uint32_t cy = static_cast<uint32_t>(fminf(fmaxf(p.y, 0.0f), static_cast<float>(max_cell)));
        uint32_t bs = (static_cast<uint32_t>(res) + NB - 1u) / NB;
        uint32_t bx = min(cx / bs, NB - 1u);
        uint32_t by = min(cy / bs, NB - 1u);
        key = by * NB + bx;
    } else {
        float fx = fminf(fmaxf(floorf(p.x), 0.0f), static_cast<float>(res - 1));
        float fy = fminf(fmaxf(floorf(p.y), 0.0f), static_cast<float>(res - 1));
        uint32_t cx = static_cast<uint32_t>(fx), cy = static_cast<uint32_t>(fy);
        key = (morton2(cx >> 3, cy >> 3) << 6) | ((cx & 7u) << 3) | (cy & 7u);
    }
    keys[i] = key;
    vals[i] = static_cast<uint32_t>(i);
}

int sort_key_bits(int res, int key_mode) {
    if (key_mode == 1) return 8;
    int tpd = (res + TILE - 1) / TILE;
    int b = 0;
    while ((1 << b) < tpd) ++b;
    return 2 * b + 6;
}

void launch_sort_keys(const float2 *x, int n, int res, int key_mode, uint32_t *keys, uint32_t *vals,
                      cudaStream_t stream) {
    if (n > 0) k_sort_keys<<<(n + 255) / 256, 256, 0, stream>>>(x, n, res, key_mode, keys, vals);
}

__global__ void __launch_bounds__(SORT_THREADS) k_hist(const uint32_t *keys, int n, int shift,
                                                       uint32_t *hist, int nblocks) {
    __shared__ uint32_t h[RADIX];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * SORT_ITEMS;
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        int i = base + r * SORT_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Sum of each SCAN_CHUNK slice.
__global__ void __launch_bounds__(256) k_chunk_sums(const uint32_t *a, int len, uint32_t *partials) {
    __shared__ uint32_t sh[8];
    uint32_t s = 0;
    int base = blockIdx.x * SCAN_CHUNK;
    for (int k = threadIdx.x; k < SCAN_CHUNK; k += 256) {
        int i = base + k;
        if (i < len) s += a[i];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        partials[blockIdx.x] = t;
    }
}

// Block-wide exclusive scan of 1024 values (4 per thread); returns the total.
__device__ uint32_t block_exclusive_scan_1024(uint32_t (&v)[4], uint32_t *sh_warp) {
    uint32_t t0 = v[0], t1 = t0 + v[1], t2 = t1 + v[2], t3 = t2 + v[3];
    uint32_t incl = t3;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sh_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < 8; ++w) {
            uint32_t c = sh_warp[w];
            sh_warp[w] = run;
            run += c;
        }
        sh_warp[8] = run;
    }
    __syncthreads();
    uint32_t excl_thread = incl - t3 + sh_warp[warp];
    v[0] = excl_thread;
    v[1] = excl_thread + t0;
    v[2] = excl_thread + t1;
    v[3] = excl_thread + t2;
    uint32_t total = sh_warp[8];
    __syncthreads();
    return total;
}

// Exclusive scan of the partials, one CTA, in slices of 1024 with a carry.
__global__ void __launch_bounds__(256) k_scan_partials(uint32_t *partials, int len) {
    __shared__ uint32_t sh[9];
    uint32_t carry = 0;
    for (int base = 0; base < len; base += SCAN_CHUNK) {
        uint32_t v[4];
        for (int k = 0; k < 4; ++k) {
            int i = base + threadIdx.x * 4 + k;
            v[k] = i < len ? partials[i] : 0u;
        }
        uint32_t total = block_exclusive_scan_1024(v, sh);
        for (int k = 0; k < 4; ++k) {
            int i = base + threadIdx.x * 4 + k;
            if (i < len) partials[i] = v[k] + carry;
        }
        carry += total;
    }
}

// Exclusive scan of each slice, offset by its scanned partial.
__global__ void __launch_bounds__(256) k_chunk_scan(uint32_t *a, int len, const uint32_t *partials) {
    __shared__ uint32_t sh[9];
    int base = blockIdx.x * SCAN_CHUNK;
    uint32_t v[4];
    for (int k = 0; k < 4; ++k) {
        int i = base + threadIdx.x * 4 + k;
        v[k] = i < len ? a[i] : 0u;
    }
    block_exclusive_scan_1024(v, sh);
    uint32_t off = partials[blockIdx.x];
    for (int k = 0; k < 4; ++k) {
        int i = base + threadIdx.x * 4 + k;
        if (i < len) a[i] = v[k] + off;
    }
}

__global__ void __launch_bounds__(SORT_THREADS) k_scatter(const uint32_t *kin, const uint32_t *vin,
                                                          uint32_t *kout, uint32_t *vout, int n,
                                                          int shift, const uint32_t *offsets,
                                                          int nblocks) {
    __shared__ uint32_t s_off[RADIX];
    __shared__ uint32_t s_run[RADIX];
    __shared__ uint32_t s_round[RADIX];
    __shared__ uint32_t s_wc[SORT_THREADS / 32][RADIX];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    s_off[tid] = offsets[tid * nblocks + blockIdx.x];
    s_run[tid] = 0;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int base = blockIdx.x * SORT_ITEMS;
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        for (int w = 0; w < SORT_THREADS / 32; ++w) s_wc[w][tid] = 0;
        __syncthreads();
        const int i = base + r * SORT_THREADS + tid;
        const bool valid = i < n;
        uint32_t key = 0, val = 0, d = RADIX;  // RADIX = sentinel for padding lanes
        if (valid) {
            key = kin[i];
            val = vin[i];
            d = (key >> shift) & 255u;
        }
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned rank_w = __popc(peers & lt_mask);
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) s_wc[warp][d] = __popc(peers);
        __syncthreads();
        {
            uint32_t run = 0;
            for (int w = 0; w < SORT_THREADS / 32; ++w) {
                uint32_t c = s_wc[w][tid];
                s_wc[w][tid] = run;
                run += c;
            }
            s_round[tid] = s_run[tid];
            s_run[tid] += run;
        }
        __syncthreads();
        if (valid) {
            uint32_t pos = s_off[d] + s_round[d] + s_wc[warp][d] + rank_w;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
    }
}

int radix_sort_pairs(SortScratch &s, int n, int key_bits, cudaStream_t stream) {
    if (n <= 1) return 0;
    const int nb = sort_blocks(n);
    const int hist_len = RADIX * nb;
    const int nchunks = (hist_len + SCAN_CHUNK - 1) / SCAN_CHUNK;
    int cur = 0;
    for (int shift = 0; shift < key_bits; shift += 8) {
        k_hist<<<nb, SORT_THREADS, 0, stream>>>(s.keys[cur], n, shift, s.hist, nb);
        k_chunk_sums<<<nchunks, 256, 0, stream>>>(s.hist, hist_len, s.partials);
        k_scan_partials<<<1, 256, 0, stream>>>(s.partials, nchunks);
        k_chunk_scan<<<nchunks, 256, 0, stream>>>(s.hist, hist_len, s.partials);
        k_scatter<<<nb, SORT_THREADS, 0, stream>>>(s.keys[cur], s.vals[cur], s.keys[cur ^ 1],
                                                   s.vals[cur ^ 1], n, shift, s.hist, nb);
        cur ^= 1;
    }
    return cur;
}

// dst slot j <- src slot i, every particle array.
__device__ __forceinline__ void copy_slot(const DevParticles &src, uint32_t i, const DevParticles &dst, int j) {
    dst.x[j] = src.x[i];
    dst.v[j] = src.v[i];
    dst.c[j] = src.c[i];
    dst.f[j] = src.f[i];
    dst.mass[j] = src.mass[i];
    dst.v0[j] = src.v0[i];
    dst.vol[j] = src.vol[i];
    dst.rho[j] = src.rho[i];
    dst.mat[j] = src.mat[i];
    dst.jp[j] = src.jp[i];
    dst.h[j] = src.h[i];
    dst.q[j] = src.q[i];
    dst.lvs[j] = src.lvs[i];
    dst.temperature[j] = src.temperature[i];
    dst.activation[j] = src.activation[i];
    dst.act_dir[j] = src.act_dir[i];
    dst.pinned[j] = src.pinned[i];
    dst.user_tag[j] = src.user_tag[i];
    dst.muscle[j] = src.muscle[i];
    dst.contact[j] = src.contact[i];
    dst.sleeping[j] = src.sleeping[i];
    dst.scalar[j] = src.scalar[i];
    dst.slot_to_index[j] = src.slot_to_index[i];
    dst.rho_dp[j] = src.rho_dp[i];
}

__global__ void k_permute(DevParticles src, DevParticles dst, const uint32_t *perm, int n) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    copy_slot(src, perm[j], dst, j);
}

// ---- batched scenes: one sort over all scenes, scene index in the key's high bits ----
constexpr int BATCH_TILE_KEY_BITS = 20;  // grids up to 1024^2 (128^2 tiles)

// Scene of compact particle index c: compact_start[s] <= c < compact_start[s + 1].
__device__ __forceinline__ int scene_of(const int *compact_start, int n_scenes, int c) {
    int lo = 0, hi = n_scenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (compact_start[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_batch_sort_keys(const SceneDesc *scenes, const int *compact_start, int n_scenes,
                                  DevParticles P, int total, uint32_t *keys, uint32_t *vals, int shape) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= total) return;
    const int s = scene_of(compact_start, n_scenes, c);
    const SceneDesc &sd = scenes[s];
    const int slot = sd.p0 + (c - compact_start[s]);
    const float2 p = P.x[slot];
    const int res = sd.g.res;
    const float fx = fminf(fmaxf(floorf(p.x), 0.0f), static_cast<float>(res - 1));
    const float fy = fminf(fmaxf(floorf(p.y), 0.0f), static_cast<float>(res - 1));
    const uint32_t cx = static_cast<uint32_t>(fx), cy = static_cast<uint32_t>(fy);
    uint32_t k;  // spatial key below 2^20 for grids up to 1024^2
    if (shape == 1)
        k = (morton2(cx >> 3, cy >> 3) << 6) | morton2(cx & 7u, cy & 7u);
    else if (shape == 2)  // 16 x 16 blocks, four 16 x 4 strips each
        k = (morton2(cx >> 4, cy >> 4) << 8) | (((cy >> 2) & 3u) << 6) | ((cx & 15u) << 2) | (cy & 3u);
    else if (shape == 3)  // 16 x 16 blocks, four 4 x 16 strips each
        k = (morton2(cx >> 4, cy >> 4) << 8) | (((cx >> 2) & 3u) << 6) | ((cy & 15u) << 2) | (cx & 3u);
    else
        k = (morton2(cx >> 3, cy >> 3) << 6) | ((cx & 7u) << 3) | (cy & 7u);
    keys[c] = (static_cast<uint32_t>(s) << BATCH_TILE_KEY_BITS) | k;
    vals[c] = static_cast<uint32_t>(slot);
}

__global__ void k_permute_batch(DevParticles src, DevParticles dst, const uint32_t *keys,
                                const uint32_t *vals, const SceneDesc *scenes, const int *compact_start,
                                int total) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= total) return;
    const int s = static_cast<int>(keys[j] >> BATCH_TILE_KEY_BITS);
    copy_slot(src, vals[j], dst, scenes[s].p0 + (j - compact_start[s]));
}

int batch_sort_key_bits(int n_scenes) {
    int b = 0;
    while ((1 << b) < n_scenes) ++b;
    return BATCH_TILE_KEY_BITS + b;
}

void launch_batch_sort_keys(const SceneDesc *scenes, const int *compact_start, int n_scenes,
                            const DevParticles &P, int total, uint32_t *keys, uint32_t *vals, int shape,
                            cudaStream_t stream) {
    if (total > 0)
        k_batch_sort_keys<<<(total + 255) / 256, 256, 0, stream>>>(scenes, compact_start, n_scenes, P, total,
                                                                  keys, vals, shape);
}

void launch_permute_batch(const DevParticles &src, const DevParticles &dst, const uint32_t *keys,
                          const uint32_t *vals, const SceneDesc *scenes, const int *compact_start, int total,
                          cudaStream_t stream) {
    if (total > 0)
        k_permute_batch<<<(total + 255) / 256, 256, 0, stream>>>(src, dst, keys, vals, scenes, compact_start,
                                                                total);
}

void launch_permute(const DevParticles &src, const DevParticles &dst, const uint32_t *perm, int n,
                    cudaStream_t stream) {
    if (n > 0) k_permute<<<(n + 255) / 256, 256, 0, stream>>>(src, dst, perm, n);
}

}  // namespace emerge
