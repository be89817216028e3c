// batch.cu -- many independent scenes advanced together (no counterpart in the reference).
//
// A batch packs the scenes of several simulations into one particle store, one pool of
// grids and one table of scene descriptors.  Every substep is one launch per kernel for
// all scenes: the particle and density passes find their scene from a CTA -> scene table,
// the grid update from a tile -> scene table, and a one-CTA controller runs each scene's
// own CFL substep schedule (a scene whose frame has ended sits out the remaining substeps
// of the batch's frame).  The frame is a CUDA graph with a conditional while node, as for
// one scene.  Scenes keep their own grid size, materials, boundaries and configuration;
// results equal the single-scene step up to float summation order.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "closure_host.h"
#include "kernels.h"

using namespace emerge;

namespace {

thread_local std::string g_batch_error;

struct Buf {
    void *p = nullptr;
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) {
        if (p) cudaFree(p);
        p = nullptr;
        return cudaMalloc(&p, bytes);
    }
};

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// The particle arrays of one scene: every pointer advanced to the scene's first slot.
DevParticles offset_particles(const DevParticles &P, size_t off) {
    DevParticles Q = P;
    Q.x += off; Q.v += off; Q.c += off; Q.f += off;
    Q.mass += off; Q.v0 += off; Q.vol += off; Q.rho += off; Q.mat += off;
    Q.jp += off; Q.h += off; Q.q += off; Q.lvs += off;
    Q.temperature += off; Q.activation += off; Q.act_dir += off; Q.pinned += off;
    Q.user_tag += off; Q.muscle += off; Q.contact += off; Q.sleeping += off; Q.scalar += off;
    Q.slot_to_index += off; Q.rho_dp += off;
    return Q;
}

struct SceneHost {
    int res, tpd, p0, n, block0, tile0, n_tiles, n_mats, density_mode;
};

}  // namespace

struct emerge_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string error;
    std::vector<SceneHost> scenes;
    int n_blocks = 0, n_tiles = 0, total = 0;
    size_t slots = 0;
    LoadFlagsHost lf;
    unsigned model_mask = 1u << M_FALLBACK;
    int any_density = 0;
    Buf pbuf, gbuf, tables, sortbuf, region, staging, states, flush;
    DevParticles P[2];
    int cur = 0;
    SceneDesc *d_desc = nullptr;
    uint16_t *d_block_scene = nullptr, *d_tile_scene = nullptr;
    int *d_compact_start = nullptr;
    StepState *d_states = nullptr;  // [scenes + 1]: the last one is the batch's own state
    StepState *h_batch = nullptr;   // pinned mirror of the batch state
    SortScratch sort;
    emerge_material_params *d_mats = nullptr;
    bool pending_valid = false, sorted_once = false;
    int use_graph = 1, aggregate = 0;
    int tile_shape = 0;   // particle order of the sort (launch_batch_sort_keys)
    int chunks = 1;       // 256-particle chunks per CTA of the particle and density passes
    int64_t sort_interval = 8;
    uint64_t steps_since_sort = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_dirty = true;
    cudaEvent_t ev[2] = {nullptr, nullptr};

    int fail(emerge_status st, const std::string &m) {
        error = m;
        return st;
    }
    BatchView view(int check_active) const {
        BatchView b;
        b.scenes = d_desc;
        b.block_scene = d_block_scene;
        b.tile_scene = d_tile_scene;
        b.n_scenes = static_cast<int>(scenes.size());
        b.check_active = check_active;
        return b;
    }
    StepState *batch_state() const { return d_states + scenes.size(); }
};

namespace {

#define BK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return static_cast<emerge_status>(b->fail(                                        \
                e_ == cudaErrorMemoryAllocation ? EMERGE_ERR_OOM : EMERGE_ERR_CUDA,           \
                std::string(#call) + ": " + cudaGetErrorString(e_)));                         \
    } while (0)

void destroy_graph(emerge_batch *b) {
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

// Stable sort of every scene's particles by (scene, tile key); each scene stays in its
// own slot range.  Changes no result beyond float summation order.
emerge_status sort_batch(emerge_batch *b) {
    b->sorted_once = true;
    b->steps_since_sort = 0;
    if (b->total < 2) return EMERGE_OK;
    const int S = static_cast<int>(b->scenes.size());
    launch_batch_sort_keys(b->d_desc, b->d_compact_start, S, b->P[b->cur], b->total, b->sort.keys[0],
                           b->sort.vals[0], b->tile_shape, b->stream);
    const int r = radix_sort_pairs(b->sort, b->total, batch_sort_key_bits(S), b->stream);
    launch_permute_batch(b->P[b->cur], b->P[b->cur ^ 1], b->sort.keys[r], b->sort.vals[r], b->d_desc,
                         b->d_compact_start, b->total, b->stream);
    b->cur ^= 1;
    b->graph_dirty = true;  // the graph's kernels hold the particle arrays
    BK(cudaGetLastError());
    return EMERGE_OK;
}

bool sort_due(const emerge_batch *b) {
    return !b->sorted_once ||
           (b->sort_interval > 0 && b->steps_since_sort >= static_cast<uint64_t>(b->sort_interval));
}

// The first substep's P2G (and density pass) of every scene, from the stored state.
emerge_status prime(emerge_batch *b) {
    const BatchView all = b->view(0);
    launch_prime_setup_batch(all, b->stream);
    launch_particle_pass_batch(b->P[b->cur], all, b->n_blocks, b->lf, b->model_mask, 0, 1,
                               b->aggregate, b->chunks, b->stream);
    if (b->any_density)
        launch_density_pass_batch(b->P[b->cur], all, b->n_blocks, b->lf, b->model_mask,
                                  b->aggregate, b->chunks, b->stream);
    BK(cudaGetLastError());
    b->pending_valid = true;
    return EMERGE_OK;
}

void enqueue_substep(emerge_batch *b, int use_cond, unsigned long long handle) {
    const BatchView live = b->view(1);
    launch_substep_begin_batch(live, b->batch_state(), use_cond, handle, 3 + b->any_density, b->stream);
    launch_grid_update_batch(live, b->n_tiles, b->stream);
    launch_particle_pass_batch(b->P[b->cur], live, b->n_blocks, b->lf, b->model_mask, 1, 1,
                               b->aggregate, b->chunks, b->stream);
    if (b->any_density)
        launch_density_pass_batch(b->P[b->cur], live, b->n_blocks, b->lf, b->model_mask,
                                  b->aggregate, b->chunks, b->stream);
}

emerge_status build_graph(emerge_batch *b) {
    destroy_graph(b);
    cudaGraph_t graph;
    BK(cudaGraphCreate(&graph, 0));
    b->graph = graph;
    BK(cudaStreamBeginCaptureToGraph(b->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_step_begin_batch(b->view(0), b->batch_state(), b->stream);
    BK(cudaStreamEndCapture(b->stream, &graph));
    size_t nn = 0;
    BK(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    BK(cudaGraphGetNodes(graph, nodes.data(), &nn));
    cudaGraphConditionalHandle handle;
    BK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    BK(cudaGraphAddNode(&wnode, graph, nodes.data(), nn, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BK(cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_substep(b, 1, static_cast<unsigned long long>(handle));
    BK(cudaStreamEndCapture(b->stream, &body));
    BK(cudaGraphInstantiate(&b->graph_exec, graph, 0));
    b->graph_dirty = false;
    return EMERGE_OK;
}

// One frame of every scene (asynchronous); sorting is due-checked by the caller.
emerge_status frame(emerge_batch *b) {
    if (!b->pending_valid) {
        emerge_status st = prime(b);
        if (st != EMERGE_OK) return st;
    }
    if (b->use_graph) {
        if (b->graph_dirty || !b->graph_exec) {
            emerge_status st = build_graph(b);
            if (st != EMERGE_OK) return st;
        }
        BK(cudaGraphLaunch(b->graph_exec, b->stream));
    } else {  // host-driven loop (the same kernels; profilers see them)
        launch_step_begin_batch(b->view(0), b->batch_state(), b->stream);
        for (;;) {
            enqueue_substep(b, 0, 0ull);
            BK(cudaMemcpyAsync(b->h_batch, b->batch_state(), sizeof(StepState), cudaMemcpyDeviceToHost, b->stream));
            BK(cudaStreamSynchronize(b->stream));
            if (!b->h_batch->cont) break;
        }
    }
    b->steps_since_sort += 1;
    BK(cudaGetLastError());
    return EMERGE_OK;
}

emerge_status read_states(emerge_batch *b, std::vector<StepState> &out) {
    out.resize(b->scenes.size() + 1);
    BK(cudaMemcpyAsync(out.data(), b->d_states, out.size() * sizeof(StepState), cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return EMERGE_OK;
}

}  // namespace

namespace {

// One autotuned setting of a batch (and its frame time in GPU ms, 0 when loaded).
struct TuneChoice {
    int sort_interval, aggregate, tile_shape, chunks;
    float ms;
};

// Cache key: device name and SM count, then each scene's grid size, particle count and model
// mask, folded into a 64-bit FNV-1a hash (with the scene count in clear text).
std::string tune_signature(const emerge_batch *b) {
    cudaDeviceProp prop{};
    std::string dev = "unknown";
    if (cudaGetDeviceProperties(&prop, b->device) == cudaSuccess)
        dev = std::string(prop.name) + "/" + std::to_string(prop.multiProcessorCount);
    for (char &ch : dev)
        if (ch == ' ') ch = '_';
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int k = 0; k < 8; ++k) {
            h ^= (v >> (8 * k)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    for (const SceneHost &sc : b->scenes) {
        mix(static_cast<uint64_t>(sc.res));
        mix(static_cast<uint64_t>(sc.n));
        mix(static_cast<uint64_t>(sc.density_mode));
    }
    mix(b->model_mask);
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%016llx", static_cast<unsigned long long>(h));
    return dev + ":" + std::to_string(b->scenes.size()) + ":" + buf;
}

// The cache is a text file of lines "key sort_interval aggregate tile_shape chunks ms".
bool cache_lookup(const char *path, const std::string &key, TuneChoice &out) {
    std::FILE *f = std::fopen(path, "r");
    if (!f) return false;
    char k[256];
    TuneChoice c{};
    bool found = false;
    while (std::fscanf(f, "%255s %d %d %d %d %f", k, &c.sort_interval, &c.aggregate, &c.tile_shape, &c.chunks,
                       &c.ms) == 6) {
        if (key == k && c.sort_interval >= 0 && (c.aggregate == 0 || c.aggregate == 1) && c.tile_shape >= 0 &&
            c.tile_shape <= 3 && (c.chunks == 1 || c.chunks == 2 || c.chunks == 4)) {
            out = c;
            found = true;  // the last matching line wins
        }
    }
    std::fclose(f);
    return found;
}

void cache_store(const char *path, const std::string &key, const TuneChoice &c) {
    std::vector<std::string> keep;
    if (std::FILE *f = std::fopen(path, "r")) {
        char line[512];
        while (std::fgets(line, sizeof(line), f)) {
            std::string l(line);
            if (l.compare(0, key.size() + 1, key + " ") != 0) keep.push_back(l);
        }
        std::fclose(f);
    }
    std::FILE *f = std::fopen(path, "w");
    if (!f) return;  // a cache that cannot be written only costs the next batch its trials
    for (const std::string &l : keep) std::fputs(l.c_str(), f);
    std::fprintf(f, "%s %d %d %d %d %.6f\n", key.c_str(), c.sort_interval, c.aggregate, c.tile_shape, c.chunks, c.ms);
    std::fclose(f);
}

}  // namespace

extern "C" {

const char *emerge_cuda_batch_last_error(const emerge_batch *b) {
    return b ? b->error.c_str() : g_batch_error.c_str();
}

emerge_status emerge_cuda_batch_create(emerge_sim *const *sims, uint32_t n_sims, emerge_batch **out) {
    if (!sims || !out || n_sims == 0 || n_sims > 4096) {
        g_batch_error = "batch_create: 1..4096 simulations";
        return EMERGE_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::vector<SimView> views;
    views.reserve(n_sims);
    for (uint32_t k = 0; k < n_sims; ++k) {
        if (!sims[k]) {
            g_batch_error = "batch_create: null simulation";
            return EMERGE_ERR_INVALID_ARG;
        }
        views.push_back(sim_view(sims[k]));
        const SimView &v = views.back();
        if (v.deterministic) {
            g_batch_error = "batch_create: scenes run the fast path (the reference-order mode is per simulation)";
            return EMERGE_ERR_UNSUPPORTED;
        }
        if (v.dcfg.n_fields > 0 || v.dcfg.asflip > 0.0f || v.cfg.sleep_threshold > 0.0f || v.dcfg.zones ||
            v.dcfg.multi) {
            g_batch_error = "batch_create: scenes with force fields, ASFLIP, a sleep partition or multi-field "
                            "contact / mixture run as single simulations";
            return EMERGE_ERR_UNSUPPORTED;
        }
        if (v.cfg.grid_res > 1024) {
            g_batch_error = "batch_create: grid_res above 1024";
            return EMERGE_ERR_UNSUPPORTED;
        }
        if (v.device != views[0].device) {
            g_batch_error = "batch_create: simulations on different devices";
            return EMERGE_ERR_INVALID_ARG;
        }
    }
    emerge_batch *b = new emerge_batch();
    auto bail = [&](emerge_status st, const char *msg) {
        g_batch_error = std::string("batch_create: ") + msg;
        emerge_cuda_batch_destroy(b);
        return st;
    };
    b->device = views[0].device;
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(EMERGE_ERR_CUDA, "stream");
    // layout: slot ranges, CTA and tile ranges, grid pool offsets
    size_t grid_bytes = 0, n_mats = 0, max_n = 0;
    std::vector<size_t> grid_off(n_sims);
    for (uint32_t k = 0; k < n_sims; ++k) {
        const SimView &v = views[k];
        SceneHost h;
        h.res = static_cast<int>(v.cfg.grid_res);
        h.tpd = (h.res + TILE - 1) / TILE;
        h.n = static_cast<int>(v.n);
        h.p0 = static_cast<int>(b->slots);
        h.block0 = b->n_blocks;
        h.tile0 = b->n_tiles;
        h.n_tiles = h.tpd * h.tpd;
        h.n_mats = static_cast<int>(v.mats.size());
        int dens = v.cfg.recompute_density_each_step ? 1 : 0;
        for (const auto &m : v.mats) {
            if (m.model == M_FLUID) dens = 1;  // needs_density_recompute (fluid.rs:261-263)
            b->model_mask |= model_bits(m);
        }
        h.density_mode = dens;
        b->any_density |= dens;
        b->lf.temperature |= v.lf.temperature;
        b->lf.activation |= v.lf.activation;
        b->lf.pinned |= v.lf.pinned;
        const int blocks = (h.n + PARTICLE_THREADS - 1) / PARTICLE_THREADS;
        b->slots += static_cast<size_t>(blocks) * PARTICLE_THREADS;
        b->n_blocks += blocks;
        b->n_tiles += h.n_tiles;
        b->total += h.n;
        grid_off[k] = grid_bytes;
        const size_t cells = static_cast<size_t>(h.n_tiles) * TILE_CELLS;
        grid_bytes += align256(cells * sizeof(float4)) + 2 * align256(cells * sizeof(float2)) + align256(h.n_tiles);
        n_mats += v.mats.size();
        max_n = std::max<size_t>(max_n, v.n);
        b->scenes.push_back(h);
    }
    if (b->n_blocks > 65535 || b->n_tiles > 65535 * 4)
        return bail(EMERGE_ERR_UNSUPPORTED, "batch too large for the 16-bit scene tables");
    // device memory
    const size_t cap = std::max<size_t>(b->slots, PARTICLE_THREADS);
    const size_t set_bytes = particle_set_size(cap);
    if (b->pbuf.alloc(2 * set_bytes) != cudaSuccess) return bail(EMERGE_ERR_OOM, "particles");
    b->P[0] = particle_set_carve(b->pbuf.p, cap);
    b->P[1] = particle_set_carve(static_cast<char *>(b->pbuf.p) + set_bytes, cap);
    if (b->gbuf.alloc(std::max<size_t>(grid_bytes, 256)) != cudaSuccess) return bail(EMERGE_ERR_OOM, "grids");
    if (cudaMemsetAsync(b->gbuf.p, 0, grid_bytes, b->stream) != cudaSuccess) return bail(EMERGE_ERR_CUDA, "grids");
    const size_t desc_bytes = align256(n_sims * sizeof(SceneDesc));
    const size_t mats_bytes = align256(std::max<size_t>(n_mats, 1) * sizeof(emerge_material_params));
    const size_t bs_bytes = align256(std::max(b->n_blocks, 1) * sizeof(uint16_t));
    const size_t ts_bytes = align256(std::max(b->n_tiles, 1) * sizeof(uint16_t));
    const size_t cs_bytes = align256((n_sims + 1) * sizeof(int));
    if (b->tables.alloc(desc_bytes + mats_bytes + bs_bytes + ts_bytes + cs_bytes) != cudaSuccess)
        return bail(EMERGE_ERR_OOM, "tables");
    char *tp = static_cast<char *>(b->tables.p);
    b->d_desc = reinterpret_cast<SceneDesc *>(tp);
    b->d_mats = reinterpret_cast<emerge_material_params *>(tp + desc_bytes);
    b->d_block_scene = reinterpret_cast<uint16_t *>(tp + desc_bytes + mats_bytes);
    b->d_tile_scene = reinterpret_cast<uint16_t *>(tp + desc_bytes + mats_bytes + bs_bytes);
    b->d_compact_start = reinterpret_cast<int *>(tp + desc_bytes + mats_bytes + bs_bytes + ts_bytes);
    if (b->states.alloc((n_sims + 1) * sizeof(StepState)) != cudaSuccess) return bail(EMERGE_ERR_OOM, "states");
    b->d_states = static_cast<StepState *>(b->states.p);
    if (cudaMallocHost(&b->h_batch, sizeof(StepState)) != cudaSuccess) return bail(EMERGE_ERR_OOM, "pinned state");
    const int sort_n = std::max(b->total, 2);
    if (b->sortbuf.alloc(sort_scratch_bytes(sort_n)) != cudaSuccess) return bail(EMERGE_ERR_OOM, "sort");
    sort_scratch_bind(b->sort, b->sortbuf.p, sort_n);
    if (b->region.alloc(region_acc_bytes()) != cudaSuccess) return bail(EMERGE_ERR_OOM, "region");
    if (b->staging.alloc(std::max<size_t>(max_n, 1) * sizeof(emerge_particle)) != cudaSuccess)
        return bail(EMERGE_ERR_OOM, "staging");
    // scene table, controller states, materials, lookup tables
    std::vector<StepState> states(n_sims + 1);
    std::memset(states.data(), 0, states.size() * sizeof(StepState));
    std::vector<emerge_material_params> mats;
    std::vector<uint16_t> block_scene(std::max(b->n_blocks, 1)), tile_scene(std::max(b->n_tiles, 1));
    std::vector<int> compact(n_sims + 1, 0);
    std::vector<SceneDesc> desc(n_sims);
    char *gp = static_cast<char *>(b->gbuf.p);
    for (uint32_t k = 0; k < n_sims; ++k) {
        const SimView &v = views[k];
        const SceneHost &h = b->scenes[k];
        StepState &st = states[k];
        st.last_step_dt = v.cfg.dt;
        st.min_mdt_bits[0] = st.min_mdt_bits[1] = 0x7f800000u;
        SceneDesc &d = desc[k];
        std::memset(&d, 0, sizeof(d));
        d.cfg = v.dcfg;
        const size_t cells = static_cast<size_t>(h.n_tiles) * TILE_CELLS;
        char *g0 = gp + grid_off[k];
        d.g.res = h.res;
        d.g.tpd = h.tpd;
        d.g.acc_a = reinterpret_cast<float4 *>(g0);
        d.g.acc_s = reinterpret_cast<float2 *>(g0 + align256(cells * sizeof(float4)));
        d.g.grid_v = reinterpret_cast<float2 *>(g0 + align256(cells * sizeof(float4)) + align256(cells * sizeof(float2)));
        d.g.tile_flag = reinterpret_cast<uint8_t *>(g0 + align256(cells * sizeof(float4)) +
                                                    2 * align256(cells * sizeof(float2)));
        d.st = b->d_states + k;
        d.mats = b->d_mats + mats.size();
        d.n_mats = h.n_mats;
        d.p0 = h.p0;
        d.n = h.n;
        d.block0 = h.block0;
        d.tile0 = h.tile0;
        d.density_mode = h.density_mode;
        mats.insert(mats.end(), v.mats.begin(), v.mats.end());
        const int blocks = (h.n + PARTICLE_THREADS - 1) / PARTICLE_THREADS;
        for (int i = 0; i < blocks; ++i) block_scene[h.block0 + i] = static_cast<uint16_t>(k);
        for (int t = 0; t < h.n_tiles; ++t) tile_scene[h.tile0 + t] = static_cast<uint16_t>(k);
        compact[k + 1] = compact[k] + h.n;
    }
    if (cudaMemcpyAsync(b->d_desc, desc.data(), n_sims * sizeof(SceneDesc), cudaMemcpyHostToDevice, b->stream) ||
        (!mats.empty() && cudaMemcpyAsync(b->d_mats, mats.data(), mats.size() * sizeof(emerge_material_params),
                                          cudaMemcpyHostToDevice, b->stream)) ||
        cudaMemcpyAsync(b->d_block_scene, block_scene.data(), block_scene.size() * sizeof(uint16_t),
                        cudaMemcpyHostToDevice, b->stream) ||
        cudaMemcpyAsync(b->d_tile_scene, tile_scene.data(), tile_scene.size() * sizeof(uint16_t),
                        cudaMemcpyHostToDevice, b->stream) ||
        cudaMemcpyAsync(b->d_compact_start, compact.data(), compact.size() * sizeof(int), cudaMemcpyHostToDevice,
                        b->stream) ||
        cudaMemcpyAsync(b->d_states, states.data(), states.size() * sizeof(StepState), cudaMemcpyHostToDevice,
                        b->stream))
        return bail(EMERGE_ERR_CUDA, "tables upload");
    // particles: each simulation's particles (reference order) into its slot range
    std::vector<emerge_particle> host;
    for (uint32_t k = 0; k < n_sims; ++k) {
        const SceneHost &h = b->scenes[k];
        if (h.n == 0) continue;
        host.resize(h.n);
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(EMERGE_ERR_CUDA, "sync");
        if (emerge_cuda_read_particles(sims[k], host.data(), h.n) != EMERGE_OK)
            return bail(EMERGE_ERR_CUDA, "read scene particles");
        if (cudaMemcpyAsync(b->staging.p, host.data(), h.n * sizeof(emerge_particle), cudaMemcpyHostToDevice,
                            b->stream) != cudaSuccess)
            return bail(EMERGE_ERR_CUDA, "upload");
        launch_append_aos(offset_particles(b->P[b->cur], h.p0), 0, h.n,
                          static_cast<const emerge_particle *>(b->staging.p), b->stream);
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess ||
        cudaEventCreate(&b->ev[0]) != cudaSuccess || cudaEventCreate(&b->ev[1]) != cudaSuccess)
        return bail(EMERGE_ERR_CUDA, "initialise");
    *out = b;
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_destroy(emerge_batch *b) {
    if (!b) return EMERGE_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    destroy_graph(b);
    for (cudaEvent_t &e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->h_batch) cudaFreeHost(b->h_batch);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_step(emerge_batch *b, uint32_t n_steps) {
    if (!b) return EMERGE_ERR_INVALID_ARG;
    for (uint32_t k = 0; k < n_steps; ++k) {
        if (sort_due(b)) {
            emerge_status st = sort_batch(b);
            if (st != EMERGE_OK) return st;
        }
        emerge_status st = frame(b);
        if (st != EMERGE_OK) return st;
    }
    BK(cudaStreamSynchronize(b->stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_time_steps(emerge_batch *b, uint32_t n_steps, int flush_l2, float *ms_total) {
    if (!b || !ms_total) return EMERGE_ERR_INVALID_ARG;
    *ms_total = 0.0f;
    const size_t flush_bytes = size_t(512) << 20;
    if (flush_l2 && !b->flush.p && b->flush.alloc(flush_bytes) != cudaSuccess)
        return static_cast<emerge_status>(b->fail(EMERGE_ERR_OOM, "flush buffer"));
    for (uint32_t k = 0; k < n_steps; ++k) {
        if (sort_due(b)) {  // before the timed region, as a single scene's bench does
            emerge_status st = sort_batch(b);
            if (st != EMERGE_OK) return st;
        }
        if (flush_l2) BK(cudaMemsetAsync(b->flush.p, static_cast<int>(k & 0xff), flush_bytes, b->stream));
        BK(cudaEventRecord(b->ev[0], b->stream));
        emerge_status st = frame(b);
        if (st != EMERGE_OK) return st;
        BK(cudaEventRecord(b->ev[1], b->stream));
        BK(cudaEventSynchronize(b->ev[1]));
        float ms = 0.0f;
        BK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
        *ms_total += ms;
    }
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_scene_count(const emerge_batch *b, uint32_t *n) {
    if (!b || !n) return EMERGE_ERR_INVALID_ARG;
    *n = static_cast<uint32_t>(b->scenes.size());
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_particle_count(const emerge_batch *b, uint32_t scene, uint64_t *n) {
    if (!b || !n || scene >= b->scenes.size()) return EMERGE_ERR_INVALID_ARG;
    *n = static_cast<uint64_t>(b->scenes[scene].n);
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_read_particles(emerge_batch *b, uint32_t scene, emerge_particle *out, uint64_t n) {
    if (!b || scene >= b->scenes.size() || (!out && n)) return EMERGE_ERR_INVALID_ARG;
    const SceneHost &h = b->scenes[scene];
    if (n != static_cast<uint64_t>(h.n))
        return static_cast<emerge_status>(b->fail(EMERGE_ERR_INVALID_ARG, "n must equal the scene's particle count"));
    if (n == 0) return EMERGE_OK;
    launch_gather_aos(offset_particles(b->P[b->cur], h.p0), h.n, static_cast<emerge_particle *>(b->staging.p),
                      b->stream);
    BK(cudaMemcpyAsync(out, b->staging.p, n * sizeof(emerge_particle), cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_region_state(emerge_batch *b, uint32_t scene, float cx, float cy, float radius,
                                             emerge_body_state *out) {
    if (!b || !out || scene >= b->scenes.size()) return EMERGE_ERR_INVALID_ARG;
    const SceneHost &h = b->scenes[scene];
    std::vector<unsigned char> acc(region_acc_bytes(), 0);
    BK(cudaMemsetAsync(b->region.p, 0, region_acc_bytes(), b->stream));
    const uint32_t zero_ordered = 0x80000000u;  // max_jp starts at the ordered encoding of 0.0f
    BK(cudaMemcpyAsync(static_cast<char *>(b->region.p) + region_acc_bytes() - 8, &zero_ordered, 4,
                       cudaMemcpyHostToDevice, b->stream));
    launch_region_state(offset_particles(b->P[b->cur], h.p0), h.n, cx, cy, radius * radius, b->region.p, b->stream);
    BK(cudaMemcpyAsync(acc.data(), b->region.p, acc.size(), cudaMemcpyDeviceToHost, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    region_acc_finalize(acc.data(), out);
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_substeps(emerge_batch *b, uint64_t *last, uint64_t *total) {
    if (!b || (!last && !total)) return EMERGE_ERR_INVALID_ARG;
    std::vector<StepState> st;
    emerge_status s = read_states(b, st);
    if (s != EMERGE_OK) return s;
    for (size_t k = 0; k < b->scenes.size(); ++k) {
        if (last) last[k] = st[k].substeps;
        if (total) total[k] = st[k].total_substeps;
    }
    return EMERGE_OK;
}

emerge_status emerge_cuda_batch_set_option(emerge_batch *b, int option, int64_t value) {
    if (!b) return EMERGE_ERR_INVALID_ARG;
    switch (option) {
    case EMERGE_OPT_USE_GRAPH: b->use_graph = value != 0; return EMERGE_OK;
    case EMERGE_OPT_SORT_INTERVAL:
        if (value < 0) return static_cast<emerge_status>(b->fail(EMERGE_ERR_INVALID_ARG, "sort interval < 0"));
        b->sort_interval = value;
        return EMERGE_OK;
    case EMERGE_OPT_P2G_AGGREGATE:  // kernel codes: 1 warp segments, 3 lane pairs / quads
        if (value < 0 || value > 2)
            return static_cast<emerge_status>(b->fail(EMERGE_ERR_INVALID_ARG, "P2G aggregation mode must be 0, 1 or 2"));
        b->aggregate = value == 2 ? 3 : static_cast<int>(value);
        b->graph_dirty = true;
        return EMERGE_OK;
    case EMERGE_OPT_TILE_SHAPE:
        if (value < 0 || value > 3)
            return static_cast<emerge_status>(b->fail(EMERGE_ERR_INVALID_ARG, "tile shape must be 0..3"));
        b->tile_shape = static_cast<int>(value);
        b->sorted_once = false;  // re-sort in the new order before the next frame
        return EMERGE_OK;
    case EMERGE_OPT_CHUNKS_PER_CTA:
        if (value != 1 && value != 2 && value != 4)
            return static_cast<emerge_status>(b->fail(EMERGE_ERR_INVALID_ARG, "chunks per CTA must be 1, 2 or 4"));
        b->chunks = static_cast<int>(value);
        b->graph_dirty = true;
        return EMERGE_OK;
    default: return static_cast<emerge_status>(b->fail(EMERGE_ERR_INVALID_ARG, "option not available for batches"));
    }
}

// Autotuner.  Four knobs change no result beyond float summation order: the particle order
// the sort gives each scene (tile shape), the particles each CTA of the particle and density
// passes takes (256 per chunk, 1, 2 or 4 chunks), the sort interval and the P2G warp
// aggregation.  Coordinate descent from the current setting: each knob in turn takes every
// value while the others keep their best so far; each trial re-sorts, runs one untimed frame
// and times steps_per_trial frames of the batch itself (the trials advance the scenes).  With a cache file, a batch of the same
// signature (device, SM count, every scene's grid size, particle count and model set) takes
// the stored choice without trials, and a tuned choice is stored.
emerge_status emerge_cuda_batch_autotune(emerge_batch *b, uint32_t steps_per_trial, const char *cache_path,
                                         emerge_batch_tune_report *rep) {
    if (!b || steps_per_trial == 0) return EMERGE_ERR_INVALID_ARG;
    emerge_batch_tune_report r;
    std::memset(&r, 0, sizeof(r));
    const std::string key = tune_signature(b);
    TuneChoice cur{static_cast<int>(b->sort_interval), b->aggregate == 3 ? 0 : b->aggregate, b->tile_shape, b->chunks, 0.0f};
    if (cache_path && cache_path[0] && cache_lookup(cache_path, key, cur)) {
        r.from_cache = 1u;
    } else {
        float best = 1e30f;
        auto trial = [&](const TuneChoice &c) -> emerge_status {
            b->sort_interval = c.sort_interval;
            b->aggregate = c.aggregate;
            b->tile_shape = c.tile_shape;
            b->chunks = c.chunks;
            b->graph_dirty = true;
            b->sorted_once = false;
            // one untimed frame rebuilds the frame graph and re-sorts in the new tile shape
            emerge_status st = emerge_cuda_batch_step(b, 1);
            if (st != EMERGE_OK) return st;
            float ms = 0.0f;
            st = emerge_cuda_batch_time_steps(b, steps_per_trial, 0, &ms);
            if (st != EMERGE_OK) return st;
            const uint32_t t = r.n_trials;
            if (t < EMERGE_TUNE_MAX_TRIALS) {
                r.trial_sort_interval[t] = c.sort_interval;
                r.trial_aggregate[t] = c.aggregate;
                r.trial_tile_shape[t] = c.tile_shape;
                r.trial_chunks[t] = c.chunks;
                r.trial_ms[t] = ms / steps_per_trial;
                r.n_trials = t + 1;
            }
            if (ms / steps_per_trial < best) {
                best = ms / steps_per_trial;
                cur = c;
                cur.ms = best;
            }
            return EMERGE_OK;
        };
        const int shapes[4] = {0, 1, 2, 3}, chunks[3] = {1, 2, 4}, intervals[3] = {4, 8, 16}, aggs[2] = {0, 1};
        for (int v : shapes) {
            TuneChoice c = cur;
            c.tile_shape = v;
            emerge_status st = trial(c);
            if (st != EMERGE_OK) return st;
        }
        for (int v : chunks) {
            TuneChoice c = cur;
            c.chunks = v;
            emerge_status st = trial(c);
            if (st != EMERGE_OK) return st;
        }
        for (int v : intervals) {
            TuneChoice c = cur;
            c.sort_interval = v;
            emerge_status st = trial(c);
            if (st != EMERGE_OK) return st;
        }
        for (int v : aggs) {
            TuneChoice c = cur;
            c.aggregate = v;
            emerge_status st = trial(c);
            if (st != EMERGE_OK) return st;
        }
        if (cache_path && cache_path[0]) cache_store(cache_path, key, cur);
    }
    b->sort_interval = cur.sort_interval;
    b->aggregate = cur.aggregate;
    b->tile_shape = cur.tile_shape;
    b->chunks = cur.chunks;
    b->graph_dirty = true;
    b->sorted_once = false;
    r.sort_interval = cur.sort_interval;
    r.aggregate = cur.aggregate;
    r.tile_shape = cur.tile_shape;
    r.chunks_per_cta = cur.chunks;
    r.best_ms = cur.ms;
    if (rep) *rep = r;
    return EMERGE_OK;
}

}  // extern "C"
