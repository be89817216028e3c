// closure_host.h -- host-side glue between the simulation runtime (sim.cu) and the
// learned-closure manager (closure.cu).
#pragma once

#include <string>
#include <vector>

#include "../../include/emerge_cuda.h"
#include "closure.cuh"
#include "kernels.h"

namespace emerge {

struct ClosureHost;  // closure.cu: networks, statistics, log buffers, master weights

// Kernel arguments of the closure (all zero when the simulation has none).
ClosureArgs closure_args(const ClosureHost *c, size_t n);
void closure_destroy(ClosureHost *c);

// sim.cu: a simulation's scene description, for building batches (batch.cu).
struct SimView {
    emerge_sim_config cfg;
    std::vector<uint64_t> bounds;
    std::vector<emerge_material_params> mats;
    LoadFlagsHost lf;
    DevConfig dcfg;
    int deterministic;
    size_t n;
    int device;
};
SimView sim_view(emerge_sim *s);
// Byte size of, and carving of, one particle set of capacity `cap` (256-byte pieces).
size_t particle_set_size(size_t cap);
DevParticles particle_set_carve(void *base, size_t cap);

// sim.cu: the pieces of a simulation the closure manager uses.
cudaStream_t sim_stream(emerge_sim *s);
size_t sim_capacity(emerge_sim *s);  // particle capacity of the device storage (at least 1)
ClosureHost *&sim_closure(emerge_sim *s);
void sim_invalidate_graph(emerge_sim *s);
emerge_status sim_fail(emerge_sim *s, emerge_status st, const std::string &msg);

}  // namespace emerge
