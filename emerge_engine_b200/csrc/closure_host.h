// closure_host.h -- host-side glue between the simulation runtime (sim.cu) and the
// learned-closure manager (closure.cu).
#pragma once

#include <string>

#include "../../include/emerge_cuda.h"
#include "closure.cuh"

namespace emerge {

struct ClosureHost;  // closure.cu: networks, statistics, log buffers, master weights

// Kernel arguments of the closure (all zero when the simulation has none).
ClosureArgs closure_args(const ClosureHost *c);
void closure_destroy(ClosureHost *c);

// sim.cu: the pieces of a simulation the closure manager uses.
cudaStream_t sim_stream(emerge_sim *s);
ClosureHost *&sim_closure(emerge_sim *s);
void sim_invalidate_graph(emerge_sim *s);
emerge_status sim_fail(emerge_sim *s, emerge_status st, const std::string &msg);

}  // namespace emerge
